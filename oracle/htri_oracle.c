/* Helmholtz layer potentials on flat triangles: CPU restatement (test
 * infrastructure only; included by fmm3d_oracle.c after the Helmholtz FMM,
 * whose core runs in triangle mode for it).
 *
 * Restated from the reference:
 *   hfmm3dtriatarg / hfmm3dtriatargmain  src/hfmm3dtria.f:133-1215
 *   h3dtriadirect                        src/hfmm3dtria.f (the O(N^2) sum)
 *   near field direct3dtritarghelms3 / direct3dtrihelms2 / direct3dtritarghelmd3
 *   / direct3dtrihelmd2 with triquadhelm2, triquadselfhelm, triquadhelmd2 and
 *   triquadselfhelmd (src/triquadflatlib.f:819-2356): the Laplace part of
 *   the kernel integrated exactly (the closed forms of ltri_oracle.c), the
 *   difference e^{ikr}/r - 1/r (and its derivatives) by a quadrature rule on
 *   the triangle, with four-term Taylor series when |k r| < 0.01, and at a
 *   triangle's own centroid the parts that the rule cannot integrate
 *   subtracted and integrated in closed form.
 *
 * With z = i k r, d = x - y, h = n.(x - v1) and
 *   g  = (e^z - 1)/r,                 grad_x g = (d/r) F/r^2,  F = e^z (z - 1) + 1,
 *   f2 = ((1 - z) e^z - 1)/r^3 = -F/r^3,   f2' = k^2 e^z / r^2 + 3 F / r^4,
 * the single layer adds int g (value) and int grad_x g; the double layer
 * (n.grad_y of the kernel) adds h int f2 and int (n f2 + h f2' d/r).  At the
 * triangle's own centroid (h = 0): the charge gradient's quadrature takes
 * grad_x g - (ik)^2/2 d/r and adds (ik)^2/2 int d/r dS = -(ik)^2/2 sum_e m_e
 * int_e r dl; the double layer's value and in-plane gradient vanish and its
 * normal gradient is int (f2 - k^2/(2r)) + (k^2/2) int 1/r.
 *
 * Quadrature: as for the Laplace triangles, collapsed Gauss-Legendre rules of
 * the reference's degrees stand in for its symmetric rules (triasymq): far
 * field norder = 2, 2, 4, 4 and near field nqtri = 2, 2, 4, 6 for iprec
 * -2, -1, 0, >= 1, else 1 and 1 (src/hfmm3dtria.f:730-751).               */

typedef struct {
    int n;
    double xi[64], eta[64], w[64];
} trule;

static trule g_trules[8];
static int g_trules_ready[8];

static const trule *get_trule(int deg)
{
    if (deg < 1) deg = 1;
    if (deg > 7) deg = 7;
    if (!g_trules_ready[deg]) {
#pragma omp critical(htri_rule)
        {
            if (!g_trules_ready[deg]) {
                g_trules[deg].n = tri_rule(deg, g_trules[deg].xi, g_trules[deg].eta, g_trules[deg].w);
                g_trules_ready[deg] = 1;
            }
        }
    }
    return &g_trules[deg];
}

static int htri_norder(int iprec) { return (iprec == -2 || iprec == -1) ? 2 : iprec >= 0 ? 4 : 1; }
static int htri_nqtri(int iprec) { return (iprec == -2 || iprec == -1) ? 2 : iprec == 0 ? 4 : iprec >= 1 ? 6 : 1; }

/* Helmholtz single layer S, grad S and double layer D, grad D (gradients in x)
 * of triangle v[9] with unit density at x. */
static void htri_near(cplx zk, const double *v, const double *x, int self, const trule *r, cplx *S, cplx *gS,
                      cplx *D, cplx *gD)
{
    double Sl, gSl[3], Dl, gDl[3];
    tri_near(v, x, self, &Sl, gSl, &Dl, gDl);
    double e1[3], e2[3], n[3];
    for (int c = 0; c < 3; c++) { e1[c] = v[3 + c] - v[c]; e2[c] = v[6 + c] - v[c]; }
    cross3(e1, e2, n);
    const double nn = sqrt(dot3(n, n)), area = 0.5 * nn;
    for (int c = 0; c < 3; c++) n[c] /= nn;
    double xv[3] = {x[0] - v[0], x[1] - v[1], x[2] - v[2]};
    const double h = self ? 0.0 : dot3(n, xv);
    const cplx ik = I * zk, ik2 = ik * ik;
    cplx sp = 0, sg[3] = {0, 0, 0}, dp = 0, dg[3] = {0, 0, 0}, dn = 0;
    for (int q = 0; q < r->n; q++) {
        double d[3];
        for (int c = 0; c < 3; c++) d[c] = x[c] - (v[c] + r->xi[q] * e1[c] + r->eta[q] * e2[c]);
        /* a node on x itself (the one-node rule at a triangle's own centroid) adds the
         * limit of the bounded difference kernel: its value ik, a zero gradient */
        const double r2 = dot3(d, d), rr = sqrt(r2), ir = rr > 0 ? 1.0 / rr : 0.0, w = r->w[q] * area;
        const cplx z = ik * rr;
        cplx g, Fr2, f2, f2p, f2s;
        if (cabs(z) < 0.01) {
            const cplx ik3 = ik2 * ik, ik4 = ik3 * ik, ik5 = ik4 * ik, ik6 = ik5 * ik;
            g = ik * (1.0 + z / 2.0 + z * z / 6.0 + z * z * z / 24.0 + z * z * z * z / 120.0);
            Fr2 = ik2 / 2.0 + rr * ik3 / 3.0 + r2 * ik4 / 8.0 + r2 * rr * ik5 / 30.0;
            f2s = -(ik3 / 3.0 + rr * ik4 / 8.0 + r2 * ik5 / 30.0 + r2 * rr * ik6 / 144.0);
            f2 = f2s - ik2 / 2.0 * ir;
            f2p = ik2 / 2.0 * ir * ir - ik4 / 8.0 - 2.0 * rr * ik5 / 30.0 - 3.0 * r2 * ik6 / 144.0;
        } else {
            const cplx E = cexp(z), F = E * (z - 1.0) + 1.0;
            g = (E - 1.0) / rr;
            Fr2 = F / r2;
            f2 = -F / (rr * r2);
            f2s = f2 + ik2 / (2.0 * rr);
            f2p = -ik2 * E / r2 + 3.0 * F / (r2 * r2);
        }
        sp += w * g;
        for (int c = 0; c < 3; c++) sg[c] += w * (d[c] * ir) * (self ? Fr2 - ik2 / 2.0 : Fr2);
        if (self) {
            dn += w * f2s;
        } else {
            dp += w * h * f2;
            for (int c = 0; c < 3; c++) dg[c] += w * (n[c] * f2 + h * f2p * d[c] * ir);
        }
    }
    *S = Sl + sp;
    for (int c = 0; c < 3; c++) gS[c] = gSl[c] + sg[c];
    *D = Dl + dp;
    for (int c = 0; c < 3; c++) gD[c] = gDl[c] + dg[c];
    if (self) {
        /* (ik)^2/2 int_T d/r dS = -(ik)^2/2 sum_e m_e int_e r dl, in the plane (h = 0) */
        double J[3] = {0, 0, 0}, dv[3][3], R[3];
        for (int k = 0; k < 3; k++) {
            for (int c = 0; c < 3; c++) dv[k][c] = v[3 * k + c] - x[c];
            R[k] = sqrt(dot3(dv[k], dv[k]));
        }
        for (int i = 0; i < 3; i++) {
            const int a = i, b = (i + 1) % 3;
            double t[3], m[3];
            for (int c = 0; c < 3; c++) t[c] = dv[b][c] - dv[a][c];
            double L = sqrt(dot3(t, t));
            for (int c = 0; c < 3; c++) t[c] /= L;
            cross3(t, n, m);
            const double sm = dot3(dv[a], t), spp = dot3(dv[b], t), pd = dot3(dv[a], m);
            const double f = (spp + sm >= 0) ? log((R[b] + spp) / (R[a] + sm)) : log((R[a] - sm) / (R[b] - spp));
            const double line = 0.5 * (spp * R[b] - sm * R[a] + pd * pd * f);
            for (int c = 0; c < 3; c++) J[c] -= m[c] * line;
        }
        for (int c = 0; c < 3; c++) gS[c] += ik2 / 2.0 * J[c];
        /* double layer: value and in-plane gradient 0, normal gradient int f2 = int f2s - (ik)^2/2 int 1/r */
        *D = 0;
        for (int c = 0; c < 3; c++) gD[c] = gDl[c] + n[c] * (dn - ik2 / 2.0 * Sl);
    }
}

static void htri_point(cplx zk, int nj, const double *tri, int ifcharge, const cplx *q, int ifdipole, const cplx *ds,
                       const double *x, long self, int iffld, int nqtri, cplx *pot, cplx *fld)
{
    const trule *r = get_trule(nqtri);
    *pot = 0;
    for (int c = 0; c < 3; c++) fld[c] = 0;
    for (int j = 0; j < nj; j++) {
        cplx S, gS[3], D, gD[3];
        htri_near(zk, tri + 9 * (size_t)j, x, j == self, r, &S, gS, &D, gD);
        if (ifcharge == 1) {
            *pot += q[j] * S;
            if (iffld) for (int c = 0; c < 3; c++) fld[c] -= q[j] * gS[c];
        }
        if (ifdipole == 1) {
            *pot += ds[j] * D;
            if (iffld) for (int c = 0; c < 3; c++) fld[c] -= ds[j] * gD[c];
        }
    }
}

void oracle_htri_near(double zkr, double zki, const double *v, int npts, const double *x, int self, int nqtri,
                      cplx *S, cplx *gS, cplx *D, cplx *gD)
{
    const trule *r = get_trule(nqtri);
    for (int i = 0; i < npts; i++)
        htri_near(zkr + I * zki, v, x + 3 * (size_t)i, self, r, S + i, gS + 3 * (size_t)i, D + i, gD + 3 * (size_t)i);
}

/* hfmm3dtriatarg (FP64): the Helmholtz FMM's core in triangle mode. */
void oracle_hfmm3dtriatarg(int *ier, int iprec, double zkr, double zki, int ns, const double *tri,
                           const double *trinorm, const double *source, int ifcharge, const cplx *charge, int ifdipole,
                           const cplx *dipstr, int ifpot, cplx *pot, int iffld, cplx *fld, int nt, const double *target,
                           int ifpottarg, cplx *pottarg, int iffldtarg, cplx *fldtarg)
{
    htri_args ta = {tri, trinorm, htri_norder(iprec), htri_nqtri(iprec)};
    hfmm_core(ier, iprec, zkr, zki, ns, source, ifcharge, charge, ifdipole, dipstr, trinorm, ifpot, pot, iffld, fld, nt,
              target, ifpottarg, pottarg, iffldtarg, fldtarg, NULL, NULL, &ta);
}

/* The direct sum at arbitrary points with the near-field integrals of degree
 * nqtri (h3dtriadirect uses those of its iprec); point k is the centroid of
 * triangle self[k] (or -1). */
void oracle_htri_direct_points(double zkr, double zki, int ns, const double *tri, int ifcharge, const cplx *charge,
                               int ifdipole, const cplx *dipstr, int npts, const double *pts, const long *self,
                               int nqtri, cplx *pot, cplx *fld)
{
    get_trule(nqtri);
#pragma omp parallel for schedule(dynamic, 8)
    for (long k = 0; k < npts; k++)
        htri_point(zkr + I * zki, ns, tri, ifcharge, charge, ifdipole, dipstr, pts + 3 * k, self ? self[k] : -1, 1,
                   nqtri, pot + k, fld + 3 * k);
}

int oracle_htri_nqtri(int iprec) { return htri_nqtri(iprec); }
