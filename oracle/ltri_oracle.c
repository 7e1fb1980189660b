/* Laplace layer potentials on flat triangles: CPU restatement (test
 * infrastructure only; included by fmm3d_oracle.c, sharing its tree, lists,
 * expansions and far-field passes).
 *
 * Restated from the reference:
 *   lfmm3dtriatarg / lfmm3dtriatargmain  src/lfmm3dtria.f:121-1160
 *   l3dtriadirect                        src/lfmm3dtria.f:1385-1560
 *   near-field integrals direct3dtritarglaps2 / direct3dtritarglapd2 and the
 *   self terms direct3dtrilaps2 / direct3dtrilapd2 (src/triquadflatlib.f:147,
 *   340, 533, 726), which integrate 1/r and its derivatives exactly over a
 *   flat triangle (triahquad, src/triahquad.f:63)
 *   far-field forms l3dformmptris2_add / l3dformmptrid2_add and the P2L
 *   forms (src/l3dtrirouts.f:803-1000): the triangle's density as point
 *   charges (dipoles along the normal) at quadrature nodes.
 *
 * The potential of triangle T with unit density at x is
 *   single layer  S(x) = int_T 1/|x-y| dS_y,          field -grad S,
 *   double layer  D(x) = int_T n.(x-y)/|x-y|^3 dS_y,  field -grad D,
 * n = (v2-v1)x(v3-v1)/|.| (the frame of tri_ini, src/trilib.f:445-520).  At
 * a triangle's own centroid the reference takes the in-plane value (iquad =
 * 0): the jump terms of the normal derivative of S and of D vanish there.
 *
 * Closed forms (this restatement's own derivation of the exact integrals the
 * reference evaluates): with h = n.(x - v1) and, per edge a -> b, unit tangent
 * t, outward in-plane normal m = t x n, s- = (a-x).t, s+ = (b-x).t,
 * p = (a-x).m, R- = |a-x|, R+ = |b-x|,
 *   f    = log((R+ + s+)/(R- + s-)),
 *   beta = atan2(p s+, p^2 + h^2 + |h| R+) - atan2(p s-, p^2 + h^2 + |h| R-),
 *   S = sum p f - |h| sum beta,   grad S = -sum m f - sign(h) n sum beta,
 *   D = sign(h) sum beta (the signed solid angle, taken in closed form below),
 *   grad D = - sum (u x w)(|u|+|w|) / (|u||w|(|u||w| + u.w)),  u = x-a, w = x-b.
 *
 * Far-field quadrature: the reference's symmetric rules (triasymq,
 * src/triasymq.f) are tabulated numbers that are not restated here; the
 * triangle's density is integrated with a collapsed Gauss-Legendre product
 * rule of the same polynomial degree instead (degree 1: the centroid; degree
 * 2k: k+1 x k+1 nodes), so the far field differs from the reference's by the
 * two rules' quadrature errors, far below the FMM truncation error at the
 * reference's degrees (nqtri = 2 for iprec -2 and -1, 4 for 0, 6 for
 * iprec >= 1, src/lfmm3dtria.f:679-701).                                    */

void oracle_legewhts(int n, double *x, double *w);

static void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* S, grad S, D, grad D of triangle v[9] (vertices v1, v2, v3) at x; self:
 * x is the triangle's own centroid (in-plane values).  The sum of the edge
 * angles beta (the solid angle) is taken in one atan2 by the formula of Van
 * Oosterom and Strackee (1983); D = sign(h) sum beta is that signed solid
 * angle, and S = sum p f - h D, grad S = -sum m f - n D. */
static void tri_near(const double *v, const double *x, int self, double *S, double *gS, double *D, double *gD)
{
    double e1[3], e2[3], n[3];
    for (int c = 0; c < 3; c++) { e1[c] = v[3 + c] - v[c]; e2[c] = v[6 + c] - v[c]; }
    cross3(e1, e2, n);
    double nn = sqrt(dot3(n, n));
    for (int c = 0; c < 3; c++) n[c] /= nn;
    double dv[3][3], R[3];
    for (int k = 0; k < 3; k++) {
        for (int c = 0; c < 3; c++) dv[k][c] = v[3 * k + c] - x[c];
        R[k] = sqrt(dot3(dv[k], dv[k]));
    }
    const double h = self ? 0.0 : -dot3(n, dv[0]);
    double om = 0;
    if (!self) {
        double bc[3];
        cross3(dv[1], dv[2], bc);
        const double num = dot3(dv[0], bc);
        const double den = R[0] * R[1] * R[2] + dot3(dv[0], dv[1]) * R[2] + dot3(dv[0], dv[2]) * R[1] +
                           dot3(dv[1], dv[2]) * R[0];
        om = 2.0 * atan2(-num, den);
    }
    double spf = 0, gm[3] = {0, 0, 0}, bs[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++) {
        const int a = i, b = (i + 1) % 3;
        double t[3], m[3];
        for (int c = 0; c < 3; c++) t[c] = dv[b][c] - dv[a][c];
        double L = sqrt(dot3(t, t));
        for (int c = 0; c < 3; c++) t[c] /= L;
        cross3(t, n, m);
        const double sm = dot3(dv[a], t), sp = dot3(dv[b], t), pd = dot3(dv[a], m);
        const double f = (sp + sm >= 0) ? log((R[b] + sp) / (R[a] + sm)) : log((R[a] - sm) / (R[b] - sp));
        spf += pd * f;
        for (int c = 0; c < 3; c++) gm[c] += m[c] * f;
        /* segment a -> b: (u x w)(|u|+|w|)/(|u||w|(|u||w|+u.w)), u = x-a = -dv[a], w = x-b = -dv[b] */
        double uw[3];
        cross3(dv[a], dv[b], uw);   /* (-u) x (-w) = u x w */
        const double co = (R[a] + R[b]) / (R[a] * R[b] * (R[a] * R[b] + dot3(dv[a], dv[b])));
        for (int c = 0; c < 3; c++) bs[c] += uw[c] * co;
    }
    *S = spf - h * om;
    for (int c = 0; c < 3; c++) gS[c] = -gm[c] - n[c] * om;
    *D = om;
    for (int c = 0; c < 3; c++) gD[c] = -bs[c];
}

/* Collapsed Gauss-Legendre rule on the reference triangle (0,0),(1,0),(0,1)
 * of polynomial degree >= norder: barycentric-free coordinates (xi, eta)
 * and weights summing to 1 (multiply by the area). */
static int tri_rule(int norder, double *xi, double *eta, double *w)
{
    if (norder <= 1) { xi[0] = eta[0] = 1.0 / 3.0; w[0] = 1.0; return 1; }
    int k = norder / 2 + 1;
    double x[16], wx[16];
    oracle_legewhts(k, x, wx);
    int q = 0;
    for (int i = 0; i < k; i++) {
        double u = 0.5 * (x[i] + 1), wu = 0.5 * wx[i];
        for (int j = 0; j < k; j++) {
            double vv = 0.5 * (x[j] + 1), wv = 0.5 * wx[j];
            xi[q] = u;
            eta[q] = (1 - u) * vv;
            w[q] = 2 * wu * wv * (1 - u);   /* the reference triangle's area is 1/2 */
            q++;
        }
    }
    return q;
}

/* nqtri per iprec, src/lfmm3dtria.f:679-701: 1 by default, 2 for iprec -2 / -1, 4 for 0, 6 for >= 1 */
static int tri_norder(int iprec)
{
    if (iprec == -2 || iprec == -1) return 2;
    if (iprec == 0) return 4;
    if (iprec >= 1) return 6;
    return 1;
}

/* nbox of lfmm3dtriatarg, src/lfmm3dtria.f:290-300 (integer divisions as written) */
int oracle_tri_nbox(int iprec, int ns, int nt)
{
    switch (iprec) {
    case -2: return 8 / 3;
    case -1: return 15 / 3;
    case 0: return 30 / 3;
    case 1: return 60 / 3;
    case 2: return 120 / 3;
    case 3: return 240 / 3;
    case 4: return 480 / 3;
    case 5: return 700 / 3;
    case 6: return ns + nt;
    }
    return -1;
}

/* Quadrature nodes of triangles tri[9*i] (i < n): positions, weights * area. */
static void tri_nodes(int n, const double *tri, int norder, double *pos, double *wt, int *nq_out)
{
    double xi[64], eta[64], w[64];
    int nq = tri_rule(norder, xi, eta, w);
    for (int i = 0; i < n; i++) {
        const double *v = tri + 9 * (size_t)i;
        double e1[3], e2[3], c[3];
        for (int d = 0; d < 3; d++) { e1[d] = v[3 + d] - v[d]; e2[d] = v[6 + d] - v[d]; }
        cross3(e1, e2, c);
        double area = 0.5 * sqrt(dot3(c, c));
        for (int k = 0; k < nq; k++) {
            for (int d = 0; d < 3; d++) pos[3 * ((size_t)i * nq + k) + d] = v[d] + xi[k] * e1[d] + eta[k] * e2[d];
            wt[(size_t)i * nq + k] = w[k] * area;
        }
    }
    *nq_out = nq;
}

void oracle_tri_rule(int norder, double *xi, double *eta, double *w, int *nq) { *nq = tri_rule(norder, xi, eta, w); }

void oracle_tri_near(const double *v, int npts, const double *x, int self, double *S, double *gS, double *D,
                     double *gD)
{
    for (int i = 0; i < npts; i++)
        tri_near(v, x + 3 * (size_t)i, self, S + i, gS + 3 * (size_t)i, D + i, gD + 3 * (size_t)i);
}

/* One evaluation point against triangles [j0, j0+nj): adds pot and fld. */
static void tri_point(int nj, const double *tri, int ifcharge, const cplx *q, int ifdipole, const cplx *ds,
                      const double *x, long self, int iffld, cplx *pot, cplx *fld)
{
    for (int j = 0; j < nj; j++) {
        double S, gS[3], D, gD[3];
        tri_near(tri + 9 * (size_t)j, x, j == self, &S, gS, &D, gD);
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

/* The direct sum at arbitrary points; point k is the centroid of triangle self[k] (or -1). */
void oracle_tri_direct_points(int ns, const double *tri, int ifcharge, const cplx *charge, int ifdipole,
                              const cplx *dipstr, int npts, const double *pts, const long *self, cplx *pot, cplx *fld)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (long k = 0; k < npts; k++) {
        cplx pv = 0, fv[3] = {0, 0, 0};
        tri_point(ns, tri, ifcharge, charge, ifdipole, dipstr, pts + 3 * k, self ? self[k] : -1, 1, &pv, fv);
        pot[k] = pv;
        for (int c = 0; c < 3; c++) fld[3 * k + c] = fv[c];
    }
}

/* l3dtriadirect: every triangle at every centroid (self by index) and target. */
void oracle_l3dtriadirect(int ns, const double *tri, const double *source, int ifcharge, const cplx *charge,
                          int ifdipole, const cplx *dipstr, int ifpot, cplx *pot, int iffld, cplx *fld, int nt,
                          const double *target, int ifpottarg, cplx *pottarg, int iffldtarg, cplx *fldtarg)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < ns + (long)nt; i++) {
        const int is_src = i < ns;
        const long k = is_src ? i : i - ns;
        if (is_src && !(ifpot == 1 || iffld == 1)) continue;
        if (!is_src && !(ifpottarg == 1 || iffldtarg == 1)) continue;
        cplx pv = 0, fv[3] = {0, 0, 0};
        tri_point(ns, tri, ifcharge, charge, ifdipole, dipstr, (is_src ? source : target) + 3 * k, is_src ? k : -1,
                  is_src ? iffld == 1 : iffldtarg == 1, &pv, fv);
        if (is_src) {
            if (ifpot == 1) pot[k] = pv;
            if (iffld == 1) for (int c = 0; c < 3; c++) fld[3 * k + c] = fv[c];
        } else {
            if (ifpottarg == 1) pottarg[k] = pv;
            if (iffldtarg == 1) for (int c = 0; c < 3; c++) fldtarg[3 * k + c] = fv[c];
        }
    }
}

/* lfmm3dtriatarg: the tree on the centroids and targets with the triangle
 * FMM's nbox, far field from the triangles' quadrature nodes (P2M, P2L over
 * list 4), STEPS 3-5 as the particle FMM, M2P / L2P at centroids and
 * targets, near field (self box and list 1) by the exact integrals. */
void oracle_lfmm3dtriatarg(int *ier, int iprec, int ns, const double *tri, const double *trinorm,
                           const double *source, int ifcharge, const cplx *charge, int ifdipole, const cplx *dipstr,
                           int ifpot, cplx *pot, int iffld, cplx *fld, int nt, const double *target, int ifpottarg,
                           cplx *pottarg, int iffldtarg, cplx *fldtarg)
{
    *ier = 0;
    double eps = oracle_lap_eps(iprec);
    int nbox = oracle_tri_nbox(iprec, ns, nt);
    if (nbox < 1 || ns < 1) { *ier = 4; return; }
    otree T;
    memset(&T, 0, sizeof T);
    build_boxes(&T, source, ns, target, nt, nbox);
    build_lists(&T);
    int p = oracle_l3dterms(eps);
    int K = (p + 1) * (p + 1), nb = T.nboxes;
    size_t ntt = nt > 0 ? nt : 1;
    double *ss = malloc(sizeof(double) * 3 * (size_t)ns), *ts = malloc(sizeof(double) * 3 * ntt);
    double *trs = malloc(sizeof(double) * 9 * (size_t)ns), *nrs = malloc(sizeof(double) * 3 * (size_t)ns);
    cplx *qs = calloc(ns, sizeof(cplx)), *dss = calloc(ns, sizeof(cplx));
    for (int i = 0; i < ns; i++) {
        int j = T.iz[i];
        memcpy(ss + 3 * (size_t)i, source + 3 * (size_t)j, 3 * sizeof(double));
        memcpy(trs + 9 * (size_t)i, tri + 9 * (size_t)j, 9 * sizeof(double));
        memcpy(nrs + 3 * (size_t)i, trinorm + 3 * (size_t)j, 3 * sizeof(double));
        if (ifcharge == 1) qs[i] = charge[j];
        if (ifdipole == 1) dss[i] = dipstr[j];
    }
    for (int i = 0; i < nt; i++) memcpy(ts + 3 * (size_t)i, target + 3 * (size_t)T.iztarg[i], 3 * sizeof(double));
    /* quadrature nodes in tree order: triangle i owns nodes [i nq, (i+1) nq) */
    double xi[64], eta[64], wr[64];
    int nq = tri_rule(tri_norder(iprec), xi, eta, wr);
    size_t nn = (size_t)ns * nq;
    double *qp = malloc(sizeof(double) * 3 * nn), *qw = malloc(sizeof(double) * nn), *qv = malloc(sizeof(double) * 3 * nn);
    cplx *qq = calloc(nn, sizeof(cplx)), *qd = calloc(nn, sizeof(cplx));
    tri_nodes(ns, trs, tri_norder(iprec), qp, qw, &nq);
    for (size_t i = 0; i < nn; i++) {
        size_t t = i / nq;
        if (ifcharge == 1) qq[i] = qs[t] * qw[i];
        if (ifdipole == 1) qd[i] = dss[t] * qw[i];
        memcpy(qv + 3 * i, nrs + 3 * t, 3 * sizeof(double));
    }
    cplx *ps = calloc(ns, sizeof(cplx)), *fs = calloc(3 * (size_t)ns, sizeof(cplx));
    cplx *pt = calloc(ntt, sizeof(cplx)), *ft = calloc(3 * ntt, sizeof(cplx));
    cplx *mpole = calloc((size_t)nb * K, sizeof(cplx)), *local = calloc((size_t)nb * K, sizeof(cplx));
#define BX(b, f) T.box[20 * (size_t)(b) + (f)]
#define LS(ty, b) T.lstart[ty][b]
#define LE(ty, b) T.lstart[ty][(b) + 1]
#define LI(ty, i) T.lidx[ty][i]
    double tm[9];
    /* STEP 1: P2M from the quadrature nodes of every childless box (src/lfmm3dtria.f:737-806) */
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        if (BX(ib, B_NSRC) == 0 || nkids(&T, ib) != 0) continue;
        size_t s0 = (size_t)BX(ib, B_SRC0) * nq;
        int n = BX(ib, B_NSRC) * nq;
        oracle_formmp(n, qp + 3 * s0, ifcharge, qq + s0, ifdipole, qd + s0, qv + 3 * s0, T.center + 3 * (size_t)ib, p,
                      mpole + (size_t)ib * K);
    }
    /* STEP 2: P2L from the nodes of list-4 boxes (the reference walks list 3 of the source box, :816-893) */
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        for (int li = LS(4, ib); li < LE(4, ib); li++) {
            int jb = LI(4, li);
            if (BX(jb, B_NSRC) == 0) continue;
            size_t s0 = (size_t)BX(jb, B_SRC0) * nq;
            int n = BX(jb, B_NSRC) * nq;
            oracle_formta(n, qp + 3 * s0, ifcharge, qq + s0, ifdipole, qd + s0, qv + 3 * s0, T.center + 3 * (size_t)ib,
                          p, local + (size_t)ib * K);
        }
    }
    far_passes(&T, p, eps, mpole, local, !(ifpot == 1 || iffld == 1), tm);
    /* STEPS 6, 7: M2P from list 3 and L2P at leaves of level >= 2, at centroids and targets (:910-1057) */
#pragma omp parallel
    {
        double *pp = malloc(sizeof(double) * (p + 2) * (p + 2)), *ppd = malloc(sizeof(double) * (p + 2) * (p + 2));
#pragma omp for schedule(dynamic)
        for (int ib = 0; ib < nb; ib++) {
            if (nkids(&T, ib) != 0) continue;
            cplx pv, fv[3];
            for (int li = LS(3, ib); li < LE(3, ib); li++) {
                int jb = LI(3, li);
                const double *cj = T.center + 3 * (size_t)jb;
                const cplx *mj = mpole + (size_t)jb * K;
                for (int i = BX(ib, B_SRC0); i < BX(ib, B_SRC0) + BX(ib, B_NSRC); i++) {
                    mpeval(cj, mj, p, ss + 3 * (size_t)i, &pv, fv, pp, ppd);
                    ps[i] += pv;
                    for (int c = 0; c < 3; c++) fs[3 * (size_t)i + c] += fv[c];
                }
                for (int i = BX(ib, B_TRG0); i < BX(ib, B_TRG0) + BX(ib, B_NTRG); i++) {
                    mpeval(cj, mj, p, ts + 3 * (size_t)i, &pv, fv, pp, ppd);
                    pt[i] += pv;
                    for (int c = 0; c < 3; c++) ft[3 * (size_t)i + c] += fv[c];
                }
            }
            if (BX(ib, B_LEV) < 2) continue;
            const double *cb = T.center + 3 * (size_t)ib;
            const cplx *lb = local + (size_t)ib * K;
            for (int i = BX(ib, B_SRC0); i < BX(ib, B_SRC0) + BX(ib, B_NSRC); i++) {
                taeval(cb, lb, p, ss + 3 * (size_t)i, &pv, fv, pp, ppd);
                ps[i] += pv;
                for (int c = 0; c < 3; c++) fs[3 * (size_t)i + c] += fv[c];
            }
            for (int i = BX(ib, B_TRG0); i < BX(ib, B_TRG0) + BX(ib, B_NTRG); i++) {
                taeval(cb, lb, p, ts + 3 * (size_t)i, &pv, fv, pp, ppd);
                pt[i] += pv;
                for (int c = 0; c < 3; c++) ft[3 * (size_t)i + c] += fv[c];
            }
        }
        free(pp); free(ppd);
    }
    /* STEP 8: near field, self box and list 1, by the exact integrals (:1067-1140) */
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        if (nkids(&T, ib) != 0) continue;
        int s0 = BX(ib, B_SRC0), nsb = BX(ib, B_NSRC), t0 = BX(ib, B_TRG0), ntg = BX(ib, B_NTRG);
        int nl = 1 + LE(1, ib) - LS(1, ib);
        for (int li = 0; li < nl; li++) {
            int jb = li == 0 ? ib : LI(1, LS(1, ib) + li - 1);
            int js0 = BX(jb, B_SRC0), jn = BX(jb, B_NSRC);
            if (jn == 0) continue;
            for (int i = s0; i < s0 + nsb; i++)
                tri_point(jn, trs + 9 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0, ss + 3 * (size_t)i,
                          jb == ib ? i - s0 : -1, 1, ps + i, fs + 3 * (size_t)i);
            for (int i = t0; i < t0 + ntg; i++)
                tri_point(jn, trs + 9 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0, ts + 3 * (size_t)i, -1, 1,
                          pt + i, ft + 3 * (size_t)i);
        }
    }
    /* unsort (l3dpsort / l3dfsort) */
    for (int i = 0; i < ns; i++) {
        int j = T.iz[i];
        if (ifpot == 1) pot[j] = ps[i];
        if (iffld == 1) for (int d = 0; d < 3; d++) fld[3 * (size_t)j + d] = fs[3 * (size_t)i + d];
    }
    for (int i = 0; i < nt; i++) {
        int j = T.iztarg[i];
        if (ifpottarg == 1) pottarg[j] = pt[i];
        if (iffldtarg == 1) for (int d = 0; d < 3; d++) fldtarg[3 * (size_t)j + d] = ft[3 * (size_t)i + d];
    }
#undef BX
#undef LS
#undef LE
#undef LI
    free(ss); free(ts); free(trs); free(nrs); free(qs); free(dss); free(qp); free(qw); free(qv); free(qq); free(qd);
    free(ps); free(fs); free(pt); free(ft); free(mpole); free(local);
    tree_free(&T);
}
