/* Laplace Hessians: CPU restatement (test infrastructure only; included by
 * fmm3d_oracle.c, sharing its tree, lists, expansions and Legendre helpers).
 *
 * Restated from the reference:
 *   lpotfld3dhess      src/laprouts3d.f:5442-5536   pair, charge
 *   lpotfld3dhess_dp   src/laprouts3d.f:5619-5735   pair, dipole
 *   l3dtaevalhessdini  src/laprouts3d.f:7613-7676   shift factors, local
 *   l3dtaevalhessd_trunc src/laprouts3d.f:7682-7906 pot/fld/hess of a local
 *   l3dmpevalhessdini  src/laprouts3d.f:7129-7188   shift factors, multipole
 *   l3dmpevalhessd_trunc src/laprouts3d.f:7194-7378 pot/fld/hess of a multipole
 * Hessians are the second derivatives of the potential, ordered dxx, dyy,
 * dzz, dxy, dxz, dyz (the layout l3dhsort unsorts, src/lfmm3drouts.f:621).
 * The FMM with Hessians (oracle_lfmm3dparttarg_hess) runs the passes of
 * lfmm3dparttargmain and adds, at every evaluation point, the Hessians of
 * the near-field pairs, of the list-3 multipoles and of the leaf's local
 * expansion with the routines above: the reference has the evaluators but no
 * particle driver that calls them.                                         */

static inline int par(int k) { return (k & 1) ? -1 : 1; }   /* (-1)**k for any integer k */

/* lpotfld3dhess: charge at s, target t (dxx, dyy, dzz, dxy, dxz, dyz) */
static void lpotfld3dhess_r(const double *s, cplx q, const double *t, cplx h[6])
{
    double xd = t[0] - s[0], yd = t[1] - s[1], zd = t[2] - s[2];
    double dd = xd * xd + yd * yd + zd * zd;
    double d = sqrt(dd), dinv = 1.0 / d, ddinv = dinv * dinv, dddinv = dinv * ddinv, d5 = ddinv * dddinv;
    cplx cd = q * d5;
    h[0] = cd * (3 * xd * xd - dd);
    h[1] = cd * (3 * yd * yd - dd);
    h[2] = cd * (3 * zd * zd - dd);
    h[3] = cd * 3 * xd * yd;
    h[4] = cd * 3 * xd * zd;
    h[5] = cd * 3 * yd * zd;
}

/* lpotfld3dhess_dp: dipole (strength ds, direction v) at s, target t */
static void lpotfld3dhess_dp_r(const double *s, cplx ds, const double *v, const double *t, cplx h[6])
{
    double rx = t[0] - s[0], ry = t[1] - s[1], rz = t[2] - s[2];
    double dd = rx * rx + ry * ry + rz * rz;
    double d = sqrt(dd), dinv = 1.0 / d, ddinv = dinv * dinv, dddinv = ddinv * dinv;
    double dot = rx * v[0] + ry * v[1] + rz * v[2];
    double d5 = ddinv * dddinv;
    double dx = rx * dinv, dy = ry * dinv, dz = rz * dinv;
    double hh[6];
    hh[0] = 3 * (dot * (5 * dx * dx - 1) - (v[0] * rx + v[0] * rx));
    hh[1] = 3 * (dot * (5 * dy * dy - 1) - (v[1] * ry + v[1] * ry));
    hh[2] = 3 * (dot * (5 * dz * dz - 1) - (v[2] * rz + v[2] * rz));
    hh[3] = 3 * (dot * (5 * dx * dy) - (v[1] * rx + v[0] * ry));
    hh[4] = 3 * (dot * (5 * dx * dz) - (v[2] * rx + v[0] * rz));
    hh[5] = 3 * (dot * (5 * dy * dz) - (v[2] * ry + v[1] * rz));
    cplx cd = ds * d5;
    for (int i = 0; i < 6; i++) h[i] = hh[i] * cd;
}

/* Hessians of the pair sum at one point (skip = excluded source index). */
static void direct_hess_one(int ns, const double *src, int ifcharge, const cplx *charge, int ifdipole,
                            const cplx *dipstr, const double *dipvec, const double *t, long skip, cplx h[6])
{
    for (int i = 0; i < 6; i++) h[i] = 0;
    cplx hp[6];
    for (long i = 0; i < ns; i++) {
        if (i == skip) continue;
        if (ifcharge == 1) {
            lpotfld3dhess_r(src + 3 * i, charge[i], t, hp);
            for (int k = 0; k < 6; k++) h[k] += hp[k];
        }
        if (ifdipole == 1) {
            lpotfld3dhess_dp_r(src + 3 * i, dipstr[i], dipvec + 3 * i, t, hp);
            for (int k = 0; k < 6; k++) h[k] += hp[k];
        }
    }
}

/* Direct Hessians at arbitrary points (skip[k] excluded at point k, or -1). */
void oracle_l3ddirect_points_hess(int nsource, const double *source, int ifcharge, const cplx *charge,
                                  int ifdipole, const cplx *dipstr, const double *dipvec, int npts,
                                  const double *pts, const long *skip, cplx *hess)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < npts; k++)
        direct_hess_one(nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, pts + 3 * k,
                        skip ? skip[k] : -1, hess + 6 * k);
}

/* l3dtaevalhessdini: factors of the shift of a local expansion to an order-2
 * expansion about the target; 10 (nterms+2)^2 entries. */
static double *taevalhess_ini(int nterms)
{
    double *sc = calloc((size_t)10 * (nterms + 2) * (nterms + 2), sizeof(double));
    double *fact = malloc(sizeof(double) * (2 * nterms + 1));
    int ldc = 2 * nterms + 1;
    double *cs = calloc((size_t)(nterms + 1) * ldc, sizeof(double));
#define CS(l, m) cs[(l) * ldc + (m) + nterms]
    double d = 1.0;
    fact[0] = d;
    for (int l = 1; l <= 2 * nterms; l++) { d = d * sqrt(l + 0.0); fact[l] = d; }
    CS(0, 0) = 1.0;
    for (int l = 1; l <= nterms; l++)
        for (int m = 0; m <= l; m++) {
            CS(l, m) = par(l) / (fact[l - m] * fact[l + m]);
            CS(l, -m) = CS(l, m);
        }
    int iuse = 0;
    for (int j = 0; j <= 2; j++)
        for (int l = j; l <= nterms; l++)
            for (int k = -j; k <= j; k++)
                for (int m = -l; m <= l; m++) {
                    int ll = l - j, mm = m - k;
                    if (abs(mm) > ll) continue;
                    double v = CS(j, k) * CS(ll, mm) / CS(l, m);
                    v = v / sqrt(2 * ll + 1.0);
                    v = v * par(ll);
                    if (m * mm < 0) v = v * par(mm);
                    if (m * mm >= 0 && abs(m) <= abs(mm)) v = v * par(k);
                    sc[iuse++] = v;
                }
#undef CS
    free(fact); free(cs);
    return sc;
}

/* l3dmpevalhessdini: factors of the shift of a multipole expansion to an
 * order-2 local expansion about the target. */
static double *mpevalhess_ini(int nterms)
{
    double *sc = calloc((size_t)10 * (nterms + 2) * (nterms + 2), sizeof(double));
    int ld = 2 * nterms + 5;
    double *c = calloc((size_t)ld * ld, sizeof(double)), *sqc = calloc((size_t)ld * ld, sizeof(double));
#define C_(l, m) c[(l) * ld + (m)]
#define SQC(l, m) sqc[(l) * ld + (m)]
    for (int l = 0; l < ld; l++) { C_(l, 0) = 1.0; SQC(l, 0) = 1.0; }
    for (int m = 1; m < ld; m++) {
        C_(m, m) = 1.0;
        SQC(m, m) = 1.0;
        for (int l = m + 1; l < ld; l++) {
            C_(l, m) = C_(l - 1, m) + C_(l - 1, m - 1);
            SQC(l, m) = sqrt(C_(l, m));
        }
    }
    int iuse = 0;
    for (int lnew = 0; lnew <= 2; lnew++)
        for (int l = 0; l <= nterms; l++)
            for (int m = -l; m <= l; m++)
                for (int mnew = -lnew; mnew <= lnew; mnew++) {
                    int ll = l + lnew, mm = mnew - m;
                    double v = SQC(ll + mm, lnew + mnew) * SQC(ll - mm, lnew - mnew);
                    v = v * par(l);
                    v = v / sqrt(2 * ll + 1.0);
                    if (m < 0 && mnew < 0) {
                        if (-mnew < -m) v = v * par(mnew);
                        if (-mnew >= -m) v = v * par(m);
                    }
                    if (m > 0 && mnew > 0) {
                        if (mnew < m) v = v * par(mnew);
                        if (mnew >= m) v = v * par(m);
                    }
                    sc[iuse++] = v;
                }
#undef C_
#undef SQC
    free(c); free(sqc);
    return sc;
}

#define L2(j, k) loc2[(j) * (j) + (j) + (k)]

/* pot, -grad and Hessian from the order-2 expansion about the target */
static void hess_out_local(const cplx *loc2, double rscale, cplx *pot, cplx *fld, cplx *hess)
{
    *pot = L2(0, 0);
    double rfac = rscale / sqrt(2.0);
    if (fld) {
        fld[2] = -L2(1, 0) * rscale;
        fld[0] = rfac * (L2(1, 1) + L2(1, -1));
        fld[1] = rfac * I * (L2(1, 1) - L2(1, -1));
    }
    if (hess) {
        rfac = rfac * rscale * sqrt(3.0);
        cplx z0 = rscale * rscale * L2(2, 0);
        hess[0] = rfac * (L2(2, 2) + L2(2, -2)) - z0;
        hess[1] = -rfac * (L2(2, 2) + L2(2, -2)) - z0;
        hess[2] = 2.0 * z0;
        hess[3] = rfac * I * (L2(2, 2) - L2(2, -2));
        hess[4] = -rfac * (L2(2, 1) + L2(2, -1));
        hess[5] = -rfac * I * (L2(2, 1) - L2(2, -1));
    }
}

/* l3dtaevalhessd_trunc: pot, fld (iffld) and Hessian (ifhess) of the local
 * expansion `loc` (orders 0..nterms) about `center` at `targ`. */
static void taevalhess(double rscale, const double *center, const cplx *loc, int nterms, const double *targ,
                       cplx *pot, int iffld, cplx *fld, int ifhess, cplx *hess, const double *sc)
{
    int ll = 0;
    if (iffld == 1) ll = 1;
    if (ifhess == 1) ll = 2;
    cplx loc2[9] = {0};
    double zd[3] = {center[0] - targ[0], center[1] - targ[1], center[2] - targ[2]}, d, th, ph;
    cart2polarl(zd, &d, &th, &ph);
    double ct = cos(th);
    cplx e1 = cos(ph) + I * sin(ph);
    int ld = nterms + 1;
    double *pw = malloc(sizeof(double) * (nterms + 2)), *pp = malloc(sizeof(double) * ld * ld);
    cplx *eps = malloc(sizeof(cplx) * (2 * nterms + 3)), *ep = eps + nterms + 1;
    cplx *ppc = malloc(sizeof(cplx) * ld * (2 * nterms + 1));
#define PPC(l, k) ppc[(l) * (2 * nterms + 1) + (k) + nterms]
    double dd = d * rscale;
    pw[0] = 1.0; pw[1] = dd;
    ep[0] = 1.0; ep[1] = e1; ep[-1] = conj(e1);
    for (int l = 2; l <= nterms + 1; l++) { pw[l] = dd * pw[l - 1]; ep[l] = ep[l - 1] * ep[1]; ep[-l] = conj(ep[l]); }
    ylgndrfw(nterms, ct, pp);
    for (int l = 0; l <= nterms; l++)
        for (int k = -l; k <= l; k++) PPC(l, k) = pp[l * ld + abs(k)] * pw[l] * ep[k];
    int iuse = 0;
    for (int l = 0; l <= nterms; l++)
        for (int m = -l; m <= l; m++) { L2(0, 0) += PPC(l, m) * sc[iuse] * loc[EI(l, m)]; iuse++; }
    if (ll >= 1)
        for (int l = 1; l <= nterms; l++) {
            int ldf = l - 1;
            for (int m = -l; m <= l - 2; m++) { L2(1, -1) += PPC(ldf, m + 1) * sc[iuse] * loc[EI(l, m)]; iuse++; }
            for (int m = -ldf; m <= ldf; m++) { L2(1, 0) += PPC(ldf, m) * sc[iuse] * loc[EI(l, m)]; iuse++; }
            for (int m = -l + 2; m <= l; m++) { L2(1, 1) += PPC(ldf, m - 1) * sc[iuse] * loc[EI(l, m)]; iuse++; }
        }
    if (ll == 2)
        for (int l = 2; l <= nterms; l++) {
            int ldf = l - 2;
            for (int m = -l; m <= l - 4; m++) { L2(2, -2) += PPC(ldf, m + 2) * sc[iuse] * loc[EI(l, m)]; iuse++; }
            for (int m = -l + 1; m <= l - 3; m++) { L2(2, -1) += PPC(ldf, m + 1) * sc[iuse] * loc[EI(l, m)]; iuse++; }
            for (int m = -ldf; m <= ldf; m++) { L2(2, 0) += PPC(ldf, m) * sc[iuse] * loc[EI(l, m)]; iuse++; }
            for (int m = -l + 3; m <= l - 1; m++) { L2(2, 1) += PPC(ldf, m - 1) * sc[iuse] * loc[EI(l, m)]; iuse++; }
            for (int m = -l + 4; m <= l; m++) { L2(2, 2) += PPC(ldf, m - 2) * sc[iuse] * loc[EI(l, m)]; iuse++; }
        }
#undef PPC
    hess_out_local(loc2, rscale, pot, iffld == 1 ? fld : NULL, ifhess == 1 ? hess : NULL);
    free(pw); free(pp); free(eps); free(ppc);
}

/* l3dmpevalhessd_trunc: pot, fld and Hessian of the multipole `mp` about
 * `center` at `targ`. */
static void mpevalhess(double rscale, const double *center, const cplx *mp, int nterms, const double *targ,
                       cplx *pot, int iffld, cplx *fld, int ifhess, cplx *hess, const double *sc)
{
    int ll = 0;
    if (iffld == 1) ll = 1;
    if (ifhess == 1) ll = 2;
    cplx loc2[9] = {0};
    double zd[3] = {center[0] - targ[0], center[1] - targ[1], center[2] - targ[2]}, d, th, ph;
    cart2polarl(zd, &d, &th, &ph);
    double ct = cos(th);
    cplx e1 = cos(ph) + I * sin(ph);
    int n2 = nterms + 2, ld = n2 + 1;
    double *pw = malloc(sizeof(double) * (nterms + 4)), *pp = malloc(sizeof(double) * ld * ld);
    cplx *eps = malloc(sizeof(cplx) * (2 * nterms + 7)), *ep = eps + nterms + 3;
    cplx *ppc = malloc(sizeof(cplx) * ld * (2 * n2 + 1));
#define PPC(l, k) ppc[(l) * (2 * n2 + 1) + (k) + n2]
    double dd = 1.0 / d;
    dd = dd / rscale;
    pw[0] = 1.0; pw[1] = dd;
    ep[0] = 1.0; ep[1] = e1; ep[-1] = conj(e1);
    for (int l = 2; l <= nterms + 3; l++) { pw[l] = dd * pw[l - 1]; ep[l] = ep[l - 1] * ep[1]; ep[-l] = conj(ep[l]); }
    ylgndrfw(n2, ct, pp);
    for (int l = 0; l <= n2; l++)
        for (int k = -l; k <= l; k++) PPC(l, k) = pp[l * ld + abs(k)] * pw[l + 1] * ep[-k];
    int iuse = 0;
    for (int l = 0; l <= nterms; l++)
        for (int m = -l; m <= l; m++) { L2(0, 0) += PPC(l, -m) * sc[iuse] * mp[EI(l, m)]; iuse++; }
    if (ll >= 1)
        for (int l = 0; l <= nterms; l++) {
            int ls = l + 1;
            for (int m = -l; m <= l; m++) {
                L2(1, -1) += PPC(ls, -1 - m) * sc[iuse] * mp[EI(l, m)];
                L2(1, 0) += PPC(ls, -m) * sc[iuse + 1] * mp[EI(l, m)];
                L2(1, 1) += PPC(ls, 1 - m) * sc[iuse + 2] * mp[EI(l, m)];
                iuse += 3;
            }
        }
    if (ll == 2)
        for (int l = 0; l <= nterms; l++) {
            int ls = l + 2;
            for (int m = -l; m <= l; m++) {
                L2(2, -2) += PPC(ls, -2 - m) * sc[iuse] * mp[EI(l, m)];
                L2(2, -1) += PPC(ls, -1 - m) * sc[iuse + 1] * mp[EI(l, m)];
                L2(2, 0) += PPC(ls, -m) * sc[iuse + 2] * mp[EI(l, m)];
                L2(2, 1) += PPC(ls, 1 - m) * sc[iuse + 3] * mp[EI(l, m)];
                L2(2, 2) += PPC(ls, 2 - m) * sc[iuse + 4] * mp[EI(l, m)];
                iuse += 5;
            }
        }
#undef PPC
    *pot = L2(0, 0) * rscale;
    if (iffld == 1) {
        double rfac = sqrt(2.0) * rscale * rscale;
        fld[0] = rfac * (L2(1, 1) + L2(1, -1)) / 2.0;
        fld[1] = rfac * I * (L2(1, 1) - L2(1, -1)) / 2.0;
        fld[2] = -L2(1, 0) * rscale * rscale;
    }
    if (ifhess == 1) {
        double rfac = rscale * rscale * rscale * sqrt(3.0) / sqrt(2.0);
        cplx z0 = rscale * rscale * rscale * L2(2, 0);
        hess[0] = rfac * (L2(2, 2) + L2(2, -2)) - z0;
        hess[1] = -rfac * (L2(2, 2) + L2(2, -2)) - z0;
        hess[2] = 2.0 * z0;
        hess[3] = rfac * I * (L2(2, 2) - L2(2, -2));
        hess[4] = -rfac * (L2(2, 1) + L2(2, -1));
        hess[5] = -rfac * I * (L2(2, 1) - L2(2, -1));
    }
    free(pw); free(pp); free(eps); free(ppc);
}
#undef L2

/* Entry points for the operator tests: one expansion, many targets. */
void oracle_taevalhess(double rscale, const double *center, const cplx *loc, int nterms, int nt, const double *targ,
                       cplx *pot, cplx *fld, cplx *hess)
{
    double *sc = taevalhess_ini(nterms);
#pragma omp parallel for
    for (int i = 0; i < nt; i++)
        taevalhess(rscale, center, loc, nterms, targ + 3 * (size_t)i, pot + i, 1, fld + 3 * (size_t)i, 1,
                   hess + 6 * (size_t)i, sc);
    free(sc);
}

void oracle_mpevalhess(double rscale, const double *center, const cplx *mp, int nterms, int nt, const double *targ,
                       cplx *pot, cplx *fld, cplx *hess)
{
    double *sc = mpevalhess_ini(nterms);
#pragma omp parallel for
    for (int i = 0; i < nt; i++)
        mpevalhess(rscale, center, mp, nterms, targ + 3 * (size_t)i, pot + i, 1, fld + 3 * (size_t)i, 1,
                   hess + 6 * (size_t)i, sc);
    free(sc);
}
