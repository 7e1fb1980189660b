/*
 * hfmm3d_oracle.c -- CPU restatement of FMMLIB3D's Helmholtz particle FMM.
 *
 * TEST INFRASTRUCTURE ONLY, like fmm3d_oracle.c, which includes this file at
 * its end so that both share the tree, the lists and the rotation recursion.
 * Only tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs
 * of bench.py load the oracle library.
 *
 * Parity status: unpinned against the reference's FMM itself (no Fortran
 * compiler, no stored outputs); pinned through the FP64 O(N^2) direct sum
 * h3dpartdirect (restated below), the accuracy contract per iprec, and the
 * special functions against independent implementations (tests).
 *
 * Each routine names the reference routine (file:line) it follows; paths are
 * relative to the FMMLIB3D source tree.
 */

/* ------------------------------------------------------------------ */
/* Spherical Hankel functions h_n(z) = j_n + i y_n, scaled by scale^n:
 * h3d01 (src/helmrouts3d.f:666-704) and h3dall (:709-809).               */
static void h3d01(cplx z, cplx *h0, cplx *h1)
{
    if (cabs(z) < 1.0e-15) { *h0 = 0; *h1 = 0; return; }
    cplx cd = I * z;
    *h0 = cexp(cd) / cd;
    *h1 = *h0 * (1.0 / z - I);
}

static void h3dall(int nterms, cplx z, double scale, cplx *hvec, int ifder, cplx *hder)
{
    if (cabs(z) < 1.0e-15) {
        for (int i = 0; i <= nterms; i++) { hvec[i] = 0; if (ifder) hder[i] = 0; }
        return;
    }
    h3d01(z, &hvec[0], &hvec[1]);
    hvec[1] = hvec[1] * scale;
    double scal2 = scale * scale;
    cplx zinv = scale / z;
    for (int i = 1; i <= nterms - 1; i++) {
        cplx ztmp = zinv * (2 * i + 1.0);
        hvec[i + 1] = ztmp * hvec[i] - scal2 * hvec[i - 1];
    }
    if (ifder) {
        hder[0] = -hvec[1] / scale;
        zinv = 1.0 / z;
        for (int i = 1; i <= nterms; i++) {
            cplx ztmp = zinv * (i + 1.0);
            hder[i] = scale * hvec[i - 1] - ztmp * hvec[i];
        }
    }
}

/* Spherical Bessel functions j_n(z)/scale^n by Miller's backward recurrence:
 * jfuns3d, src/cdjseval3d.f:15-197.  fjs needs lwfjs+2 entries, iscale
 * lwfjs+2.  Returns the reference's ier (8: the upward sweep never grew past
 * the bound within lwfjs terms).                                          */
static int jfuns3d(int nterms, cplx z, double scale, cplx *fjs, int ifder, cplx *fjder, int lwfjs, int *iscale)
{
    const double upbound2 = 1.0e40, upbound2inv = 1.0e-40, tiny = 1.0e-200;
    if (cabs(z) < tiny) {
        fjs[0] = 1;
        for (int i = 1; i <= nterms; i++) fjs[i] = 0;
        if (ifder) {
            for (int i = 0; i <= nterms; i++) fjder[i] = 0;
            fjder[1] = 1.0 / (3 * scale);
        }
        return 0;
    }
    int ntop = 0;
    cplx zinv = 1.0 / z;
    fjs[nterms] = 1;
    fjs[nterms - 1] = 0;
    for (int i = nterms; i <= lwfjs; i++) {
        double dcoef = 2 * i + 1.0;
        cplx ztmp = dcoef * zinv * fjs[i] - fjs[i - 1];
        fjs[i + 1] = ztmp;
        double dd = creal(ztmp) * creal(ztmp) + cimag(ztmp) * cimag(ztmp);
        if (dd > upbound2) { ntop = i + 1; break; }
    }
    if (ntop == 0) return 8;
    for (int i = 0; i <= ntop; i++) iscale[i] = 0;
    fjs[ntop] = 0;
    fjs[ntop - 1] = 1;
    for (int i = ntop - 1; i >= 1; i--) {
        double dcoef = 2 * i + 1.0;
        cplx ztmp = dcoef * zinv * fjs[i] - fjs[i + 1];
        fjs[i - 1] = ztmp;
        double dd = creal(ztmp) * creal(ztmp) + cimag(ztmp) * cimag(ztmp);
        if (dd > upbound2) {
            fjs[i] = fjs[i] * upbound2inv;
            fjs[i - 1] = fjs[i - 1] * upbound2inv;
            iscale[i] = 1;
        }
    }
    double scalinv = 1.0 / scale, sctot = 1.0;
    for (int i = 1; i <= ntop; i++) {
        sctot = sctot * scalinv;
        if (iscale[i - 1] == 1) sctot = sctot * upbound2inv;
        fjs[i] = fjs[i] * sctot;
    }
    cplx fj0 = csin(z) * zinv;
    cplx fj1 = fj0 * zinv - ccos(z) * zinv;
    cplx zscale = cabs(fj1) > cabs(fj0) ? fj1 / (fjs[1] * scale) : fj0 / fjs[0];
    for (int i = 0; i <= nterms; i++) fjs[i] = fjs[i] * zscale;
    if (ifder) {
        fjs[nterms + 1] = fjs[nterms + 1] * zscale;
        fjder[0] = -fjs[1] * scale;
        for (int i = 1; i <= nterms; i++) {
            double dc1 = i / (2 * i + 1.0), dc2 = 1.0 - dc1;
            dc1 = dc1 * scalinv;
            dc2 = dc2 * scale;
            fjder[i] = dc1 * fjs[i - 1] - dc2 * fjs[i + 1];
        }
    }
    return 0;
}

/* Test hooks for the special functions. */
void oracle_h3dall(int nterms, double zr, double zi, double scale, cplx *hvec, cplx *hder)
{
    h3dall(nterms, zr + I * zi, scale, hvec, 1, hder);
}
int oracle_jfuns3d(int nterms, double zr, double zi, double scale, cplx *fjs, cplx *fjder)
{
    int lw = nterms + 1000;
    cplx *f = malloc(sizeof(cplx) * (lw + 2));
    int *isc = malloc(sizeof(int) * (lw + 2));
    int ier = jfuns3d(nterms, zr + I * zi, scale, f, 1, fjder, lw, isc);
    memcpy(fjs, f, sizeof(cplx) * (nterms + 2));
    free(f); free(isc);
    return ier;
}

/* ------------------------------------------------------------------ */
/* Expansion orders: h3dterms (src/h3dterms.f:28-102), h3dterms_eval
 * (:508-598, itype 1 is the same formula), h3dterms_list2 (:192-344).   */
static int hterms_core(cplx zk, double size, double eps, double fac_h, int *ier)
{
    enum { NT = 1000, LW = 2000 };
    cplx *hfun = malloc(sizeof(cplx) * (NT + 2)), *jfun = malloc(sizeof(cplx) * (LW + 2));
    int *isc = malloc(sizeof(int) * (LW + 2));
    cplx fhder[2];
    *ier = 0;
    cplx z1 = (zk * size) * fac_h;
    double rscale = 1.0;
    if (cabs(zk * size) < 1.0) rscale = cabs(zk * size);
    h3dall(NT, z1, rscale, hfun, 0, fhder);
    cplx z2 = (zk * size) * sqrt(3.0) / 2.0;
    int nterms = 1000;
    if (jfuns3d(NT, z2, rscale, jfun, 0, NULL, LW, isc) == 8) { *ier = 11; nterms = 0; goto done; }
    double xtemp0 = cabs(jfun[0] * hfun[0]) + cabs(jfun[1] * hfun[1]);
    for (int j = 2; j <= NT; j++) {
        double xtemp = cabs(jfun[j] * hfun[j]) + cabs(jfun[j - 1] * hfun[j - 1]);
        if (xtemp < eps * xtemp0) { nterms = j + 1; goto done; }
    }
    *ier = 13;
done:
    free(hfun); free(jfun); free(isc);
    return nterms;
}

int oracle_h3dterms(double size, double zkr, double zki, double eps, int *ier)
{
    return hterms_core(zkr + I * zki, size, eps, 1.5, ier);
}

void oracle_h3dterms_list2(double size, double zkr, double zki, double eps, int *itable, int *ier)
{
    int tab[2][4][4];
    *ier = 0;
    for (int ii = 2; ii <= 3; ii++)
        for (int jj = 0; jj <= 3; jj++)
            for (int kk = 0; kk <= 3; kk++) {
                double dx = ii, dy = jj, dz = kk;
                if (dx > 0) dx -= .5;
                if (dy > 0) dy -= .5;
                if (dz > 0) dz -= .5;
                double rr = sqrt(dx * dx + dy * dy + dz * dz);
                int e;
                tab[ii - 2][jj][kk] = hterms_core(zkr + I * zki, size, eps, rr, &e);
                if (e) *ier = e;
            }
    for (int i = 0; i < 343; i++) itable[i] = 0;
    for (int k = -3; k <= 3; k++)
        for (int i = -3; i <= 3; i++)
            for (int j = -3; j <= 3; j++) {
                int v = 0, ai = abs(i), aj = abs(j), ak = abs(k);
                if (ai > 1) v = tab[ai - 2][aj][ak];
                else if (aj > 1) v = tab[aj - 2][ai][ak];
                if (ai <= 1 && aj <= 1 && ak > 1) v = ai >= aj ? tab[ak - 2][ai][aj] : tab[ak - 2][aj][ai];
                itable[((i + 3) * 7 + (j + 3)) * 7 + (k + 3)] = v;
            }
}

/* Gauss-Legendre nodes and weights on [-1,1] (the quadrature legewhts of
 * src/legeexps.f:288-355 returns): Newton's method on P_n from the
 * three-term recurrence, started at cos(pi (i - 1/4) / (n + 1/2)).        */
void oracle_legewhts(int n, double *x, double *w)
{
    for (int i = 0; i < n; i++) {
        double t = cos(M_PI * (i + 0.75) / (n + 0.5)), pd = 1;
        for (int it = 0; it < 100; it++) {
            double p0 = 1, p1 = t;
            for (int k = 2; k <= n; k++) { double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
            pd = n * (t * p1 - p0) / (t * t - 1);
            double dt = p1 / pd;
            t -= dt;
            if (fabs(dt) < 1e-16) break;
        }
        double p0 = 1, p1 = t;
        for (int k = 2; k <= n; k++) { double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
        pd = n * (t * p1 - p0) / (t * t - 1);
        x[n - 1 - i] = t;
        w[n - 1 - i] = 2.0 / ((1 - t * t) * pd * pd);
    }
}

/* Legendre functions with the sqrt(2n+1) factor of ylgndr / ylgndr2s
 * (src/yrecursion.f:189-238, :298-385): the unit-normalized ones above
 * times sqrt(2n+1).                                                       */
static void ylgndrfw(int nmax, double x, double *y)
{
    int ld = nmax + 1;
    ylgndru(nmax, x, y);
    for (int n = 0; n <= nmax; n++) {
        double s = sqrt(2 * n + 1.0);
        for (int m = 0; m <= n; m++) y[n * ld + m] *= s;
    }
}
static void ylgndr2sfw(int nmax, double x, double *y, double *d)
{
    int ld = nmax + 1;
    ylgndru2s(nmax, x, y, d);
    for (int n = 0; n <= nmax; n++) {
        double s = sqrt(2 * n + 1.0);
        for (int m = 0; m <= n; m++) { y[n * ld + m] *= s; d[n * ld + m] *= s; }
    }
}

/* ------------------------------------------------------------------ */
/* Pairwise kernels: hpotfld3d (src/helmrouts3d.f:1335-1417) and
 * hpotfld3d_dp (:1844-1924).                                              */
static inline void hpotfld3d(int iffld, const double *s, cplx q, const double *t, cplx zk, cplx *pot, cplx *fld)
{
    double xd = t[0] - s[0], yd = t[1] - s[1], zd = t[2] - s[2];
    double dd = xd * xd + yd * yd + zd * zd, d = sqrt(dd);
    *pot = q * cexp(I * zk * d) / d;
    if (iffld == 1) {
        cplx cd = (1 - I * zk * d) * *pot / dd;
        fld[0] = cd * xd; fld[1] = cd * yd; fld[2] = cd * zd;
    }
}

static inline void hpotfld3d_dp(int iffld, const double *s, cplx ds, const double *v, const double *t, cplx zk,
                                cplx *pot, cplx *fld)
{
    double xd = t[0] - s[0], yd = t[1] - s[1], zd = t[2] - s[2];
    double dd = xd * xd + yd * yd + zd * zd, d = sqrt(dd);
    cplx h0, h1;
    h3d01(d * zk, &h0, &h1);
    cplx ewavek = I * zk;
    double dinv = 1.0 / d;
    cplx cd = h1 * dinv * ewavek * zk * ds;
    double dot = xd * v[0] + yd * v[1] + zd * v[2];
    *pot = cd * dot;
    if (iffld == 1) {
        double dinv2 = dinv * dinv;
        cd = h0 * ewavek * ds;
        cd = cd * dot;
        cplx z1 = dinv * (dinv - ewavek);
        double z2 = -3 * dinv2 * dinv;
        cplx z3 = 2.0 * ewavek * dinv2;
        cd = cd * (ewavek * z1 + z2 + z3) * dinv;
        fld[0] = -cd * xd; fld[1] = -cd * yd; fld[2] = -cd * zd;
        cd = h1 * dinv * ewavek * zk * ds;
        fld[0] -= cd * v[0]; fld[1] -= cd * v[1]; fld[2] -= cd * v[2];
    }
}

static void hdirect_one(cplx zk, int ns, const double *src, int ifcharge, const cplx *charge, int ifdipole,
                        const cplx *dipstr, const double *dipvec, const double *t, int skip, int iffld, cplx *pot,
                        cplx fld[3])
{
    cplx p = 0, f0 = 0, f1 = 0, f2 = 0, pv, fv[3] = {0, 0, 0};
    for (int i = 0; i < ns; i++) {
        if (i == skip) continue;
        if (ifcharge == 1) {
            hpotfld3d(iffld, src + 3 * (size_t)i, charge[i], t, zk, &pv, fv);
            p += pv;
            if (iffld == 1) { f0 += fv[0]; f1 += fv[1]; f2 += fv[2]; }
        }
        if (ifdipole == 1) {
            hpotfld3d_dp(iffld, src + 3 * (size_t)i, dipstr[i], dipvec + 3 * (size_t)i, t, zk, &pv, fv);
            p += pv;
            if (iffld == 1) { f0 += fv[0]; f1 += fv[1]; f2 += fv[2]; }
        }
    }
    *pot = p;
    fld[0] = f0; fld[1] = f1; fld[2] = f2;
}

/* h3dpartdirect, src/hfmm3dpart.f:1268-1401. */
void oracle_h3dpartdirect(double zkr, double zki, int nsource, const double *source, int ifcharge,
                          const cplx *charge, int ifdipole, const cplx *dipstr, const double *dipvec, int ifpot,
                          cplx *pot, int iffld, cplx *fld, int ntarget, const double *target, int ifpottarg,
                          cplx *pottarg, int iffldtarg, cplx *fldtarg)
{
    cplx zk = zkr + I * zki;
#pragma omp parallel for schedule(dynamic, 64)
    for (int j = 0; j < nsource; j++) {
        if (!(ifpot == 1 || iffld == 1)) continue;
        cplx pv, fv[3];
        hdirect_one(zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, source + 3 * (size_t)j, j, iffld,
                    &pv, fv);
        if (ifpot == 1) pot[j] = pv;
        if (iffld == 1) for (int d = 0; d < 3; d++) fld[3 * (size_t)j + d] = fv[d];
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int j = 0; j < ntarget; j++) {
        if (!(ifpottarg == 1 || iffldtarg == 1)) continue;
        cplx pv, fv[3];
        hdirect_one(zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, target + 3 * (size_t)j, -1,
                    iffldtarg, &pv, fv);
        if (ifpottarg == 1) pottarg[j] = pv;
        if (iffldtarg == 1) for (int d = 0; d < 3; d++) fldtarg[3 * (size_t)j + d] = fv[d];
    }
}

/* Direct sum at selected evaluation points (pot and field), skip[k] the
 * source index excluded at point k (-1 for none).                        */
void oracle_h3ddirect_points(double zkr, double zki, int nsource, const double *source, int ifcharge,
                             const cplx *charge, int ifdipole, const cplx *dipstr, const double *dipvec, int npts,
                             const double *pts, const long *skip, cplx *pot, cplx *fld)
{
    cplx zk = zkr + I * zki;
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < npts; k++)
        hdirect_one(zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, pts + 3 * (size_t)k,
                    skip ? (int)skip[k] : -1, 1, pot + k, fld + 3 * (size_t)k);
}

/* ------------------------------------------------------------------ */
/* Per-thread scratch for the point operators below.                     */
typedef struct {
    int p, lw;
    double *pp, *ppd;
    cplx *f, *fd, *em;
    int *isc;
} hwork;

static void hwork_init(hwork *w, int p)
{
    w->p = p;
    w->lw = p + 1000;
    w->pp = malloc(sizeof(double) * (p + 2) * (p + 2));
    w->ppd = malloc(sizeof(double) * (p + 2) * (p + 2));
    w->f = malloc(sizeof(cplx) * (w->lw + 2));
    w->fd = malloc(sizeof(cplx) * (w->lw + 2));
    w->em = malloc(sizeof(cplx) * (2 * p + 5));
    w->isc = malloc(sizeof(int) * (w->lw + 2));
}
static void hwork_free(hwork *w) { free(w->pp); free(w->ppd); free(w->f); free(w->fd); free(w->em); free(w->isc); }

/* e^{i m phi}, m = -p-1..p+1, by repeated products as the reference does;
 * em[m + p + 1].  `inv_by_div` selects 1/e^{i phi} (h3dformta_trunc0)
 * instead of the conjugate for the negative powers.                      */
static void hphases(cplx e1, int p, cplx *em, int inv_by_div)
{
    cplx *e = em + p + 1, einv = inv_by_div ? 1.0 / e1 : conj(e1);
    e[0] = 1; e[1] = e1; e[-1] = einv;
    for (int i = 2; i <= p + 1; i++) { e[i] = e[i - 1] * e1; e[-i] = e[-i + 1] * einv; }
}

/* P2M of one charge, without the final factor ik: h3dformmp_trunc0,
 * src/helmrouts3d.f:3119-3230.                                            */
static void hformmp_charge(cplx zk, double rscale, const double *s, cplx q, const double *c, int p, cplx *mp, hwork *w)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th);
    hphases(cos(ph) + I * sin(ph), p, w->em, 0);
    const cplx *e = w->em + p + 1;
    ylgndrfw(p, ct, w->pp);
    cplx *f = w->f;
    if (jfuns3d(p, zk * r, rscale, f, 0, NULL, w->lw, w->isc)) return;
    for (int n = 0; n <= p; n++) f[n] = f[n] * q;
    int ld = p + 1;
    mp[0] += f[0];
    for (int n = 1; n <= p; n++) {
        mp[EI(n, 0)] += w->pp[n * ld] * f[n];
        for (int m = 1; m <= n; m++) {
            cplx z = w->pp[n * ld + m] * f[n];
            mp[EI(n, m)] += z * conj(e[m]);
            mp[EI(n, -m)] += z * conj(e[-m]);
        }
    }
}

/* P2M of one dipole, without the factor ik: h3dformmp0_dp_trunc,
 * src/helmrouts3d.f:3648-3760.                                             */
static void hformmp_dipole(cplx zk, double rscale, const double *s, cplx ds, const double *v, const double *c, int p,
                           cplx *mp, hwork *w)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    hphases(cp + I * sp, p, w->em, 0);
    const cplx *e = w->em + p + 1;
    double rx = st * cp, thx = ct * cp, phx = -sp, ry = st * sp, thy = ct * sp, phy = cp, rz = ct, thz = -st;
    ylgndr2sfw(p, ct, w->pp, w->ppd);
    cplx *f = w->f, *fd = w->fd;
    if (jfuns3d(p, zk * r, rscale, f, 1, fd, w->lw, w->isc)) return;
    for (int i = 0; i <= p; i++) fd[i] = fd[i] * zk;
    int ld = p + 1;
    const double *pp = w->pp, *ppd = w->ppd;
#define HDOT(ur, ut, up) (v[0] * ((ur) * rx + (ut) * thx + (up) * phx) + v[1] * ((ur) * ry + (ut) * thy + (up) * phy) + \
                          v[2] * ((ur) * rz + (ut) * thz))
    mp[0] += HDOT(pp[0] * fd[0], 0.0, 0.0) * ds;
    for (int n = 1; n <= p; n++) {
        cplx fu = f[n + 1] * rscale + f[n - 1] / rscale;
        fu = zk * fu / (2 * n + 1.0);
        mp[EI(n, 0)] += HDOT(pp[n * ld] * fd[n], -fu * ppd[n * ld] * st, 0.0) * ds;
        for (int m = 1; m <= n; m++) {
            cplx ur = fd[n] * pp[n * ld + m] * st * e[-m], ut = -e[-m] * fu * ppd[n * ld + m];
            cplx up = -I * (double)m * e[-m] * fu * pp[n * ld + m];
            mp[EI(n, m)] += HDOT(ur, ut, up) * ds;
            ur = fd[n] * pp[n * ld + m] * st * e[m];
            ut = -e[m] * fu * ppd[n * ld + m];
            up = I * (double)m * e[m] * fu * pp[n * ld + m];
            mp[EI(n, -m)] += HDOT(ur, ut, up) * ds;
        }
    }
}

/* P2L of one charge, without the factor ik: h3dformta_trunc0,
 * src/helmrouts3d.f:3370-3440.                                             */
static void hformta_charge(cplx zk, double rscale, const double *s, cplx q, const double *c, int p, cplx *lo, hwork *w)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th);
    hphases(cos(ph) + I * sin(ph), p, w->em, 1);
    const cplx *e = w->em + p + 1;
    ylgndrfw(p, ct, w->pp);
    cplx z = zk * r, *f = w->f, fdum[2];
    if (cabs(z) < 1.0e-15) return;
    h3dall(p, z, rscale, f, 0, fdum);
    for (int n = 0; n <= p; n++) f[n] = f[n] * q;
    int ld = p + 1;
    lo[0] += f[0];
    for (int n = 1; n <= p; n++) {
        lo[EI(n, 0)] += w->pp[n * ld] * f[n];
        for (int m = 1; m <= n; m++) {
            cplx zt = w->pp[n * ld + m] * f[n];
            lo[EI(n, m)] += zt * e[-m];
            lo[EI(n, -m)] += zt * e[m];
        }
    }
}

/* P2L of one dipole, without the factor ik: h3dformta0_dp_trunc,
 * src/helmrouts3d.f:4123-4250.                                             */
static void hformta_dipole(cplx zk, double rscale, const double *s, cplx ds, const double *v, const double *c, int p,
                           cplx *lo, hwork *w)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    hphases(cp + I * sp, p, w->em, 1);
    const cplx *e = w->em + p + 1;
    double rx = st * cp, thx = ct * cp / r, phx = -sp / r, ry = st * sp, thy = ct * sp / r, phy = cp / r, rz = ct,
           thz = -st / r;
    ylgndr2sfw(p, ct, w->pp, w->ppd);
    cplx *f = w->f, *fd = w->fd;
    h3dall(p, zk * r, rscale, f, 1, fd);
    for (int i = 0; i <= p; i++) fd[i] = fd[i] * zk;
    int ld = p + 1;
    const double *pp = w->pp, *ppd = w->ppd;
    lo[0] += HDOT(pp[0] * fd[0], 0.0, 0.0) * ds;
    for (int n = 1; n <= p; n++) {
        lo[EI(n, 0)] += HDOT(pp[n * ld] * fd[n], -f[n] * ppd[n * ld] * st, 0.0) * ds;
        for (int m = 1; m <= n; m++) {
            cplx ur = fd[n] * pp[n * ld + m] * st * e[-m], ut = -e[-m] * f[n] * ppd[n * ld + m];
            cplx up = -I * (double)m * e[-m] * f[n] * pp[n * ld + m];
            lo[EI(n, m)] += HDOT(ur, ut, up) * ds;
            ur = fd[n] * pp[n * ld + m] * st * e[m];
            ut = -e[m] * f[n] * ppd[n * ld + m];
            up = I * (double)m * e[m] * f[n] * pp[n * ld + m];
            lo[EI(n, -m)] += HDOT(ur, ut, up) * ds;
        }
    }
}
#undef HDOT

/* M2P with field: h3dmpeval_trunc0, src/helmrouts3d.f:2405-2543.  Returns
 * nonzero (no value) at the expansion center.                              */
static int hmpeval(cplx zk, double rscale, const double *c, const cplx *mp, int p, const double *t, cplx *pot,
                   cplx fld[3], hwork *w)
{
    double zd[3] = {t[0] - c[0], t[1] - c[1], t[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    if (cabs(zk * r) < 1.0e-15) return 8;
    hphases(cp + I * sp, p, w->em, 0);
    const cplx *e = w->em + p + 1;
    double rx = st * cp, thx = ct * cp / r, phx = -sp / r, ry = st * sp, thy = ct * sp / r, phy = cp / r, rz = ct,
           thz = -st / r;
    ylgndr2sfw(p, ct, w->pp, w->ppd);
    cplx *f = w->f, *fd = w->fd;
    h3dall(p, zk * r, rscale, f, 1, fd);
    for (int i = 0; i <= p; i++) fd[i] = fd[i] * zk;
    int ld = p + 1;
    const double *y = w->pp, *yd = w->ppd;
    cplx ur = mp[0] * fd[0], ut = 0, up = 0, pt = mp[0] * f[0];
    for (int n = 1; n <= p; n++) {
        pt += mp[EI(n, 0)] * f[n] * y[n * ld];
        ur += fd[n] * y[n * ld] * mp[EI(n, 0)];
        ut -= mp[EI(n, 0)] * f[n] * yd[n * ld] * st;
        for (int m = 1; m <= n; m++) {
            cplx z1 = f[n] * y[n * ld + m] * st, z2 = mp[EI(n, m)] * e[m], z3 = mp[EI(n, -m)] * e[-m], zs = z2 + z3;
            pt += z1 * zs;
            ur += fd[n] * y[n * ld + m] * st * zs;
            ut -= zs * f[n] * yd[n * ld + m];
            zs = I * (double)m * (z2 - z3);
            up += f[n] * y[n * ld + m] * zs;
        }
    }
    *pot = pt;
    fld[0] = -(ur * rx + ut * thx + up * phx);
    fld[1] = -(ur * ry + ut * thy + up * phy);
    fld[2] = -(ur * rz + ut * thz);
    return 0;
}

/* L2P with field: h3dtaeval_trunc0, src/helmrouts3d.f:2732-2900. */
static int htaeval(cplx zk, double rscale, const double *c, const cplx *lo, int p, const double *t, cplx *pot,
                   cplx fld[3], hwork *w)
{
    double zd[3] = {t[0] - c[0], t[1] - c[1], t[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    hphases(cp + I * sp, p, w->em, 0);
    const cplx *e = w->em + p + 1;
    double rx = st * cp, thx = ct * cp, phx = -sp, ry = st * sp, thy = ct * sp, phy = cp, rz = ct, thz = -st;
    ylgndr2sfw(p, ct, w->pp, w->ppd);
    cplx *f = w->f, *fd = w->fd;
    if (jfuns3d(p, zk * r, rscale, f, 1, fd, w->lw, w->isc)) return 8;
    for (int i = 0; i <= p; i++) fd[i] = fd[i] * zk;
    int ld = p + 1;
    const double *y = w->pp, *yd = w->ppd;
    cplx pt = lo[0] * f[0], ur = lo[0] * fd[0], ut = 0, up = 0;
    for (int n = 1; n <= p; n++) {
        pt += lo[EI(n, 0)] * f[n] * y[n * ld];
        ur += fd[n] * y[n * ld] * lo[EI(n, 0)];
        cplx fu = f[n + 1] * rscale + f[n - 1] / rscale;
        fu = zk * fu / (2 * n + 1.0);
        ut -= lo[EI(n, 0)] * fu * yd[n * ld] * st;
        for (int m = 1; m <= n; m++) {
            cplx z1 = f[n] * y[n * ld + m] * st, z2 = lo[EI(n, m)] * e[m], z3 = lo[EI(n, -m)] * e[-m], zs = z2 + z3;
            pt += z1 * zs;
            ur += fd[n] * y[n * ld + m] * st * zs;
            ut -= zs * fu * yd[n * ld + m];
            zs = I * (double)m * (z2 - z3);
            up += fu * y[n * ld + m] * zs;
        }
    }
    *pot = pt;
    fld[0] = -(ur * rx + ut * thx + up * phx);
    fld[1] = -(ur * ry + ut * thy + up * phy);
    fld[2] = -(ur * rz + ut * thz);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Translations along z by evaluation on a sphere and projection.
 * `a` holds the rotated source expansion (degrees <= n1), `out` receives the
 * target expansion (degrees <= n2); x/w are the nq Gauss-Legendre nodes.   */

/* M2M: h3dmpmpzshift_fast (src/h3dtrans.f:630-717) = h3dmpevalspherenm_fast
 * (src/projections.f:1611-1695), h3dprojlocnmsep_fast (:1277-1352),
 * h3drescalemp (:556-609).                                                  */
static void hzshift_m2m(cplx zk, double sc1, const cplx *a, int n1, double sc2, cplx *out, int n2, double radius,
                        double zshift, const double *x, const double *w, int nq)
{
    int pm = n1 > n2 ? n1 : n2, wm = 2 * n1 + 1;
    cplx *phi = calloc((size_t)nq * wm, sizeof(cplx)), *fh = malloc(sizeof(cplx) * (pm + 2)), fd[2];
    double *y = malloc(sizeof(double) * (pm + 2) * (pm + 2));
    for (int jj = 0; jj < nq; jj++) {
        double ct = x[jj], st = sqrt(1.0 - ct * ct);
        double rj = sqrt((zshift + radius * ct) * (zshift + radius * ct) + (radius * st) * (radius * st));
        double ctj = (zshift + radius * ct) / rj;
        ylgndrfw(n1, ctj, y);
        h3dall(n1, zk * rj, sc1, fh, 0, fd);
        for (int m = -n1; m <= n1; m++) {
            int am = abs(m);
            cplx s = phi[(size_t)jj * wm + m + n1];
            for (int n = am; n <= n1; n++) s += a[EI(n, m)] * fh[n] * y[n * (n1 + 1) + am];
            phi[(size_t)jj * wm + m + n1] = s;
        }
    }
    for (int l = 0; l <= n2; l++) for (int m = -l; m <= l; m++) out[EI(l, m)] = 0;
    for (int jj = 0; jj < nq; jj++) {
        ylgndrfw(n2, x[jj], y);
        for (int m = -n1; m <= n1; m++) {
            cplx zm = phi[(size_t)jj * wm + m + n1] * w[jj] / 2;
            for (int l = abs(m); l <= n2; l++) out[EI(l, m)] += zm * y[l * (n2 + 1) + abs(m)];
        }
    }
    h3dall(n2, zk * radius, sc2, fh, 0, fd);
    for (int l = 0; l <= n2; l++) for (int m = -l; m <= l; m++) out[EI(l, m)] = out[EI(l, m)] / fh[l];
    free(phi); free(fh); free(y);
}

/* Projection of values and normal derivatives, then the stabilised
 * rescaling: h3dprojlocsepstab_fast (src/projections.f:2292-2385) and
 * h3drescalestab (:679-752).  Frees phi/phin.                              */
static void hproject_stab(cplx zk, cplx *phi, cplx *phin, int ntold, double sc2, cplx *out, int n2, double radius,
                          const double *x, const double *w, int nq)
{
    int wm = 2 * ntold + 1, K2 = (n2 + 1) * (n2 + 1), lw = n2 + 1000;
    cplx *lo2 = calloc(K2, sizeof(cplx)), *fj = malloc(sizeof(cplx) * (lw + 2)), *fjd = malloc(sizeof(cplx) * (n2 + 2));
    int *isc = malloc(sizeof(int) * (lw + 2));
    double *y = malloc(sizeof(double) * (n2 + 2) * (n2 + 2));
    for (int k = 0; k < K2; k++) out[k] = 0;
    for (int jj = 0; jj < nq; jj++) {
        ylgndrfw(n2, x[jj], y);
        for (int m = -ntold; m <= ntold; m++) {
            cplx zm = phi[(size_t)jj * wm + m + ntold] * w[jj] / 2.0;
            for (int l = abs(m); l <= n2; l++) out[EI(l, m)] += zm * y[l * (n2 + 1) + abs(m)];
            zm = phin[(size_t)jj * wm + m + ntold] * w[jj] / 2.0;
            for (int l = abs(m); l <= n2; l++) lo2[EI(l, m)] += zm * y[l * (n2 + 1) + abs(m)];
        }
    }
    if (jfuns3d(n2, zk * radius, sc2, fj, 1, fjd, lw, isc) == 0) {
        for (int l = 0; l <= n2; l++) {
            cplx zh = fj[l], zhn = fjd[l] * zk, zm = zh * zh + zhn * zhn;
            for (int m = -l; m <= l; m++) out[EI(l, m)] = (zh * out[EI(l, m)] + zhn * lo2[EI(l, m)]) / zm;
        }
    }
    free(lo2); free(fj); free(fjd); free(isc); free(y); free(phi); free(phin);
}

/* M2L: h3dmploczshiftstab_fast (src/h3dtrans.f:1715-1798) =
 * h3dmpevalspherenmstab_fast (src/projections.f:1917-2033) + projection. */
static void hzshift_m2l(cplx zk, double sc1, const cplx *a, int n1, double sc2, cplx *out, int n2, double radius,
                        double zshift, const double *x, const double *w, int nq)
{
    int wm = 2 * n1 + 1, ld = n1 + 1;
    cplx *phi = calloc((size_t)nq * wm, sizeof(cplx)), *phin = calloc((size_t)nq * wm, sizeof(cplx));
    cplx *fh = malloc(sizeof(cplx) * (n1 + 2)), *fhd = malloc(sizeof(cplx) * (n1 + 2));
    double *y = malloc(sizeof(double) * (n1 + 2) * (n1 + 2)), *yd = malloc(sizeof(double) * (n1 + 2) * (n1 + 2));
    for (int jj = 0; jj < nq; jj++) {
        double ct = x[jj], st = sqrt(1.0 - ct * ct);
        double rj = sqrt((zshift + radius * ct) * (zshift + radius * ct) + (radius * st) * (radius * st));
        double ctj = (zshift + radius * ct) / rj, stj = sqrt(1.0 - ctj * ctj);
        double rn = stj * st + ctj * ct, thn = (ctj * st - ct * stj) / rj;
        ylgndr2sfw(n1, ctj, y, yd);
        h3dall(n1, zk * rj, sc1, fh, 1, fhd);
        for (int i = 0; i <= n1; i++) fhd[i] = fhd[i] * zk;
        for (int n = 1; n <= n1; n++) for (int m = 1; m <= n; m++) y[n * ld + m] *= stj;
        cplx *pv = phi + (size_t)jj * wm + n1, *pn = phin + (size_t)jj * wm + n1;
        pv[0] = a[0] * fh[0];
        pn[0] = a[0] * fhd[0] * rn;
        for (int n = 1; n <= n1; n++) {
            pv[0] += a[EI(n, 0)] * fh[n] * y[n * ld];
            cplx u1 = fhd[n] * rn, u2 = fh[n] * thn, u3 = u1 * y[n * ld] - u2 * yd[n * ld] * stj;
            pn[0] += u3 * a[EI(n, 0)];
            for (int m = 1; m <= n; m++) {
                cplx z1 = fh[n] * y[n * ld + m];
                pv[m] += a[EI(n, m)] * z1;
                pv[-m] += a[EI(n, -m)] * z1;
                u3 = u1 * y[n * ld + m] - u2 * yd[n * ld + m];
                pn[m] += u3 * a[EI(n, m)];
                pn[-m] += u3 * a[EI(n, -m)];
            }
        }
    }
    free(fh); free(fhd); free(y); free(yd);
    hproject_stab(zk, phi, phin, n1, sc2, out, n2, radius, x, w, nq);
}

/* L2L: h3dlocloczshiftstab_fast (src/h3dtrans.f:2151-2245) =
 * h3dlocevalspherestab_fast (src/projections.f:901-1045) + projection.   */
static void hzshift_l2l(cplx zk, double sc1, const cplx *a, int n1, double sc2, cplx *out, int n2, double radius,
                        double zshift, const double *x, const double *w, int nq)
{
    int wm = 2 * n2 + 1, ld = n1 + 1, lw = n1 + 1000;
    cplx *phi = calloc((size_t)nq * wm, sizeof(cplx)), *phin = calloc((size_t)nq * wm, sizeof(cplx));
    cplx *fj = malloc(sizeof(cplx) * (lw + 2)), *fjd = malloc(sizeof(cplx) * (n1 + 2));
    int *isc = malloc(sizeof(int) * (lw + 2));
    double *y = malloc(sizeof(double) * (n1 + 2) * (n1 + 2)), *yd = malloc(sizeof(double) * (n1 + 2) * (n1 + 2));
    for (int jj = 0; jj < nq; jj++) {
        double ct = x[jj], st = sqrt(1.0 - ct * ct);
        double rj = sqrt((zshift + radius * ct) * (zshift + radius * ct) + (radius * st) * (radius * st));
        double ctj = (zshift + radius * ct) / rj, stj = sqrt(1.0 - ctj * ctj);
        double rn = stj * st + ctj * ct, thn = (ctj * st - stj * ct) / rj;
        ylgndr2sfw(n1, ctj, y, yd);
        if (jfuns3d(n1, zk * rj, sc1, fj, 1, fjd, lw, isc)) continue;
        for (int i = 0; i <= n1; i++) fjd[i] = fjd[i] * zk;
        for (int n = 1; n <= n1; n++) for (int m = 1; m <= n; m++) y[n * ld + m] *= stj;
        cplx *pv = phi + (size_t)jj * wm + n2, *pn = phin + (size_t)jj * wm + n2;
        pv[0] = a[0] * fj[0];
        pn[0] = a[0] * fjd[0] * rn;
        for (int n = 1; n <= n1; n++) {
            pv[0] += a[EI(n, 0)] * fj[n] * y[n * ld];
            cplx u1 = fjd[n] * rn, u2 = fj[n] * thn, u3 = u1 * y[n * ld] - u2 * yd[n * ld] * stj;
            pn[0] += u3 * a[EI(n, 0)];
            int mm = n < n2 ? n : n2;
            for (int m = 1; m <= mm; m++) {
                cplx z1 = fj[n] * y[n * ld + m];
                pv[m] += a[EI(n, m)] * z1;
                pv[-m] += a[EI(n, -m)] * z1;
                u3 = u1 * y[n * ld + m] - u2 * yd[n * ld + m];
                pn[m] += u3 * a[EI(n, m)];
                pn[-m] += u3 * a[EI(n, -m)];
            }
        }
    }
    free(fj); free(fjd); free(isc); free(y); free(yd);
    hproject_stab(zk, phi, phin, n2, sc2, out, n2, radius, x, w, nq);
}

/* Rotation matrices for the directions the translations use, cached by
 * polar angle (many offsets share one).                                   */
typedef struct {
    int n, cap, ldm;
    double *theta;
    double **mat;
} rotcache;

static const double *rotcache_get(rotcache *c, double theta)
{
    const double *r = NULL;
#pragma omp critical(hrotcache)
    {
        for (int i = 0; i < c->n; i++)
            if (fabs(c->theta[i] - theta) < 1e-13) { r = c->mat[i]; break; }
        if (!r) {
            if (c->n == c->cap) {
                c->cap = c->cap ? 2 * c->cap : 64;
                c->theta = realloc(c->theta, sizeof(double) * c->cap);
                c->mat = realloc(c->mat, sizeof(double *) * c->cap);
            }
            double *m = malloc(sizeof(double) * (size_t)(c->ldm + 1) * (c->ldm + 1) * (2 * c->ldm + 1));
            rot_init(m, c->ldm, theta);
            c->theta[c->n] = theta;
            c->mat[c->n] = m;
            c->n++;
            r = m;
        }
    }
    return r;
}
static void rotcache_free(rotcache *c)
{
    for (int i = 0; i < c->n; i++) free(c->mat[i]);
    free(c->theta); free(c->mat);
}

/* ---- rotation by projection, rotviaprojf90 (src/rotproj.f:883-940), used
 * by the reference's Helmholtz translations for orders >= 30
 * (src/h3dtrans.f:318-345, 1335-1362, 2102-2131).                          */

/* next235_cproj (src/rotproj.f:123-149): the smallest even 2^a 3^b 5^c >= base */
static int next235(double base)
{
    int n = 2 * (int)(base / 2.0 + .9999);
    if (n <= 0) n = 2;
    for (;;) {
        int d = n;
        while (d % 2 == 0) d /= 2;
        while (d % 3 == 0) d /= 3;
        while (d % 5 == 0) d /= 5;
        if (d == 1) return n;
        n += 2;
    }
}

/* ylgndrini (src/yrecursion.f:679-711) */
static void ylgndrini_r(int nmax, double *rat1, double *rat2)
{
    int ld = nmax + 1;
#define R1(n, m) rat1[(n) * ld + (m)]
#define R2(n, m) rat2[(n) * ld + (m)]
    R1(0, 0) = 1; R2(0, 0) = 1;
    for (int m = 0; m <= nmax; m++) {
        if (m > 0) { R1(m, m) = sqrt((2 * m - 1.0) / (2 * m)); R2(m, m) = 1; }
        if (m < nmax) { R1(m + 1, m) = sqrt(2 * m + 1.0); R2(m + 1, m) = 1; }
        for (int n = m + 2; n <= nmax; n++) {
            R1(n, m) = (2 * n - 1) / sqrt((double)(n - m) * (n + m));
            R2(n, m) = sqrt((n + m - 1.0) * (n - m - 1.0)) / sqrt((double)(n - m) * (n + m));
        }
    }
}

/* ylgndru2sf (src/yrecursion.f:909-980): y(n,m) = sqrt((n-m)!/(n+m)!) P_n^m(x),
 * for m > 0 divided by sqrt(1-x^2); d = dy/dx, for m > 0 times sqrt(1-x^2) */
static void ylgndru2sf_r(int nmax, double x, double *y, double *d, const double *rat1, const double *rat2)
{
    int ld = nmax + 1;
#define Y_(n, m) y[(n) * ld + (m)]
#define D_(n, m) d[(n) * ld + (m)]
    double u = -sqrt((1 - x) * (1 + x)), u2 = (1 - x) * (1 + x);
    Y_(0, 0) = 1; D_(0, 0) = 0;
    if (0 < nmax) { Y_(1, 0) = x * Y_(0, 0) * R1(1, 0); D_(1, 0) = (x * D_(0, 0) + Y_(0, 0)) * R1(1, 0); }
    for (int n = 2; n <= nmax; n++) {
        Y_(n, 0) = R1(n, 0) * x * Y_(n - 1, 0) - R2(n, 0) * Y_(n - 2, 0);
        D_(n, 0) = R1(n, 0) * (x * D_(n - 1, 0) + Y_(n - 1, 0)) - R2(n, 0) * D_(n - 2, 0);
    }
    for (int m = 1; m <= nmax; m++) {
        if (m == 1) Y_(m, m) = Y_(m - 1, m - 1) * (-1) * R1(m, m);
        else Y_(m, m) = Y_(m - 1, m - 1) * u * R1(m, m);
        D_(m, m) = Y_(m, m) * (-m) * x;
        if (m < nmax) {
            Y_(m + 1, m) = x * Y_(m, m) * R1(m + 1, m);
            D_(m + 1, m) = (x * D_(m, m) + u2 * Y_(m, m)) * R1(m + 1, m);
        }
        for (int n = m + 2; n <= nmax; n++) {
            Y_(n, m) = R1(n, m) * x * Y_(n - 1, m) - R2(n, m) * Y_(n - 2, m);
            D_(n, m) = R1(n, m) * (x * D_(n - 1, m) + u2 * Y_(n - 1, m)) - R2(n, m) * D_(n - 2, m);
        }
    }
}

/* ylgndr2pm_opt (src/yrecursion.f:1871-1903): the values of ylgndru2sf at -x */
static void ylgndr2pm_r(int nterms, double *y, double *d)
{
    int ld = nterms + 1;
    for (int n = 0; n <= nterms; n += 2) {
        for (int m = 0; m <= n; m += 2) D_(n, m) = -D_(n, m);
        for (int m = 1; m <= n; m += 2) Y_(n, m) = -Y_(n, m);
    }
    for (int n = 1; n <= nterms; n += 2) {
        for (int m = 0; m <= n; m += 2) Y_(n, m) = -Y_(n, m);
        for (int m = 1; m <= n; m += 2) D_(n, m) = -D_(n, m);
    }
}

/* Forward DFT c_k = sum_j x_j e^{-2 pi i jk/n}, the transform of FFTPACK's
 * zfftf (src/dfft.f:942; the reference computes it by a mixed-radix FFT):
 * here a textbook recursive mixed-radix (2, 3, 5) decimation in time, n being
 * 2^a 3^b 5^c (next235).  tw[j] = e^{-2 pi i j / N} for the full size N.    */
static void fft235(int n, const cplx *x, int stride, cplx *out, const cplx *tw, int N)
{
    if (n == 1) { out[0] = x[0]; return; }
    const int r = (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : 5, m = n / r, step = N / n;
    cplx *sub = malloc(sizeof(cplx) * n);
    for (int q = 0; q < r; q++) fft235(m, x + (size_t)q * stride, stride * r, sub + (size_t)q * m, tw, N);
    for (int k = 0; k < m; k++)
        for (int s2 = 0; s2 < r; s2++) {
            cplx acc = 0;
            for (int q = 0; q < r; q++) {
                long e = ((long)q * (k + (long)m * s2)) % n;
                acc += sub[(size_t)q * m + k] * tw[e * step];
            }
            out[k + (size_t)m * s2] = acc;
        }
    free(sub);
}

static void dft_forward(int n, const cplx *x, cplx *c)
{
    cplx *tw = malloc(sizeof(cplx) * n);
    for (int k = 0; k < n; k++) {
        double a = -2 * M_PI * (double)k / n;
        tw[k] = cos(a) + I * sin(a);
    }
    fft235(n, x, 1, c, tw, n);
    free(tw);
}

/* rotviaproj0 (src/rotproj.f:152-219) with getmeridian (:222-283), evalall2
 * (:507-705) and projectonynm2 (:798-875): rotation of the expansion `in`
 * (degrees 0..nterms) by beta about the y axis into `out`.  The expansion and
 * its derivative along the rotated meridians are evaluated at nquad
 * equispaced nodes of the rotated equator (half of them by the reflection
 * x -> -x), and projected onto the spherical harmonics by a transform along
 * the equator.                                                             */
static void rotviaproj(double beta, int nterms, const cplx *in, cplx *out)
{
    const int nquad = next235(2.0 * nterms + 2), ld = nterms + 1;
    double *ct = malloc(sizeof(double) * 4 * nquad), *stt = ct + nquad, *cph = stt + nquad, *sph = cph + nquad;
    /* getmeridian */
    {
        double ca = cos(beta), sa = sin(beta);
        for (int i = 0; i < nquad; i++) {
            double phi = 2 * M_PI * i / nquad, theta = M_PI / 2.0;
            double xp = cos(phi) * sin(theta), yp = sin(phi) * sin(theta), zp = cos(theta);
            double x = ca * xp + sa * zp, y = yp, z = -sa * xp + ca * zp;
            double proj = sqrt(x * x + y * y);
            if (proj <= 1.0e-16) { cph[i] = 1.0; sph[i] = 0.0; }
            else { cph[i] = x / proj; sph[i] = y / proj; }
            ct[i] = z;
            stt[i] = proj;
        }
    }
    double *rat1 = calloc((size_t)ld * ld, sizeof(double)), *rat2 = calloc((size_t)ld * ld, sizeof(double));
    double *y = calloc((size_t)ld * ld, sizeof(double)), *d = calloc((size_t)ld * ld, sizeof(double));
    cplx *uval = calloc((size_t)nquad * ld, sizeof(cplx)), *uder = calloc((size_t)nquad * ld, sizeof(cplx));
    cplx *epm = malloc(sizeof(cplx) * (2 * nterms + 3)), *eph = epm + nterms + 1;
    /* evalall2 */
    {
        double cbeta = cos(beta), sbeta = -sin(beta);
        ylgndrini_r(nterms, rat1, rat2);
        int nquad2 = nquad / 2, nquad4 = nquad2 / 2 + 1;
        for (int jj = 1; jj <= nquad4; jj++) {
            for (int pass = 0; pass < 2; pass++) {
                int col;
                double ctheta, stheta, cphi, sphi;
                if (pass == 0) {
                    col = jj;
                    ctheta = ct[jj - 1]; stheta = stt[jj - 1]; cphi = cph[jj - 1]; sphi = sph[jj - 1];
                    ylgndru2sf_r(nterms, ctheta, y, d, rat1, rat2);
                } else {
                    int reflect = !(jj == 1 || (jj == nquad4 && nquad2 % 2 == 0));
                    if (!reflect) break;
                    col = nquad2 - jj + 2;
                    ylgndr2pm_r(nterms, y, d);
                    ctheta = -ct[jj - 1]; stheta = stt[jj - 1]; cphi = -cph[jj - 1]; sphi = sph[jj - 1];
                }
                double dir1 = -sbeta, dir2 = 0, dir3 = cbeta;
                double proj2 = (cphi * ctheta) * dir1 + (sphi * ctheta) * dir2 + (-stheta) * dir3;
                double proj1 = (-sphi) * dir1 + cphi * dir2 + 0 * dir3;
                cplx e1 = cphi + I * sphi;
                eph[0] = 1;
                eph[1] = e1; eph[-1] = conj(e1);
                for (int i = 2; i <= nterms; i++) { eph[i] = eph[i - 1] * e1; eph[-i] = conj(eph[i]); }
                for (int n = 0; n <= nterms; n++) {
                    cplx uv = 0, ut = 0, up = 0;
                    for (int m = 1; m <= n; m++) {
                        cplx z1 = eph[m] * in[EI(n, m)], z2 = eph[-m] * in[EI(n, -m)];
                        cplx zs = z1 + z2, zd = z1 - z2;
                        uv += Y_(n, m) * zs;
                        ut += D_(n, m) * zs;
                        up -= Y_(n, m) * m * zd;
                    }
                    uv = stheta * uv + Y_(n, 0) * in[EI(n, 0)];
                    ut = ut + D_(n, 0) * stheta * in[EI(n, 0)];
                    cplx v = uv, dv = ut * proj2 + up * I * proj1;
                    uval[(size_t)n * nquad + col - 1] = v;
                    uder[(size_t)n * nquad + col - 1] = dv;
                    uval[(size_t)n * nquad + col - 1 + nquad / 2] = (n % 2 == 0) ? v : -v;
                    uder[(size_t)n * nquad + col - 1 + nquad / 2] = (n % 2 == 0) ? -dv : dv;
                }
            }
        }
    }
    /* projectonynm2 */
    {
        double h = 1.0 / nquad;
        ylgndru2sf_r(nterms, 0.0, y, d, rat1, rat2);
        cplx *av = malloc(sizeof(cplx) * 2 * nquad), *cv = av + nquad;
        for (int n = 0; n <= nterms; n++) {
            double dn = sqrt(2 * n + 1.0);
            for (int i = 0; i < nquad; i++) av[i] = uval[(size_t)n * nquad + i] * dn + uder[(size_t)n * nquad + i];
            dft_forward(nquad, av, cv);
            for (int m = -n; m <= n; m++) {
                cplx alpha = (m >= 0 ? cv[m] : cv[nquad + m]) * h;
                int am = m < 0 ? -m : m;
                out[EI(n, m)] = alpha / (Y_(n, am) * dn - D_(n, am));
            }
        }
        free(av);
    }
#undef R1
#undef R2
#undef Y_
#undef D_
    free(ct); free(rat1); free(rat2); free(y); free(d); free(uval); free(uder); free(epm);
}

void oracle_rotviaproj(double beta, int nterms, const cplx *in, cplx *out) { rotviaproj(beta, nterms, in, out); }

void oracle_rotviarecur(double beta, int nterms, const cplx *in, cplx *out)
{
    size_t sz = (size_t)(nterms + 1) * (nterms + 1) * (2 * nterms + 1);
    double *r = malloc(sz * sizeof(double));
    rot_init(r, nterms, beta);
    rot_apply(r, nterms, nterms, in, out);
    free(r);
}

/* One translation: phases e^{i m phi}, rotation by theta, z-shift, rotation
 * by -theta, phases e^{-i m phi}, added into `out`: h3dmpmpquad0
 * (src/h3dtrans.f:211-363), h3dmplocquad_trunc0 (:1229-1376) and
 * h3dloclocquad0 (:1998-2150).  kind 0 M2M, 1 M2L, 2 L2L; nin / nout are the
 * source and target degrees.                                               */
static void htranslate(int kind, cplx zk, const double *c_from, const double *c_to, const cplx *in, int nin, double sc1,
                       int nout, double sc2, double radius, const double *x, const double *w, int nq, cplx *out,
                       rotcache *rc)
{
    double rv[3] = {c_to[0] - c_from[0], c_to[1] - c_from[1], c_to[2] - c_from[2]}, d, th, ph;
    cart2polarl(rv, &d, &th, &ph);
    int pm = nin > nout ? nin : nout, K = (pm + 1) * (pm + 1);
    cplx *em = malloc(sizeof(cplx) * (2 * pm + 5)), *e = em + pm + 1;
    e[0] = 1; e[1] = cexp(I * ph); e[-1] = conj(e[1]);
    for (int l = 1; l <= pm; l++) { e[l + 1] = e[l] * e[1]; e[-1 - l] = conj(e[l + 1]); }
    cplx *a = calloc(K, sizeof(cplx)), *b = calloc(K, sizeof(cplx)), *cz = calloc(K, sizeof(cplx));
    for (int l = 0; l <= nin; l++) for (int m = -l; m <= l; m++) a[EI(l, m)] = in[EI(l, m)] * e[m];
    /* orders >= 30 rotate by projection (rotviaprojf90), lower ones by the
     * recursion (rotviarecur3f90): forward on the source order for M2M and
     * M2L, on the target order for L2L; backward on the target order
     * (src/h3dtrans.f:318, 340, 1335, 1356, 2102, 2127)                   */
    if ((kind == 2 ? nout : nin) >= 30) rotviaproj(th, nin, a, b);
    else rot_apply(rotcache_get(rc, th), rc->ldm, nin, a, b);
    if (kind == 0) hzshift_m2m(zk, sc1, b, nin, sc2, cz, nout, radius, d, x, w, nq);
    else if (kind == 1) hzshift_m2l(zk, sc1, b, nin, sc2, cz, nout, radius, d, x, w, nq);
    else hzshift_l2l(zk, sc1, b, nin, sc2, cz, nout, radius, d, x, w, nq);
    if (nout >= 30) rotviaproj(-th, nout, cz, a);
    else rot_apply(rotcache_get(rc, -th), rc->ldm, nout, cz, a);
    for (int l = 0; l <= nout; l++) for (int m = -l; m <= l; m++) out[EI(l, m)] += e[-m] * a[EI(l, m)];
    free(em); free(a); free(b); free(cz);
}

/* Single-operator entry points for the oracle's own tests (the box's sum
 * times ik, as h3dformmp_add_trunc / h3dformta_add_trunc add it).         */
void oracle_hformmp(double zkr, double zki, double rscale, int ns, const double *src, int ifcharge, const cplx *q,
                    int ifdipole, const cplx *ds, const double *dv, const double *c, int p, cplx *mp)
{
    cplx zk = zkr + I * zki;
    int K = (p + 1) * (p + 1);
    cplx *tmp = calloc(K, sizeof(cplx));
    hwork w;
    hwork_init(&w, p);
    for (int pass = 0; pass < 2; pass++) {
        if ((pass == 0 && ifcharge != 1) || (pass == 1 && ifdipole != 1)) continue;
        memset(tmp, 0, sizeof(cplx) * K);
        for (int i = 0; i < ns; i++) {
            if (pass == 0) hformmp_charge(zk, rscale, src + 3 * (size_t)i, q[i], c, p, tmp, &w);
            else hformmp_dipole(zk, rscale, src + 3 * (size_t)i, ds[i], dv + 3 * (size_t)i, c, p, tmp, &w);
        }
        for (int k = 0; k < K; k++) mp[k] += tmp[k] * I * zk;
    }
    hwork_free(&w);
    free(tmp);
}

void oracle_hformta(double zkr, double zki, double rscale, int ns, const double *src, int ifcharge, const cplx *q,
                    int ifdipole, const cplx *ds, const double *dv, const double *c, int p, cplx *lo)
{
    cplx zk = zkr + I * zki;
    int K = (p + 1) * (p + 1);
    cplx *tmp = calloc(K, sizeof(cplx));
    hwork w;
    hwork_init(&w, p);
    for (int pass = 0; pass < 2; pass++) {
        if ((pass == 0 && ifcharge != 1) || (pass == 1 && ifdipole != 1)) continue;
        memset(tmp, 0, sizeof(cplx) * K);
        for (int i = 0; i < ns; i++) {
            if (pass == 0) hformta_charge(zk, rscale, src + 3 * (size_t)i, q[i], c, p, tmp, &w);
            else hformta_dipole(zk, rscale, src + 3 * (size_t)i, ds[i], dv + 3 * (size_t)i, c, p, tmp, &w);
        }
        for (int k = 0; k < K; k++) lo[k] += tmp[k] * I * zk;
    }
    hwork_free(&w);
    free(tmp);
}

void oracle_hmpeval(double zkr, double zki, double rscale, const double *c, const cplx *mp, int p, int nt,
                    const double *t, cplx *pot, cplx *fld)
{
    hwork w;
    hwork_init(&w, p);
    for (int i = 0; i < nt; i++) hmpeval(zkr + I * zki, rscale, c, mp, p, t + 3 * i, pot + i, fld + 3 * i, &w);
    hwork_free(&w);
}

void oracle_htaeval(double zkr, double zki, double rscale, const double *c, const cplx *lo, int p, int nt,
                    const double *t, cplx *pot, cplx *fld)
{
    hwork w;
    hwork_init(&w, p);
    for (int i = 0; i < nt; i++) htaeval(zkr + I * zki, rscale, c, lo, p, t + 3 * i, pot + i, fld + 3 * i, &w);
    hwork_free(&w);
}

void oracle_htranslate(int kind, double zkr, double zki, const double *c_from, const double *c_to, const cplx *in,
                       int nin, double sc1, int nout, double sc2, double radius, int nq, cplx *out)
{
    double *x = malloc(sizeof(double) * nq), *w = malloc(sizeof(double) * nq);
    oracle_legewhts(nq, x, w);
    rotcache rc = {0, 0, nin > nout ? nin : nout, NULL, NULL};
    htranslate(kind, zkr + I * zki, c_from, c_to, in, nin, sc1, nout, sc2, radius, x, w, nq, out, &rc);
    rotcache_free(&rc);
    free(x); free(w);
}

/* ------------------------------------------------------------------ */
/* hfmm3dparttarg (src/hfmm3dpart.f:141-539) with hfmm3dparttargmain
 * (:545-1086) and hfmm3d_list2 (src/hfmm3drouts.f:153-564).  `tinfo`
 * (optional) receives the wall time of the tree and of steps 1..8;
 * `nterms_out` (optional, 200 ints) the expansion order of every level.   */
/* Triangle mode of the Helmholtz FMM (hfmm3dtriatarg, src/hfmm3dtria.f:133-1215):
 * the sources are flat triangles, the tree's points their centroids (source);
 * the far field runs on the triangles' quadrature nodes (degree norder), the
 * near field integrates over each triangle (htri_oracle.c, degree nqtri). */
typedef struct {
    const double *tri, *trinorm;
    int norder, nqtri;
} htri_args;
static void htri_point(cplx zk, int nj, const double *tri, int ifcharge, const cplx *q, int ifdipole, const cplx *ds,
                       const double *x, long self, int iffld, int nqtri, cplx *pot, cplx *fld);

static void hfmm_core(int *ier, int iprec, double zkr, double zki, int nsource, const double *source,
                      int ifcharge, const cplx *charge, int ifdipole, const cplx *dipstr, const double *dipvec,
                      int ifpot, cplx *pot, int iffld, cplx *fld, int ntarget, const double *target,
                      int ifpottarg, cplx *pottarg, int iffldtarg, cplx *fldtarg, double *tinfo,
                      int *nterms_out, const htri_args *ta)
{
    *ier = 0;
    cplx zk = zkr + I * zki;
    double eps = oracle_lap_eps(iprec);
    int nbox = ta ? oracle_tri_nbox(iprec, nsource, ntarget) : oracle_lap_nbox(iprec, nsource, ntarget);
    if (nbox < 0 || nsource < 1) { *ier = 4; return; }
    double tt0 = omp_get_wtime();
    otree T;
    memset(&T, 0, sizeof T);
    build_boxes(&T, source, nsource, target, ntarget, nbox);
    build_lists(&T);
    double tt1 = omp_get_wtime();
    if (tinfo) tinfo[0] = tt1 - tt0;
    int nlev = T.nlev, nb = T.nboxes;
    double scale[202], bsize[202];
    int nterms[202];
    for (int i = 0; i <= nlev; i++) {
        scale[i] = 1.0;
        /* zk is implicitly real*8 in hfmm3dparttarg (src/hfmm3dpart.f:145, no
         * complex declaration), so this rule reads only Re(zk) (:337-341) */
        /* hfmm3dtriatarg declares zk complex*16: there the rule sees |zk| (src/hfmm3dtria.f:248, 350-355) */
        double bs = ta ? cabs((T.size / pow(2.0, i)) * zk) : fabs((T.size / pow(2.0, i)) * creal(zk));
        if (bs < 1) scale[i] = bs;
        bsize[i] = T.size / pow(2.0, i);
        int e;
        nterms[i] = oracle_h3dterms(bsize[i], zkr, zki, eps, &e);
        if (nterms_out) nterms_out[i] = nterms[i];
    }
    int pmax = 1;
    for (int i = 2; i <= nlev; i++) if (nterms[i] > pmax) pmax = nterms[i];
    int K = (pmax + 1) * (pmax + 1);
    double *ss = malloc(sizeof(double) * 3 * (size_t)nsource);
    double *ts = malloc(sizeof(double) * 3 * (size_t)(ntarget > 0 ? ntarget : 1));
    cplx *qs = calloc((size_t)nsource, sizeof(cplx)), *dss = calloc((size_t)nsource, sizeof(cplx));
    double *dvs = calloc(3 * (size_t)nsource, sizeof(double));
    for (int i = 0; i < nsource; i++) {
        int j = T.iz[i];
        memcpy(ss + 3 * (size_t)i, source + 3 * (size_t)j, 3 * sizeof(double));
        if (ifcharge == 1) qs[i] = charge[j];
        if (ifdipole == 1) { dss[i] = dipstr[j]; memcpy(dvs + 3 * (size_t)i, dipvec + 3 * (size_t)j, 3 * sizeof(double)); }
    }
    for (int i = 0; i < ntarget; i++) memcpy(ts + 3 * (size_t)i, target + 3 * (size_t)T.iztarg[i], 3 * sizeof(double));
    /* triangles: sorted vertices, and the far field's quadrature nodes in tree order */
    double *trs = NULL, *qp = NULL, *qw = NULL, *qv = NULL;
    cplx *qq = NULL, *qd = NULL;
    int nq = 1;
    if (ta) {
        trs = malloc(sizeof(double) * 9 * (size_t)nsource);
        for (int i = 0; i < nsource; i++) memcpy(trs + 9 * (size_t)i, ta->tri + 9 * (size_t)T.iz[i], 9 * sizeof(double));
        double xi[64], eta[64], wr[64];
        nq = tri_rule(ta->norder, xi, eta, wr);
        size_t nn = (size_t)nsource * nq;
        qp = malloc(sizeof(double) * 3 * nn); qw = malloc(sizeof(double) * nn); qv = malloc(sizeof(double) * 3 * nn);
        qq = calloc(nn, sizeof(cplx)); qd = calloc(nn, sizeof(cplx));
        tri_nodes(nsource, trs, ta->norder, qp, qw, &nq);
        for (size_t i = 0; i < nn; i++) {
            size_t t = i / nq;
            if (ifcharge == 1) qq[i] = qs[t] * qw[i];
            if (ifdipole == 1) qd[i] = dss[t] * qw[i];
            memcpy(qv + 3 * i, ta->trinorm + 3 * (size_t)T.iz[t], 3 * sizeof(double));
        }
    }
    cplx *ps = calloc((size_t)nsource, sizeof(cplx)), *fs = calloc(3 * (size_t)nsource, sizeof(cplx));
    cplx *pt = calloc((size_t)(ntarget > 0 ? ntarget : 1), sizeof(cplx));
    cplx *ft = calloc(3 * (size_t)(ntarget > 0 ? ntarget : 1), sizeof(cplx));
    cplx *mpole = calloc((size_t)nb * K, sizeof(cplx)), *local = calloc((size_t)nb * K, sizeof(cplx));
    rotcache rc = {0, 0, pmax, NULL, NULL};
    double *xq = malloc(sizeof(double) * (3 * pmax + 8)), *wq = malloc(sizeof(double) * (3 * pmax + 8));
#define BX(b, f) T.box[20 * (size_t)(b) + (f)]
#define LS(ty, b) T.lstart[ty][b]
#define LE(ty, b) T.lstart[ty][(b) + 1]
#define LI(ty, i) T.lidx[ty][i]
#define CEN(b) (T.center + 3 * (size_t)(b))
#define RAD(lev) (sqrt(3.0) / 2.0 * bsize[lev])
    double tm[9];
    /* STEP 1: P2M at leaves of level >= 2 with sources (src/hfmm3dpart.f:696-760) */
    tm[0] = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        int lev = BX(ib, B_LEV);
        if (lev < 2 || BX(ib, B_NSRC) == 0 || nkids(&T, ib) != 0) continue;
        int s0 = BX(ib, B_SRC0), n = BX(ib, B_NSRC);
        if (ta) {
            size_t q0 = (size_t)s0 * nq;
            oracle_hformmp(zkr, zki, scale[lev], n * nq, qp + 3 * q0, ifcharge, qq + q0, ifdipole, qd + q0, qv + 3 * q0,
                           CEN(ib), nterms[lev], mpole + (size_t)ib * K);
        } else {
            oracle_hformmp(zkr, zki, scale[lev], n, ss + 3 * (size_t)s0, ifcharge, qs + s0, ifdipole, dss + s0,
                           dvs + 3 * (size_t)s0, CEN(ib), nterms[lev], mpole + (size_t)ib * K);
        }
    }
    /* STEP 2: P2L of a leaf's sources into its list-3 boxes (src/hfmm3dpart.f:775-846),
     * gathered here per receiving box through the dual list 4.           */
    tm[1] = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        int lev = BX(ib, B_LEV);
        for (int li = LS(4, ib); li < LE(4, ib); li++) {
            int jb = LI(4, li);
            int n = BX(jb, B_NSRC);
            if (n == 0) continue;
            int s0 = BX(jb, B_SRC0);
            if (ta) {
                size_t q0 = (size_t)s0 * nq;
                oracle_hformta(zkr, zki, scale[lev], n * nq, qp + 3 * q0, ifcharge, qq + q0, ifdipole, qd + q0,
                               qv + 3 * q0, CEN(ib), nterms[lev], local + (size_t)ib * K);
            } else {
                oracle_hformta(zkr, zki, scale[lev], n, ss + 3 * (size_t)s0, ifcharge, qs + s0, ifdipole, dss + s0,
                               dvs + 3 * (size_t)s0, CEN(ib), nterms[lev], local + (size_t)ib * K);
            }
        }
    }
    /* STEP 3: M2M into parents of levels nlev-1..2 (src/hfmm3drouts.f:209-289) */
    tm[2] = omp_get_wtime();
    for (int lev = nlev - 1; lev >= 2; lev--) {
        int nq = (int)(nterms[lev] * 2.5);
        if (nq < 6) nq = 6;
        oracle_legewhts(nq, xq, wq);
        int b0 = T.laddr[2 * lev], b1 = b0 + T.laddr[2 * lev + 1];
#pragma omp parallel for schedule(dynamic)
        for (int ib = b0; ib < b1; ib++) {
            if (BX(ib, B_NSRC) == 0 || nkids(&T, ib) == 0) continue;
            cplx *mo = mpole + (size_t)ib * K;
            memset(mo, 0, sizeof(cplx) * K);
            for (int k = 0; k < 8; k++) {
                int jb = BX(ib, B_KID + k);
                if (jb < 0) continue;
                htranslate(0, zk, CEN(jb), CEN(ib), mpole + (size_t)jb * K, nterms[lev + 1], scale[lev + 1],
                           nterms[lev], scale[lev], RAD(lev), xq, wq, nq, mo, &rc);
            }
        }
    }
    /* STEP 4: M2L over list 2, levels 2..nlev (src/hfmm3drouts.f:337-470) */
    tm[3] = omp_get_wtime();
    int ifprune = !(ifpot == 1 || iffld == 1);
    for (int lev = 2; lev <= nlev; lev++) {
        int itable[343], e;
        oracle_h3dterms_list2(bsize[lev], zkr, zki, eps, itable, &e);
        int nq = (int)((float)nterms[lev] * 1.2f); /* a default-real product in the reference */
        if (nq < 6) nq = 6;
        oracle_legewhts(nq, xq, wq);
        int b0 = T.laddr[2 * lev], b1 = b0 + T.laddr[2 * lev + 1];
#pragma omp parallel for schedule(dynamic)
        for (int ib = b0; ib < b1; ib++) {
            for (int li = LS(2, ib); li < LE(2, ib); li++) {
                int jb = LI(2, li);
                if (BX(jb, B_NSRC) == 0) continue;
                if (BX(ib, B_NTRG) == 0 && ifprune) continue;
                int ii = BX(jb, B_I) - BX(ib, B_I), jj = BX(jb, B_J) - BX(ib, B_J), kk = BX(jb, B_K) - BX(ib, B_K);
                int nt = itable[((ii + 3) * 7 + (jj + 3)) * 7 + (kk + 3)];
                if (nt > nterms[lev]) nt = nterms[lev];
                htranslate(1, zk, CEN(jb), CEN(ib), mpole + (size_t)jb * K, nt, scale[lev], nt, scale[lev], RAD(lev),
                           xq, wq, nq, local + (size_t)ib * K, &rc);
            }
        }
    }
    /* STEP 5: L2L from parents of levels 2..nlev-1 (src/hfmm3drouts.f:485-548) */
    tm[4] = omp_get_wtime();
    for (int lev = 2; lev <= nlev - 1; lev++) {
        int nq = 2 * nterms[lev];
        if (nq < 6) nq = 6;
        oracle_legewhts(nq, xq, wq);
        int b0 = T.laddr[2 * lev], b1 = b0 + T.laddr[2 * lev + 1];
#pragma omp parallel for schedule(dynamic)
        for (int ib = b0; ib < b1; ib++) {
            if (nkids(&T, ib) == 0) continue;
            for (int k = 0; k < 8; k++) {
                int jb = BX(ib, B_KID + k);
                if (jb < 0) continue;
                htranslate(2, zk, CEN(ib), CEN(jb), local + (size_t)ib * K, nterms[lev], scale[lev], nterms[lev + 1],
                           scale[lev + 1], RAD(lev + 1), xq, wq, nq, local + (size_t)jb * K, &rc);
            }
        }
    }
    /* STEP 6: M2P from list-3 boxes (src/hfmm3dpart.f:870-935, there per
     * source box through list 4); STEP 7: L2P at leaves of level >= 2.   */
    tm[5] = omp_get_wtime();
#pragma omp parallel
    {
        hwork w;
        hwork_init(&w, pmax);
#pragma omp for schedule(dynamic)
        for (int ib = 0; ib < nb; ib++) {
            for (int li = LS(3, ib); li < LE(3, ib); li++) {
                int jb = LI(3, li), lj = BX(jb, B_LEV);
                if (BX(jb, B_NSRC) == 0) continue;
                const cplx *mj = mpole + (size_t)jb * K;
                cplx pv, fv[3];
                for (int i = BX(ib, B_SRC0); i < BX(ib, B_SRC0) + BX(ib, B_NSRC); i++) {
                    if (hmpeval(zk, scale[lj], CEN(jb), mj, nterms[lj], ss + 3 * (size_t)i, &pv, fv, &w)) continue;
                    if (ifpot == 1) ps[i] += pv;
                    if (iffld == 1) for (int d = 0; d < 3; d++) fs[3 * (size_t)i + d] += fv[d];
                }
                for (int i = BX(ib, B_TRG0); i < BX(ib, B_TRG0) + BX(ib, B_NTRG); i++) {
                    if (hmpeval(zk, scale[lj], CEN(jb), mj, nterms[lj], ts + 3 * (size_t)i, &pv, fv, &w)) continue;
                    if (ifpottarg == 1) pt[i] += pv;
                    if (iffldtarg == 1) for (int d = 0; d < 3; d++) ft[3 * (size_t)i + d] += fv[d];
                }
            }
        }
#pragma omp for schedule(dynamic)
        for (int ib = 0; ib < nb; ib++) {
            int lev = BX(ib, B_LEV);
            if (nkids(&T, ib) != 0 || lev < 2) continue;
            const cplx *lb = local + (size_t)ib * K;
            cplx pv, fv[3];
            for (int i = BX(ib, B_SRC0); i < BX(ib, B_SRC0) + BX(ib, B_NSRC); i++) {
                if (htaeval(zk, scale[lev], CEN(ib), lb, nterms[lev], ss + 3 * (size_t)i, &pv, fv, &w)) continue;
                if (ifpot == 1) ps[i] += pv;
                if (iffld == 1) for (int d = 0; d < 3; d++) fs[3 * (size_t)i + d] += fv[d];
            }
            for (int i = BX(ib, B_TRG0); i < BX(ib, B_TRG0) + BX(ib, B_NTRG); i++) {
                if (htaeval(zk, scale[lev], CEN(ib), lb, nterms[lev], ts + 3 * (size_t)i, &pv, fv, &w)) continue;
                if (ifpottarg == 1) pt[i] += pv;
                if (iffldtarg == 1) for (int d = 0; d < 3; d++) ft[3 * (size_t)i + d] += fv[d];
            }
        }
        hwork_free(&w);
    }
    /* STEP 8: P2P, self and list 1 (src/hfmm3dpart.f:1046-1080) */
    tm[6] = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        if (nkids(&T, ib) != 0) continue;
        int s0 = BX(ib, B_SRC0), ns = BX(ib, B_NSRC), t0 = BX(ib, B_TRG0), ntg = BX(ib, B_NTRG);
        int nl = 1 + LE(1, ib) - LS(1, ib);
        for (int li = 0; li < nl; li++) {
            int jb = li == 0 ? ib : LI(1, LS(1, ib) + li - 1);
            int js0 = BX(jb, B_SRC0), jn = BX(jb, B_NSRC);
            if (jn == 0) continue;
            cplx pv, fv[3];
            if (ifpot == 1 || iffld == 1)
                for (int i = s0; i < s0 + ns; i++) {
                    if (ta)
                        htri_point(zk, jn, trs + 9 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0,
                                   ss + 3 * (size_t)i, jb == ib ? i - s0 : -1, iffld, ta->nqtri, &pv, fv);
                    else
                        hdirect_one(zk, jn, ss + 3 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0,
                                    dvs + 3 * (size_t)js0, ss + 3 * (size_t)i, jb == ib ? i - s0 : -1, iffld, &pv, fv);
                    if (ifpot == 1) ps[i] += pv;
                    if (iffld == 1) for (int d = 0; d < 3; d++) fs[3 * (size_t)i + d] += fv[d];
                }
            if (ifpottarg == 1 || iffldtarg == 1)
                for (int i = t0; i < t0 + ntg; i++) {
                    if (ta)
                        htri_point(zk, jn, trs + 9 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0,
                                   ts + 3 * (size_t)i, -1, iffldtarg, ta->nqtri, &pv, fv);
                    else
                        hdirect_one(zk, jn, ss + 3 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0,
                                    dvs + 3 * (size_t)js0, ts + 3 * (size_t)i, -1, iffldtarg, &pv, fv);
                    if (ifpottarg == 1) pt[i] += pv;
                    if (iffldtarg == 1) for (int d = 0; d < 3; d++) ft[3 * (size_t)i + d] += fv[d];
                }
        }
    }
    tm[7] = omp_get_wtime();
    if (tinfo) for (int i = 0; i < 7; i++) tinfo[1 + i] = tm[i + 1] - tm[i];
    for (int i = 0; i < nsource; i++) {
        int j = T.iz[i];
        if (ifpot == 1) pot[j] = ps[i];
        if (iffld == 1) for (int d = 0; d < 3; d++) fld[3 * (size_t)j + d] = fs[3 * (size_t)i + d];
    }
    for (int i = 0; i < ntarget; i++) {
        int j = T.iztarg[i];
        if (ifpottarg == 1) pottarg[j] = pt[i];
        if (iffldtarg == 1) for (int d = 0; d < 3; d++) fldtarg[3 * (size_t)j + d] = ft[3 * (size_t)i + d];
    }
#undef BX
#undef LS
#undef LE
#undef LI
#undef CEN
#undef RAD
    rotcache_free(&rc);
    free(xq); free(wq);
    free(ss); free(ts); free(qs); free(dss); free(dvs); free(ps); free(fs); free(pt); free(ft);
    free(mpole); free(local);
    free(trs); free(qp); free(qw); free(qv); free(qq); free(qd);
    tree_free(&T);
}

void oracle_hfmm3dparttarg(int *ier, int iprec, double zkr, double zki, int nsource, const double *source,
                           int ifcharge, const cplx *charge, int ifdipole, const cplx *dipstr, const double *dipvec,
                           int ifpot, cplx *pot, int iffld, cplx *fld, int ntarget, const double *target,
                           int ifpottarg, cplx *pottarg, int iffldtarg, cplx *fldtarg, double *tinfo,
                           int *nterms_out)
{
    hfmm_core(ier, iprec, zkr, zki, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, pot, iffld,
              fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg, tinfo, nterms_out, NULL);
}
