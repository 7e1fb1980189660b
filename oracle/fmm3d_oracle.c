/*
 * fmm3d_oracle.c -- CPU restatement of FMMLIB3D's Laplace particle FMM.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library in fmmlib3d_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it; nothing in the
 * product path links, calls or falls back to it.
 *
 * Parity status: the reference (Fortran 77/90) cannot be compiled in this
 * environment (no Fortran compiler) and ships no golden output files, so this
 * restatement is pinned only through (a) the FP64 O(N^2) direct sum
 * (l3dpartdirect), which it also restates, and (b) the accuracy contract of
 * each iprec (src/lfmm3dpart.f:156-165).  Relative to the reference's FMM
 * itself, parity is unpinned.
 *
 * Every routine below names the reference routine (file:line) whose
 * arithmetic it follows.  Paths are relative to the FMMLIB3D source tree.
 * The layout of data differs (0-based ids, CSR lists, compact expansion
 * index n*n+n+m) but the arithmetic, the tree, the lists, the expansion
 * orders and the order of the passes are the reference's.
 */
#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

/* ------------------------------------------------------------------ */
/* Deterministic inputs: LAPACK dlaran as vendored in examples/dlaran.f:48-84,
 * driven by examples/hkrand.f:3-19.                                       */
static int hk_seed[4] = {0, 0, 0, 1};

double oracle_dlaran(int *iseed)
{
    const int m1 = 494, m2 = 322, m3 = 2508, m4 = 2549, ipw2 = 4096;
    const double r = 1.0 / ipw2;
    int it4 = iseed[3] * m4;
    int it3 = it4 / ipw2;
    it4 -= ipw2 * it3;
    it3 += iseed[2] * m4 + iseed[3] * m3;
    int it2 = it3 / ipw2;
    it3 -= ipw2 * it2;
    it2 += iseed[1] * m4 + iseed[2] * m3 + iseed[3] * m2;
    int it1 = it2 / ipw2;
    it2 -= ipw2 * it1;
    it1 += iseed[0] * m4 + iseed[1] * m3 + iseed[2] * m2 + iseed[3] * m1;
    it1 %= ipw2;
    iseed[0] = it1; iseed[1] = it2; iseed[2] = it3; iseed[3] = it4;
    return r * ((double)it1 + r * ((double)it2 + r * ((double)it3 + r * ((double)it4))));
}

double oracle_hkrand(int iseed_hk)
{
    if (iseed_hk != 0) {
        hk_seed[0] = 0; hk_seed[1] = 0; hk_seed[2] = 0;
        hk_seed[3] = (2 * iseed_hk + 1) % 4096;
    }
    return oracle_dlaran(hk_seed);
}

void oracle_hkrand_reset(void)
{
    hk_seed[0] = 0; hk_seed[1] = 0; hk_seed[2] = 0; hk_seed[3] = 1;
}

/* ------------------------------------------------------------------ */
/* Pairwise kernels: lpotfld3d (src/laprouts3d.f:1308-1368) and
 * lpotfld3d_dp (src/laprouts3d.f:1962-2035).                           */
static inline void lpotfld3d(int iffld, const double *s, cplx q, const double *t,
                             cplx *pot, cplx fld[3])
{
    double xd = t[0] - s[0], yd = t[1] - s[1], zd = t[2] - s[2];
    double dd = xd * xd + yd * yd + zd * zd;
    double d = sqrt(dd);
    double dinv = 1.0 / d;
    *pot = q * dinv;
    if (iffld == 1) {
        double dinv2 = dinv * dinv, dinv3 = dinv * dinv2;
        fld[0] = q * xd * dinv3;
        fld[1] = q * yd * dinv3;
        fld[2] = q * zd * dinv3;
    }
}

static inline void lpotfld3d_dp(int iffld, const double *s, cplx ds, const double *v,
                                const double *t, cplx *pot, cplx fld[3])
{
    double xd = t[0] - s[0], yd = t[1] - s[1], zd = t[2] - s[2];
    double dd = xd * xd + yd * yd + zd * zd;
    double d = sqrt(dd);
    double dinv = 1.0 / d, dinv2 = dinv * dinv, dinv3 = dinv * dinv2;
    double dot = xd * v[0] + yd * v[1] + zd * v[2];
    *pot = ds * (dot * dinv3);
    if (iffld == 1) {
        double dinv5 = dinv3 * dinv2;
        double rt = 3.0 * dot * dinv5;
        fld[0] = ds * (rt * xd - dinv3 * v[0]);
        fld[1] = ds * (rt * yd - dinv3 * v[1]);
        fld[2] = ds * (rt * zd - dinv3 * v[2]);
    }
}

/* Sum of all sources (skipping index `skip`) at one evaluation point: the
 * inner loop of l3dpartdirect (src/lfmm3dpart.f:1451-1476).              */
static void direct_one(int ns, const double *src, int ifcharge, const cplx *charge,
                       int ifdipole, const cplx *dipstr, const double *dipvec,
                       const double *t, long skip, int iffld, cplx *pot, cplx fld[3])
{
    cplx p = 0, f0 = 0, f1 = 0, f2 = 0, pt, ft[3];
    for (long i = 0; i < ns; i++) {
        if (i == skip) continue;
        if (ifcharge == 1) {
            lpotfld3d(iffld, src + 3 * i, charge[i], t, &pt, ft);
            p += pt;
            if (iffld == 1) { f0 += ft[0]; f1 += ft[1]; f2 += ft[2]; }
        }
        if (ifdipole == 1) {
            lpotfld3d_dp(iffld, src + 3 * i, dipstr[i], dipvec + 3 * i, t, &pt, ft);
            p += pt;
            if (iffld == 1) { f0 += ft[0]; f1 += ft[1]; f2 += ft[2]; }
        }
    }
    *pot = p; fld[0] = f0; fld[1] = f1; fld[2] = f2;
}

/* l3dpartdirect, src/lfmm3dpart.f:1391-1523. */
void oracle_l3dpartdirect(int nsource, const double *source, int ifcharge, const cplx *charge,
                          int ifdipole, const cplx *dipstr, const double *dipvec,
                          int ifpot, cplx *pot, int iffld, cplx *fld,
                          int ntarget, const double *target, int ifpottarg, cplx *pottarg,
                          int iffldtarg, cplx *fldtarg)
{
    if (ifpot == 1 || iffld == 1) {
#pragma omp parallel for schedule(dynamic, 16)
        for (long j = 0; j < nsource; j++) {
            cplx p, f[3];
            direct_one(nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec,
                       source + 3 * j, j, iffld, &p, f);
            if (ifpot == 1) pot[j] = p;
            if (iffld == 1) { fld[3 * j] = f[0]; fld[3 * j + 1] = f[1]; fld[3 * j + 2] = f[2]; }
        }
    }
    if (ifpottarg == 1 || iffldtarg == 1) {
#pragma omp parallel for schedule(dynamic, 16)
        for (long j = 0; j < ntarget; j++) {
            cplx p, f[3];
            direct_one(nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec,
                       target + 3 * j, -1, iffldtarg, &p, f);
            if (ifpottarg == 1) pottarg[j] = p;
            if (iffldtarg == 1) { fldtarg[3 * j] = f[0]; fldtarg[3 * j + 1] = f[1]; fldtarg[3 * j + 2] = f[2]; }
        }
    }
}

/* Direct sum at selected evaluation points, the sampled form of
 * l3dpartdirecttime (src/lfmm3dpart.f:1529-1661).  `skip[k]` is the source
 * index excluded at evaluation point k (-1 for none).                      */
void oracle_l3ddirect_points(int nsource, const double *source, int ifcharge, const cplx *charge,
                             int ifdipole, const cplx *dipstr, const double *dipvec,
                             int npts, const double *pts, const long *skip,
                             cplx *pot, cplx *fld)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < npts; k++) {
        cplx p, f[3];
        direct_one(nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec,
                   pts + 3 * k, skip ? skip[k] : -1, 1, &p, f);
        pot[k] = p;
        fld[3 * k] = f[0]; fld[3 * k + 1] = f[1]; fld[3 * k + 2] = f[2];
    }
}

/* ------------------------------------------------------------------ */
/* Octree, src/d3tstrcr.f.  Box fields follow the 20-int record documented
 * at src/d3tstrcr.f:1286-1313; ids are 0-based, absent children are -1.  */
enum { B_LEV = 0, B_I = 1, B_J = 2, B_K = 3, B_PAR = 4, B_KID = 5, B_SRC0 = 13, B_NSRC = 14,
       B_TRG0 = 15, B_NTRG = 16, B_STYPE = 17, B_TTYPE = 18 };

typedef struct {
    int nboxes, nlev, cap;
    int *box;          /* 20 per box */
    double *center;    /* 3 per box  */
    double center0[3], size;
    int *iz, *iztarg;  /* sorted position -> original index */
    int laddr[2 * 202];/* per level: first box, count */
    /* lists 1..5 in CSR (index 0 unused) */
    int *lstart[6], *lidx[6];
    int ier;
} otree;

/* d3tcentf, src/d3tstrcr.f:1671-1700 (center of box (i,j,k) on a level). */
static void d3tcentf(const double *c0, double size, int level, int i, int j, int k, double *c)
{
    double side = size / (double)(1L << level);
    double side2 = side / 2;
    double x0 = c0[0] - size / 2, y0 = c0[1] - size / 2, z0 = c0[2] - size / 2;
    c[0] = x0 + (i - 1) * side + side2;
    c[1] = y0 + (j - 1) * side + side2;
    c[2] = z0 + (k - 1) * side + side2;
}

/* Stable 8-way split of a point range, equivalent to the three stable
 * passes of d3tsepa1/d3tsepa0 (src/d3tstrcr.f:1705-1890): a point goes to
 * the upper half of an axis iff its coordinate is strictly greater than the
 * center.  Child order is z-major then y then x (src/d3tstrcr.f:1250-1251). */
static void sepa8(const double *c, const double *z, int *iz, int n, int *work, int is[8], int ns[8])
{
    int cnt[8] = {0};
    for (int i = 0; i < n; i++) {
        const double *p = z + 3 * (long)iz[i];
        int d = (p[2] > c[2]) * 4 + (p[1] > c[1]) * 2 + (p[0] > c[0]);
        cnt[d]++;
    }
    int off[8], s = 0;
    for (int d = 0; d < 8; d++) { off[d] = s; is[d] = s; ns[d] = cnt[d]; s += cnt[d]; }
    for (int i = 0; i < n; i++) {
        const double *p = z + 3 * (long)iz[i];
        int d = (p[2] > c[2]) * 4 + (p[1] > c[1]) * 2 + (p[0] > c[0]);
        work[off[d]++] = iz[i];
    }
    memcpy(iz, work, sizeof(int) * n);
}

static void tree_grow(otree *t, int need)
{
    if (need <= t->cap) return;
    int nc = t->cap * 2;
    if (nc < need) nc = need;
    t->box = realloc(t->box, sizeof(int) * 20 * (size_t)nc);
    t->cap = nc;
}

/* d3tallbem (src/d3tstrcr.f:1242-1583): a box splits unless it holds at most
 * nbox sources and nbox targets and lies at minlevel or below (:1490-1491);
 * only a box over nbox is marked subdivided (:1495-1498); levels stop at
 * min(198, maxlevel) (:1450-1451); empty children are kept when ifempty = 1
 * (:1529-1530).  d3tstrcr uses ifempty=0, minlevel=0, maxlevel=100
 * (src/d3tstrcr.f:181-182).                                               */
static void build_boxes_em(otree *t, const double *z, int n, const double *zt, int nt, int nbox, int ifempty,
                           int minlevel, int maxlevel)
{
    double xmin = z[0], xmax = z[0], ymin = z[1], ymax = z[1], zmin = z[2], zmax = z[2];
    for (int i = 0; i < n; i++) {
        const double *p = z + 3 * (long)i;
        if (p[0] < xmin) xmin = p[0];
        if (p[0] > xmax) xmax = p[0];
        if (p[1] < ymin) ymin = p[1];
        if (p[1] > ymax) ymax = p[1];
        if (p[2] < zmin) zmin = p[2];
        if (p[2] > zmax) zmax = p[2];
    }
    for (int i = 0; i < nt; i++) {
        const double *p = zt + 3 * (long)i;
        if (p[0] < xmin) xmin = p[0];
        if (p[0] > xmax) xmax = p[0];
        if (p[1] < ymin) ymin = p[1];
        if (p[1] > ymax) ymax = p[1];
        if (p[2] < zmin) zmin = p[2];
        if (p[2] > zmax) zmax = p[2];
    }
    double size = xmax - xmin, sy = ymax - ymin, sz = zmax - zmin;
    if (sy > size) size = sy;
    if (sz > size) size = sz;
    t->size = size;
    t->center0[0] = (xmin + xmax) / 2;
    t->center0[1] = (ymin + ymax) / 2;
    t->center0[2] = (zmin + zmax) / 2;

    t->cap = 1024;
    t->box = malloc(sizeof(int) * 20 * (size_t)t->cap);
    int *b = t->box;
    memset(b, 0, sizeof(int) * 20);
    b[B_LEV] = 0; b[B_I] = b[B_J] = b[B_K] = 1; b[B_PAR] = -1;
    for (int c = 0; c < 8; c++) b[B_KID + c] = -1;
    b[B_SRC0] = 0; b[B_NSRC] = n; b[B_TRG0] = 0; b[B_NTRG] = nt;
    b[B_STYPE] = n > 0; b[B_TTYPE] = nt > 0;
    t->iz = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    t->iztarg = malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
    for (int i = 0; i < n; i++) t->iz[i] = i;
    for (int i = 0; i < nt; i++) t->iztarg[i] = i;
    int *work = malloc(sizeof(int) * (size_t)((n > nt ? n : nt) + 1));
    t->laddr[0] = 0; t->laddr[1] = 1;
    int nboxes = 1, nlev = 0;
    int maxlev = maxlevel < 198 ? maxlevel : 198;
    for (int level = 0; level < maxlev; level++) {
        int d0 = t->laddr[2 * level], d1 = d0 + t->laddr[2 * level + 1];
        t->laddr[2 * (level + 1)] = nboxes;
        int nson = 0;
        for (int dad = d0; dad < d1; dad++) {
            int *bd = t->box + 20 * (size_t)dad;
            int np = bd[B_NSRC], ntp = bd[B_NTRG];
            if (np <= nbox && ntp <= nbox && level >= minlevel) continue;
            if (np > nbox || ntp > nbox) {
                if (bd[B_STYPE] == 1) bd[B_STYPE] = 2;
                if (bd[B_TTYPE] == 1) bd[B_TTYPE] = 2;
            }
            double c[3];
            d3tcentf(t->center0, t->size, level, bd[B_I], bd[B_J], bd[B_K], c);
            int is[8], ns[8], ist[8], nst[8];
            int s0 = bd[B_SRC0], t0 = bd[B_TRG0];
            sepa8(c, z, t->iz + s0, np, work, is, ns);
            sepa8(c, zt, t->iztarg + t0, ntp, work, ist, nst);
            int ii = bd[B_I], jj = bd[B_J], kk = bd[B_K];
            int slot = 0;
            for (int d = 0; d < 8; d++) {
                if (ns[d] == 0 && nst[d] == 0 && ifempty != 1) continue;
                tree_grow(t, nboxes + 1);
                bd = t->box + 20 * (size_t)dad;
                int *bs = t->box + 20 * (size_t)nboxes;
                memset(bs, 0, sizeof(int) * 20);
                bs[B_LEV] = level + 1;
                bs[B_I] = (ii - 1) * 2 + 1 + (d & 1);
                bs[B_J] = (jj - 1) * 2 + 1 + ((d >> 1) & 1);
                bs[B_K] = (kk - 1) * 2 + 1 + ((d >> 2) & 1);
                bs[B_PAR] = dad;
                for (int cc = 0; cc < 8; cc++) bs[B_KID + cc] = -1;
                bs[B_SRC0] = s0 + is[d]; bs[B_NSRC] = ns[d];
                bs[B_TRG0] = t0 + ist[d]; bs[B_NTRG] = nst[d];
                bs[B_STYPE] = ns[d] > 0; bs[B_TTYPE] = nst[d] > 0;
                bd[B_KID + slot++] = nboxes;
                nboxes++; nson++;
                nlev = level + 1;
            }
        }
        t->laddr[2 * (level + 1) + 1] = nson;
        if (nson == 0) break;
    }
    free(work);
    t->nboxes = nboxes;
    t->nlev = nlev;
    /* d3tcentc, src/d3tstrcr.f:1589-1669 */
    t->center = malloc(sizeof(double) * 3 * (size_t)nboxes);
    for (int i = 0; i < nboxes; i++) {
        int *bi = t->box + 20 * (size_t)i;
        double x00 = t->center0[0] - t->size / 2, y00 = t->center0[1] - t->size / 2,
               z00 = t->center0[2] - t->size / 2;
        double side = t->size / (double)(1L << bi[B_LEV]), side2 = side / 2;
        t->center[3 * i] = x00 + (bi[B_I] - 1) * side + side2;
        t->center[3 * i + 1] = y00 + (bi[B_J] - 1) * side + side2;
        t->center[3 * i + 2] = z00 + (bi[B_K] - 1) * side + side2;
    }
}

static void build_boxes(otree *t, const double *z, int n, const double *zt, int nt, int nbox)
{
    build_boxes_em(t, z, n, zt, nt, nbox, 0, 0, 100);
}

/* d3tifint (src/d3tstrcr.f:1075-1172): do two boxes intersect or touch,
 * with the reference's slack eps = (smallest side)/10000.                */
static int d3tifint(const otree *t, int b1, int b2)
{
    double s1 = t->size / (double)(1L << t->box[20 * (size_t)b1 + B_LEV]);
    double s2 = t->size / (double)(1L << t->box[20 * (size_t)b2 + B_LEV]);
    const double *c1 = t->center + 3 * (size_t)b1, *c2 = t->center + 3 * (size_t)b2;
    double mn1[3], mx1[3], mn2[3], mx2[3];
    for (int d = 0; d < 3; d++) {
        mn1[d] = c1[d] - s1 / 2; mx1[d] = mn1[d] + s1;
        mn2[d] = c2[d] - s2 / 2; mx2[d] = mn2[d] + s2;
    }
    double eps = mx1[0] - mn1[0];
    if (eps > mx2[0] - mn2[0]) eps = mx2[0] - mn2[0];
    if (eps > mx2[1] - mn2[1]) eps = mx2[1] - mn2[1];
    if (eps > mx2[2] - mn2[2]) eps = mx2[2] - mn2[2];
    if (eps > mx1[1] - mn1[1]) eps = mx1[1] - mn1[1];
    if (eps > mx1[2] - mn1[2]) eps = mx1[2] - mn1[2];
    eps = eps / 10000;
    for (int d = 0; d < 3; d++) {
        if (mn1[d] > mx2[d] + eps) return 0;
        if (mn2[d] > mx1[d] + eps) return 0;
    }
    return 1;
}

typedef struct { int *a; int n, cap; } ivec;
static void ivpush(ivec *v, int x)
{
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 8; v->a = realloc(v->a, sizeof(int) * v->cap); }
    v->a[v->n++] = x;
}

static int nkids(const otree *t, int b)
{
    int c = 0;
    for (int k = 0; k < 8; k++) c += t->box[20 * (size_t)b + B_KID + k] >= 0;
    return c;
}

/* d3tlst31 (src/d3tstrcr.f:912-1069): lists 1 and 3 of leaf ibox from the
 * subtree of its colleague jbox0.                                          */
static void lst31(const otree *t, int ibox, int jbox0, ivec *L)
{
    int stack[256], top = 0;
    stack[top++] = jbox0;
    while (top) {
        int j = stack[--top];
        if (!d3tifint(t, ibox, j)) {
            ivpush(&L[(size_t)6 * ibox + 3], j);
            continue;
        }
        if (nkids(t, j) == 0) {
            ivpush(&L[(size_t)6 * ibox + 1], j);
            if (t->box[20 * (size_t)j + B_LEV] != t->box[20 * (size_t)ibox + B_LEV])
                ivpush(&L[(size_t)6 * j + 1], ibox);
            continue;
        }
        for (int k = 7; k >= 0; k--) {
            int c = t->box[20 * (size_t)j + B_KID + k];
            if (c >= 0) stack[top++] = c;
        }
    }
}

/* d3tlsts (src/d3tstrcr.f:695-906): lists 5 and 2 for every non-root box,
 * lists 1 and 3 for every non-root leaf, list 4 as the dual of list 3.    */
static void build_lists(otree *t)
{
    int nb = t->nboxes;
    ivec *L = calloc((size_t)6 * nb, sizeof(ivec));
    L[0].a = NULL;
    for (int ib = 1; ib < nb; ib++) {
        int dad = t->box[20 * (size_t)ib + B_PAR];
        int ncoll = 1 + L[(size_t)6 * dad + 5].n;
        for (int ci = 0; ci < ncoll; ci++) {
            int coll = ci == 0 ? dad : L[(size_t)6 * dad + 5].a[ci - 1];
            for (int k = 0; k < 8; k++) {
                int kid = t->box[20 * (size_t)coll + B_KID + k];
                if (kid < 0) break;
                if (kid == ib) continue;
                if (d3tifint(t, kid, ib)) ivpush(&L[(size_t)6 * ib + 5], kid);
                else ivpush(&L[(size_t)6 * ib + 2], kid);
            }
        }
    }
    for (int i = 0; i < nb; i++) {
        if (t->box[20 * (size_t)i + B_KID] >= 0) continue;
        if (t->box[20 * (size_t)i + B_LEV] == 0) continue;
        int n5 = L[(size_t)6 * i + 5].n;
        for (int j = 0; j < n5; j++) lst31(t, i, L[(size_t)6 * i + 5].a[j], L);
    }
    for (int ib = 0; ib < nb; ib++) {
        ivec *l3 = &L[(size_t)6 * ib + 3];
        for (int j = 0; j < l3->n; j++) ivpush(&L[(size_t)6 * l3->a[j] + 4], ib);
    }
    for (int ty = 1; ty <= 5; ty++) {
        t->lstart[ty] = malloc(sizeof(int) * ((size_t)nb + 1));
        long tot = 0;
        for (int ib = 0; ib < nb; ib++) { t->lstart[ty][ib] = (int)tot; tot += L[(size_t)6 * ib + ty].n; }
        t->lstart[ty][nb] = (int)tot;
        t->lidx[ty] = malloc(sizeof(int) * (size_t)(tot > 0 ? tot : 1));
        for (int ib = 0; ib < nb; ib++)
            if (L[(size_t)6 * ib + ty].n)
                memcpy(t->lidx[ty] + t->lstart[ty][ib], L[(size_t)6 * ib + ty].a,
                       sizeof(int) * L[(size_t)6 * ib + ty].n);
    }
    for (size_t i = 0; i < (size_t)6 * nb; i++) free(L[i].a);
    free(L);
}

static void tree_free(otree *t)
{
    free(t->box); free(t->center); free(t->iz); free(t->iztarg);
    for (int ty = 1; ty <= 5; ty++) { free(t->lstart[ty]); free(t->lidx[ty]); }
}

/* Tree export for the parity tests: boxes (20 ints each), centers, the two
 * permutations and the five lists.  Returns an opaque handle.             */
void *oracle_tree_build(int n, const double *z, int nt, const double *zt, int nbox)
{
    otree *t = calloc(1, sizeof(otree));
    build_boxes(t, z, n, zt, nt, nbox);
    build_lists(t);
    return t;
}

/* d3tstrcrem (src/d3tstrcr.f:264-460): the same tree with its refinement options. */
void *oracle_tree_build_em(int n, const double *z, int nt, const double *zt, int nbox, int ifempty, int minlevel,
                           int maxlevel)
{
    otree *t = calloc(1, sizeof(otree));
    build_boxes_em(t, z, n, zt, nt, nbox, ifempty, minlevel, maxlevel);
    build_lists(t);
    return t;
}
int oracle_tree_nboxes(void *h) { return ((otree *)h)->nboxes; }
int oracle_tree_nlev(void *h) { return ((otree *)h)->nlev; }
void oracle_tree_geometry(void *h, double *center0_size)
{
    otree *t = h;
    center0_size[0] = t->center0[0]; center0_size[1] = t->center0[1];
    center0_size[2] = t->center0[2]; center0_size[3] = t->size;
}
void oracle_tree_boxes(void *h, int *box20, double *centers, int *iz, int *iztarg, int n, int nt)
{
    otree *t = h;
    memcpy(box20, t->box, sizeof(int) * 20 * (size_t)t->nboxes);
    memcpy(centers, t->center, sizeof(double) * 3 * (size_t)t->nboxes);
    memcpy(iz, t->iz, sizeof(int) * (size_t)n);
    if (nt > 0) memcpy(iztarg, t->iztarg, sizeof(int) * (size_t)nt);
}
int oracle_tree_list_len(void *h, int ty) { otree *t = h; return t->lstart[ty][t->nboxes]; }
void oracle_tree_list(void *h, int ty, int *start, int *idx)
{
    otree *t = h;
    memcpy(start, t->lstart[ty], sizeof(int) * ((size_t)t->nboxes + 1));
    memcpy(idx, t->lidx[ty], sizeof(int) * (size_t)t->lstart[ty][t->nboxes]);
}
void oracle_tree_free(void *h) { tree_free(h); free(h); }

/* ------------------------------------------------------------------ */
/* Expansion orders, src/l3dterms.f.                                    */
int oracle_l3dterms(double eps)                     /* l3dterms :34-77 */
{
    double z1 = 1.5, z2 = sqrt(3.0) / 2.0;
    double jfun = z2, hfun = 1.0 / (z1 * z1);
    for (int j = 2; j <= 1000; j++) {
        hfun = hfun / z1;
        jfun = jfun * z2;
        if (jfun * hfun < eps) return j;
    }
    return 1;
}

void oracle_l3dterms_list2(double eps, int *itable /* 7*7*7, [i+3][j+3][k+3] */)
{                                               /* l3dterms_list2 :136-248 */
    int tab[2][4][4];
    for (int ii = 2; ii <= 3; ii++)
        for (int jj = 0; jj <= 3; jj++)
            for (int kk = 0; kk <= 3; kk++) {
                double dx = ii, dy = jj, dz = kk;
                if (dx > 0) dx -= .5;
                if (dy > 0) dy -= .5;
                if (dz > 0) dz -= .5;
                double rr = sqrt(dx * dx + dy * dy + dz * dz);
                double z1 = rr, z2 = sqrt(3.0) / 2.0, jfun = z2, hfun = 1.0 / (z1 * z1);
                int nterms = 1;
                for (int j = 2; j <= 1000; j++) {
                    hfun = hfun / z1;
                    jfun = jfun * z2;
                    if (jfun * hfun < eps) { nterms = j; break; }
                }
                tab[ii - 2][jj][kk] = nterms;
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

/* iprec tables of lfmm3dparttarg, src/lfmm3dpart.f:277-300. */
double oracle_lap_eps(int iprec)
{
    static const double e[] = {.5e0, .5e-1, .5e-2, .5e-3, .5e-6, .5e-9, .5e-12, .5e-15, 0.0};
    if (iprec < -2 || iprec > 6) return -1;
    return e[iprec + 2];
}
int oracle_lap_nbox(int iprec, int ns, int nt)
{
    static const int nb[] = {40, 50, 80, 160, 400, 800, 1200, 1400};
    if (iprec == 6) return ns + nt;
    if (iprec < -2 || iprec > 6) return -1;
    return nb[iprec + 2];
}

/* ------------------------------------------------------------------ */
/* Normalized Legendre functions Y_n^m = sqrt((n-m)!/(n+m)!) P_n^m:
 * ylgndru (src/yrecursion.f:386-430) and the scaled pair with derivatives
 * ylgndru2s (src/yrecursion.f:495-580).  Layout y[n*(nmax+1)+m].          */
static void ylgndru(int nmax, double x, double *y)
{
    int ld = nmax + 1;
    double u = -sqrt((1 - x) * (1 + x));
    y[0] = 1;
    for (int m = 0; m <= nmax; m++) {
        if (m > 0) y[m * ld + m] = y[(m - 1) * ld + m - 1] * u * sqrt((2 * m - 1.0) / (2 * m));
        if (m < nmax) y[(m + 1) * ld + m] = x * y[m * ld + m] * sqrt(2 * m + 1.0);
        for (int n = m + 2; n <= nmax; n++)
            y[n * ld + m] = ((2 * n - 1) * x * y[(n - 1) * ld + m] -
                             sqrt((n + m - 1.0) * (n - m - 1.0)) * y[(n - 2) * ld + m]) /
                            sqrt((n - m + 0.0) * (n + m));
    }
}

static void ylgndru2s(int nmax, double x, double *y, double *d)
{
    int ld = nmax + 1;
    double u = -sqrt((1 - x) * (1 + x)), u2 = (1 - x) * (1 + x);
    y[0] = 1; d[0] = 0;
    int m = 0;
    if (m < nmax) { y[ld] = x * y[0] * sqrt(1.0); d[ld] = (x * d[0] + y[0]) * sqrt(1.0); }
    for (int n = 2; n <= nmax; n++) {
        double a = sqrt((n + m - 1.0) * (n - m - 1.0)), b = sqrt((n - m + 0.0) * (n + m));
        y[n * ld] = ((2 * n - 1) * x * y[(n - 1) * ld] - a * y[(n - 2) * ld]) / b;
        d[n * ld] = ((2 * n - 1) * (x * d[(n - 1) * ld] + y[(n - 1) * ld]) - a * d[(n - 2) * ld]) / b;
    }
    for (m = 1; m <= nmax; m++) {
        if (m == 1) y[m * ld + m] = y[(m - 1) * ld + m - 1] * (-1) * sqrt((2 * m - 1.0) / (2 * m));
        if (m > 1) y[m * ld + m] = y[(m - 1) * ld + m - 1] * u * sqrt((2 * m - 1.0) / (2 * m));
        d[m * ld + m] = y[m * ld + m] * (-m) * x;
        if (m < nmax) {
            y[(m + 1) * ld + m] = x * y[m * ld + m] * sqrt(2 * m + 1.0);
            d[(m + 1) * ld + m] = (x * d[m * ld + m] + u2 * y[m * ld + m]) * sqrt(2 * m + 1.0);
        }
        for (int n = m + 2; n <= nmax; n++) {
            double a = sqrt((n + m - 1.0) * (n - m - 1.0)), b = sqrt((n - m + 0.0) * (n + m));
            y[n * ld + m] = ((2 * n - 1) * x * y[(n - 1) * ld + m] - a * y[(n - 2) * ld + m]) / b;
            d[n * ld + m] = ((2 * n - 1) * (x * d[(n - 1) * ld + m] + u2 * y[(n - 1) * ld + m]) -
                             a * d[(n - 2) * ld + m]) / b;
        }
    }
}

/* cart2polarl, src/laprouts3d.f:1416-1451 */
static void cart2polarl(const double *z, double *r, double *theta, double *phi)
{
    *r = sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
    double proj = sqrt(z[0] * z[0] + z[1] * z[1]);
    *theta = atan2(proj, z[2]);
    if (fabs(z[0]) == 0 && fabs(z[1]) == 0) *phi = 0;
    else *phi = atan2(z[1], z[0]);
}

#define EI(n, m) ((n) * (n) + (n) + (m)) /* compact index of coefficient (n,m) */

/* P2M for one charge: l3dformmp_trunc0, src/laprouts3d.f:3348-3450 (rscale=1). */
static void formmp_charge(const double *s, cplx q, const double *c, int p, cplx *mp, double *pp)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th);
    cplx e1 = cos(ph) + I * sin(ph);
    ylgndru(p, ct, pp);
    double fr = 1.0;
    cplx em = 1.0;
    mp[EI(0, 0)] += q;
    for (int n = 1; n <= p; n++) {
        fr *= r;
        cplx frq = fr * q;
        mp[EI(n, 0)] += pp[n * (p + 1)] * frq;
        em = 1.0;
        for (int m = 1; m <= n; m++) {
            em *= e1;
            cplx z = pp[n * (p + 1) + m] * frq;
            mp[EI(n, m)] += z * conj(em);
            mp[EI(n, -m)] += z * em;
        }
    }
}

/* P2M for one dipole: l3dformmp0_dp_trunc, src/laprouts3d.f:3970-4130. */
static void formmp_dipole(const double *s, cplx ds, const double *v, const double *c, int p,
                          cplx *mp, double *pp, double *ppd)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    cplx e1 = cp + I * sp;
    double fr[200], frder[200];
    fr[0] = 1.0;
    for (int i = 1; i <= p + 1; i++) fr[i] = fr[i - 1] * r;
    frder[0] = 0;
    for (int i = 1; i <= p + 1; i++) frder[i] = i * fr[i - 1];
    double rx = st * cp, thx = ct * cp, phx = -sp;
    double ry = st * sp, thy = ct * sp, phy = cp;
    double rz = ct, thz = -st, phz = 0.0;
    ylgndru2s(p, ct, pp, ppd);
    int ld = p + 1;
    double rf1 = v[0] * rx + v[1] * ry + v[2] * rz;
    double rf2 = v[0] * thx + v[1] * thy + v[2] * thz;
    double rf3 = v[0] * phx + v[1] * phy + v[2] * phz;
    mp[EI(0, 0)] += (rf1 * pp[0] * frder[0]) * ds;
    cplx em = 1.0;
    for (int n = 1; n <= p; n++) {
        double fu = fr[n - 1];
        cplx ur = pp[n * ld] * frder[n];
        cplx ut = -fu * ppd[n * ld] * st;
        mp[EI(n, 0)] += (rf1 * ur + rf2 * ut) * ds;
        em = 1.0;
        for (int m = 1; m <= n; m++) {
            em *= e1;
            cplx urm = frder[n] * pp[n * ld + m] * st;
            cplx utm = -fu * ppd[n * ld + m];
            cplx upm = -I * (double)m * fu * pp[n * ld + m];
            cplx zz = (rf1 * urm + rf2 * utm + rf3 * upm) * conj(em);
            mp[EI(n, m)] += zz * ds;
            mp[EI(n, -m)] += conj(zz) * ds;
        }
    }
}

/* P2L for one charge: l3dformta_trunc0, src/laprouts3d.f:3689-3764. */
static void formta_charge(const double *s, cplx q, const double *c, int p, cplx *lo, double *pp)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th);
    cplx e1 = cos(ph) + I * sin(ph);
    ylgndru(p, ct, pp);
    double d = 1.0 / r, fr = d;
    lo[EI(0, 0)] += fr * q;
    for (int n = 1; n <= p; n++) {
        fr *= d;
        cplx frq = fr * q;
        lo[EI(n, 0)] += pp[n * (p + 1)] * frq;
        cplx em = 1.0;
        for (int m = 1; m <= n; m++) {
            em *= e1;
            cplx z = pp[n * (p + 1) + m] * frq;
            lo[EI(n, m)] += z * conj(em);
            lo[EI(n, -m)] += z * em;
        }
    }
}

/* P2L for one dipole: l3dformta0_dp_trunc, src/laprouts3d.f:4355-4500. */
static void formta_dipole(const double *s, cplx ds, const double *v, const double *c, int p,
                          cplx *lo, double *pp, double *ppd)
{
    double zd[3] = {s[0] - c[0], s[1] - c[1], s[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    cplx e1 = cp + I * sp;
    double fr[202], frder[202];
    double d = 1.0 / r;
    fr[0] = d;
    for (int i = 1; i <= p + 1; i++) fr[i] = fr[i - 1] * d;
    for (int i = 0; i <= p; i++) frder[i] = -(i + 1.0) * fr[i + 1];
    double rx = st * cp, thx = ct * cp / r, phx = -sp / r;
    double ry = st * sp, thy = ct * sp / r, phy = cp / r;
    double rz = ct, thz = -st / r, phz = 0.0;
    ylgndru2s(p, ct, pp, ppd);
    int ld = p + 1;
    double rf1 = v[0] * rx + v[1] * ry + v[2] * rz;
    double rf2 = v[0] * thx + v[1] * thy + v[2] * thz;
    double rf3 = v[0] * phx + v[1] * phy + v[2] * phz;
    lo[EI(0, 0)] += (rf1 * pp[0] * frder[0]) * ds;
    for (int n = 1; n <= p; n++) {
        cplx ur = pp[n * ld] * frder[n];
        cplx ut = -fr[n] * ppd[n * ld] * st;
        lo[EI(n, 0)] += (rf1 * ur + rf2 * ut) * ds;
        cplx em = 1.0;
        for (int m = 1; m <= n; m++) {
            em *= e1;
            cplx urm = frder[n] * pp[n * ld + m] * st;
            cplx utm = -fr[n] * ppd[n * ld + m];
            cplx upm = -I * (double)m * fr[n] * pp[n * ld + m];
            cplx zz = (rf1 * urm + rf2 * utm + rf3 * upm) * conj(em);
            lo[EI(n, m)] += zz * ds;
            lo[EI(n, -m)] += conj(zz) * ds;
        }
    }
}

/* M2P with field: l3dmpeval_trunc0, src/laprouts3d.f:2606-2765. */
static void mpeval(const double *c, const cplx *mp, int p, const double *t, cplx *pot, cplx fld[3],
                   double *pp, double *ppd)
{
    double zd[3] = {t[0] - c[0], t[1] - c[1], t[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    cplx e1 = cp + I * sp;
    double fr[202], frder[202], d = 1.0 / r;
    fr[0] = d;
    for (int i = 1; i <= p + 1; i++) fr[i] = fr[i - 1] * d;
    for (int i = 0; i <= p; i++) frder[i] = -(i + 1.0) * fr[i + 1];
    double rx = st * cp, thx = ct * cp / r, phx = -sp / r;
    double ry = st * sp, thy = ct * sp / r, phy = cp / r;
    double rz = ct, thz = -st / r;
    ylgndru2s(p, ct, pp, ppd);
    int ld = p + 1;
    cplx ur = mp[EI(0, 0)] * frder[0], ut = 0, up = 0;
    cplx pt = mp[EI(0, 0)] * fr[0];
    for (int n = 1; n <= p; n++) {
        pt += mp[EI(n, 0)] * fr[n] * pp[n * ld];
        ur += frder[n] * pp[n * ld] * mp[EI(n, 0)];
        ut -= mp[EI(n, 0)] * fr[n] * ppd[n * ld] * st;
        cplx em = 1.0;
        for (int m = 1; m <= n; m++) {
            em *= e1;
            double z1 = fr[n] * pp[n * ld + m] * st;
            cplx z2 = mp[EI(n, m)] * em, z3 = mp[EI(n, -m)] * conj(em), zs = z2 + z3;
            pt += z1 * zs;
            ur += frder[n] * pp[n * ld + m] * st * zs;
            ut -= zs * fr[n] * ppd[n * ld + m];
            up += fr[n] * pp[n * ld + m] * (I * (double)m * (z2 - z3));
        }
    }
    *pot = pt;
    fld[0] = -(ur * rx + ut * thx + up * phx);
    fld[1] = -(ur * ry + ut * thy + up * phy);
    fld[2] = -(ur * rz + ut * thz);
}

/* L2P with field: l3dtaeval_trunc0, src/laprouts3d.f:2941-3111. */
static void taeval(const double *c, const cplx *lo, int p, const double *t, cplx *pot, cplx fld[3],
                   double *pp, double *ppd)
{
    double zd[3] = {t[0] - c[0], t[1] - c[1], t[2] - c[2]}, r, th, ph;
    cart2polarl(zd, &r, &th, &ph);
    double ct = cos(th), st = sqrt(1.0 - ct * ct), cp = cos(ph), sp = sin(ph);
    cplx e1 = cp + I * sp;
    double fr[202], frder[202];
    fr[0] = 1.0;
    for (int i = 1; i <= p + 1; i++) fr[i] = fr[i - 1] * r;
    frder[0] = 0;
    for (int i = 1; i <= p + 1; i++) frder[i] = i * fr[i - 1];
    double rx = st * cp, thx = ct * cp, phx = -sp;
    double ry = st * sp, thy = ct * sp, phy = cp;
    double rz = ct, thz = -st;
    ylgndru2s(p, ct, pp, ppd);
    int ld = p + 1;
    cplx pt = lo[EI(0, 0)], ur = 0, ut = 0, up = 0;
    for (int n = 1; n <= p; n++) {
        pt += lo[EI(n, 0)] * fr[n] * pp[n * ld];
        ur += frder[n] * pp[n * ld] * lo[EI(n, 0)];
        double fu = fr[n - 1];
        ut -= lo[EI(n, 0)] * fu * ppd[n * ld] * st;
        cplx em = 1.0;
        for (int m = 1; m <= n; m++) {
            em *= e1;
            double z1 = fr[n] * pp[n * ld + m] * st;
            cplx z2 = lo[EI(n, m)] * em, z3 = lo[EI(n, -m)] * conj(em), zs = z2 + z3;
            pt += z1 * zs;
            ur += frder[n] * pp[n * ld + m] * st * zs;
            ut -= zs * fu * ppd[n * ld + m];
            up += fu * pp[n * ld + m] * (I * (double)m * (z2 - z3));
        }
    }
    *pot = pt;
    fld[0] = -(ur * rx + ut * thx + up * phx);
    fld[1] = -(ur * ry + ut * thy + up * phy);
    fld[2] = -(ur * rz + ut * thz);
}

/* ------------------------------------------------------------------ */
/* Rotation about the y axis: rotviarecur3p_init (src/rotviarecur3.f:717-869)
 * builds rotmat(mp, ij, m) for 0<=mp<=ij, -ij<=m<=ij; stored here as
 * rot[(ij*(ldc+1)+mp)*(2*ldc+1) + m+ldc].                                  */
static void rot_init(double *rot, int ldc, double theta)
{
    const double precis = 1.0e-20, ww = 1 / sqrt(2.0);
    int w2 = 2 * ldc + 1;
#define RD1(mp, m) rd1[(mp) * w2 + (m) + ldc]
#define RD2(mp, m) rd2[(mp) * w2 + (m) + ldc]
#define ROT(mp, ij, m) rot[((size_t)(ij) * (ldc + 1) + (mp)) * w2 + (m) + ldc]
    double *rd1 = calloc((size_t)(ldc + 1) * w2, sizeof(double));
    double *rd2 = calloc((size_t)(ldc + 1) * w2, sizeof(double));
    double *sqc1 = malloc(sizeof(double) * (2 * ldc + 1));
    double *sqc2 = malloc(sizeof(double) * (2 * ldc + 1));
    for (int m = 0; m <= 2 * ldc; m++) sqc1[m] = sqrt(m + 0.0);
    sqc2[0] = 0.0;
    if (ldc > 0) sqc2[1] = 0.0;
    for (int m = 2; m <= 2 * ldc; m++) sqc2[m] = sqrt((m + 0.0) * (m - 1) / 2.0);
    double ct = cos(theta);
    if (fabs(ct) <= precis) ct = 0.0;
    double st = sin(-theta);
    if (fabs(st) <= precis) st = 0.0;
    double hst = ww * st;
    double ctp = 2.0 * ww * pow(cos(theta / 2.0), 2), ctn = -2.0 * ww * pow(sin(theta / 2.0), 2);
    RD1(0, 0) = 1.0;
    ROT(0, 0, 0) = 1.0;
    for (int ij = 1; ij <= ldc; ij++) {
        for (int im = -ij; im <= -1; im++) {
            RD2(0, im) = -sqc2[ij - im] * RD1(0, im + 1);
            if (im > 1 - ij) RD2(0, im) += sqc2[ij + im] * RD1(0, im - 1);
            RD2(0, im) *= hst;
            if (im > -ij) RD2(0, im) += RD1(0, im) * ct * sqc1[ij + im] * sqc1[ij - im];
            RD2(0, im) /= ij;
        }
        RD2(0, 0) = RD1(0, 0) * ct;
        if (ij > 1) RD2(0, 0) += hst * sqc2[ij] * (2 * RD1(0, -1)) / ij;
        for (int im = 1; im <= ij; im++) {
            RD2(0, im) = RD2(0, -im);
            RD2(im, 0) = (im % 2 == 0) ? RD2(0, im) : -RD2(0, im);
        }
        for (int imp = 1; imp <= ij; imp++) {
            double sc = ww / sqc2[ij + imp];
            for (int im = imp; im <= ij; im++) {
                RD2(imp, im) = RD1(imp - 1, im - 1) * (ctp * sqc2[ij + im]);
                RD2(imp, -im) = RD1(imp - 1, -im + 1) * (ctn * sqc2[ij + im]);
                if (im < ij - 1) {
                    RD2(imp, im) -= RD1(imp - 1, im + 1) * (ctn * sqc2[ij - im]);
                    RD2(imp, -im) -= RD1(imp - 1, -im - 1) * (ctp * sqc2[ij - im]);
                }
                if (im < ij) {
                    double d = st * sqc1[ij + im] * sqc1[ij - im];
                    RD2(imp, im) += RD1(imp - 1, im) * d;
                    RD2(imp, -im) += RD1(imp - 1, -im) * d;
                }
                RD2(imp, im) *= sc;
                RD2(imp, -im) *= sc;
                if (im > imp) {
                    double sg = ((imp + im) % 2 == 0) ? 1.0 : -1.0;
                    RD2(im, imp) = sg * RD2(imp, im);
                    RD2(im, -imp) = sg * RD2(imp, -im);
                }
            }
        }
        for (int m = -ij; m <= ij; m++)
            for (int mp = 0; mp <= ij; mp++) {
                RD1(mp, m) = RD2(mp, m);
                ROT(mp, ij, m) = RD2(mp, m);
            }
    }
    free(rd1); free(rd2); free(sqc1); free(sqc2);
}

/* rotviarecur3p_apply, src/rotviarecur3.f:873-950 (degrees 0..nt). */
static void rot_apply(const double *rot, int ldc, int nt, const cplx *a, cplx *b)
{
    int w2 = 2 * ldc + 1;
    for (int ij = 0; ij <= nt; ij++)
        for (int m = -ij; m <= ij; m++) {
            cplx s = a[EI(ij, 0)] * ROT(0, ij, m);
            for (int mp = 1; mp <= ij; mp++)
                s += a[EI(ij, mp)] * ROT(mp, ij, m) + a[EI(ij, -mp)] * ROT(mp, ij, -m);
            b[EI(ij, m)] = s;
        }
}
#undef RD1
#undef RD2
#undef ROT

/* sqrt of binomial coefficients, the dc array of the z-shift routines. */
static double *make_dc(int nmax)
{
    int ld = 2 * nmax + 1;
    double *car = calloc((size_t)ld * ld, sizeof(double)), *dc = calloc((size_t)ld * ld, sizeof(double));
    for (int l = 0; l <= 2 * nmax; l++) { car[l * ld] = 1; dc[l * ld] = 1; }
    for (int m = 1; m <= 2 * nmax; m++) {
        car[m * ld + m] = 1; dc[m * ld + m] = 1;
        for (int l = m + 1; l <= 2 * nmax; l++) {
            car[l * ld + m] = car[(l - 1) * ld + m] + car[(l - 1) * ld + m - 1];
            dc[l * ld + m] = sqrt(car[l * ld + m]);
        }
    }
    free(car);
    return dc;
}

/* One translation "rotate, shift along z, rotate back" with the phase
 * factors of l3dmpmpquad0 (src/l3dtrans.f:223-345), l3dmplocquad2_trunc0
 * (src/l3dtrans.f:1260-1387) and l3dloclocquad0 (src/l3dtrans.f:1676-1792).
 * kind 0: M2M with l3dmpmpzshift (:351-431); 1: M2L with
 * l3dmploczshiftstab_fast (:1439-1534) truncated to nt; 2: L2L with
 * l3dlocloczshift (:1798-1880).  Adds the result into `out`.               */
static void translate(int kind, const double *c_from, const double *c_to, const cplx *in, int p,
                      int nt, cplx *out, const double *dc, int ldc_dc, const double *rotf,
                      const double *rotb)
{
    double rv[3] = {c_to[0] - c_from[0], c_to[1] - c_from[1], c_to[2] - c_from[2]}, d, th, ph;
    cart2polarl(rv, &d, &th, &ph);
    int K = (p + 1) * (p + 1);
    cplx *a = calloc(K, sizeof(cplx)), *b = calloc(K, sizeof(cplx)), *cz = calloc(K, sizeof(cplx));
    /* powers e^{i m phi} by repeated multiplication, as the reference's ephi
     * arrays (src/l3dtrans.f:1329-1340) */
    cplx ephi_store[2 * 202 + 3], *ephi = ephi_store + 202 + 1;
    ephi[0] = 1.0;
    ephi[1] = cexp(I * ph);
    ephi[-1] = conj(ephi[1]);
    for (int l = 1; l <= p; l++) {
        ephi[l + 1] = ephi[l] * ephi[1];
        ephi[-1 - l] = conj(ephi[l + 1]);
    }
    for (int l = 0; l <= nt; l++)
        for (int m = -l; m <= l; m++) a[EI(l, m)] = in[EI(l, m)] * ephi[m];
    double *rf = NULL, *rb = NULL;
    if (rotf) { rf = (double *)rotf; rb = (double *)rotb; }
    else {
        size_t sz = (size_t)(p + 1) * (p + 1) * (2 * p + 1);
        rf = malloc(sz * sizeof(double)); rb = malloc(sz * sizeof(double));
        rot_init(rf, p, th); rot_init(rb, p, -th);
    }
    int ldr = p;
    rot_apply(rf, ldr, nt, a, b);
#define DC(l, m) dc[(l) * (2 * ldc_dc + 1) + (m)]
    if (kind == 0) {
        double fr[202]; fr[0] = 1; for (int l = 1; l <= p + 1; l++) fr[l] = fr[l - 1] * d;
        for (int j = 0; j <= p; j++)
            for (int k = -j; k <= j; k++) {
                cplx s = 0;
                int l0 = j - p > 0 ? j - p : 0;
                for (int l = l0; l <= j - abs(k); l++)
                    s += b[EI(j - l, k)] * fr[l] * DC(j - k, l) * DC(j + k, l) * ((l % 2) ? -1.0 : 1.0);
                cz[EI(j, k)] = s;
            }
    } else if (kind == 1) {
        double fr[402]; fr[0] = 1.0 / d; for (int l = 1; l <= 2 * nt + 1; l++) fr[l] = fr[l - 1] / d;
        for (int j = 0; j <= nt; j++)
            for (int k = -j; k <= j; k++) {
                cplx s = 0;
                double sg = ((abs(j + k)) % 2 == 1) ? -1.0 : 1.0;
                for (int l = abs(k); l <= nt; l++) {
                    int ll = l + j;
                    s += sg * b[EI(l, k)] * (fr[ll] * DC(ll, l - k) * DC(ll, l + k));
                }
                cz[EI(j, k)] = s;
            }
    } else {
        double fr[202]; fr[0] = 1; for (int l = 1; l <= p + 1; l++) fr[l] = fr[l - 1] * d;
        for (int j = 0; j <= p; j++)
            for (int k = -j; k <= j; k++) {
                cplx s = b[EI(j, k)];
                for (int l = 1; l <= p - j; l++) {
                    int ll = l + j;
                    s += b[EI(ll, k)] * fr[l] * DC(ll + k, l) * DC(ll - k, l);
                }
                cz[EI(j, k)] = s;
            }
    }
#undef DC
    int nout = kind == 1 ? nt : p;
    rot_apply(rb, ldr, nout, cz, a);
    for (int l = 0; l <= nout; l++)
        for (int m = -l; m <= l; m++) out[EI(l, m)] += ephi[-m] * a[EI(l, m)];
    if (!rotf) { free(rf); free(rb); }
    free(a); free(b); free(cz);
}

/* Single-operator entry points for the per-operator parity tests. */
void oracle_formmp(int ns, const double *src, int ifcharge, const cplx *q, int ifdipole, const cplx *ds,
                   const double *dv, const double *c, int p, cplx *mp)
{
    double *pp = malloc(sizeof(double) * (p + 2) * (p + 2)), *ppd = malloc(sizeof(double) * (p + 2) * (p + 2));
    for (int i = 0; i < ns; i++) {
        if (ifcharge == 1) formmp_charge(src + 3 * i, q[i], c, p, mp, pp);
        if (ifdipole == 1) formmp_dipole(src + 3 * i, ds[i], dv + 3 * i, c, p, mp, pp, ppd);
    }
    free(pp); free(ppd);
}
void oracle_formta(int ns, const double *src, int ifcharge, const cplx *q, int ifdipole, const cplx *ds,
                   const double *dv, const double *c, int p, cplx *lo)
{
    double *pp = malloc(sizeof(double) * (p + 2) * (p + 2)), *ppd = malloc(sizeof(double) * (p + 2) * (p + 2));
    for (int i = 0; i < ns; i++) {
        if (ifcharge == 1) formta_charge(src + 3 * i, q[i], c, p, lo, pp);
        if (ifdipole == 1) formta_dipole(src + 3 * i, ds[i], dv + 3 * i, c, p, lo, pp, ppd);
    }
    free(pp); free(ppd);
}
void oracle_mpeval(const double *c, const cplx *mp, int p, int nt, const double *t, cplx *pot, cplx *fld)
{
    double *pp = malloc(sizeof(double) * (p + 2) * (p + 2)), *ppd = malloc(sizeof(double) * (p + 2) * (p + 2));
    for (int i = 0; i < nt; i++) mpeval(c, mp, p, t + 3 * i, pot + i, fld + 3 * i, pp, ppd);
    free(pp); free(ppd);
}
void oracle_taeval(const double *c, const cplx *lo, int p, int nt, const double *t, cplx *pot, cplx *fld)
{
    double *pp = malloc(sizeof(double) * (p + 2) * (p + 2)), *ppd = malloc(sizeof(double) * (p + 2) * (p + 2));
    for (int i = 0; i < nt; i++) taeval(c, lo, p, t + 3 * i, pot + i, fld + 3 * i, pp, ppd);
    free(pp); free(ppd);
}
void oracle_translate(int kind, const double *c_from, const double *c_to, const cplx *in, int p, int nt, cplx *out)
{
    double *dc = make_dc(2 * p + 2);
    translate(kind, c_from, c_to, in, p, nt, out, dc, 2 * p + 2, NULL, NULL);
    free(dc);
}

/* ------------------------------------------------------------------ */
/* lfmm3dparttarg (src/lfmm3dpart.f:138-522) with lfmm3dparttargmain
 * (:528-1169) and lfmm3d_list2 (src/lfmm3drouts.f:148-566).  `tinfo`
 * (optional) receives the wall time of the tree and of steps 1..8.        */
static double *taevalhess_ini(int nterms);
static double *mpevalhess_ini(int nterms);
static void taevalhess(double rscale, const double *center, const cplx *loc, int nterms, const double *targ,
                       cplx *pot, int iffld, cplx *fld, int ifhess, cplx *hess, const double *sc);
static void mpevalhess(double rscale, const double *center, const cplx *mp, int nterms, const double *targ,
                       cplx *pot, int iffld, cplx *fld, int ifhess, cplx *hess, const double *sc);
static void direct_hess_one(int ns, const double *src, int ifcharge, const cplx *charge, int ifdipole,
                            const cplx *dipstr, const double *dipvec, const double *t, long skip, cplx h[6]);

/* STEPS 3-5 of lfmm3dparttargmain (M2M, M2L over list 2, L2L), shared by the
 * particle and the triangle FMM (src/lfmm3dtria.f:904 calls the same
 * lfmm3d_list2).  tm[2..4] receive the pass start times. */
static void far_passes(const otree *tp, int p, double eps, cplx *mpole, cplx *local, int ifprune, double *tm)
{
    const otree T = *tp;
    const int K = (p + 1) * (p + 1);
    (void)K;
#define BX(b, f) T.box[20 * (size_t)(b) + (f)]
#define LS(ty, b) T.lstart[ty][b]
#define LE(ty, b) T.lstart[ty][(b) + 1]
#define LI(ty, i) T.lidx[ty][i]
    /* STEP 3: M2M, levels nlev-1..2 (src/lfmm3drouts.f:195-258) */
    tm[2] = omp_get_wtime();
    double *dc = make_dc(2 * p + 2);
    int ldc = 2 * p + 2;
    for (int lev = T.nlev - 1; lev >= 2; lev--) {
        int b0 = T.laddr[2 * lev], b1 = b0 + T.laddr[2 * lev + 1];
#pragma omp parallel for schedule(dynamic)
        for (int ib = b0; ib < b1; ib++) {
            if (BX(ib, B_NSRC) == 0 || nkids(&T, ib) == 0) continue;
            cplx *mo = mpole + (size_t)ib * K;
            memset(mo, 0, sizeof(cplx) * K);
            for (int k = 0; k < 8; k++) {
                int jb = BX(ib, B_KID + k);
                if (jb < 0) continue;
                translate(0, T.center + 3 * (size_t)jb, T.center + 3 * (size_t)ib, mpole + (size_t)jb * K, p, p,
                          mo, dc, ldc, NULL, NULL);
            }
        }
    }
    /* STEP 4: M2L over list 2, levels 2..nlev (src/lfmm3drouts.f:347-483),
     * with precomputed rotations per offset (:297-337).                  */
    tm[3] = omp_get_wtime();
    int itable[343];
    oracle_l3dterms_list2(eps, itable);
    size_t rsz = (size_t)(p + 1) * (p + 1) * (2 * p + 1);
    double *rotf = malloc(rsz * 343 * sizeof(double)), *rotb = malloc(rsz * 343 * sizeof(double));
#pragma omp parallel for
    for (int o = 0; o < 343; o++) {
        int i = o / 49 - 3, j = (o / 7) % 7 - 3, k = o % 7 - 3;
        if (i == 0 && j == 0 && k == 0) continue;
        double rv[3] = {i, j, k}, d, th, ph;
        cart2polarl(rv, &d, &th, &ph);
        rot_init(rotf + rsz * o, p, th);
        rot_init(rotb + rsz * o, p, -th);
    }
    for (int lev = 2; lev <= T.nlev; lev++) {
        int b0 = T.laddr[2 * lev], b1 = b0 + T.laddr[2 * lev + 1];
#pragma omp parallel for schedule(dynamic)
        for (int ib = b0; ib < b1; ib++) {
            for (int li = LS(2, ib); li < LE(2, ib); li++) {
                int jb = LI(2, li);
                if (BX(jb, B_NSRC) == 0) continue;
                if (BX(ib, B_NTRG) == 0 && ifprune) continue;
                int ii = BX(jb, B_I) - BX(ib, B_I), jj = BX(jb, B_J) - BX(ib, B_J), kk = BX(jb, B_K) - BX(ib, B_K);
                int nt = itable[((ii + 3) * 7 + (jj + 3)) * 7 + (kk + 3)];
                if (nt > p) nt = p;
                int o = ((-ii + 3) * 7 + (-jj + 3)) * 7 + (-kk + 3);
                translate(1, T.center + 3 * (size_t)jb, T.center + 3 * (size_t)ib, mpole + (size_t)jb * K, p, nt,
                          local + (size_t)ib * K, dc, ldc, rotf + rsz * o, rotb + rsz * o);
            }
        }
    }
    free(rotf); free(rotb);
    /* STEP 5: L2L, levels 2..nlev-1 (src/lfmm3drouts.f:498-558) */
    tm[4] = omp_get_wtime();
    for (int lev = 2; lev <= T.nlev - 1; lev++) {
        int b0 = T.laddr[2 * lev], b1 = b0 + T.laddr[2 * lev + 1];
#pragma omp parallel for schedule(dynamic)
        for (int ib = b0; ib < b1; ib++) {
            if (nkids(&T, ib) == 0) continue;
            for (int k = 0; k < 8; k++) {
                int jb = BX(ib, B_KID + k);
                if (jb < 0) continue;
                translate(2, T.center + 3 * (size_t)ib, T.center + 3 * (size_t)jb, local + (size_t)ib * K, p, p,
                          local + (size_t)jb * K, dc, ldc, NULL, NULL);
            }
        }
    }
    free(dc);
#undef BX
#undef LS
#undef LE
#undef LI
}

/* lfmm3dparttarg with optional Hessian outputs (ifhess / ifhesstarg, 6 per
 * point).  Potentials and fields are computed exactly as without them; the
 * Hessians add, at each evaluation point, the list-3 multipoles
 * (l3dmpevalhessd_trunc), the leaf's local (l3dtaevalhessd_trunc) and the
 * near pairs (lpotfld3dhess, lpotfld3dhess_dp), all with rscale = 1.     */
static void lfmm_core(int *ier, int iprec, int nsource, const double *source, int ifcharge,
                      const cplx *charge, int ifdipole, const cplx *dipstr, const double *dipvec,
                      int ifpot, cplx *pot, int iffld, cplx *fld, int ifhess, cplx *hess, int ntarget,
                      const double *target, int ifpottarg, cplx *pottarg, int iffldtarg, cplx *fldtarg,
                      int ifhesstarg, cplx *hesstarg, double *tinfo)
{
    *ier = 0;
    double eps = oracle_lap_eps(iprec);
    int nbox = oracle_lap_nbox(iprec, nsource, ntarget);
    if (nbox < 0 || nsource < 1) { *ier = 4; return; }
    double tt0 = omp_get_wtime();
    otree T;
    memset(&T, 0, sizeof T);
    build_boxes(&T, source, nsource, target, ntarget, nbox);
    build_lists(&T);
    double tt1 = omp_get_wtime();
    if (tinfo) tinfo[0] = tt1 - tt0;
    int p = oracle_l3dterms(eps);
    int K = (p + 1) * (p + 1);
    int nb = T.nboxes;
    /* sorted copies: l3dreorder / l3dreordertarg, src/lfmm3drouts.f:667-708 */
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
    cplx *ps = calloc((size_t)nsource, sizeof(cplx)), *fs = calloc(3 * (size_t)nsource, sizeof(cplx));
    cplx *pt = calloc((size_t)(ntarget > 0 ? ntarget : 1), sizeof(cplx));
    cplx *ft = calloc(3 * (size_t)(ntarget > 0 ? ntarget : 1), sizeof(cplx));
    cplx *mpole = calloc((size_t)nb * K, sizeof(cplx)), *local = calloc((size_t)nb * K, sizeof(cplx));
    cplx *hs = ifhess == 1 ? calloc(6 * (size_t)nsource, sizeof(cplx)) : NULL;
    cplx *ht = ifhesstarg == 1 ? calloc(6 * (size_t)(ntarget > 0 ? ntarget : 1), sizeof(cplx)) : NULL;
    double *scm = (ifhess == 1 || ifhesstarg == 1) ? mpevalhess_ini(p) : NULL;
    double *sct = (ifhess == 1 || ifhesstarg == 1) ? taevalhess_ini(p) : NULL;
#define BX(b, f) T.box[20 * (size_t)(b) + (f)]
#define LS(ty, b) T.lstart[ty][b]
#define LE(ty, b) T.lstart[ty][(b) + 1]
#define LI(ty, i) T.lidx[ty][i]
    double tm[9];
    /* STEP 1: P2M at every leaf with sources (src/lfmm3dpart.f:700-769) */
    tm[0] = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        if (BX(ib, B_NSRC) == 0 || nkids(&T, ib) != 0) continue;
        int s0 = BX(ib, B_SRC0), n = BX(ib, B_NSRC);
        oracle_formmp(n, ss + 3 * (size_t)s0, ifcharge, qs + s0, ifdipole, dss + s0, dvs + 3 * (size_t)s0,
                      T.center + 3 * (size_t)ib, p, mpole + (size_t)ib * K);
    }
    /* STEP 2: P2L from the sources of list-4 boxes (src/lfmm3dpart.f:788-869) */
    tm[1] = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
    for (int ib = 0; ib < nb; ib++) {
        for (int li = LS(4, ib); li < LE(4, ib); li++) {
            int jb = LI(4, li);
            int n = BX(jb, B_NSRC);
            if (n == 0) continue;
            int s0 = BX(jb, B_SRC0);
            oracle_formta(n, ss + 3 * (size_t)s0, ifcharge, qs + s0, ifdipole, dss + s0, dvs + 3 * (size_t)s0,
                          T.center + 3 * (size_t)ib, p, local + (size_t)ib * K);
        }
    }
    far_passes(&T, p, eps, mpole, local, !(ifpot == 1 || iffld == 1 || ifhess == 1), tm);
    /* STEP 6: M2P from list-3 boxes (src/lfmm3dpart.f:907-984) */
    tm[5] = omp_get_wtime();
#pragma omp parallel
    {
        double *pp = malloc(sizeof(double) * (p + 2) * (p + 2)), *ppd = malloc(sizeof(double) * (p + 2) * (p + 2));
#pragma omp for schedule(dynamic)
        for (int ib = 0; ib < nb; ib++) {
            for (int li = LS(3, ib); li < LE(3, ib); li++) {
                int jb = LI(3, li);
                const double *cj = T.center + 3 * (size_t)jb;
                const cplx *mj = mpole + (size_t)jb * K;
                cplx pv, fv[3];
                cplx hv[6], ph, fh[3];
                for (int i = BX(ib, B_SRC0); i < BX(ib, B_SRC0) + BX(ib, B_NSRC); i++) {
                    mpeval(cj, mj, p, ss + 3 * (size_t)i, &pv, fv, pp, ppd);
                    if (ifpot == 1) ps[i] += pv;
                    if (iffld == 1) { fs[3 * (size_t)i] += fv[0]; fs[3 * (size_t)i + 1] += fv[1]; fs[3 * (size_t)i + 2] += fv[2]; }
                    if (ifhess == 1) {
                        mpevalhess(1.0, cj, mj, p, ss + 3 * (size_t)i, &ph, 0, fh, 1, hv, scm);
                        for (int k = 0; k < 6; k++) hs[6 * (size_t)i + k] += hv[k];
                    }
                }
                for (int i = BX(ib, B_TRG0); i < BX(ib, B_TRG0) + BX(ib, B_NTRG); i++) {
                    mpeval(cj, mj, p, ts + 3 * (size_t)i, &pv, fv, pp, ppd);
                    if (ifpottarg == 1) pt[i] += pv;
                    if (iffldtarg == 1) { ft[3 * (size_t)i] += fv[0]; ft[3 * (size_t)i + 1] += fv[1]; ft[3 * (size_t)i + 2] += fv[2]; }
                    if (ifhesstarg == 1) {
                        mpevalhess(1.0, cj, mj, p, ts + 3 * (size_t)i, &ph, 0, fh, 1, hv, scm);
                        for (int k = 0; k < 6; k++) ht[6 * (size_t)i + k] += hv[k];
                    }
                }
            }
        }
        /* STEP 7: L2P at leaves of level >= 2 (src/lfmm3dpart.f:1003-1056) */
#pragma omp for schedule(dynamic)
        for (int ib = 0; ib < nb; ib++) {
            if (nkids(&T, ib) != 0 || BX(ib, B_LEV) < 2) continue;
            const double *cb = T.center + 3 * (size_t)ib;
            const cplx *lb = local + (size_t)ib * K;
            cplx pv, fv[3], hv[6], ph, fh[3];
            for (int i = BX(ib, B_SRC0); i < BX(ib, B_SRC0) + BX(ib, B_NSRC); i++) {
                taeval(cb, lb, p, ss + 3 * (size_t)i, &pv, fv, pp, ppd);
                if (ifpot == 1) ps[i] += pv;
                if (iffld == 1) { fs[3 * (size_t)i] += fv[0]; fs[3 * (size_t)i + 1] += fv[1]; fs[3 * (size_t)i + 2] += fv[2]; }
                if (ifhess == 1) {
                    taevalhess(1.0, cb, lb, p, ss + 3 * (size_t)i, &ph, 0, fh, 1, hv, sct);
                    for (int k = 0; k < 6; k++) hs[6 * (size_t)i + k] += hv[k];
                }
            }
            for (int i = BX(ib, B_TRG0); i < BX(ib, B_TRG0) + BX(ib, B_NTRG); i++) {
                taeval(cb, lb, p, ts + 3 * (size_t)i, &pv, fv, pp, ppd);
                if (ifpottarg == 1) pt[i] += pv;
                if (iffldtarg == 1) { ft[3 * (size_t)i] += fv[0]; ft[3 * (size_t)i + 1] += fv[1]; ft[3 * (size_t)i + 2] += fv[2]; }
                if (ifhesstarg == 1) {
                    taevalhess(1.0, cb, lb, p, ts + 3 * (size_t)i, &ph, 0, fh, 1, hv, sct);
                    for (int k = 0; k < 6; k++) ht[6 * (size_t)i + k] += hv[k];
                }
            }
        }
        free(pp); free(ppd);
    }
    /* STEP 8: P2P, self and list 1 (src/lfmm3dpart.f:1076-1141) */
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
            cplx pv, fv[3], hv[6];
            if (ifpot == 1 || iffld == 1)
                for (int i = s0; i < s0 + ns; i++) {
                    direct_one(jn, ss + 3 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0, dvs + 3 * (size_t)js0,
                               ss + 3 * (size_t)i, jb == ib ? i - s0 : -1, iffld, &pv, fv);
                    if (ifpot == 1) ps[i] += pv;
                    if (iffld == 1) { fs[3 * (size_t)i] += fv[0]; fs[3 * (size_t)i + 1] += fv[1]; fs[3 * (size_t)i + 2] += fv[2]; }
                }
            if (ifhess == 1)
                for (int i = s0; i < s0 + ns; i++) {
                    direct_hess_one(jn, ss + 3 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0,
                                    dvs + 3 * (size_t)js0, ss + 3 * (size_t)i, jb == ib ? i - s0 : -1, hv);
                    for (int k = 0; k < 6; k++) hs[6 * (size_t)i + k] += hv[k];
                }
            if (ifpottarg == 1 || iffldtarg == 1)
                for (int i = t0; i < t0 + ntg; i++) {
                    direct_one(jn, ss + 3 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0, dvs + 3 * (size_t)js0,
                               ts + 3 * (size_t)i, -1, iffldtarg, &pv, fv);
                    if (ifpottarg == 1) pt[i] += pv;
                    if (iffldtarg == 1) { ft[3 * (size_t)i] += fv[0]; ft[3 * (size_t)i + 1] += fv[1]; ft[3 * (size_t)i + 2] += fv[2]; }
                }
            if (ifhesstarg == 1)
                for (int i = t0; i < t0 + ntg; i++) {
                    direct_hess_one(jn, ss + 3 * (size_t)js0, ifcharge, qs + js0, ifdipole, dss + js0,
                                    dvs + 3 * (size_t)js0, ts + 3 * (size_t)i, -1, hv);
                    for (int k = 0; k < 6; k++) ht[6 * (size_t)i + k] += hv[k];
                }
        }
    }
    tm[7] = omp_get_wtime();
    if (tinfo) for (int i = 0; i < 7; i++) tinfo[1 + i] = tm[i + 1] - tm[i];
    /* unsort: l3dpsort / l3dfsort, src/lfmm3drouts.f:583-615 */
    for (int i = 0; i < nsource; i++) {
        int j = T.iz[i];
        if (ifpot == 1) pot[j] = ps[i];
        if (iffld == 1) for (int d = 0; d < 3; d++) fld[3 * (size_t)j + d] = fs[3 * (size_t)i + d];
        if (ifhess == 1) for (int d = 0; d < 6; d++) hess[6 * (size_t)j + d] = hs[6 * (size_t)i + d];
    }
    for (int i = 0; i < ntarget; i++) {
        int j = T.iztarg[i];
        if (ifpottarg == 1) pottarg[j] = pt[i];
        if (iffldtarg == 1) for (int d = 0; d < 3; d++) fldtarg[3 * (size_t)j + d] = ft[3 * (size_t)i + d];
        if (ifhesstarg == 1) for (int d = 0; d < 6; d++) hesstarg[6 * (size_t)j + d] = ht[6 * (size_t)i + d];
    }
#undef BX
#undef LS
#undef LE
#undef LI
    free(ss); free(ts); free(qs); free(dss); free(dvs); free(ps); free(fs); free(pt); free(ft);
    free(mpole); free(local); free(hs); free(ht); free(scm); free(sct);
    tree_free(&T);
}

void oracle_lfmm3dparttarg(int *ier, int iprec, int nsource, const double *source, int ifcharge,
                           const cplx *charge, int ifdipole, const cplx *dipstr, const double *dipvec,
                           int ifpot, cplx *pot, int iffld, cplx *fld, int ntarget, const double *target,
                           int ifpottarg, cplx *pottarg, int iffldtarg, cplx *fldtarg, double *tinfo)
{
    lfmm_core(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, pot, iffld, fld, 0,
              NULL, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg, 0, NULL, tinfo);
}

void oracle_lfmm3dparttarg_hess(int *ier, int iprec, int nsource, const double *source, int ifcharge,
                                const cplx *charge, int ifdipole, const cplx *dipstr, const double *dipvec,
                                int ifpot, cplx *pot, int iffld, cplx *fld, int ifhess, cplx *hess, int ntarget,
                                const double *target, int ifpottarg, cplx *pottarg, int iffldtarg, cplx *fldtarg,
                                int ifhesstarg, cplx *hesstarg)
{
    lfmm_core(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, pot, iffld, fld, ifhess,
              hess, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg, ifhesstarg, hesstarg, NULL);
}

/* Laplace layer potentials on flat triangles (lfmm3dtriatarg). */
#include "ltri_oracle.c"

/* The Helmholtz restatement shares the tree, lists and rotations above. */
#include "hfmm3d_oracle.c"

/* Laplace Hessians (pair, local and multipole evaluators, FMM driver). */
#include "lhess_oracle.c"

/* Helmholtz layer potentials on flat triangles (hfmm3dtriatarg). */
#include "htri_oracle.c"
