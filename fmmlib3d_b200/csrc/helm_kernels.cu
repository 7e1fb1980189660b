// Helmholtz FMM kernels (FP64): special functions, P2M/P2L, L2P/M2P,
// z-shift operators, rotate-shift-rotate translations, P2P and the direct sum.
#include <mutex>

#include "helm_kernels.cuh"

namespace fmm {

// ================================================================ complex helpers
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b)
{
    // Smith's algorithm
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    double r = b.x / b.y, d = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double cabsd(double2 a) { return hypot(a.x, a.y); }
// e^{i z}
__device__ __forceinline__ double2 cexpi(double2 z)
{
    double s, c;
    sincos(z.x, &s, &c);
    double e = exp(-z.y);
    return make_double2(e * c, e * s);
}

// ================================================================ special functions
// Scaled spherical Hankel functions h_n(z) scale^n, n = 0..nt, and (if hd)
// their derivatives: h3dall (src/helmrouts3d.f:709-809), stored with stride
// hs.  Needs nt >= 1.
__device__ void hank_dev(int nt, double2 z, double scale, double2 *h, double2 *hd, int hs = 1)
{
    if (cabsd(z) < 1.0e-15) {
        for (int i = 0; i <= nt; i++) { h[i * hs] = cmk(0, 0); if (hd) hd[i * hs] = cmk(0, 0); }
        return;
    }
    // h0 = e^{iz} / (iz), h1 = h0 (1/z - i)   (h3d01, :666-704)
    double2 iz = cmk(-z.y, z.x);
    double2 h0 = cdiv(cexpi(z), iz);
    double2 zi = cdiv(cmk(1, 0), z);
    double2 h1 = cmul(h0, cmk(zi.x, zi.y - 1.0));
    h[0] = h0;
    h[hs] = cscal(scale, h1);
    double s2 = scale * scale;
    double2 zs = cscal(scale, zi);
    for (int i = 1; i <= nt - 1; i++) {
        double2 t = cscal(2 * i + 1.0, zs);
        h[(i + 1) * hs] = csub(cmul(t, h[i * hs]), cscal(s2, h[(i - 1) * hs]));
    }
    if (hd) {
        hd[0] = cscal(-1.0 / scale, h[hs]);
        for (int i = 1; i <= nt; i++) hd[i * hs] = csub(cscal(scale, h[(i - 1) * hs]), cmul(cscal(i + 1.0, zi), h[i * hs]));
    }
}

// Scaled spherical Bessel functions j_n(z) / scale^n, n = 0..nt+1, by the
// backward recurrence of jfuns3d (src/cdjseval3d.f:15-197): the upward
// sweep from n = nt finds the start ntop (first |f|^2 > 1e40, at most
// nt + 1000 terms), the downward sweep rescales by 1e-40 when it grows past
// that bound, and the values are normalized against sin z / z or its
// successor.  Only entries 0..nt+1 are stored (with stride fs).  fd
// (optional) receives the derivatives of entries 0..nt.  Returns 8 if the
// upward sweep never grew.
__device__ int bess_dev(int nt, double2 z, double scale, double2 *f, double2 *fd, int fs = 1)
{
    const double ub = 1.0e40, ubinv = 1.0e-40;
    if (cabsd(z) < 1.0e-200) {
        f[0] = cmk(1, 0);
        for (int i = 1; i <= nt + 1; i++) f[i * fs] = cmk(0, 0);
        if (fd) {
            for (int i = 0; i <= nt; i++) fd[i * fs] = cmk(0, 0);
            if (nt >= 1) fd[fs] = cmk(1.0 / (3 * scale), 0);
        }
        return 0;
    }
    double2 zi = cdiv(cmk(1, 0), z);
    int ntop = 0;
    {
        double2 fm = cmk(0, 0), fc = cmk(1, 0);
        for (int i = nt; i <= nt + 1000; i++) {
            double2 fn = csub(cmul(cscal(2 * i + 1.0, zi), fc), fm);
            if (cabs2(fn) > ub) { ntop = i + 1; break; }
            fm = fc;
            fc = fn;
        }
    }
    if (ntop == 0) return 8;
    unsigned long long fl[4] = {0ull, 0ull, 0ull, 0ull};  // rescale events at index i <= 255
    if (ntop <= nt + 1) f[ntop * fs] = cmk(0, 0);
    double2 a = cmk(0, 0), b = cmk(1, 0);    // f(i+1), f(i)
    for (int i = ntop - 1; i >= 1; i--) {
        double2 c = csub(cmul(cscal(2 * i + 1.0, zi), b), a);
        if (cabs2(c) > ub) {
            b = cscal(ubinv, b);
            c = cscal(ubinv, c);
            if (i < 256) fl[i >> 6] |= 1ull << (i & 63);
        }
        if (i <= nt + 1) f[i * fs] = b;
        a = b;
        b = c;
    }
    f[0] = b;
    double sinv = 1.0 / scale, sct = 1.0;
    for (int i = 1; i <= nt + 1; i++) {
        sct *= sinv;
        int k = i - 1;
        if ((fl[k >> 6] >> (k & 63)) & 1ull) sct *= ubinv;
        f[i * fs] = cscal(sct, f[i * fs]);
    }
    // sin z / z and (sin z / z - cos z) / z
    double sx, cx;
    sincos(z.x, &sx, &cx);
    double ch = cosh(z.y), sh = sinh(z.y);
    double2 sz = cmk(sx * ch, cx * sh), cz = cmk(cx * ch, -sx * sh);
    double2 j0 = cmul(sz, zi);
    double2 j1 = csub(cmul(j0, zi), cmul(cz, zi));
    double2 zs = cabsd(j1) > cabsd(j0) ? cdiv(j1, cscal(scale, f[fs])) : cdiv(j0, f[0]);
    for (int i = 0; i <= nt + 1; i++) f[i * fs] = cmul(f[i * fs], zs);
    if (fd) {
        fd[0] = cscal(-scale, f[fs]);
        for (int i = 1; i <= nt; i++) {
            double d1 = i / (2 * i + 1.0), d2 = 1.0 - d1;
            fd[i * fs] = csub(cscal(d1 * sinv, f[(i - 1) * fs]), cscal(d2 * scale, f[(i + 1) * fs]));
        }
    }
    return 0;
}

// Column m of the Legendre functions with the sqrt(2n+1) factor at x, for
// n = m..nmax, in the scaled form of ylgndr2s (src/yrecursion.f:298-385):
// y[n] = Y_n^m / sin(theta) and d[n] = -dY_n^m/dtheta for m >= 1, and
// y[n] = Y_n^0, d[n] = dY_n^0/dx for m = 0.  Arrays are indexed by n - m.
// `regular` multiplies y by sin(theta) (giving Y_n^m) and turns d into
// dY/dtheta for every m.  d may be null.
__device__ void legendre_col(int m, int nmax, double x, double *y, double *d, bool regular)
{
    double u2 = (1 - x) * (1 + x), st = sqrt(u2), u = -st;
    double ym, dm;
    if (m == 0) { ym = 1; dm = 0; }
    else {
        ym = -sqrt(0.5);
        for (int k = 2; k <= m; k++) ym *= u * sqrt((2 * k - 1.0) / (2 * k));
        dm = ym * (-m) * x;
    }
    const double w = m == 0 ? 1.0 : u2;
    double y1 = 0, d1 = 0, y2 = 0, d2 = 0;  // values at n-1 and n-2
    for (int n = m; n <= nmax; n++) {
        double yn, dn;
        if (n == m) { yn = ym; dn = dm; }
        else if (n == m + 1) {
            yn = x * y1 * sqrt(2 * m + 1.0);
            dn = (x * d1 + w * y1) * sqrt(2 * m + 1.0);
        } else {
            double a = sqrt((n + m - 1.0) * (n - m - 1.0)), b = sqrt((n - m + 0.0) * (n + m));
            yn = ((2 * n - 1) * x * y1 - a * y2) / b;
            dn = ((2 * n - 1) * (x * d1 + w * y1) - a * d2) / b;
        }
        y[n - m] = yn;
        if (d) d[n - m] = dn;
        y2 = y1; d2 = d1;
        y1 = yn; d1 = dn;
    }
    for (int n = m; n <= nmax; n++) {
        double s = sqrt(2 * n + 1.0);
        y[n - m] *= s;
        if (regular && m > 0) y[n - m] *= st;
        if (d) {
            d[n - m] *= s;
            if (regular) d[n - m] = m == 0 ? -st * d[n - m] : -d[n - m];
        }
    }
}

// ================================================================ z-shift operators
// For one block (kind, degrees nin -> nout, shift zshift along z, sphere
// radius, quadrature x_j, w_j of nq Gauss-Legendre nodes) the reference
// evaluates the rotated source expansion at the nodes of the target sphere
// (h3dmpevalspherenm_fast / h3dmpevalspherenmstab_fast /
// h3dlocevalspherestab_fast, src/projections.f:1611, 1917, 901), projects
// on Y_l^m (h3dprojlocnmsep_fast / h3dprojlocsepstab_fast, :1277, 2292) and
// rescales (h3drescalemp / h3drescalestab, :556, 679).  The composition is
// linear and diagonal in m, depends on |m| only, and is built here entry by
// entry:
//   A[l][n] = sum_j w_j/2 Y_l^m(x_j) f_n(k r_j) Y_n^m(cos t_j)
//   B[l][n] = sum_j w_j/2 Y_l^m(x_j) (k f'_n(k r_j) rn_j Y_n^m + f_n thn_j dY_n^m/dtheta)
// with f = h (M2M, M2L) or j (L2L) scaled by sc1, and
//   M2M:   Z = A / h_l(k R)                 (scaled by sc2)
//   stab:  Z = (j_l A + k j'_l B) / (j_l^2 + (k j'_l)^2)   at k R, scaled by sc2.
__device__ __forceinline__ void hz_node(const HZBlock &B, const double *xw, int j, double &ctj, double &stj,
                                        double &rn, double &thn, double &rj)
{
    double ct = xw[2 * (B.qoff + j)], st = sqrt(1.0 - ct * ct);
    double a = B.zshift + B.radius * ct, c = B.radius * st;
    rj = sqrt(a * a + c * c);
    ctj = a / rj;
    stj = sqrt(1.0 - ctj * ctj);
    rn = stj * st + ctj * ct;
    thn = (ctj * st - ct * stj) / rj;
}

__global__ void k_hz_radial(const HZBlock *blk, const double *xw, double2 zk, int pmax, double2 *rad)
{
    const HZBlock B = blk[blockIdx.x];
    const int j = blockIdx.y * blockDim.x + threadIdx.x;
    if (j > B.nq) return;
    const int W = pmax + 2;
    double2 *R = rad + B.roff + (size_t)j * 2 * W, *Rd = R + W;
    if (j < B.nq) {
        double ctj, stj, rn, thn, rj;
        hz_node(B, xw, j, ctj, stj, rn, thn, rj);
        double2 z = cscal(rj, zk);
        int nt = B.nin > 1 ? B.nin : 1;
        if (B.kind == 2) {
            if (bess_dev(nt, z, B.sc1, R, Rd))
                for (int i = 0; i <= nt + 1; i++) { R[i] = cmk(0, 0); Rd[i] = cmk(0, 0); }
        } else {
            hank_dev(nt, z, B.sc1, R, B.kind == 1 ? Rd : nullptr);
        }
        if (B.kind != 0)
            for (int i = 0; i <= nt; i++) Rd[i] = cmul(Rd[i], zk);
    } else {
        double2 z = cscal(B.radius, zk);
        int nt = B.nout > 1 ? B.nout : 1;
        if (B.kind == 0) hank_dev(nt, z, B.sc2, R, nullptr);
        else {
            if (bess_dev(nt, z, B.sc2, R, Rd))
                for (int i = 0; i <= nt + 1; i++) { R[i] = cmk(0, 0); Rd[i] = cmk(0, 0); }
            for (int i = 0; i <= nt; i++) Rd[i] = cmul(Rd[i], zk);
        }
    }
}

constexpr int kHzThreads = 256, kHzNodes = 32, kHzPer = 4;

__global__ void __launch_bounds__(kHzThreads) k_hz_build(const HZBlock *blk, const double *xw, int pmax,
                                                         const double2 *rad, double2 *Z)
{
    extern __shared__ double hzs[];
    const HZBlock B = blk[blockIdx.x];
    const int m = blockIdx.y;
    const int mmax = B.nin < B.nout ? B.nin : B.nout;
    if (m > mmax) return;
    const int W = pmax + 2, LD = pmax + 1;
    double *Yt = hzs;                          // [node][l - m]
    double *Ys = Yt + kHzNodes * LD;           // [node][n - m]
    double *dYs = Ys + kHzNodes * LD;
    double *gw = dYs + kHzNodes * LD;          // w/2, rn, thn per node
    const int nr = B.nout + 1 - m, ncol = B.nin + 1 - m, ne = nr * ncol;
    long long mo = 0;
    for (int k = 0; k < m; k++) mo += (long long)(B.nout + 1 - k) * (B.nin + 1 - k);
    double2 *Zm = Z + B.zoff + mo;
    const double2 *Rt = rad + B.roff + (size_t)B.nq * 2 * W, *Rtd = Rt + W;
    for (int e0 = 0; e0 < ne; e0 += kHzThreads * kHzPer) {
        double2 A[kHzPer], Bv[kHzPer];
#pragma unroll
        for (int q = 0; q < kHzPer; q++) { A[q] = cmk(0, 0); Bv[q] = cmk(0, 0); }
        for (int j0 = 0; j0 < B.nq; j0 += kHzNodes) {
            const int nj = min(kHzNodes, B.nq - j0);
            __syncthreads();
            if (threadIdx.x < nj) {
                int j = j0 + threadIdx.x;
                double ctj, stj, rn, thn, rj;
                hz_node(B, xw, j, ctj, stj, rn, thn, rj);
                legendre_col(m, B.nin, ctj, Ys + threadIdx.x * LD, B.kind == 0 ? nullptr : dYs + threadIdx.x * LD,
                             true);
                gw[3 * threadIdx.x] = 0.5 * xw[2 * (B.qoff + j) + 1];
                gw[3 * threadIdx.x + 1] = rn;
                gw[3 * threadIdx.x + 2] = thn;
            } else if (threadIdx.x >= 32 && threadIdx.x < 32 + nj) {
                int t = threadIdx.x - 32;
                legendre_col(m, B.nout, xw[2 * (B.qoff + j0 + t)], Yt + t * LD, nullptr, true);
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < kHzPer; q++) {
                int e = e0 + q * kHzThreads + threadIdx.x;
                if (e >= ne) continue;
                int li = e / ncol, ni = e % ncol, n = ni + m;
                for (int jj = 0; jj < nj; jj++) {
                    const double2 *R = rad + B.roff + (size_t)(j0 + jj) * 2 * W;
                    double wt = gw[3 * jj] * Yt[jj * LD + li];
                    double ys = Ys[jj * LD + ni];
                    crfma(A[q], wt * ys, R[n]);
                    if (B.kind != 0) {
                        crfma(Bv[q], wt * ys * gw[3 * jj + 1], R[W + n]);
                        crfma(Bv[q], wt * dYs[jj * LD + ni] * gw[3 * jj + 2], R[n]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kHzPer; q++) {
            int e = e0 + q * kHzThreads + threadIdx.x;
            if (e >= ne) continue;
            int l = e / ncol + m;
            double2 v;
            if (B.kind == 0) v = cdiv(A[q], Rt[l]);
            else {
                double2 zh = Rt[l], zhn = Rtd[l];
                double2 zm = cadd(cmul(zh, zh), cmul(zhn, zhn));
                v = cdiv(cadd(cmul(zh, A[q]), cmul(zhn, Bv[q])), zm);
            }
            Zm[e] = v;
        }
    }
}

void build_hz(int nblk, const HZBlock *d_blk, const HZBlock *h_blk, const double *d_xw, double2 zk, int pmax,
              double2 *rad, double2 *Z, cudaStream_t s, Status &st)
{
    if (!st.ok() || nblk == 0) return;
    int maxq = 0;
    for (int b = 0; b < nblk; b++) maxq = std::max(maxq, h_blk[b].nq + 1);
    dim3 g1(nblk, div_up(maxq, 64));
    k_hz_radial<<<g1, 64, 0, s>>>(d_blk, d_xw, zk, pmax, rad); FMM_COUNT_LAUNCH();
    size_t sm = sizeof(double) * (3 * kHzNodes * (pmax + 1) + 3 * kHzNodes);
    FMM_TRY(st, smem_allow(k_hz_build, (int)sm));
    dim3 g2(nblk, pmax + 1);
    k_hz_build<<<g2, kHzThreads, sm, s>>>(d_blk, d_xw, pmax, rad, Z); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// ================================================================ translations
// h3dmpmpquad0 (M2M), h3dmplocquad_trunc0 (M2L) and h3dloclocquad0 (L2L)
// (src/h3dtrans.f:211, 1229, 1998), batched as the Laplace translations: a
// CTA owns up to KT targets of one (level, octant) group; per source slot it
// gathers the sources, applies e^{i m phi}, the rotation D(theta), the
// z-shift operator of the slot (per |m| dense block), D(theta)^T and
// e^{-i m phi}, and accumulates in shared memory.
constexpr int kHTransThreads = 256;
constexpr size_t kHTransSmemMax = 200 * 1024;   // larger buffers go to global scratch

__device__ __forceinline__ int hsrc_of(int kind, const TreeView &tv, int t, const HSlot &sl)
{
    if (kind == 0) return tv.child[8L * t + sl.oct];
    if (kind == 2) return tv.parent[t];
    int P = tv.parent[t];
    if (P < 0) return -1;
    int C = tv.coll[27L * P + sl.coll];
    if (C < 0) return -1;
    return tv.child[8L * C + sl.oct];
}

__device__ __forceinline__ int deg_of(int e)
{
    int n = (int)sqrtf((float)e);
    while (n * n > e) n--;
    while ((n + 1) * (n + 1) <= e) n++;
    return n;
}

// gs: null, or global scratch of gridDim.x x 3 KT (pmax+1)^2 entries for the
// three expansion buffers (orders whose buffers do not fit in shared memory);
// the CTAs then walk the tiles with a grid stride.
template <int KIND, int KT, bool GS>
__global__ void __launch_bounds__(kHTransThreads) k_htranslate(const Tile *tiles, int ntiles, const int *grouped,
                                                               const HSlot *slots, TreeView tv, int pmax,
                                                               const double *rot, const double2 *Z,
                                                               const double2 *in, double2 *out, int prune,
                                                               double2 *gs)
{
    extern __shared__ double2 sm[];
    const int NC = (pmax + 1) * (pmax + 1);
    double2 *acc = GS ? gs + (size_t)blockIdx.x * 3 * KT * NC : sm;
    double2 *bA = acc + (size_t)KT * NC;
    double2 *bB = bA + (size_t)KT * NC;
    double2 *eph = GS ? sm : bB + (size_t)KT * NC;  // e^{i m phi}, m = 0..pmax
    __shared__ int tg[8], sv[8];
    __shared__ int anyv;
    for (int tix = blockIdx.x; tix < (GS ? ntiles : blockIdx.x + 1); tix += gridDim.x) {
    if (GS) __syncthreads();
    const Tile tile = tiles[tix];
    if (threadIdx.x < 8) {
        int t = threadIdx.x < tile.count ? grouped[tile.first + threadIdx.x] : -1;
        if (t >= 0 && KIND == 0 && tv.nchild[t] == 0) t = -1;
        if (t >= 0 && KIND == 0 && tv.nsrc[t] == 0) t = -1;  // sourceless boxes keep a zero multipole
        tg[threadIdx.x] = t;
    }
    for (int i = threadIdx.x; i < KT * NC; i += kHTransThreads) acc[i] = cmk(0, 0);
    const size_t csz = rot_class_size(pmax);
    for (int si = 0; si < tile.nslot; si++) {
        const HSlot sl = slots[tile.slot0 + si];
        __syncthreads();
        if (threadIdx.x == 0) anyv = 0;
        __syncthreads();
        if (threadIdx.x < KT) {
            int t = tg[threadIdx.x];
            int sb = -1;
            if (t >= 0) {
                sb = hsrc_of(KIND, tv, t, sl);
                if (sb >= 0 && KIND != 2 && tv.nsrc[sb] == 0) sb = -1;
                if (KIND == 1 && prune && tv.ntrg[t] == 0) sb = -1;
            }
            sv[threadIdx.x] = sb;
            if (sb >= 0) atomicOr(&anyv, 1);
        }
        if (threadIdx.x == 32) {
            double2 e1 = cmk(sl.ex, sl.ey), e = cmk(1, 0);
            for (int m = 0; m <= pmax; m++) { eph[m] = e; e = cmul(e, e1); }
        }
        __syncthreads();
        if (!anyv) continue;
        const int nin = sl.nin, nout = sl.nout, mmax = sl.mmax;
        const int Rin = (nin + 1) * (nin + 1), Rout = (nout + 1) * (nout + 1);
        // phase 1: gather, times e^{i m phi}
        for (int i = threadIdx.x; i < KT * Rin; i += kHTransThreads) {
            int k = i / Rin, e = i % Rin;
            int sb = sv[k];
            double2 v = cmk(0, 0);
            if (sb >= 0) {
                int n = deg_of(e), m = e - n * n - n;
                double2 ph = m >= 0 ? eph[m] : cconj(eph[-m]);
                v = cmul(in[(size_t)sb * NC + e], ph);
            }
            bA[(size_t)k * NC + e] = v;
        }
        __syncthreads();
        const double *R = rot + csz * sl.cls;
        // phase 2: bB[n][m'] = sum_m bA[n][m] D^n[m][m']
        for (int row = threadIdx.x; row < Rin; row += kHTransThreads) {
            int n = deg_of(row), mp = row - n * n - n;
            const double *Dn = R + (size_t)n * (4 * n * n - 1) / 3;
            int w = 2 * n + 1;
            double2 a[KT];
            _Pragma("unroll") for (int k = 0; k < KT; k++) a[k] = cmk(0, 0);
            for (int m = -n; m <= n; m++) {
                double d = Dn[(m + n) * w + (mp + n)];
                _Pragma("unroll") for (int k = 0; k < KT; k++) crfma(a[k], d, bA[(size_t)k * NC + eidx(n, m)]);
            }
            _Pragma("unroll") for (int k = 0; k < KT; k++) bB[(size_t)k * NC + row] = a[k];
        }
        __syncthreads();
        // phase 3: z-shift, bA[l][m] = sum_n Z_|m|[l][n] bB[n][m]
        const double2 *Zb = Z + sl.zoff;
        for (int row = threadIdx.x; row < Rout; row += kHTransThreads) {
            int l = deg_of(row), m = row - l * l - l, am = m < 0 ? -m : m;
            double2 a[KT];
            _Pragma("unroll") for (int k = 0; k < KT; k++) a[k] = cmk(0, 0);
            if (am <= mmax) {
                long long mo = 0;
                for (int q = 0; q < am; q++) mo += (long long)(nout + 1 - q) * (nin + 1 - q);
                const double2 *zr = Zb + mo + (long long)(l - am) * (nin + 1 - am) - am;
                for (int n = am; n <= nin; n++) {
                    double2 z = zr[n];
                    _Pragma("unroll") for (int k = 0; k < KT; k++) cfma(a[k], z, bB[(size_t)k * NC + eidx(n, m)]);
                }
            }
            _Pragma("unroll") for (int k = 0; k < KT; k++) bA[(size_t)k * NC + row] = a[k];
        }
        __syncthreads();
        // phase 4: back rotation, times e^{-i m phi}, accumulate
        for (int row = threadIdx.x; row < Rout; row += kHTransThreads) {
            int n = deg_of(row), m = row - n * n - n;
            const double *Dn = R + (size_t)n * (4 * n * n - 1) / 3 + (size_t)(m + n) * (2 * n + 1);
            double2 a[KT];
            _Pragma("unroll") for (int k = 0; k < KT; k++) a[k] = cmk(0, 0);
            for (int mp = -n; mp <= n; mp++) {
                double d = Dn[mp + n];
                _Pragma("unroll") for (int k = 0; k < KT; k++) crfma(a[k], d, bA[(size_t)k * NC + eidx(n, mp)]);
            }
            double2 ph = m >= 0 ? cconj(eph[m]) : eph[-m];
            _Pragma("unroll") for (int k = 0; k < KT; k++)
                if (sv[k] >= 0) acc[(size_t)k * NC + row] = cadd(acc[(size_t)k * NC + row], cmul(a[k], ph));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < KT * NC; i += kHTransThreads) {
        int k = i / NC, e = i % NC;
        int t = tg[k];
        if (t < 0) continue;
        double2 *o = out + (size_t)t * NC + e;
        if (KIND == 0) *o = acc[i];
        else *o = cadd(*o, acc[i]);
    }
    }
}

template <int KIND>
static void launch_htranslate_kind(const Tile *tiles, int ntiles, const int *grouped, const HSlot *slots,
                                   const TreeView &tv, int pmax, const double *rot, const double2 *Z,
                                   const double2 *in, double2 *out, int prune, int kt, size_t sm, int grid,
                                   double2 *gs, cudaStream_t s, Status &st)
{
#define FMM_HTR(KTV)                                                                                           \
    do {                                                                                                       \
        if (gs) {                                                                                              \
            FMM_TRY(st, smem_allow(k_htranslate<KIND, KTV, true>,                                    \
                                             (int)sm));           \
            k_htranslate<KIND, KTV, true><<<grid, kHTransThreads, sm, s>>>(tiles, ntiles, grouped, slots, tv,  \
                                                                           pmax, rot, Z, in, out, prune, gs);  \
        } else {                                                                                               \
            FMM_TRY(st, smem_allow(k_htranslate<KIND, KTV, false>,                                   \
                                             (int)sm));           \
            k_htranslate<KIND, KTV, false><<<grid, kHTransThreads, sm, s>>>(tiles, ntiles, grouped, slots, tv, \
                                                                            pmax, rot, Z, in, out, prune, gs); \
        }                                                                                                      \
        FMM_COUNT_LAUNCH();                                                                                    \
    } while (0)
    if (kt == 8) FMM_HTR(8);
    else if (kt == 4) FMM_HTR(4);
    else if (kt == 2) FMM_HTR(2);
    else FMM_HTR(1);
#undef FMM_HTR
}

void launch_htranslate(int kind, const Tile *tiles, int ntiles, const int *grouped, const HSlot *slots,
                       const TreeView &tv, int pmax, const double *rot, const double2 *Z, const double2 *in,
                       double2 *out, int prune, int kt, cudaStream_t s, Status &st)
{
    if (ntiles == 0 || !st.ok()) return;
    int NC = (pmax + 1) * (pmax + 1);
    size_t sm = (size_t)3 * kt * NC * sizeof(double2) + (pmax + 1) * sizeof(double2);
    int grid = ntiles;
    DBuf<double2> gs;
    if (sm > kHTransSmemMax) {
        // high orders: the three buffers in global scratch, one slice per CTA of a grid-stride launch
        grid = std::min(ntiles, 2 * 148);
        if (!gs.alloc((size_t)grid * 3 * kt * NC, s, st)) return;
        sm = (pmax + 1) * sizeof(double2);
    }
    if (kind == 0) launch_htranslate_kind<0>(tiles, ntiles, grouped, slots, tv, pmax, rot, Z, in, out, prune, kt, sm, grid, gs.p, s, st);
    else if (kind == 1) launch_htranslate_kind<1>(tiles, ntiles, grouped, slots, tv, pmax, rot, Z, in, out, prune, kt, sm, grid, gs.p, s, st);
    else launch_htranslate_kind<2>(tiles, ntiles, grouped, slots, tv, pmax, rot, Z, in, out, prune, kt, sm, grid, gs.p, s, st);
    FMM_LAUNCH_CHECK(st);
}

// ================================================================ point operators
// Legendre recurrence coefficients for the column recurrences in registers:
// g_ha[n][m] = sqrt((n+m-1)(n-m-1)), g_hb[n][m] = 1/sqrt((n-m)(n+m)),
// g_hs[n] = sqrt(2n+1), g_hc[m] = sqrt((2m-1)/(2m)); the weights of the radial
// derivative of j_n, g_hq[n] = n/(2n+1), and g_hr[n] = 1/(2n+1).
constexpr int kHTab = kHelmMaxP + 3;
__device__ double g_ha[kHTab * kHTab], g_hb[kHTab * kHTab], g_hs[kHTab], g_hc[kHTab], g_hq[kHTab], g_hr[kHTab];

__global__ void k_htab_init()
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kHTab) {
        g_hs[i] = sqrt(2 * i + 1.0);
        g_hc[i] = i > 0 ? sqrt((2 * i - 1.0) / (2 * i)) : 0.0;
        g_hq[i] = i / (2 * i + 1.0);
        g_hr[i] = 1.0 / (2 * i + 1.0);
    }
    if (i >= kHTab * kHTab) return;
    int n = i / kHTab, m = i % kHTab;
    g_ha[i] = (n >= m + 2) ? sqrt((n + m - 1.0) * (n - m - 1.0)) : 0.0;
    g_hb[i] = (n > m) ? 1.0 / sqrt((n - m + 0.0) * (n + m)) : 0.0;
}

static void htab_init(cudaStream_t s, Status &st)
{
    static std::mutex mu;  // several host threads may make their first call at once
    std::lock_guard<std::mutex> lk(mu);
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done[dev]) return;
    k_htab_init<<<div_up(kHTab * kHTab, 256), 256, 0, s>>>(); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    FMM_TRY(st, cudaStreamSynchronize(s));  // other threads' streams may read the tables next
    if (st.ok() && dev >= 0 && dev < 64) done[dev] = true;
}

// One step of the scaled column recurrence (2s form, src/yrecursion.f:298):
// y1, d1 hold degree n-1 and y2, d2 degree n-2 of column m.
struct LegCol {
    double x, w, y1, d1, y2, d2;
    int m;
    __device__ __forceinline__ void start(int m_, double x_, double u)
    {
        m = m_;
        x = x_;
        w = m == 0 ? 1.0 : u * u;
        double y;
        if (m == 0) y = 1;
        else {
            y = -sqrt(0.5);
            for (int k = 2; k <= m; k++) y *= u * sqrt((2 * k - 1.0) / (2 * k));
        }
        y1 = y;
        d1 = m == 0 ? 0.0 : y * (-m) * x;
        y2 = 0;
        d2 = 0;
    }
    // advance from degree n-1 to n (n > m)
    __device__ __forceinline__ void step(int n)
    {
        double yn, dn;
        if (n == m + 1) {
            double s = __ldg(&g_hs[m]);
            yn = x * y1 * s;
            dn = (x * d1 + w * y1) * s;
        } else {
            double a = __ldg(&g_ha[n * kHTab + m]), b = __ldg(&g_hb[n * kHTab + m]);
            yn = ((2 * n - 1) * x * y1 - a * y2) * b;
            dn = ((2 * n - 1) * (x * d1 + w * y1) - a * d2) * b;
        }
        y2 = y1; d2 = d1;
        y1 = yn; d1 = dn;
    }
};

// Geometry of one point relative to an expansion center (cart2polar,
// src/helmrouts3d.f:627-662).
struct PtGeo {
    double r, ct, st, cp, sp;
};
__device__ __forceinline__ PtGeo pt_geo(double dx, double dy, double dz)
{
    PtGeo g;
    g.r = sqrt(dx * dx + dy * dy + dz * dz);
    double proj = sqrt(dx * dx + dy * dy);
    double th = atan2(proj, dz);
    g.ct = cos(th);
    g.st = sqrt(1.0 - g.ct * g.ct);
    double ph = (dx == 0 && dy == 0) ? 0.0 : atan2(dy, dx);
    sincos(ph, &g.sp, &g.cp);
    return g;
}

// P2M / P2L.  CTA per receiving box and range of 1024 coefficients, each
// thread owning up to kHFormPer coefficients in registers.  Sources are taken in chunks of CH: per chunk
// the sources' radial functions, e^{-i m phi} powers, diagonal Legendre
// values and full Legendre tables (2s form, one column per (source, m) task)
// are built in shared memory, then every thread adds the chunk's
// contributions to its coefficients.  The sum is multiplied by ik at the end
// (h3dformmp_add_trunc / h3dformta_add_trunc, src/helmrouts3d.f:2972, 3299;
// dipoles h3dformmp_dp_add_trunc :3580, h3dformta_dp_add_trunc :3978).
constexpr int kHFormThreads = 256, kHFormPer = 4;
// Source set-up in batches of kHFormSetA x kHFormSetCH (32) sources, tables per kHFormSetCH.
constexpr int kHFormSetCH = 8, kHFormSetA = 4;

template <int CH, bool DIP, int AX = 1>
struct HFormSmem {
    // sizes in doubles for expansion order p
    static __host__ __device__ size_t doubles(int p)
    {
        size_t W = p + 2, T = (size_t)(p + 1) * (p + 2) / 2;
        size_t d = AX * CH * (2 * W + 2 * (p + 1) + (p + 1) + 16) + CH * T;  // f, e^{-im phi}, diagonal, scalars; Y
        if (DIP) d += CH * T + AX * CH * 4 * (p + 1);                         // D; fd, fu
        return d;
    }
};

template <bool IRREG, bool CHG, bool DIP, int CH, int AX = 1>
__global__ void __launch_bounds__(kHFormThreads) k_hform(const int *boxes, TreeView tv, PointsSoA src, HLevels lv,
                                                        int NC, double2 zk, double2 *exps)
{
    extern __shared__ double hsd[];
    const int b = boxes[blockIdx.x];
    const int lev = tv.level[b];
    if (lev < 2) return;
    if (!IRREG && (tv.nchild[b] != 0 || tv.nsrc[b] == 0)) return;
    if (IRREG && tv.l4_start[b + 1] == tv.l4_start[b]) return;
    const int p = lv.p[lev];
    const double sc = lv.sc[lev];
    const int W = p + 2, P1 = p + 1, TS = (p + 1) * (p + 2) / 2, K = (p + 1) * (p + 1);
    // per-source arrays for AX CH sources (set up together in phase A), the
    // Legendre tables for CH (phases B and C run on AX sub-chunks in turn)
    double2 *F = (double2 *)hsd;                 // [AX CH][W]
    double2 *Em = F + AX * CH * W;               // [AX CH][P1]   e^{-i m phi}
    double *Dg = (double *)(Em + AX * CH * P1);  // [AX CH][P1]   diagonal Y_m^m (2s form)
    double *Y = Dg + AX * CH * P1;               // [CH][TS]
    double *Sc = Y + CH * TS;                    // [AX CH][16]   per-source scalars
    double *D = Sc + AX * CH * 16;               // [CH][TS]      (dipoles)
    double2 *Fd = (double2 *)(D + (DIP ? CH * TS : 0));  // [AX CH][P1]
    double2 *Fu = Fd + (DIP ? AX * CH * P1 : 0);         // [AX CH][P1]
    const int e0 = blockIdx.y * kHFormThreads * kHFormPer;  // this CTA's coefficient range
    if (e0 >= K) return;
    double2 acc[kHFormPer];
    int en[kHFormPer], em_[kHFormPer];
#pragma unroll
    for (int q = 0; q < kHFormPer; q++) {
        acc[q] = cmk(0, 0);
        int e = e0 + threadIdx.x + q * kHFormThreads;
        int n = 0;
        while ((n + 1) * (n + 1) <= e) n++;
        en[q] = e < K ? n : -1;
        em_[q] = e - n * n - n;
    }
    const double *c = tv.center + 3L * b;
    const int nsb = IRREG ? tv.l4_start[b + 1] - tv.l4_start[b] : 1;
    for (int si = 0; si < nsb; si++) {
        const int sb = IRREG ? tv.l4_idx[tv.l4_start[b] + si] : b;
        const int s0 = tv.src0[sb], ns = tv.nsrc[sb];
        for (int c0 = 0; c0 < ns; c0 += AX * CH) {
            const int nba = min(AX * CH, ns - c0);
            __syncthreads();
            // phase A: per source, radial functions, phases, diagonal, scalars
            if (threadIdx.x < nba) {
                const int j = threadIdx.x, i = s0 + c0 + j;
                const PtGeo g = pt_geo(src.x[i] - c[0], src.y[i] - c[1], src.z[i] - c[2]);
                double2 *f = F + j * W;
                const double2 z = cscal(g.r, zk);
                bool ok = true;
                if (IRREG) {
                    if (cabsd(z) < 1.0e-15) ok = false;
                    else hank_dev(p > 1 ? p : 1, z, sc, f, nullptr);
                } else {
                    ok = bess_dev(p > 1 ? p : 1, z, sc, f, nullptr) == 0;
                }
                if (!ok)  // the reference skips such a source (ier 4 / 16)
                    for (int n = 0; n < W; n++) f[n] = cmk(0, 0);
                const double2 e1 = cmk(g.cp, -g.sp);  // e^{-i phi}
                double2 e = cmk(1, 0);
                double dg = 1.0;
                const double u = -g.st;
                for (int m = 0; m <= p; m++) {
                    if (m > 0) e = cmul(e, e1);
                    if (m == 1) dg = -sqrt(0.5);
                    else if (m > 1) dg *= u * __ldg(&g_hc[m]);
                    Em[j * P1 + m] = e;
                    Dg[j * P1 + m] = dg;
                }
                double *S = Sc + j * 16;
                const double2 qv = (CHG && ok) ? src.q[i] : cmk(0, 0), dv = (DIP && ok) ? src.dq[i] : cmk(0, 0);
                S[0] = g.ct; S[1] = g.st; S[2] = qv.x; S[3] = qv.y; S[4] = dv.x; S[5] = dv.y;
                if (DIP) {
                    const double vx = src.vx[i], vy = src.vy[i], vz = src.vz[i];
                    S[6] = vx * g.st * g.cp + vy * g.st * g.sp + vz * g.ct;  // v . r-hat
                    S[7] = vx * g.ct * g.cp + vy * g.ct * g.sp - vz * g.st;  // v . theta-hat
                    S[8] = -vx * g.sp + vy * g.cp;                           // v . phi-hat
                    // radial derivative (times k) and the 1/r angular radial factor
                    const double2 zi = IRREG && ok ? cdiv(cmk(1, 0), z) : cmk(0, 0);
                    for (int n = 0; n <= p; n++) {
                        double2 fd, fu;
                        if (IRREG) {
                            fd = n == 0 ? cscal(-1.0 / sc, f[1]) : csub(cscal(sc, f[n - 1]), cmul(cscal(n + 1.0, zi), f[n]));
                            fu = ok ? cscal(1.0 / g.r, f[n]) : cmk(0, 0);
                        } else {
                            double d1 = n / (2 * n + 1.0), d2 = 1.0 - d1;
                            fd = n == 0 ? cscal(-sc, f[1]) : csub(cscal(d1 / sc, f[n - 1]), cscal(d2 * sc, f[n + 1]));
                            fu = n == 0 ? cmk(0, 0)
                                        : cscal(1.0 / (2 * n + 1.0), cmul(zk, cadd(cscal(sc, f[n + 1]), cscal(1.0 / sc, f[n - 1]))));
                        }
                        Fd[j * P1 + n] = cmul(fd, zk);
                        Fu[j * P1 + n] = fu;
                    }
                }
            }
            __syncthreads();
            for (int sub = 0; sub < AX; sub++) {
                const int jb = sub * CH, nb = min(CH, nba - jb);
                if (nb <= 0) break;
                if (sub > 0) __syncthreads();   // the previous sub-chunk's tables are read
                const double2 *Fs = F + jb * W, *Ems = Em + jb * P1;
                const double *Dgs = Dg + jb * P1, *Scs = Sc + jb * 16;
                const double2 *Fds = Fd + (DIP ? jb * P1 : 0), *Fus = Fu + (DIP ? jb * P1 : 0);
                // phase B: Legendre columns, one (source, m) task per thread
                for (int task = threadIdx.x; task < nb * P1; task += kHFormThreads) {
                    const int j = task / P1, m = task % P1;
                    const double x = Scs[j * 16], u = -Scs[j * 16 + 1];
                    LegCol L;
                    L.x = x; L.m = m; L.w = m == 0 ? 1.0 : u * u;
                    L.y1 = Dgs[j * P1 + m];
                    L.d1 = m == 0 ? 0.0 : L.y1 * (-m) * x;
                    L.y2 = 0; L.d2 = 0;
                    for (int n = m; n <= p; n++) {
                        if (n > m) L.step(n);
                        const double sn = __ldg(&g_hs[n]);
                        Y[j * TS + tidx(n, m)] = L.y1 * sn;
                        if (DIP) D[j * TS + tidx(n, m)] = L.d1 * sn;
                    }
                }
                __syncthreads();
                // phase C: accumulate into this thread's coefficients
    #pragma unroll
                for (int q = 0; q < kHFormPer; q++) {
                    const int n = en[q];
                    if (n < 0) continue;
                    const int m = em_[q], am = m < 0 ? -m : m, ti = tidx(n, am);
                    for (int j = 0; j < nb; j++) {
                        const double *S = Scs + j * 16;
                        const double st = S[1];
                        double2 E = Ems[j * P1 + am];
                        if (m < 0) E = cconj(E);
                        const double ys = Y[j * TS + ti];
                        if (CHG) {
                            const double yr = am == 0 ? ys : ys * st;
                            cfma(acc[q], cmul(cmk(S[2], S[3]), cscal(yr, Fs[j * W + n])), E);
                        }
                        if (DIP) {
                            const double dd = D[j * TS + ti];
                            const double2 fd = Fds[j * P1 + n], fu = Fus[j * P1 + n];
                            double2 A, B = cmk(0, 0);
                            if (am == 0) A = csub(cscal(ys * S[6], fd), cscal(dd * st * S[7], fu));
                            else {
                                A = csub(cscal(ys * st * S[6], fd), cscal(dd * S[7], fu));
                                B = cscal((m > 0 ? am : -am) * ys * S[8], fu);
                            }
                            // ds E (A - i sgn(m) B)
                            const double2 AB = cmk(A.x + B.y, A.y - B.x);
                            cfma(acc[q], cmul(cmk(S[4], S[5]), AB), E);
                        }
                    }
                }
            }
        }
    }
    double2 *o = exps + (size_t)b * NC;
    const double2 ik = cmk(-zk.y, zk.x);
#pragma unroll
    for (int q = 0; q < kHFormPer; q++) {
        const int e = e0 + threadIdx.x + q * kHFormThreads;
        if (e < K) o[e] = cadd(o[e], cmul(acc[q], ik));
    }
}

__host__ __device__ static int max_p(const HLevels &lv)
{
    int pm = 1;
    for (int l = 0; l <= kMaxLevel; l++) pm = lv.p[l] > pm ? lv.p[l] : pm;
    return pm;
}

void launch_hform(bool irreg, const int *boxes, int nboxes, const TreeView &tv, const PointsSoA &src,
                  int ifcharge, int ifdipole, HLevels lv, int NC, double2 zk, double2 *exps, cudaStream_t s,
                  Status &st)
{
    if (nboxes == 0 || !st.ok()) return;
    bool c = ifcharge == 1, d = ifdipole == 1;
    if (!c && !d) return;
    htab_init(s, st);
    const int pm = max_p(lv);
    const dim3 grid(nboxes, div_up((pm + 1) * (pm + 1), kHFormThreads * kHFormPer));
#define FMM_HF2(IR, C, D, CHV, AXV)                                                                           \
    do {                                                                                                      \
        size_t sm = sizeof(double) * HFormSmem<CHV, D, AXV>::doubles(pm);                                    \
        FMM_TRY(st, smem_allow(k_hform<IR, C, D, CHV, AXV>, (int)sm));                                       \
        k_hform<IR, C, D, CHV, AXV><<<grid, kHFormThreads, sm, s>>>(boxes, tv, src, lv, NC, zk, exps);      \
        FMM_COUNT_LAUNCH();                                                                                   \
    } while (0)
#define FMM_HF(IR, C, D, CHV) FMM_HF2(IR, C, D, CHV, 1)
    // chunks of 8 or 16 sources; 4, 2 or 1 at orders whose staging would not
    // fit (above ~54, ~80, ~110).  The chunk size does not change the order of
    // any sum.
    // The sources' set-up (phase A) runs one thread per source, so it takes 32 sources
    // at a time where that fits two CTAs per SM (the tables stay per 8 sources; phases
    // B and C walk the four sub-chunks in order, so no sum changes order).
#define FMM_HF_FIT(IR, C, D, CHV)                                                                             \
    do {                                                                                                      \
        if (sizeof(double) * HFormSmem<kHFormSetCH, D, kHFormSetA>::doubles(pm) <= 110 * 1024)               \
            FMM_HF2(IR, C, D, kHFormSetCH, kHFormSetA);                                                       \
        else if (sizeof(double) * HFormSmem<CHV, D>::doubles(pm) <= 226 * 1024) FMM_HF(IR, C, D, CHV);      \
        else if (sizeof(double) * HFormSmem<4, D>::doubles(pm) <= 226 * 1024) FMM_HF(IR, C, D, 4);          \
        else if (sizeof(double) * HFormSmem<2, D>::doubles(pm) <= 226 * 1024) FMM_HF(IR, C, D, 2);          \
        else FMM_HF(IR, C, D, 1);                                                                             \
    } while (0)
    if (irreg) {
        if (c && d) FMM_HF_FIT(true, true, true, 8);
        else if (c) FMM_HF_FIT(true, true, false, 16);
        else FMM_HF_FIT(true, false, true, 8);
    } else {
        if (c && d) FMM_HF_FIT(false, true, true, 8);
        else if (c) FMM_HF_FIT(false, true, false, 16);
        else FMM_HF_FIT(false, false, true, 8);
    }
#undef FMM_HF_FIT
#undef FMM_HF
#undef FMM_HF2
    FMM_LAUNCH_CHECK(st);
}

// L2P (h3dtaeval_trunc0, src/helmrouts3d.f:2732) at the leaf's own local
// expansion when its level is >= 2, and M2P (h3dmpeval_trunc0, :2405) of the
// multipoles of its list-3 boxes, at the leaf's sources and targets.  CTA per
// leaf, one evaluation point per thread; per expansion the coefficients are
// staged in shared memory and read by all threads of a warp at once
// (broadcast), each thread keeps its point's radial functions in a shared
// column, and walks the orders m (outer) and degrees n (inner) with the
// Legendre column recurrence in registers.
constexpr int kHEvalThreads = 128, kHM2PThreads = 64;

// T threads per CTA: 128, or 32 at orders whose radial columns of 128 points
// would not fit in shared memory beside the coefficients.
template <int T>
__global__ void __launch_bounds__(T) k_heval(const int *leaves, TreeView tv, const double *sx,
                                                        const double *sy, const double *sz, const double *tx,
                                                        const double *ty, const double *tz, HLevels lv, int NC,
                                                        double2 zk, const double2 *mpole, const double2 *local,
                                                        OutSoA outs, OutSoA outt, int do_src, int do_trg,
                                                        int with_l3)
{
    extern __shared__ double2 hsm[];
    const int b = leaves[blockIdx.x];
    const int blev = tv.level[b];
    if (!with_l3 && blev < 2) return;
    const int ns = do_src ? tv.nsrc[b] : 0, nt = do_trg ? tv.ntrg[b] : 0, ne = ns + nt;
    if (ne == 0) return;
    const int pm = max_p(lv);
    const int KM = (pm + 1) * (pm + 1);
    double2 *E = hsm;
    double2 *Fs = hsm + KM;  // radial functions, [n][thread]
    const int t = threadIdx.x;
    const int l3a = tv.l3_start[b], nl3 = with_l3 ? tv.l3_start[b + 1] - l3a : 0;
    // CTA (leaf, y) serves the leaf's point chunks y, y + gridDim.y, ... of T points
    for (int c0 = blockIdx.y * T; c0 < ne; c0 += gridDim.y * T)
    for (int xi = -1; xi < nl3; xi++) {
        int eb;
        const bool isloc = xi < 0;
        if (isloc) {
            if (blev < 2) continue;
            eb = b;
        } else {
            eb = tv.l3_idx[l3a + xi];
            if (tv.nsrc[eb] == 0) continue;
        }
        const int lev = tv.level[eb], p = lv.p[lev];
        const double sc = lv.sc[lev];
        const int K = (p + 1) * (p + 1);
        const double2 *ex = (isloc ? local : mpole) + (size_t)eb * NC;
        __syncthreads();
        for (int i = t; i < K; i += T) E[i] = ex[i];
        __syncthreads();
        const double *c = tv.center + 3L * eb;
        {
            const int e = c0 + t;
            if (e >= ne) continue;
            const bool is_src = e < ns;
            const int i = is_src ? tv.src0[b] + e : tv.trg0[b] + e - ns;
            double px = is_src ? sx[i] : tx[i], py = is_src ? sy[i] : ty[i], pz = is_src ? sz[i] : tz[i];
            const PtGeo g = pt_geo(px - c[0], py - c[1], pz - c[2]);
            double2 *f = Fs + t;
            const double2 z = cscal(g.r, zk);
            if (isloc) {
                if (bess_dev(p > 1 ? p : 1, z, sc, f, nullptr, T)) continue;
            } else {
                if (cabsd(z) < 1.0e-15) continue;
                hank_dev(p > 1 ? p : 1, z, sc, f, nullptr, T);
            }
            const double r = g.r, ct = g.ct, st = g.st, u = -st;
            const double isc = 1.0 / sc, ir = 1.0 / r;
            const double2 zi = cdiv(cmk(1, 0), z), e1 = cmk(g.cp, g.sp);
            double2 pot = cmk(0, 0), ur = cmk(0, 0), ut = cmk(0, 0), up = cmk(0, 0);
            double2 em = cmk(1, 0);
            double ymm = 1.0;
            for (int m = 0; m <= p; m++) {
                if (m == 1) ymm = -sqrt(0.5);
                else if (m > 1) ymm *= u * __ldg(&g_hc[m]);
                if (m > 0) em = cmul(em, e1);
                LegCol L;
                L.x = ct;
                L.m = m;
                L.w = m == 0 ? 1.0 : u * u;
                L.y1 = ymm;
                L.d1 = m == 0 ? 0.0 : ymm * (-m) * ct;
                L.y2 = 0;
                L.d2 = 0;
                for (int n = m; n <= p; n++) {
                    if (n > m) L.step(n);
                    const double sn = __ldg(&g_hs[n]);
                    const double y = L.y1 * sn, dd = L.d1 * sn;
                    const double2 fn = f[n * T];
                    double2 fd, fu;
                    if (isloc) {
                        if (n == 0) { fd = cscal(-sc, f[T]); fu = cmk(0, 0); }
                        else {
                            // j_n' = [n j_{n-1} - (n+1) j_{n+1}] / (2n+1) in the scaled functions
                            const double2 fm = f[(n - 1) * T], fp = f[(n + 1) * T];
                            const double d1 = __ldg(&g_hq[n]), d2 = 1.0 - d1;
                            fd = csub(cscal(d1 * isc, fm), cscal(d2 * sc, fp));
                            fu = cscal(__ldg(&g_hr[n]), cmul(zk, cadd(cscal(sc, fp), cscal(isc, fm))));
                        }
                    } else {
                        fd = n == 0 ? cscal(-isc, f[T]) : csub(cscal(sc, f[(n - 1) * T]), cmul(cscal(n + 1.0, zi), fn));
                        fu = cscal(ir, fn);
                    }
                    fd = cmul(fd, zk);
                    if (m == 0) {
                        const double2 a = E[eidx(n, 0)];
                        cfma(pot, fn, cscal(y, a));
                        cfma(ur, fd, cscal(y, a));
                        cfma(ut, fu, cscal(-dd * st, a));
                    } else {
                        const double2 z2 = cmul(E[eidx(n, m)], em), z3 = cmul(E[eidx(n, -m)], cconj(em));
                        const double2 zs = cadd(z2, z3), zd = csub(z2, z3);
                        cfma(pot, fn, cscal(y * st, zs));
                        cfma(ur, fd, cscal(y * st, zs));
                        cfma(ut, fu, cscal(-dd, zs));
                        cfma(up, fu, cscal(y * m, cmk(-zd.y, zd.x)));  // i m (z2 - z3)
                    }
                }
            }
            // fld = -(ur r-hat + ut theta-hat + up phi-hat)
            const double cp = g.cp, sp = g.sp;
            const double2 fx = cadd(cadd(cscal(st * cp, ur), cscal(ct * cp, ut)), cscal(-sp, up));
            const double2 fy = cadd(cadd(cscal(st * sp, ur), cscal(ct * sp, ut)), cscal(cp, up));
            const double2 fz = csub(cscal(ct, ur), cscal(st, ut));
            double2 *po = is_src ? outs.pot : outt.pot;
            double2 *ox = is_src ? outs.fx : outt.fx, *oy = is_src ? outs.fy : outt.fy, *oz = is_src ? outs.fz : outt.fz;
            if (po) po[i] = cadd(po[i], pot);
            if (ox) {
                ox[i] = csub(ox[i], fx);
                oy[i] = csub(oy[i], fy);
                oz[i] = csub(oz[i], fz);
            }
        }
    }
}

// M2P of the list-3 boxes (h3dmpeval_trunc0, src/helmrouts3d.f:2405) apart from the
// local expansions.  List 3 is very uneven on adaptive trees (on a sphere surface
// most leaves have none and a few have over a hundred), so the work is cut into
// items of one leaf, one chunk of T of its points and one group of at most
// kHM2PGroup of its list-3 boxes, one CTA each.  An item writes its points' sums
// over its group to its own slot of a scratch array; k_hm2p_add then adds the
// groups' sums to the outputs in group order, so results do not depend on the
// schedule.  The scaled Hankel functions f_n = h_n(z) scale^n of h3dall (the
// upward recurrence f_{n+1} = (2n+1) scale/z f_n - scale^2 f_{n-1} of hank_dev,
// from f_0 = e^{iz}/(iz) and f_1) are regenerated along each order's run of
// degrees from the pair (f_{m-1}, f_m) that the previous order's run passed, so
// every value is the one hank_dev stores and shared memory holds only the staged
// multipole.
constexpr int kHM2PGroup = 16;

__global__ void k_hm2p_count(const int *leaves, int nleaves, TreeView tv, int do_src, int do_trg, int *cnt)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nleaves) return;
    const int b = leaves[l];
    const int ne = (do_src ? tv.nsrc[b] : 0) + (do_trg ? tv.ntrg[b] : 0);
    const int nl3 = tv.l3_start[b + 1] - tv.l3_start[b];
    cnt[l] = (ne > 0 && nl3 > 0) ? ((ne + kHM2PThreads - 1) / kHM2PThreads) * ((nl3 + kHM2PGroup - 1) / kHM2PGroup)
                                 : 0;
}

// The leaf of work item `item`: the last l with off[l] <= item (leaves without items
// share their offset with the next leaf).
__device__ __forceinline__ int hm2p_leaf(const int *off, int nleaves, int item)
{
    int lo = 0, hi = nleaves - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int T>
__global__ void __launch_bounds__(T) k_hm2p(const int *leaves, int nleaves, const int *off, TreeView tv,
                                             const double *sx, const double *sy, const double *sz, const double *tx,
                                             const double *ty, const double *tz, HLevels lv, int NC, double2 zk,
                                             const double2 *mpole, int do_src, int do_trg, double *part)
{
    extern __shared__ double2 hsm[];
    const int item = blockIdx.x;
    const int l = hm2p_leaf(off, nleaves, item), b = leaves[l];
    const int ns = do_src ? tv.nsrc[b] : 0, nt = do_trg ? tv.ntrg[b] : 0, ne = ns + nt;
    const int l3a = tv.l3_start[b], nl3 = tv.l3_start[b + 1] - l3a;
    const int ngr = (nl3 + kHM2PGroup - 1) / kHM2PGroup;
    const int local = item - off[l], ck = local / ngr, grp = local - ck * ngr;
    const int c0 = ck * T, x1 = min(nl3, (grp + 1) * kHM2PGroup);
    double2 *E = hsm;
    const int t = threadIdx.x;
    // this item's sums at its point: pot, then -fld (x, y, z)
    double2 spot = cmk(0, 0), sfx = cmk(0, 0), sfy = cmk(0, 0), sfz = cmk(0, 0);
    for (int xi = grp * kHM2PGroup; xi < x1; xi++) {
        const int eb = tv.l3_idx[l3a + xi];
        if (tv.nsrc[eb] == 0) continue;
        const int lev = tv.level[eb], p = lv.p[lev];
        const double sc = lv.sc[lev];
        const int K = (p + 1) * (p + 1);
        const double2 *ex = mpole + (size_t)eb * NC;
        __syncthreads();
        for (int i = t; i < K; i += T) E[i] = ex[i];
        __syncthreads();
        const double *c = tv.center + 3L * eb;
        {
            const int e = c0 + t;
            if (e >= ne) continue;
            const bool is_src = e < ns;
            const int i = is_src ? tv.src0[b] + e : tv.trg0[b] + e - ns;
            double px = is_src ? sx[i] : tx[i], py = is_src ? sy[i] : ty[i], pz = is_src ? sz[i] : tz[i];
            const PtGeo g = pt_geo(px - c[0], py - c[1], pz - c[2]);
            const double2 z = cscal(g.r, zk);
            if (cabsd(z) < 1.0e-15) continue;
            const double r = g.r, ct = g.ct, st = g.st, u = -st;
            const double isc = 1.0 / sc, ir = 1.0 / r;
            const double2 zi = cdiv(cmk(1, 0), z), e1 = cmk(g.cp, g.sp);
            // f_0, f_1 as hank_dev (h3d01, src/helmrouts3d.f:666-704)
            const double2 h0 = cdiv(cexpi(z), cmk(-z.y, z.x));
            const double2 f1 = cscal(sc, cmul(h0, cmk(zi.x, zi.y - 1.0)));
            const double s2 = sc * sc;
            const double2 zs = cscal(sc, zi);
            double2 pot = cmk(0, 0), ur = cmk(0, 0), ut = cmk(0, 0), up = cmk(0, 0);
            double2 em = cmk(1, 0);
            double ymm = 1.0;
            double2 sa = cmk(0, 0), sb = h0;   // f_{m-1}, f_m at the start of order m
            for (int m = 0; m <= p; m++) {
                if (m == 1) ymm = -sqrt(0.5);
                else if (m > 1) ymm *= u * __ldg(&g_hc[m]);
                if (m > 0) em = cmul(em, e1);
                LegCol L;
                L.x = ct;
                L.m = m;
                L.w = m == 0 ? 1.0 : u * u;
                L.y1 = ymm;
                L.d1 = m == 0 ? 0.0 : ymm * (-m) * ct;
                L.y2 = 0;
                L.d2 = 0;
                double2 fa = sa, fb = sb;      // f_{n-1}, f_n
                for (int n = m; n <= p; n++) {
                    if (n > m) L.step(n);
                    const double sn = __ldg(&g_hs[n]);
                    const double y = L.y1 * sn, dd = L.d1 * sn;
                    const double2 fn = fb;
                    double2 fd = n == 0 ? cscal(-isc, f1) : csub(cscal(sc, fa), cmul(cscal(n + 1.0, zi), fn));
                    const double2 fu = cscal(ir, fn);
                    fd = cmul(fd, zk);
                    if (m == 0) {
                        const double2 a = E[eidx(n, 0)];
                        cfma(pot, fn, cscal(y, a));
                        cfma(ur, fd, cscal(y, a));
                        cfma(ut, fu, cscal(-dd * st, a));
                    } else {
                        const double2 z2 = cmul(E[eidx(n, m)], em), z3 = cmul(E[eidx(n, -m)], cconj(em));
                        const double2 zs2 = cadd(z2, z3), zd = csub(z2, z3);
                        cfma(pot, fn, cscal(y * st, zs2));
                        cfma(ur, fd, cscal(y * st, zs2));
                        cfma(ut, fu, cscal(-dd, zs2));
                        cfma(up, fu, cscal(y * m, cmk(-zd.y, zd.x)));  // i m (z2 - z3)
                    }
                    if (n < p) {
                        const double2 fc = n == 0 ? f1 : csub(cmul(cscal(2 * n + 1.0, zs), fb), cscal(s2, fa));
                        fa = fb;
                        fb = fc;
                        if (n == m) { sa = fa; sb = fb; }   // (f_m, f_{m+1}) start order m + 1
                    }
                }
            }
            const double cp = g.cp, sp = g.sp;
            spot = cadd(spot, pot);
            sfx = csub(sfx, cadd(cadd(cscal(st * cp, ur), cscal(ct * cp, ut)), cscal(-sp, up)));
            sfy = csub(sfy, cadd(cadd(cscal(st * sp, ur), cscal(ct * sp, ut)), cscal(cp, up)));
            sfz = csub(sfz, csub(cscal(ct, ur), cscal(st, ut)));
        }
    }
    double *o = part + (size_t)item * 8 * T + t;
    o[0] = spot.x; o[T] = spot.y; o[2 * T] = sfx.x; o[3 * T] = sfx.y;
    o[4 * T] = sfy.x; o[5 * T] = sfy.y; o[6 * T] = sfz.x; o[7 * T] = sfz.y;
}

// Adds the list-3 groups' sums of a leaf to its outputs, group by group.
template <int T>
__global__ void k_hm2p_add(const int *leaves, const int *off, TreeView tv, OutSoA outs, OutSoA outt, int do_src,
                           int do_trg, const double *part)
{
    const int l = blockIdx.x, b = leaves[l];
    const int ns = do_src ? tv.nsrc[b] : 0, nt = do_trg ? tv.ntrg[b] : 0, ne = ns + nt;
    const int nl3 = tv.l3_start[b + 1] - tv.l3_start[b];
    if (ne == 0 || nl3 == 0) return;
    const int ngr = (nl3 + kHM2PGroup - 1) / kHM2PGroup, nch = (ne + T - 1) / T;
    for (int ck = blockIdx.y; ck < nch; ck += gridDim.y) {
        const int e = ck * T + threadIdx.x;
        if (e >= ne) continue;
        const bool is_src = e < ns;
        const int i = is_src ? tv.src0[b] + e : tv.trg0[b] + e - ns;
        double2 *po = is_src ? outs.pot : outt.pot;
        double2 *ox = is_src ? outs.fx : outt.fx, *oy = is_src ? outs.fy : outt.fy, *oz = is_src ? outs.fz : outt.fz;
        double2 vp = po ? po[i] : cmk(0, 0), vx = ox ? ox[i] : cmk(0, 0), vy = ox ? oy[i] : cmk(0, 0),
                vz = ox ? oz[i] : cmk(0, 0);
        for (int g = 0; g < ngr; g++) {
            const double *q = part + (size_t)(off[l] + ck * ngr + g) * 8 * T + threadIdx.x;
            vp = cadd(vp, cmk(q[0], q[T]));
            vx = cadd(vx, cmk(q[2 * T], q[3 * T]));
            vy = cadd(vy, cmk(q[4 * T], q[5 * T]));
            vz = cadd(vz, cmk(q[6 * T], q[7 * T]));
        }
        if (po) po[i] = vp;
        if (ox) {
            ox[i] = vx;
            oy[i] = vy;
            oz[i] = vz;
        }
    }
}

// L2P of the leaves' local expansions (h3dtaeval_trunc0, src/helmrouts3d.f:2732)
// with half a warp per point.  A warp takes its points in batches of
// kHL2PBatch: first each of 16 lanes builds one point's scaled Bessel column
// (Miller's downward recurrence, so stored) in shared memory, then each half-warp
// evaluates one point at a time, its 16 lanes sharing the orders m (lane l
// takes m = l and 31 - l, mod 32, so the triangle of degrees splits evenly),
// and the lanes' sums are added by shuffles.  The coefficients are staged
// diagonal-major, entry (s = n - m, m) holding E(n, m) and E(n, -m), so lanes at
// the same step read consecutive entries.  Shared memory per point is one
// radial column instead of one per thread, which doubles the CTAs per SM.
constexpr int kHL2PWarps = 4, kHL2PBatch = 16;

static size_t hl2p_smem(int pm)
{
    return (size_t)(pm + 1) * (pm + 2) * sizeof(double2) +
           (size_t)kHL2PWarps * kHL2PBatch * ((pm + 2) * sizeof(double2) + sizeof(int));
}

__global__ void __launch_bounds__(32 * kHL2PWarps) k_hl2p(const int *leaves, TreeView tv, const double *sx,
                                                        const double *sy, const double *sz, const double *tx,
                                                        const double *ty, const double *tz, HLevels lv, int NC,
                                                        double2 zk, const double2 *local, OutSoA outs, OutSoA outt,
                                                        int do_src, int do_trg, int pm)
{
    extern __shared__ double2 hsm[];
    const int b = leaves[blockIdx.x];
    const int lev = tv.level[b];
    if (lev < 2) return;
    const int ns = do_src ? tv.nsrc[b] : 0, nt = do_trg ? tv.ntrg[b] : 0, ne = ns + nt;
    if (ne == 0) return;
    const int p = lv.p[lev], P1 = p + 1, P2 = pm + 2;
    const double sc = lv.sc[lev], isc = 1.0 / sc;
    const int ntri = (p + 1) * (p + 2) / 2;
    double2 *Ep = hsm;                                          // [ntri][2]
    double2 *Fall = hsm + (size_t)(pm + 1) * (pm + 2);          // [warps][batch][pm + 2]
    int *okall = (int *)(Fall + (size_t)kHL2PWarps * kHL2PBatch * P2);
    // diagonal index d(s, m) = base(s) + m, base(s) = s (p + 1) - s (s - 1) / 2
    const double2 *ex = local + (size_t)b * NC;
    for (int d = threadIdx.x; d < ntri; d += blockDim.x) {
        int sd = 0;
        while (sd + 1 <= p && (sd + 1) * P1 - (sd + 1) * sd / 2 <= d) sd++;
        const int m = d - (sd * P1 - sd * (sd - 1) / 2), n = m + sd;
        Ep[2 * d] = ex[eidx(n, m)];
        Ep[2 * d + 1] = ex[eidx(n, -m)];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
    double2 *F = Fall + (size_t)warp * kHL2PBatch * P2;
    int *okp = okall + warp * kHL2PBatch;
    const double *c = tv.center + 3L * b;
    auto point = [&](int e, double &px, double &py, double &pz) {
        const bool is_src = e < ns;
        const int i = is_src ? tv.src0[b] + e : tv.trg0[b] + e - ns;
        px = is_src ? sx[i] : tx[i];
        py = is_src ? sy[i] : ty[i];
        pz = is_src ? sz[i] : tz[i];
        return i;
    };
    for (int base = warp * kHL2PBatch; base < ne; base += kHL2PWarps * kHL2PBatch) {
        if (lane < kHL2PBatch) {
            const int e = base + lane;
            int ok = 0;
            if (e < ne) {
                double px, py, pz;
                point(e, px, py, pz);
                const PtGeo g = pt_geo(px - c[0], py - c[1], pz - c[2]);
                ok = bess_dev(p > 1 ? p : 1, cscal(g.r, zk), sc, F + lane * P2, nullptr, 1) == 0;
            }
            okp[lane] = ok;
        }
        __syncwarp();
        for (int it = 0; it < kHL2PBatch / 2; it++) {
            const int pt = 2 * it + half, e = base + pt;
            const bool act = e < ne && okp[pt];
            double2 pot = cmk(0, 0), ur = cmk(0, 0), ut = cmk(0, 0), up = cmk(0, 0);
            PtGeo g = {1.0, 1.0, 0.0, 1.0, 0.0};
            int oi = 0;
            if (act) {
                double px, py, pz;
                oi = point(e, px, py, pz);
                g = pt_geo(px - c[0], py - c[1], pz - c[2]);
                const double ct = g.ct, st = g.st, u = -st;
                const double2 e1 = cmk(g.cp, g.sp);
                const double2 *f = F + pt * P2;
                for (int mb = 0; mb <= p; mb += 32) {
#pragma unroll 1
                    for (int which = 0; which < 2; which++) {
                        const int m = mb + (which == 0 ? hl : 31 - hl);
                        if (m > p) continue;
                        double ymm = 1.0;
                        if (m >= 1) {
                            ymm = -sqrt(0.5);
                            for (int k = 2; k <= m; k++) ymm *= u * __ldg(&g_hc[k]);
                        }
                        double2 em = cmk(1, 0), bp = e1;   // e^{i m phi} by binary powers
                        for (int t = m; t; t >>= 1) {
                            if (t & 1) em = cmul(em, bp);
                            bp = cmul(bp, bp);
                        }
                        LegCol L;
                        L.x = ct;
                        L.m = m;
                        L.w = m == 0 ? 1.0 : u * u;
                        L.y1 = ymm;
                        L.d1 = m == 0 ? 0.0 : ymm * (-m) * ct;
                        L.y2 = 0;
                        L.d2 = 0;
                        int d = m;
                        for (int n = m; n <= p; n++) {
                            if (n > m) {
                                L.step(n);
                                d += P1 - (n - m - 1);
                            }
                            const double sn = __ldg(&g_hs[n]);
                            const double y = L.y1 * sn, dd = L.d1 * sn;
                            const double2 fn = f[n];
                            double2 fd, fu;
                            if (n == 0) {
                                fd = cscal(-sc, f[1]);
                                fu = cmk(0, 0);
                            } else {
                                // j_n' = [n j_{n-1} - (n+1) j_{n+1}] / (2n+1) in the scaled functions
                                const double2 fm = f[n - 1], fp = f[n + 1];
                                const double d1 = __ldg(&g_hq[n]), d2 = 1.0 - d1;
                                fd = csub(cscal(d1 * isc, fm), cscal(d2 * sc, fp));
                                fu = cscal(__ldg(&g_hr[n]), cmul(zk, cadd(cscal(sc, fp), cscal(isc, fm))));
                            }
                            fd = cmul(fd, zk);
                            if (m == 0) {
                                const double2 a = Ep[2 * d];
                                cfma(pot, fn, cscal(y, a));
                                cfma(ur, fd, cscal(y, a));
                                cfma(ut, fu, cscal(-dd * st, a));
                            } else {
                                const double2 z2 = cmul(Ep[2 * d], em), z3 = cmul(Ep[2 * d + 1], cconj(em));
                                const double2 zs = cadd(z2, z3), zd = csub(z2, z3);
                                cfma(pot, fn, cscal(y * st, zs));
                                cfma(ur, fd, cscal(y * st, zs));
                                cfma(ut, fu, cscal(-dd, zs));
                                cfma(up, fu, cscal(y * m, cmk(-zd.y, zd.x)));  // i m (z2 - z3)
                            }
                        }
                    }
                }
            }
            // the half-warp's sums (offsets below 16 stay within the half)
#pragma unroll
            for (int o = 8; o >= 1; o >>= 1) {
                pot.x += __shfl_xor_sync(0xffffffffu, pot.x, o);
                pot.y += __shfl_xor_sync(0xffffffffu, pot.y, o);
                ur.x += __shfl_xor_sync(0xffffffffu, ur.x, o);
                ur.y += __shfl_xor_sync(0xffffffffu, ur.y, o);
                ut.x += __shfl_xor_sync(0xffffffffu, ut.x, o);
                ut.y += __shfl_xor_sync(0xffffffffu, ut.y, o);
                up.x += __shfl_xor_sync(0xffffffffu, up.x, o);
                up.y += __shfl_xor_sync(0xffffffffu, up.y, o);
            }
            if (act && hl == 0) {
                const double ct = g.ct, st = g.st, cp = g.cp, sp = g.sp;
                const double2 fx = cadd(cadd(cscal(st * cp, ur), cscal(ct * cp, ut)), cscal(-sp, up));
                const double2 fy = cadd(cadd(cscal(st * sp, ur), cscal(ct * sp, ut)), cscal(cp, up));
                const double2 fz = csub(cscal(ct, ur), cscal(st, ut));
                const bool is_src = e < ns;
                double2 *po = is_src ? outs.pot : outt.pot;
                double2 *ox = is_src ? outs.fx : outt.fx, *oy = is_src ? outs.fy : outt.fy,
                        *oz = is_src ? outs.fz : outt.fz;
                if (po) po[oi] = cadd(po[oi], pot);
                if (ox) {
                    ox[oi] = csub(ox[oi], fx);
                    oy[oi] = csub(oy[oi], fy);
                    oz[oi] = csub(oz[oi], fz);
                }
            }
        }
        __syncwarp();
    }
}

void launch_heval(const int *leaves, int nleaves, const TreeView &tv, const double *sx, const double *sy,
                  const double *sz, const double *tx, const double *ty, const double *tz, HLevels lv, int NC,
                  double2 zk, const double2 *mpole, const double2 *local, OutSoA outs, OutSoA outt, int do_src,
                  int do_trg, cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok() || (!do_src && !do_trg)) return;
    htab_init(s, st);
    int pm = max_p(lv);
    // L2P (the leaves' own local expansions) first, then M2P of list 3
    size_t sm = sizeof(double2) * ((size_t)(pm + 1) * (pm + 1) + (size_t)(pm + 2) * kHEvalThreads);
    if (hl2p_smem(pm) <= 100 * 1024) {
        const size_t sl = hl2p_smem(pm);
        FMM_TRY(st, smem_allow(k_hl2p, (int)sl));
        k_hl2p<<<nleaves, 32 * kHL2PWarps, sl, s>>>(leaves, tv, sx, sy, sz, tx, ty, tz, lv, NC, zk, local, outs, outt,
                                                    do_src, do_trg, pm);
    } else if (sm <= 226 * 1024) {
        FMM_TRY(st, smem_allow(k_heval<kHEvalThreads>, (int)sm));
        k_heval<kHEvalThreads><<<dim3(nleaves, 2), kHEvalThreads, sm, s>>>(leaves, tv, sx, sy, sz, tx, ty, tz, lv,
                                                                           NC, zk, mpole, local, outs, outt, do_src,
                                                                           do_trg, 0);
    } else {
        sm = sizeof(double2) * ((size_t)(pm + 1) * (pm + 1) + (size_t)(pm + 2) * 32);
        FMM_TRY(st, smem_allow(k_heval<32>, (int)sm));
        k_heval<32><<<dim3(nleaves, 8), 32, sm, s>>>(leaves, tv, sx, sy, sz, tx, ty, tz, lv, NC, zk, mpole, local,
                                                     outs, outt, do_src, do_trg, 0);
    }
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    // M2P work items: (leaf, chunk of points, group of list-3 boxes)
    DBuf<int> cnt, off;
    if (!cnt.alloc(nleaves, s, st) || !off.alloc(nleaves, s, st)) return;
    k_hm2p_count<<<div_up(nleaves, 256), 256, 0, s>>>(leaves, nleaves, tv, do_src, do_trg, cnt.p);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    int nitems = 0;
    scan_exclusive_int(cnt.p, off.p, nleaves, s, st, &nitems);
    if (!st.ok() || nitems == 0) return;
    DBuf<double> part;
    if (!part.alloc((size_t)nitems * 8 * kHM2PThreads, s, st)) return;
    sm = sizeof(double2) * (size_t)(pm + 1) * (pm + 1);
    FMM_TRY(st, smem_allow(k_hm2p<kHM2PThreads>, (int)sm));
    k_hm2p<kHM2PThreads><<<nitems, kHM2PThreads, sm, s>>>(leaves, nleaves, off.p, tv, sx, sy, sz, tx, ty, tz, lv, NC,
                                                          zk, mpole, do_src, do_trg, part.p);
    FMM_COUNT_LAUNCH();
    k_hm2p_add<kHM2PThreads><<<dim3(nleaves, 4), kHM2PThreads, 0, s>>>(leaves, off.p, tv, outs, outt, do_src, do_trg,
                                                                       part.p);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// ================================================================ near field
// One source at one evaluation point: hpotfld3d (src/helmrouts3d.f:1335-1417)
// and hpotfld3d_dp (:1844-1924) in closed form,
//   g = e^{ikr}/r,  charge: pot q g,  fld q g (1 - ikr) / r^2 (x - y)
//   dipole: pot d (1 - ikr) g / r^2 (v . (x - y)),
//           fld -d [g (3ik/r^2 + k^2/r - 3/r^3)/r (v . (x - y)) (x - y) + (1 - ikr) g / r^2 v]
template <bool CHG, bool DIP>
__device__ __forceinline__ void hpair(double dx, double dy, double dz, double2 zk, double2 k2, double2 q, double2 ds,
                                      double vx, double vy, double vz, double2 &pot, double2 &fx, double2 &fy,
                                      double2 &fz)
{
    double r2 = dx * dx + dy * dy + dz * dz;
    // 1/r from one reciprocal square root (within an ulp of 1/sqrt), r = r^2 / r
    double ri = rsqrt(r2), r = r2 * ri, ri2 = ri * ri;
    double s, c;
    sincos(zk.x * r, &s, &c);
    double ee = zk.y == 0.0 ? ri : exp(-zk.y * r) * ri;
    double2 g = cmk(c * ee, s * ee);
    // (1 - ikr) g / r^2
    double2 h = cscal(ri2, cmul(cmk(1.0 + zk.y * r, -zk.x * r), g));
    if (CHG) {
        cfma(pot, q, g);
        double2 qh = cmul(q, h);
        crfma(fx, dx, qh);
        crfma(fy, dy, qh);
        crfma(fz, dz, qh);
    }
    if (DIP) {
        double dot = dx * vx + dy * vy + dz * vz;
        double2 dh = cmul(ds, h);
        crfma(pot, dot, dh);
        // 3ik/r^2 + k^2/r - 3/r^3
        double2 t = cadd(cscal(3 * ri2, cmk(-zk.y, zk.x)), cscal(ri, k2));
        t.x -= 3 * ri2 * ri;
        double2 F = cscal(ri * dot, cmul(cmul(ds, g), t));
        fx = csub(fx, cadd(cscal(dx, F), cscal(vx, dh)));
        fy = csub(fy, cadd(cscal(dy, F), cscal(vy, dh)));
        fz = csub(fz, cadd(cscal(dz, F), cscal(vz, dh)));
    }
}

constexpr int kHP2PThreads = 128;

// P2P: hfmm3dpart_direct_self / _targ (src/hfmm3dpart.f:1092-1262).  CTA per
// leaf, one evaluation point (sources, then targets) per thread, source boxes
// self and list 1 staged through shared memory, the self pair skipped by index.
template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kHP2PThreads) k_hp2p(const int *leaves, TreeView tv, PointsSoA src,
                                                      const double *tx, const double *ty, const double *tz,
                                                      double2 zk, OutSoA outs, OutSoA outt, int do_src, int do_trg)
{
    __shared__ double sx[kHP2PThreads], sy[kHP2PThreads], sz[kHP2PThreads];
    __shared__ double2 sq[kHP2PThreads], sd[kHP2PThreads];
    __shared__ double svx[kHP2PThreads], svy[kHP2PThreads], svz[kHP2PThreads];
    const int b = leaves[blockIdx.x];
    const int s0 = tv.src0[b], ns = do_src ? tv.nsrc[b] : 0;
    const int t0 = tv.trg0[b], nt = do_trg ? tv.ntrg[b] : 0;
    const int ne = ns + nt;
    const int l1a = tv.l1_start[b], nl = 1 + tv.l1_start[b + 1] - l1a;
    const double2 k2 = cmul(zk, zk);
    // CTA (leaf, y) serves the leaf's point chunks y, y + gridDim.y, ...
    for (int e0 = blockIdx.y * kHP2PThreads; e0 < ne; e0 += gridDim.y * kHP2PThreads) {
        const int e = e0 + threadIdx.x;
        const bool act = e < ne;
        const bool is_src = e < ns;
        double ex = 0, ey = 0, ez = 0;
        int self = -1;
        if (act) {
            if (is_src) { int i = s0 + e; ex = src.x[i]; ey = src.y[i]; ez = src.z[i]; self = i; }
            else { int i = t0 + e - ns; ex = tx[i]; ey = ty[i]; ez = tz[i]; }
        }
        double2 pot = cmk(0, 0), fx = cmk(0, 0), fy = cmk(0, 0), fz = cmk(0, 0);
        for (int j = 0; j < nl; j++) {
            const int jb = j == 0 ? b : tv.l1_idx[l1a + j - 1];
            const int js0 = tv.src0[jb], jn = tv.nsrc[jb];
            for (int c0 = 0; c0 < jn; c0 += kHP2PThreads) {
                const int cn = min(kHP2PThreads, jn - c0);
                __syncthreads();
                if (threadIdx.x < cn) {
                    int i = js0 + c0 + threadIdx.x;
                    sx[threadIdx.x] = src.x[i]; sy[threadIdx.x] = src.y[i]; sz[threadIdx.x] = src.z[i];
                    if (CHG) sq[threadIdx.x] = src.q[i];
                    if (DIP) {
                        sd[threadIdx.x] = src.dq[i];
                        svx[threadIdx.x] = src.vx[i]; svy[threadIdx.x] = src.vy[i]; svz[threadIdx.x] = src.vz[i];
                    }
                }
                __syncthreads();
                if (!act) continue;
                const int selfk = self - (js0 + c0);
                // the self pair adds exact zeros (no strength, unit offset) instead of a branch,
                // so consecutive pairs interleave
#pragma unroll 2
                for (int k = 0; k < cn; k++) {
                    const bool me = k == selfk;
                    hpair<CHG, DIP>(me ? 1.0 : ex - sx[k], me ? 0.0 : ey - sy[k], me ? 0.0 : ez - sz[k], zk, k2,
                                    CHG && !me ? sq[k] : cmk(0, 0), DIP && !me ? sd[k] : cmk(0, 0),
                                    DIP && !me ? svx[k] : 0.0, DIP && !me ? svy[k] : 0.0, DIP && !me ? svz[k] : 0.0,
                                    pot, fx, fy, fz);
                }
            }
        }
        if (act) {
            double2 *po = is_src ? outs.pot : outt.pot;
            double2 *ox = is_src ? outs.fx : outt.fx, *oy = is_src ? outs.fy : outt.fy, *oz = is_src ? outs.fz : outt.fz;
            int i = is_src ? s0 + e : t0 + e - ns;
            if (po) po[i] = cadd(po[i], pot);
            if (ox) {
                ox[i] = cadd(ox[i], fx);
                oy[i] = cadd(oy[i], fy);
                oz[i] = cadd(oz[i], fz);
            }
        }
    }
}

void launch_hp2p(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                 const double *ty, const double *tz, double2 zk, OutSoA outs, OutSoA outt, int ifcharge,
                 int ifdipole, int ifpot, int iffld, int ifpottarg, int iffldtarg, cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok()) return;
    int do_src = (ifpot == 1 || iffld == 1), do_trg = (ifpottarg == 1 || iffldtarg == 1);
    bool c = ifcharge == 1, d = ifdipole == 1;
    if (!c && !d) return;
    if (c && d) k_hp2p<true, true><<<dim3(nleaves, 4), kHP2PThreads, 0, s>>>(leaves, tv, src, tx, ty, tz, zk, outs, outt, do_src, do_trg);
    else if (c) k_hp2p<true, false><<<dim3(nleaves, 4), kHP2PThreads, 0, s>>>(leaves, tv, src, tx, ty, tz, zk, outs, outt, do_src, do_trg);
    else k_hp2p<false, true><<<dim3(nleaves, 4), kHP2PThreads, 0, s>>>(leaves, tv, src, tx, ty, tz, zk, outs, outt, do_src, do_trg);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// Direct sum (h3dpartdirect, src/hfmm3dpart.f:1268-1401): blockIdx.x tiles
// the evaluation points, blockIdx.y the sources; partial sums per source chunk
// go to scratch and are reduced in chunk order.
constexpr int kHDirThreads = 128;

template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kHDirThreads) k_hdirect(int nsrc, PointsSoA src, int neval, const double *ex,
                                                         const double *ey, const double *ez, const int *skip,
                                                         int self, double2 zk, int chunk, double2 *part)
{
    __shared__ double sx[kHDirThreads], sy[kHDirThreads], sz[kHDirThreads];
    __shared__ double2 sq[kHDirThreads], sd[kHDirThreads];
    __shared__ double svx[kHDirThreads], svy[kHDirThreads], svz[kHDirThreads];
    const int e = blockIdx.x * kHDirThreads + threadIdx.x;
    const bool act = e < neval;
    const int j0 = blockIdx.y * chunk, j1 = min(nsrc, j0 + chunk);
    double px = act ? ex[e] : 0, py = act ? ey[e] : 0, pz = act ? ez[e] : 0;
    int sk = act ? (skip ? skip[e] : (self ? e : -1)) : -1;
    const double2 k2 = cmul(zk, zk);
    double2 pot = cmk(0, 0), fx = cmk(0, 0), fy = cmk(0, 0), fz = cmk(0, 0);
    for (int c0 = j0; c0 < j1; c0 += kHDirThreads) {
        const int cn = min(kHDirThreads, j1 - c0);
        __syncthreads();
        if (threadIdx.x < cn) {
            int i = c0 + threadIdx.x;
            sx[threadIdx.x] = src.x[i]; sy[threadIdx.x] = src.y[i]; sz[threadIdx.x] = src.z[i];
            if (CHG) sq[threadIdx.x] = src.q[i];
            if (DIP) {
                sd[threadIdx.x] = src.dq[i];
                svx[threadIdx.x] = src.vx[i]; svy[threadIdx.x] = src.vy[i]; svz[threadIdx.x] = src.vz[i];
            }
        }
        __syncthreads();
        if (!act) continue;
        for (int k = 0; k < cn; k++) {
            if (c0 + k == sk) continue;
            hpair<CHG, DIP>(px - sx[k], py - sy[k], pz - sz[k], zk, k2, CHG ? sq[k] : cmk(0, 0),
                            DIP ? sd[k] : cmk(0, 0), DIP ? svx[k] : 0.0, DIP ? svy[k] : 0.0, DIP ? svz[k] : 0.0,
                            pot, fx, fy, fz);
        }
    }
    if (act) {
        double2 *o = part + ((size_t)blockIdx.y * neval + e) * 4;
        o[0] = pot; o[1] = fx; o[2] = fy; o[3] = fz;
    }
}

__global__ void k_hdirect_reduce(int neval, int nchunk, const double2 *part, OutSoA out)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= neval) return;
    double2 a[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    for (int c = 0; c < nchunk; c++)
        for (int q = 0; q < 4; q++) a[q] = cadd(a[q], part[((size_t)c * neval + e) * 4 + q]);
    if (out.pot) out.pot[e] = a[0];
    if (out.fx) { out.fx[e] = a[1]; out.fy[e] = a[2]; out.fz[e] = a[3]; }
}

void launch_hdirect(int nsrc, const PointsSoA &src, int ifcharge, int ifdipole, int neval, const double *ex,
                    const double *ey, const double *ez, const int *skip, int self, double2 zk, OutSoA out,
                    cudaStream_t s, Status &st)
{
    if (neval == 0 || !st.ok()) return;
    bool c = ifcharge == 1, d = ifdipole == 1;
    int gx = div_up(neval, kHDirThreads);
    // enough source chunks to fill the GPU (about 4 CTAs per SM), at least 1024 sources each
    int nchunk = std::max(1, std::min(div_up(std::max(nsrc, 1), 1024), div_up(148 * 4, gx)));
    int chunk = div_up(std::max(nsrc, 1), nchunk);
    nchunk = div_up(std::max(nsrc, 1), chunk);
    DBuf<double2> part;
    if (!part.alloc((size_t)nchunk * neval * 4, s, st)) return;
    if ((!c && !d) || nsrc == 0) part.zero(st);
    dim3 g(gx, nchunk);
    if (nsrc > 0) {
        if (c && d) { k_hdirect<true, true><<<g, kHDirThreads, 0, s>>>(nsrc, src, neval, ex, ey, ez, skip, self, zk, chunk, part.p); FMM_COUNT_LAUNCH(); }
        else if (c) { k_hdirect<true, false><<<g, kHDirThreads, 0, s>>>(nsrc, src, neval, ex, ey, ez, skip, self, zk, chunk, part.p); FMM_COUNT_LAUNCH(); }
        else if (d) { k_hdirect<false, true><<<g, kHDirThreads, 0, s>>>(nsrc, src, neval, ex, ey, ez, skip, self, zk, chunk, part.p); FMM_COUNT_LAUNCH(); }
    }
    k_hdirect_reduce<<<div_up(neval, 256), 256, 0, s>>>(neval, nchunk, part.p, out); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

}  // namespace fmm
