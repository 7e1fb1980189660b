// Laplace Hessians on the GPU (FP64).
//
// Near field: pair formulas of lpotfld3dhess / lpotfld3dhess_dp
// (src/laprouts3d.f:5442-5536, 5619-5735), one evaluation point per thread,
// sources staged through shared memory, self excluded by index as in
// lfmm3dpart_direct_self (src/lfmm3dpart.f:1193).
//
// Far field: the reference shifts the expansion to an order-2 local
// expansion about the point (l3dtaevalhessd_trunc, src/laprouts3d.f:7682;
// l3dmpevalhessd_trunc, :7194) and reads the Hessian from its degree-2
// coefficients.  Here each derivative is applied to the coefficients instead:
// d/dz, D+ = d/dx + i d/dy and D- = d/dx - i d/dy map the coefficients of a
// local expansion of order p to those of a local expansion of order p - 1
// (a multipole: order p + 1) by one ladder step per coefficient, so the five
// second derivatives d2/dz2, D+D+, D-D-, d/dz D+, d/dz D- are five
// coefficient arrays, each dotted with the point's solid harmonics:
//   dxx = ((D+D+ + D-D-)/2 - dzz)/2,   dyy = (-(D+D+ + D-D-)/2 - dzz)/2,
//   dxy = (D+D+ - D-D-)/(4i),   dxz = (dzD+ + dzD-)/2,   dyz = (dzD+ - dzD-)/(2i)
// (dxx + dyy = -dzz for a harmonic function).  The coefficient arrays are
// built in shared memory per source box, in as many phases as shared memory
// requires, and every point's harmonics are generated on the fly.
#include "hess.cuh"

#include <algorithm>
#include <mutex>

namespace fmm {

// ---------------------------------------------------------------- tables
constexpr int kHTabP = kHessMaxP + 2;
constexpr int kHTabN = (kHTabP + 1) * (kHTabP + 2) / 2;
__constant__ double h_ra[kHTabN], h_rb[kHTabN], h_cm[kHTabP + 1], h_sq[kHTabP + 1];

void hess_init_constants(Status &st)
{
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    static std::vector<double> ra, rb, cm, sq;
    if (ra.empty()) {
        ra.assign(kHTabN, 0.0);
        rb.assign(kHTabN, 0.0);
        cm.assign(kHTabP + 1, 0.0);
        sq.assign(kHTabP + 1, 0.0);
        for (int n = 0; n <= kHTabP; n++)
            for (int m = 0; m <= n; m++)
                if (n >= m + 2) {
                    double den = sqrt((double)(n - m) * (n + m));
                    ra[tidx(n, m)] = (2.0 * n - 1) / den;
                    rb[tidx(n, m)] = sqrt((double)(n + m - 1) * (n - m - 1)) / den;
                }
        for (int m = 1; m <= kHTabP; m++) cm[m] = sqrt((2.0 * m - 1) / (2.0 * m));
        for (int m = 0; m <= kHTabP; m++) sq[m] = sqrt(2.0 * m + 1);
    }
    int dev = 0;
    cudaGetDevice(&dev);
    static bool uploaded[64] = {false};
    if (dev < 64 && uploaded[dev]) return;
    FMM_TRY(st, cudaMemcpyToSymbol(h_ra, ra.data(), sizeof(double) * ra.size()));
    FMM_TRY(st, cudaMemcpyToSymbol(h_rb, rb.data(), sizeof(double) * rb.size()));
    FMM_TRY(st, cudaMemcpyToSymbol(h_cm, cm.data(), sizeof(double) * cm.size()));
    FMM_TRY(st, cudaMemcpyToSymbol(h_sq, sq.data(), sizeof(double) * sq.size()));
    if (st.ok() && dev < 64) uploaded[dev] = true;
}

// ---------------------------------------------------------------- near field
constexpr int kP2PHThreads = 128;

template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kP2PHThreads) k_p2p_hess(const int *leaves, TreeView tv, PointsSoA src,
                                                            const double *tx, const double *ty, const double *tz,
                                                            HessSoA hs, HessSoA ht, int do_src, int do_trg)
{
    __shared__ double sx[kP2PHThreads], sy[kP2PHThreads], sz[kP2PHThreads];
    __shared__ double2 sq[kP2PHThreads], sd[kP2PHThreads];
    __shared__ double svx[kP2PHThreads], svy[kP2PHThreads], svz[kP2PHThreads];
    const int b = leaves[blockIdx.x];
    const int s0 = tv.src0[b], ns = do_src ? tv.nsrc[b] : 0;
    const int t0 = tv.trg0[b], nt = do_trg ? tv.ntrg[b] : 0;
    const int ne = ns + nt;
    const int l1a = tv.l1_start[b], nl = 1 + tv.l1_start[b + 1] - l1a;
    for (int e0 = 0; e0 < ne; e0 += kP2PHThreads) {
        const int e = e0 + threadIdx.x;
        const bool act = e < ne;
        const bool is_src = e < ns;
        double ex = 0, ey = 0, ez = 0;
        int self = -1;
        if (act) {
            if (is_src) { int i = s0 + e; ex = src.x[i]; ey = src.y[i]; ez = src.z[i]; self = i; }
            else { int i = t0 + e - ns; ex = tx[i]; ey = ty[i]; ez = tz[i]; }
        }
        double hr[6] = {0, 0, 0, 0, 0, 0}, hi[6] = {0, 0, 0, 0, 0, 0};
        for (int j = 0; j < nl; j++) {
            const int jb = j == 0 ? b : tv.l1_idx[l1a + j - 1];
            const int js0 = tv.src0[jb], jn = tv.nsrc[jb];
            for (int c0 = 0; c0 < jn; c0 += kP2PHThreads) {
                const int cn = min(kP2PHThreads, jn - c0);
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
                for (int k = 0; k < cn; k++) {
                    if (k == selfk) continue;
                    const double dx = ex - sx[k], dy = ey - sy[k], dz = ez - sz[k];
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    const double ri = rsqrt(r2), ri2 = ri * ri, ri5 = ri2 * ri2 * ri;
                    if (CHG) {
                        // q (3 d d^T - r^2 I) / r^5
                        const double2 q = sq[k];
                        const double t[6] = {(3 * dx * dx - r2) * ri5, (3 * dy * dy - r2) * ri5,
                                             (3 * dz * dz - r2) * ri5, 3 * dx * dy * ri5,
                                             3 * dx * dz * ri5, 3 * dy * dz * ri5};
#pragma unroll
                        for (int c = 0; c < 6; c++) { hr[c] = fma(q.x, t[c], hr[c]); hi[c] = fma(q.y, t[c], hi[c]); }
                    }
                    if (DIP) {
                        // 3 ds [ (v.d)(5 d d^T / r^2 - I) - (v d^T + d v^T) ] / r^5
                        const double2 d = sd[k];
                        const double vx = svx[k], vy = svy[k], vz = svz[k];
                        const double dot = dx * vx + dy * vy + dz * vz;
                        const double f = 5 * dot * ri2, c3 = 3 * ri5;
                        const double t[6] = {c3 * (f * dx * dx - dot - 2 * vx * dx), c3 * (f * dy * dy - dot - 2 * vy * dy),
                                             c3 * (f * dz * dz - dot - 2 * vz * dz), c3 * (f * dx * dy - (vy * dx + vx * dy)),
                                             c3 * (f * dx * dz - (vz * dx + vx * dz)),
                                             c3 * (f * dy * dz - (vz * dy + vy * dz))};
#pragma unroll
                        for (int c = 0; c < 6; c++) { hr[c] = fma(d.x, t[c], hr[c]); hi[c] = fma(d.y, t[c], hi[c]); }
                    }
                }
            }
        }
        if (act) {
            HessSoA &o = is_src ? hs : ht;
            const int i = is_src ? s0 + e : t0 + e - ns;
#pragma unroll
            for (int c = 0; c < 6; c++) o.h[c][i] = cadd(o.h[c][i], cmk(hr[c], hi[c]));
        }
    }
}

void launch_p2p_hess(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                     const double *ty, const double *tz, HessSoA hs, HessSoA ht, int ifcharge, int ifdipole,
                     int do_src, int do_trg, cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok() || !(do_src || do_trg)) return;
    const bool c = ifcharge == 1, d = ifdipole == 1;
    if (c && d)
        k_p2p_hess<true, true><<<nleaves, kP2PHThreads, 0, s>>>(leaves, tv, src, tx, ty, tz, hs, ht, do_src, do_trg);
    else if (c)
        k_p2p_hess<true, false><<<nleaves, kP2PHThreads, 0, s>>>(leaves, tv, src, tx, ty, tz, hs, ht, do_src, do_trg);
    else if (d)
        k_p2p_hess<false, true><<<nleaves, kP2PHThreads, 0, s>>>(leaves, tv, src, tx, ty, tz, hs, ht, do_src, do_trg);
    else
        return;
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// ---------------------------------------------------------------- coefficient arrays
// Derivative arrays, by kind: 0 the expansion itself, 1 d/dz, 2 D+, 3 D-,
// 4 d2/dz2, 5 D+D+, 6 D-D-, 7 d/dz D+, 8 d/dz D-.
constexpr int kNumKinds = 9;
__host__ __device__ __forceinline__ int kind_order(int q) { return q == 0 ? 0 : q <= 3 ? 1 : 2; }
__device__ __forceinline__ int kind_step(int q, int i)   // i-th ladder step (0: d/dz, 1: D+, 2: D-), -1 none
{
    const int a[kNumKinds] = {-1, 0, 1, 2, 0, 1, 2, 0, 0};
    const int b[kNumKinds] = {-1, -1, -1, -1, 0, 1, 2, 1, 2};
    return i == 0 ? b[q] : a[q];
}

// One ladder step: the coefficient (k, mu) of the derivative t of an
// expansion is f times the expansion's coefficient (k', mu'); local
// expansions: k' = k + 1, multipoles: k' = k - 1.  (k, mu) become (k', mu');
// false when that coefficient does not exist.
__device__ __forceinline__ bool ladder(bool loc, int t, int &k, int &mu, double &f)
{
    if (loc) {
        if (t == 0) f = sqrt((double)(k + 1 + mu) * (k + 1 - mu));
        else if (t == 1) { f = (mu <= 0 ? -1.0 : 1.0) * sqrt((double)(k + 2 - mu) * (k + 1 - mu)); mu -= 1; }
        else { f = (mu >= 0 ? -1.0 : 1.0) * sqrt((double)(k + 2 + mu) * (k + 1 + mu)); mu += 1; }
        k += 1;
    } else {
        if (t == 0) f = -sqrt(fmax((double)(k + mu) * (k - mu), 0.0));
        else if (t == 1) { f = (mu <= 0 ? -1.0 : 1.0) * sqrt(fmax((double)(k + mu - 1) * (k + mu), 0.0)); mu -= 1; }
        else { f = (mu >= 0 ? -1.0 : 1.0) * sqrt(fmax((double)(k - mu - 1) * (k - mu), 0.0)); mu += 1; }
        k -= 1;
    }
    return k >= 0 && mu <= k && -mu <= k;
}

// Coefficient (k, mu) of derivative array q of the expansion C (orders 0..p,
// index eidx).  getc(n, m) reads C's coefficient.
template <class Get>
__device__ __forceinline__ double2 deriv_coef(bool loc, int p, int q, int k, int mu, const Get &getc)
{
    double f = 1.0;
    for (int i = 0; i < 2; i++) {
        const int t = kind_step(q, i);
        if (t < 0) continue;
        double g;
        if (!ladder(loc, t, k, mu, g)) return cmk(0, 0);
        f *= g;
    }
    if (k > p) return cmk(0, 0);
    return cscal(f, getc(k, mu));
}

// Degree range [lo, hi] of derivative array q of an order-p expansion.
__device__ __forceinline__ void kind_range(bool loc, int p, int q, int &lo, int &hi)
{
    const int d = kind_order(q);
    if (loc) { lo = 0; hi = p - d; }
    else { lo = d; hi = p + d; }
}

// Dots the arrays staged for kinds [Q0, Q1] (slot[q] >= 0: at arr + slot[q] ld)
// with the solid harmonics of u up to degree nmax: regular ones for a local
// expansion, irregular for a multipole (the harmonics of the first
// derivative evaluation, l3dtaeval / l3dmpeval conventions).
template <int Q0, int Q1>
__device__ __forceinline__ void dot_arrays(bool loc, int nmax, double ux, double uy, double uz, const double2 *arr,
                                           int ld, const int (&slot)[kNumKinds], const int (&lo)[kNumKinds],
                                           const int (&hi)[kNumKinds], double2 (&acc)[kNumKinds])
{
    const double r2 = ux * ux + uy * uy + uz * uz;
    const double ir2 = loc ? 1.0 : 1.0 / r2;
    const double zz = loc ? uz : uz * ir2, rr = loc ? r2 : ir2;
    double2 diag = cmk(loc ? 1.0 : sqrt(ir2), 0.0);
    for (int m = 0; m <= nmax; m++) {
        if (m > 0) {
            const double cc = -h_cm[m] * ir2;
            diag = cmk(cc * (ux * diag.x + uy * diag.y), cc * (ux * diag.y - uy * diag.x));
        }
        double2 r1 = cmk(0, 0), r0 = diag;
        for (int n = m; n <= nmax; n++) {
            double2 h;
            if (n == m) h = diag;
            else if (n == m + 1) h = cscal(h_sq[m] * zz, diag);
            else {
                const double a = h_ra[tidx(n, m)] * zz, bb = h_rb[tidx(n, m)] * rr;
                h = cmk(a * r0.x - bb * r1.x, a * r0.y - bb * r1.y);
            }
            if (n > m) { r1 = r0; r0 = h; }
            const double2 hc = cconj(h);
            const int ip = eidx(n, m), im = eidx(n, -m);
#pragma unroll
            for (int q = Q0; q <= Q1; q++) {
                if (slot[q] < 0 || n < lo[q] || n > hi[q]) continue;
                const double2 *A = arr + slot[q] * ld;
                cfma(acc[q], A[ip], hc);
                if (m > 0) cfma(acc[q], A[im], h);
            }
        }
    }
}

// The six Hessian components from the second-derivative sums (kinds 4..8).
__device__ __forceinline__ void hess_from_ladders(const double2 (&a)[kNumKinds], double sc, double2 (&h)[6])
{
    const double2 zz = a[4], pp = a[5], mm = a[6], zp = a[7], zm = a[8];
    const double2 s = cscal(0.5, cadd(pp, mm)), d = csub(pp, mm), u = cadd(zp, zm), v = csub(zp, zm);
    h[0] = cadd(h[0], cscal(0.5 * sc, csub(s, zz)));
    h[1] = csub(h[1], cscal(0.5 * sc, cadd(s, zz)));
    h[2] = cadd(h[2], cscal(sc, zz));
    h[3] = cadd(h[3], cscal(0.25 * sc, cmk(d.y, -d.x)));   // d / (4i)
    h[4] = cadd(h[4], cscal(0.5 * sc, u));
    h[5] = cadd(h[5], cscal(0.5 * sc, cmk(v.y, -v.x)));    // v / (2i)
}

// Stages the arrays of kinds list[first .. first + n) for expansion C into
// arr (stride ld = (p + 3)^2) and records their slots.
template <int Q0, int Q1, class Get>
__device__ __forceinline__ void stage_phase(bool loc, int p, int first, int n, const int *list, double2 *arr, int ld,
                                            const Get &getc, int (&slot)[kNumKinds])
{
#pragma unroll
    for (int q = Q0; q <= Q1; q++) slot[q] = -1;
    for (int j = 0; j < n; j++) {
        const int q = list[first + j];
#pragma unroll
        for (int r = Q0; r <= Q1; r++)
            if (r == q) slot[r] = j;
    }
    const int D = p + 2;
    const int cnt = (D + 1) * (D + 1);
    for (int i = threadIdx.x; i < n * cnt; i += blockDim.x) {
        const int j = i / cnt, e = i - j * cnt;
        int k = (int)sqrtf((float)e);
        while (k * k > e) k--;
        while ((k + 1) * (k + 1) <= e) k++;
        const int mu = e - k * k - k;
        arr[j * ld + e] = deriv_coef(loc, p, list[first + j], k, mu, getc);
    }
}

// ---------------------------------------------------------------- far field of the FMM
constexpr int kEvalHThreads = 128;

// Side of box b: its instance's root side (forests) or the tree's, halved per level.
__device__ __forceinline__ double hbox_side(const TreeView &tv, int b)
{
    const double size = tv.binst ? tv.inst_geom[4 * tv.binst[b] + 3] : tv.size;
    return size / (double)(1L << tv.level[b]);
}

__global__ void __launch_bounds__(kEvalHThreads) k_eval_hess(const int *leaves, TreeView tv, const double *sx,
                                                              const double *sy, const double *sz, const double *tx,
                                                              const double *ty, const double *tz, int p,
                                                              const double2 *mpole, const double2 *local,
                                                              HessSoA hs, HessSoA ht, int do_src, int do_trg,
                                                              int per_phase)
{
    extern __shared__ double2 sm[];
    const int ld = (p + 3) * (p + 3), K = (p + 1) * (p + 1);
    const int list[5] = {4, 5, 6, 7, 8};
    const int b = leaves[blockIdx.x];
    const int lev = tv.level[b];
    const int s0 = tv.src0[b], ns = do_src ? tv.nsrc[b] : 0;
    const int t0 = tv.trg0[b], nt = do_trg ? tv.ntrg[b] : 0;
    const int ne = ns + nt;
    const int l3a = tv.l3_start[b], nl3 = tv.l3_start[b + 1] - l3a;
    const bool has_local = lev >= 2;
    const int nsrcbox = (has_local ? 1 : 0) + nl3;
    for (int e0 = 0; e0 < ne; e0 += kEvalHThreads) {
        const int e = e0 + threadIdx.x;
        const bool act = e < ne;
        const bool is_src = e < ns;
        double px = 0, py = 0, pz = 0;
        if (act) {
            if (is_src) { px = sx[s0 + e]; py = sy[s0 + e]; pz = sz[s0 + e]; }
            else { px = tx[t0 + e - ns]; py = ty[t0 + e - ns]; pz = tz[t0 + e - ns]; }
        }
        double2 h[6] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
        for (int ib = 0; ib < nsrcbox; ib++) {
            const bool loc = has_local && ib == 0;
            const int c = loc ? b : tv.l3_idx[l3a + ib - (has_local ? 1 : 0)];
            const double s = hbox_side(tv, c), is = 1.0 / s;
            const double2 *coef = loc ? local + (size_t)c * K : mpole + (size_t)c * K;
            const double ux = (px - tv.center[3L * c]) * is, uy = (py - tv.center[3L * c + 1]) * is,
                         uz = (pz - tv.center[3L * c + 2]) * is;
            int lo[kNumKinds], hi[kNumKinds], slot[kNumKinds];
#pragma unroll
            for (int q = 4; q <= 8; q++) kind_range(loc, p, q, lo[q], hi[q]);
            double2 acc[kNumKinds];
#pragma unroll
            for (int q = 4; q <= 8; q++) acc[q] = cmk(0, 0);
            const int nmax = loc ? p - 2 : p + 2;
            for (int f = 0; f < 5; f += per_phase) {
                const int n = min(per_phase, 5 - f);
                __syncthreads();
                stage_phase<4, 8>(loc, p, f, n, list, sm, ld, [&](int k, int mu) { return coef[eidx(k, mu)]; }, slot);
                __syncthreads();
                if (act && nmax >= 0) dot_arrays<4, 8>(loc, nmax, ux, uy, uz, sm, ld, slot, lo, hi, acc);
            }
            if (act) hess_from_ladders(acc, is * is * is, h);
        }
        if (act) {
            HessSoA &o = is_src ? hs : ht;
            const int i = is_src ? s0 + e : t0 + e - ns;
#pragma unroll
            for (int c = 0; c < 6; c++) o.h[c][i] = cadd(o.h[c][i], h[c]);
        }
    }
}

static constexpr size_t kHessSmemMax = 200 * 1024;

void launch_eval_hess(const int *leaves, int nleaves, const TreeView &tv, const double *sx, const double *sy,
                      const double *sz, const double *tx, const double *ty, const double *tz, int p,
                      const double2 *mpole, const double2 *local, HessSoA hs, HessSoA ht, int do_src, int do_trg,
                      cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok() || !(do_src || do_trg)) return;
    if (p > kHessMaxP) { st.err = cudaErrorInvalidValue; st.where = "Hessian: expansion order above the table"; return; }
    const size_t arr = (size_t)(p + 3) * (p + 3) * sizeof(double2);
    const int per_phase = (int)std::min<size_t>(5, kHessSmemMax / arr);
    const size_t smem = per_phase * arr;
    FMM_TRY(st, smem_allow(k_eval_hess, (int)smem));
    if (!st.ok()) return;
    k_eval_hess<<<nleaves, kEvalHThreads, smem, s>>>(leaves, tv, sx, sy, sz, tx, ty, tz, p, mpole, local, hs, ht,
                                                     do_src, do_trg, per_phase);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

__global__ void k_scatter_hess(int n, const int *perm, HessSoA h, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long j = perm ? perm[i] : i;
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const double2 v = h.h[c][i];
        out[12 * j + 2 * c] = v.x;
        out[12 * j + 2 * c + 1] = v.y;
    }
}

void launch_scatter_hess(int n, const int *perm, HessSoA h, double *out, cudaStream_t s, Status &st)
{
    if (n <= 0 || !st.ok() || !out) return;
    k_scatter_hess<<<(n + 255) / 256, 256, 0, s>>>(n, perm, h, out);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// ---------------------------------------------------------------- one expansion, many points
// Every CTA stages the derivative arrays of the one expansion (in phases) and
// evaluates them at its chunk of points, grid-striding over the rest.
constexpr int kExpEvalThreads = 128;

__global__ void __launch_bounds__(kExpEvalThreads) k_expeval_hess(int loc_, double rscale, double cx, double cy,
                                                                   double cz, const double *coef, int nterms,
                                                                   int npts, const double *pts, double *pot,
                                                                   double *fld, double *hess, int nk, int per_phase)
{
    extern __shared__ double2 sm[];
    const bool loc = loc_ != 0;
    const int p = nterms, ld = (p + 3) * (p + 3);
    int list[kNumKinds];
    for (int q = 0; q < nk; q++) list[q] = q == 0 ? 0 : (nk == 4 ? q : nk == 6 ? q + 3 : q);
    // kinds in use: nk == 9 all; nk == 4 pot + gradient; nk == 6 pot + Hessian
    auto getc = [&](int k, int mu) {
        const double *c = coef + 2 * ((size_t)k + (size_t)(mu + nterms) * (nterms + 1));
        return cmk(c[0], c[1]);
    };
    int lo[kNumKinds], hi[kNumKinds], slot[kNumKinds];
#pragma unroll
    for (int q = 0; q < kNumKinds; q++) kind_range(loc, p, q, lo[q], hi[q]);
    int dmax = 0;
    for (int q = 0; q < nk; q++) dmax = max(dmax, kind_order(list[q]));
    const int nmax = loc ? p : p + dmax;
    // output scale per derivative order d: rscale^d (local), rscale^(d+1) (multipole)
    const double f0 = loc ? 1.0 : rscale, f1 = f0 * rscale, f2 = f1 * rscale;
    for (int base = blockIdx.x * kExpEvalThreads; base < npts; base += gridDim.x * kExpEvalThreads) {
        const int i = base + threadIdx.x;
        const bool act = i < npts;
        double ux = 0, uy = 0, uz = 0;
        if (act) {
            ux = (pts[3L * i] - cx) * rscale;
            uy = (pts[3L * i + 1] - cy) * rscale;
            uz = (pts[3L * i + 2] - cz) * rscale;
        }
        double2 acc[kNumKinds];
#pragma unroll
        for (int q = 0; q < kNumKinds; q++) acc[q] = cmk(0, 0);
        for (int f = 0; f < nk; f += per_phase) {
            const int n = min(per_phase, nk - f);
            __syncthreads();
            stage_phase<0, 8>(loc, p, f, n, list, sm, ld, getc, slot);
            __syncthreads();
            if (act) dot_arrays<0, 8>(loc, nmax, ux, uy, uz, sm, ld, slot, lo, hi, acc);
        }
        if (!act) continue;
        const double2 pv = cscal(f0, acc[0]);
        pot[2L * i] = pv.x;
        pot[2L * i + 1] = pv.y;
        if (fld) {
            // -gradient: d/dx = (D+ + D-)/2, d/dy = (D+ - D-)/(2i)
            const double2 gx = cscal(0.5 * f1, cadd(acc[2], acc[3]));
            const double2 dd = csub(acc[2], acc[3]);
            const double2 gy = cscal(0.5 * f1, cmk(dd.y, -dd.x));
            const double2 gz = cscal(f1, acc[1]);
            double *o = fld + 6L * i;
            o[0] = -gx.x; o[1] = -gx.y; o[2] = -gy.x; o[3] = -gy.y; o[4] = -gz.x; o[5] = -gz.y;
        }
        if (hess) {
            double2 h[6] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
            hess_from_ladders(acc, f2, h);
            double *o = hess + 12L * i;
#pragma unroll
            for (int c = 0; c < 6; c++) { o[2 * c] = h[c].x; o[2 * c + 1] = h[c].y; }
        }
    }
}

void launch_expeval_hess(bool loc, double rscale, const double *center, const double *coef, int nterms, int npts,
                         const double *pts, double *pot, int iffld, double *fld, int ifhess, double *hess,
                         cudaStream_t s, Status &st)
{
    if (npts <= 0 || !st.ok()) return;
    if (nterms < 0 || nterms > kHessMaxP) {
        st.err = cudaErrorInvalidValue;
        st.where = "Hessian evaluation: nterms outside 0..74";
        return;
    }
    hess_init_constants(st);
    if (!st.ok()) return;
    const bool f = iffld == 1, h = ifhess == 1;
    const int nk = f && h ? 9 : f ? 4 : h ? 6 : 1;
    const size_t arr = (size_t)(nterms + 3) * (nterms + 3) * sizeof(double2);
    const int per_phase = (int)std::min<size_t>(nk, kHessSmemMax / arr);
    const size_t smem = per_phase * arr;
    FMM_TRY(st, smem_allow(k_expeval_hess, (int)smem));
    if (!st.ok()) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::max(1, std::min((npts + kExpEvalThreads - 1) / kExpEvalThreads, 4 * sms));
    k_expeval_hess<<<grid, kExpEvalThreads, smem, s>>>(loc ? 1 : 0, rscale, center[0], center[1], center[2], coef,
                                                        nterms, npts, pts, pot, f ? fld : nullptr, h ? hess : nullptr,
                                                        nk, per_phase);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

}  // namespace fmm
