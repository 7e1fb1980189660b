// Mixed-precision form of the two dominant passes (iprec <= 1 only).
//
// P2P: the evaluation box's own sources in FP64; the list-1 sources in FP32,
// with evaluation and source points taken relative to the centre of the
// evaluation box in FP64 and stored as hi + lo float pairs, so pair
// differences keep FP64-level accuracy even for close pairs; the pair terms
// of a chunk are summed in FP32 and each chunk sum is folded into an FP32
// (value, error) pair with Knuth's TwoSum, i.e. compensated summation across
// chunks.  The pair formulas are those of lpotfld3d /
// lpotfld3d_dp (src/laprouts3d.f:1308-1368, 1962-2035).
//
// M2L in FP32 on the CUDA cores (k_m2l_dense32, used when the tensor-core
// M2L of tc_m2l.cu is switched off): the dense per-offset operators
// (m2l_dense.cu) rounded to FP32, box-scaled multipoles (all O(1)) rounded to
// FP32 on load, FP32 accumulation, and the tile added to the FP64 local
// expansion.
#include "lap_kernels.cuh"
#include "m2l_dense.cuh"

namespace fmm {

__device__ __forceinline__ void two_sum_acc(float &hi, float &lo, float x)
{
    float s = hi + x;
    float bb = s - hi;
    float e = (hi - (s - bb)) + (x - bb);
    hi = s;
    lo += e;
}

// Pair term in FP32 from double-float coordinate differences: every
// coordinate is stored as hi + lo floats relative to the evaluation box
// centre, and dx = (e.hi - s.hi) + (e.lo - s.lo).  For close pairs the hi
// difference is exact (Sterbenz), so close-pair differences keep FP64-level
// accuracy and only r^2, 1/r and the products are FP32.
__device__ __forceinline__ float rsqrt_approx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

template <bool CHG, bool DIP>
__device__ __forceinline__ void pair32(float exh, float eyh, float ezh, float exl, float eyl, float ezl,
                                       float sxh, float syh, float szh, float sxl, float syl, float szl, float2 q,
                                       float2 d, float vx, float vy, float vz, float *a)
{
    float dx = (exh - sxh) + (exl - sxl), dy = (eyh - syh) + (eyl - syl), dz = (ezh - szh) + (ezl - szl);
    float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float ri = rsqrt_approx(r2);
    float ri2 = ri * ri, ri3 = ri * ri2;
    if (CHG && !DIP) {
        a[0] = fmaf(q.x, ri, a[0]);
        a[1] = fmaf(q.y, ri, a[1]);
        float qx = q.x * ri3, qy = q.y * ri3;
        a[2] = fmaf(qx, dx, a[2]); a[3] = fmaf(qy, dx, a[3]);
        a[4] = fmaf(qx, dy, a[4]); a[5] = fmaf(qy, dy, a[5]);
        a[6] = fmaf(qx, dz, a[6]); a[7] = fmaf(qy, dz, a[7]);
    } else {
        // pot = (q + d t) / r with t = (v.dx)/r^2;  fld = [(q + 3 d t) dx - d v] / r^3
        float t = fmaf(dx, vx, fmaf(dy, vy, dz * vz)) * ri2;
        float ax = CHG ? fmaf(d.x, t, q.x) : d.x * t, ay = CHG ? fmaf(d.y, t, q.y) : d.y * t;
        a[0] = fmaf(ax, ri, a[0]);
        a[1] = fmaf(ay, ri, a[1]);
        float t3 = 3.0f * t;
        float bx = (CHG ? fmaf(d.x, t3, q.x) : d.x * t3) * ri3, by = (CHG ? fmaf(d.y, t3, q.y) : d.y * t3) * ri3;
        float dxr = d.x * ri3, dyr = d.y * ri3;
        a[2] = fmaf(bx, dx, fmaf(-dxr, vx, a[2])); a[3] = fmaf(by, dx, fmaf(-dyr, vx, a[3]));
        a[4] = fmaf(bx, dy, fmaf(-dxr, vy, a[4])); a[5] = fmaf(by, dy, fmaf(-dyr, vy, a[5]));
        a[6] = fmaf(bx, dz, fmaf(-dxr, vz, a[6])); a[7] = fmaf(by, dz, fmaf(-dyr, vz, a[7]));
    }
}

// The same pair term with dipoles, the field factored as r^-3 [(q + 3 d t) dx - d v]
// and the products -d v of the source (nv: re x, y, z, then im x, y, z) computed
// once when the source is staged: 38 operations per pair instead of 42.
template <bool CHG>
__device__ __forceinline__ void pair32_dip(float exh, float eyh, float ezh, float exl, float eyl, float ezl,
                                           float sxh, float syh, float szh, float sxl, float syl, float szl,
                                           float2 q, float2 d, float vx, float vy, float vz, const float *nv,
                                           float *a)
{
    float dx = (exh - sxh) + (exl - sxl), dy = (eyh - syh) + (eyl - syl), dz = (ezh - szh) + (ezl - szl);
    float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float ri = rsqrt_approx(r2);
    float ri2 = ri * ri, ri3 = ri * ri2;
    float t = fmaf(dx, vx, fmaf(dy, vy, dz * vz)) * ri2;
    float ax = CHG ? fmaf(d.x, t, q.x) : d.x * t, ay = CHG ? fmaf(d.y, t, q.y) : d.y * t;
    a[0] = fmaf(ax, ri, a[0]);
    a[1] = fmaf(ay, ri, a[1]);
    float t3 = 3.0f * t;
    float bx = CHG ? fmaf(d.x, t3, q.x) : d.x * t3, by = CHG ? fmaf(d.y, t3, q.y) : d.y * t3;
    a[2] = fmaf(ri3, fmaf(bx, dx, nv[0]), a[2]); a[3] = fmaf(ri3, fmaf(by, dx, nv[3]), a[3]);
    a[4] = fmaf(ri3, fmaf(bx, dy, nv[1]), a[4]); a[5] = fmaf(ri3, fmaf(by, dy, nv[4]), a[5]);
    a[6] = fmaf(ri3, fmaf(bx, dz, nv[2]), a[6]); a[7] = fmaf(ri3, fmaf(by, dz, nv[5]), a[7]);
}

__device__ __forceinline__ void split_df(double v, float &hi, float &lo)
{
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

// Pair term in FP64 (the evaluation box's own sources): lpotfld3d /
// lpotfld3d_dp (src/laprouts3d.f:1308-1368, 1962-2035).
template <bool CHG, bool DIP>
__device__ __forceinline__ void pair64(double dx, double dy, double dz, double2 q, double2 d, double vx, double vy,
                                       double vz, double *a)
{
    // fused multiply-adds written out, so that every instantiation (points per lane) rounds alike
    double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
    double ri = rsqrt(r2);
    double ri2 = ri * ri, ri3 = ri * ri2;
    if (CHG) {
        a[0] = fma(q.x, ri, a[0]);
        a[1] = fma(q.y, ri, a[1]);
        double qx = q.x * ri3, qy = q.y * ri3;
        a[2] = fma(qx, dx, a[2]); a[3] = fma(qy, dx, a[3]);
        a[4] = fma(qx, dy, a[4]); a[5] = fma(qy, dy, a[5]);
        a[6] = fma(qx, dz, a[6]); a[7] = fma(qy, dz, a[7]);
    }
    if (DIP) {
        double dot = fma(dx, vx, fma(dy, vy, dz * vz));
        double t = dot * ri3;
        a[0] = fma(d.x, t, a[0]);
        a[1] = fma(d.y, t, a[1]);
        double rt = 3.0 * t * ri2;
        double gx = fma(rt, dx, -(ri3 * vx)), gy = fma(rt, dy, -(ri3 * vy)), gz = fma(rt, dz, -(ri3 * vz));
        a[2] = fma(d.x, gx, a[2]); a[3] = fma(d.y, gx, a[3]);
        a[4] = fma(d.x, gy, a[4]); a[5] = fma(d.y, gy, a[5]);
        a[6] = fma(d.x, gz, a[6]); a[7] = fma(d.y, gz, a[7]);
    }
}

// Warp-synchronous mixed-precision near field.  A CTA is one warp and serves
// one childless box in passes of 32, 64 or 128 evaluation points (one, two or
// four per lane: e, e+32, e+64, e+96), chosen from the points left.  First the box's own sources, which carry
// the largest and most cancellation-prone terms, are summed in FP64 straight
// from global memory (L1 broadcast) and added to the outputs; their
// accumulators are then dead.  The sources of list 1 follow in FP32: they
// are streamed through a 32-entry shared buffer of float4 records (double-
// float coordinates relative to the box centre, charge, dipole), the next
// chunk being fetched into registers while the current one is used, each
// chunk is summed in FP32 and folded into an FP32 (value, error) pair with
// TwoSum (the pairs live in shared memory, one slot per lane, to keep the
// register count at 128), and the result is added to the outputs.
constexpr int kP2P32Threads = 32, kEPT = 4;   // at most four evaluation points per lane

template <bool CHG, bool DIP, int kEPT>
__device__ __forceinline__ void p2p32_pass(int e0, int b, const TreeView &tv, const PointsSoA &src,
                                           const double *tx, const double *ty, const double *tz, OutSoA &outs,
                                           OutSoA &outt, int do_src, int do_trg, int want_fs, int want_ft,
                                           int want_ps, int want_pt, float4 *wA, float4 *wB, float4 *wC,
                                           float4 *wD, float4 *wE, float (*whi)[32], float (*wlo)[32])
{
    const int lane = threadIdx.x;
    const double cx = tv.center[3L * b], cy = tv.center[3L * b + 1], cz = tv.center[3L * b + 2];
    const int s0 = tv.src0[b], nsb = tv.nsrc[b], ns = do_src ? nsb : 0;
    const int t0 = tv.trg0[b], nt = do_trg ? tv.ntrg[b] : 0;
    const int ne = ns + nt;
    const int l1a = tv.l1_start[b], nl = 1 + tv.l1_start[b + 1] - l1a;
    auto add_out = [&](int e, const double *r) {
        if (e < ns) {
            int i = s0 + e;
            if (want_ps) outs.pot[i] = cadd(outs.pot[i], cmk(r[0], r[1]));
            if (want_fs) {
                outs.fx[i] = cadd(outs.fx[i], cmk(r[2], r[3]));
                outs.fy[i] = cadd(outs.fy[i], cmk(r[4], r[5]));
                outs.fz[i] = cadd(outs.fz[i], cmk(r[6], r[7]));
            }
        } else {
            int i = t0 + e - ns;
            if (want_pt) outt.pot[i] = cadd(outt.pot[i], cmk(r[0], r[1]));
            if (want_ft) {
                outt.fx[i] = cadd(outt.fx[i], cmk(r[2], r[3]));
                outt.fy[i] = cadd(outt.fy[i], cmk(r[4], r[5]));
                outt.fz[i] = cadd(outt.fz[i], cmk(r[6], r[7]));
            }
        }
    };
    {
        bool act[kEPT];
        float eh[kEPT][3], el[kEPT][3];
        {
            // the box's own sources in FP64
            int self[kEPT];
            double ed[kEPT][3], a64[kEPT][8];
#pragma unroll
            for (int u = 0; u < kEPT; u++) {
                const int e = e0 + lane + 32 * u;
                act[u] = e < ne;
                self[u] = -1;
                double x = 0, y = 0, z = 0;
                if (act[u]) {
                    if (e < ns) { int i = s0 + e; x = src.x[i]; y = src.y[i]; z = src.z[i]; self[u] = i; }
                    else { int i = t0 + e - ns; x = tx[i]; y = ty[i]; z = tz[i]; }
                }
                ed[u][0] = x - cx; ed[u][1] = y - cy; ed[u][2] = z - cz;
#pragma unroll
                for (int c = 0; c < 8; c++) a64[u][c] = 0.0;
            }
            for (int k = 0; k < nsb; k++) {
                const int i = s0 + k;
                const double sx = src.x[i] - cx, sy = src.y[i] - cy, sz = src.z[i] - cz;
                const double2 q = CHG ? src.q[i] : cmk(0, 0), d = DIP ? src.dq[i] : cmk(0, 0);
                const double vx = DIP ? src.vx[i] : 0, vy = DIP ? src.vy[i] : 0, vz = DIP ? src.vz[i] : 0;
#pragma unroll
                for (int u = 0; u < kEPT; u++)
                    if (act[u] && i != self[u])
                        pair64<CHG, DIP>(ed[u][0] - sx, ed[u][1] - sy, ed[u][2] - sz, q, d, vx, vy, vz, a64[u]);
            }
#pragma unroll
            for (int u = 0; u < kEPT; u++) {
                if (act[u]) add_out(e0 + lane + 32 * u, a64[u]);
#pragma unroll
                for (int c = 0; c < 3; c++) split_df(ed[u][c], eh[u][c], el[u][c]);
            }
        }
        if (nl <= 1) return;
        // list-1 sources in FP32, streamed per warp
#pragma unroll
        for (int c = 0; c < kEPT * 8; c++) { whi[c][lane] = 0.f; wlo[c][lane] = 0.f; }
        int j = 1, c0 = 0, js0 = 0, jn = 0;
        { int jb = tv.l1_idx[l1a]; js0 = tv.src0[jb]; jn = tv.nsrc[jb]; }
        auto advance = [&]() {
            while (j < nl && c0 >= jn) {
                j++;
                c0 = 0;
                if (j < nl) { int jb = tv.l1_idx[l1a + j - 1]; js0 = tv.src0[jb]; jn = tv.nsrc[jb]; }
            }
        };
        advance();
        float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa, pc = pa, pd = pa, pe = pa;
        auto fetch = [&]() {
            int i = c0 + lane;
            if (j < nl && i < jn) {
                i += js0;
                split_df(src.x[i] - cx, pa.x, pb.x);
                split_df(src.y[i] - cy, pa.y, pb.y);
                split_df(src.z[i] - cz, pa.z, pb.z);
                if (DIP) {
                    pa.w = (float)src.vx[i];
                    pb.w = (float)src.vy[i];
                    const float vz = (float)src.vz[i];
                    const double2 d = src.dq[i];
                    const double2 q = CHG ? src.q[i] : cmk(0, 0);
                    pc = make_float4((float)q.x, (float)q.y, (float)d.x, (float)d.y);
                    // -d v (FP32 products of the FP32 operands), re then im
                    pd = make_float4(vz, -pc.z * pa.w, -pc.z * pb.w, -pc.z * vz);
                    pe = make_float4(-pc.w * pa.w, -pc.w * pb.w, -pc.w * vz, 0.f);
                } else {
                    const double2 q = src.q[i];
                    pa.w = (float)q.x;
                    pb.w = (float)q.y;
                }
            }
        };
        fetch();
        while (j < nl) {
            const int cn = min(32, jn - c0);
            __syncwarp();
            if (lane < cn) {
                wA[lane] = pa;
                wB[lane] = pb;
                if (DIP) { wC[lane] = pc; wD[lane] = pd; wE[lane] = pe; }
            }
            __syncwarp();
            c0 += 32;
            advance();
            fetch();  // next chunk in flight while this one is used
            float a[kEPT][8];
#pragma unroll
            for (int u = 0; u < kEPT; u++)
#pragma unroll
                for (int c = 0; c < 8; c++) a[u][c] = 0.f;
#pragma unroll 2
            for (int k = 0; k < cn; k++) {
                const float4 A = wA[k], B = wB[k];
                if (DIP) {
                    const float4 C = wC[k], D = wD[k], E = wE[k];
                    const float nv[6] = {D.y, D.z, D.w, E.x, E.y, E.z};
#pragma unroll
                    for (int u = 0; u < kEPT; u++)
                        pair32_dip<CHG>(eh[u][0], eh[u][1], eh[u][2], el[u][0], el[u][1], el[u][2], A.x, A.y, A.z,
                                        B.x, B.y, B.z, make_float2(C.x, C.y), make_float2(C.z, C.w), A.w, B.w, D.x,
                                        nv, a[u]);
                } else {
#pragma unroll
                    for (int u = 0; u < kEPT; u++)
                        pair32<CHG, false>(eh[u][0], eh[u][1], eh[u][2], el[u][0], el[u][1], el[u][2], A.x, A.y,
                                           A.z, B.x, B.y, B.z, make_float2(A.w, B.w), make_float2(0.f, 0.f), 0.f,
                                           0.f, 0.f, a[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < kEPT; u++)
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    float h = whi[8 * u + c][lane], l = wlo[8 * u + c][lane];
                    two_sum_acc(h, l, a[u][c]);
                    whi[8 * u + c][lane] = h;
                    wlo[8 * u + c][lane] = l;
                }
        }
#pragma unroll
        for (int u = 0; u < kEPT; u++) {
            if (!act[u]) continue;
            double r[8];
#pragma unroll
            for (int c = 0; c < 8; c++) r[c] = (double)whi[8 * u + c][lane] + (double)wlo[8 * u + c][lane];
            add_out(e0 + lane + 32 * u, r);
        }
    }
}

template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kP2P32Threads, 16) k_p2p32(const int *leaves, TreeView tv, PointsSoA src,
                                                          const double *tx, const double *ty, const double *tz,
                                                          OutSoA outs, OutSoA outt, int do_src, int do_trg,
                                                          int want_fs, int want_ft, int want_ps, int want_pt,
                                                          int max_ept)
{
    // per source: A = (x hi, y hi, z hi, charge re | vx), B = (x lo, y lo, z lo, charge im | vy),
    // C = (charge re, charge im, dipstr re, dipstr im), D = (vz, -d v re x, y, z),
    // E = (-d v im x, y, z, 0)   (C, D, E with dipoles only)
    __shared__ float4 wA[32], wB[32], wC[32], wD[32], wE[32];
    __shared__ float whi[kEPT * 8][32], wlo[kEPT * 8][32];   // TwoSum pairs, [component][lane]
    const int b = leaves[blockIdx.x];
    const int ne = (do_src ? tv.nsrc[b] : 0) + (do_trg ? tv.ntrg[b] : 0);
    // passes of 32, 64 or 128 evaluation points (one, two or four per lane, at most
    // max_ept); every point's sums run over the same sources in the same order
    // CTA (leaf, y) runs the leaf's passes y, y + gridDim.y, ... of the same sequence
    for (int e0 = 0, pass = 0; e0 < ne; pass++) {
        const int left = ne - e0;
        const bool mine = pass % gridDim.y == blockIdx.y;
        if (left <= 32 || max_ept == 1) {
            if (mine)
                p2p32_pass<CHG, DIP, 1>(e0, b, tv, src, tx, ty, tz, outs, outt, do_src, do_trg, want_fs, want_ft,
                                        want_ps, want_pt, wA, wB, wC, wD, wE, whi, wlo);
            e0 += 32;
        } else if (left <= 64 || max_ept == 2) {
            if (mine)
                p2p32_pass<CHG, DIP, 2>(e0, b, tv, src, tx, ty, tz, outs, outt, do_src, do_trg, want_fs, want_ft,
                                        want_ps, want_pt, wA, wB, wC, wD, wE, whi, wlo);
            e0 += 64;
        } else {
            if (mine)
                p2p32_pass<CHG, DIP, 4>(e0, b, tv, src, tx, ty, tz, outs, outt, do_src, do_trg, want_fs, want_ft,
                                        want_ps, want_pt, wA, wB, wC, wD, wE, whi, wlo);
            e0 += 128;
        }
    }
}

void launch_p2p32(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                  const double *ty, const double *tz, OutSoA outs, OutSoA outt, int ifcharge, int ifdipole,
                  int ifpot, int iffld, int ifpottarg, int iffldtarg, int max_ept, cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok()) return;
    int do_src = (ifpot == 1 || iffld == 1), do_trg = (ifpottarg == 1 || iffldtarg == 1);
    bool c = ifcharge == 1, d = ifdipole == 1;
    if (max_ept != 1 && max_ept != 2) max_ept = 4;
    if (c && d) {
        k_p2p32<true, true><<<dim3(nleaves, 3), kP2P32Threads, 0, s>>>(leaves, tv, src, tx, ty, tz, outs, outt, do_src,
                                                             do_trg, iffld == 1, iffldtarg == 1, ifpot == 1,
                                                             ifpottarg == 1, max_ept); FMM_COUNT_LAUNCH();
    } else if (c) {
        k_p2p32<true, false><<<dim3(nleaves, 3), kP2P32Threads, 0, s>>>(leaves, tv, src, tx, ty, tz, outs, outt, do_src,
                                                              do_trg, iffld == 1, iffldtarg == 1, ifpot == 1,
                                                              ifpottarg == 1, max_ept); FMM_COUNT_LAUNCH();
    } else if (d) {
        k_p2p32<false, true><<<dim3(nleaves, 3), kP2P32Threads, 0, s>>>(leaves, tv, src, tx, ty, tz, outs, outt, do_src,
                                                              do_trg, iffld == 1, iffldtarg == 1, ifpot == 1,
                                                              ifpottarg == 1, max_ept); FMM_COUNT_LAUNCH();
    }
    FMM_LAUNCH_CHECK(st);
}

// ---------------------------------------------------------------- FP32 dense M2L
__device__ __forceinline__ void cfmaf(float2 &acc, float2 a, float2 b)
{
    acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
    acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}

__global__ void k_to_f32(long long n, const double2 *in, float2 *out)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

constexpr int k32TM = 64, k32TN = 64, k32TK = 16, k32Threads = 256;

__global__ void __launch_bounds__(k32Threads, 3) k_m2l_dense32(const Tile *tiles, const int *grouped,
                                                               const Slot *slots, const long long *slot_toff,
                                                               const float2 *T, TreeView tv, int p,
                                                               const double2 *in, double2 *out, int prune)
{
    __shared__ float2 As[k32TK][k32TM];
    __shared__ float2 Bs[k32TK][k32TN];
    __shared__ int tg[k32TN], sv[k32TN];
    __shared__ int anyv;
    const Tile tile = tiles[blockIdx.x];
    const int row0 = blockIdx.y * k32TM;
    const int NC = (p + 1) * (p + 1);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    if (threadIdx.x < k32TN) tg[threadIdx.x] = threadIdx.x < tile.count ? grouped[tile.first + threadIdx.x] : -1;
    float2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = make_float2(0.f, 0.f);
    for (int si = 0; si < tile.nslot; si++) {
        const Slot sl = slots[tile.slot0 + si];
        const int R = (sl.pt + 1) * (sl.pt + 1);
        if (row0 >= R) continue;
        __syncthreads();
        if (threadIdx.x == 0) anyv = 0;
        __syncthreads();
        if (threadIdx.x < k32TN) {
            int t = tg[threadIdx.x], sb = -1;
            if (t >= 0 && !(prune && tv.ntrg[t] == 0)) {
                int P = tv.parent[t];
                int C = P >= 0 ? tv.coll[27L * P + sl.coll] : -1;
                sb = C >= 0 ? tv.child[8L * C + sl.oct] : -1;
                if (sb >= 0 && tv.nsrc[sb] == 0) sb = -1;
            }
            sv[threadIdx.x] = sb;
            if (sb >= 0) atomicOr(&anyv, 1);
        }
        __syncthreads();
        if (!anyv) continue;
        const float2 *Tu = T + slot_toff[tile.slot0 + si];
        for (int k0 = 0; k0 < R; k0 += k32TK) {
            {
                int r = threadIdx.x & 63, c = (threadIdx.x >> 6) * 4;
                int gr = row0 + r;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    int gc = k0 + c + q;
                    As[c + q][r] = (gr < R && gc < R) ? Tu[(size_t)gc * R + gr] : make_float2(0.f, 0.f);
                }
            }
            {
                int j = threadIdx.x & 63, c = (threadIdx.x >> 6) * 4;
                int sb = sv[j];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    int gc = k0 + c + q;
                    float2 v = make_float2(0.f, 0.f);
                    if (sb >= 0 && gc < R) {
                        double2 d = in[(size_t)sb * NC + gc];
                        v = make_float2((float)d.x, (float)d.y);
                    }
                    Bs[c + q][j] = v;
                }
            }
            __syncthreads();
#pragma unroll 4
            for (int k = 0; k < k32TK; k++) {
                float2 a[4], b[4];
#pragma unroll
                for (int q = 0; q < 4; q++) { a[q] = As[k][ty + 16 * q]; b[q] = Bs[k][tx + 16 * q]; }
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) cfmaf(acc[x][y], a[x], b[y]);
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int y = 0; y < 4; y++) {
        int t = tg[tx + 16 * y];
        if (t < 0) continue;
#pragma unroll
        for (int x = 0; x < 4; x++) {
            int r = row0 + ty + 16 * x;
            if (r < NC) {
                double2 *o = out + (size_t)t * NC + r;
                *o = cadd(*o, make_double2((double)acc[x][y].x, (double)acc[x][y].y));
            }
        }
    }
}

void convert_f32(long long n, const double2 *in, float2 *out, cudaStream_t s, Status &st)
{
    if (!st.ok() || n == 0) return;
    k_to_f32<<<(int)((n + 255) / 256), 256, 0, s>>>(n, in, out); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

void launch_m2l_dense32(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                        const long long *slot_toff, const float2 *T, const TreeView &tv, int p, const double2 *in,
                        double2 *out, int prune, cudaStream_t s, Status &st)
{
    if (!st.ok() || ntiles == 0) return;
    dim3 g(ntiles, div_up((p + 1) * (p + 1), k32TM));
    k_m2l_dense32<<<g, k32Threads, 0, s>>>(tiles, grouped, slots, slot_toff, T, tv, p, in, out, prune); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

}  // namespace fmm
