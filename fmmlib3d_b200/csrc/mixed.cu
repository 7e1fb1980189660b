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
// M2L in FP32: the dense per-offset operators (m2l_dense.cu) rounded to FP32,
// box-scaled multipoles (all O(1)) rounded to FP32 on load, FP32
// accumulation, and the tile added to the FP64 local expansion.
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
    double r2 = dx * dx + dy * dy + dz * dz;
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
        double dot = dx * vx + dy * vy + dz * vz;
        double t = dot * ri3;
        a[0] = fma(d.x, t, a[0]);
        a[1] = fma(d.y, t, a[1]);
        double rt = 3.0 * t * ri2;
        double gx = rt * dx - ri3 * vx, gy = rt * dy - ri3 * vy, gz = rt * dz - ri3 * vz;
        a[2] = fma(d.x, gx, a[2]); a[3] = fma(d.y, gx, a[3]);
        a[4] = fma(d.x, gy, a[4]); a[5] = fma(d.y, gy, a[5]);
        a[6] = fma(d.x, gz, a[6]); a[7] = fma(d.y, gz, a[7]);
    }
}

// Warp-synchronous mixed-precision near field.  A CTA of two warps serves
// one childless box; each lane owns two evaluation points (e, e+32 of its
// warp's 64).  The box's own sources, which carry the largest and most
// cancellation-prone terms, are summed in FP64 straight from global memory
// (L1 broadcast); the sources of list 1 are streamed through a per-warp
// 32-entry shared buffer in double-float coordinates and summed in FP32
// with TwoSum-compensated accumulation across chunks, the next chunk being
// prefetched into registers.  No block-wide barrier is needed.
constexpr int kP2P32Threads = 64, kP2P32Warps = kP2P32Threads / 32, kEPT = 2;

template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kP2P32Threads) k_p2p32(const int *leaves, TreeView tv, PointsSoA src,
                                                          const double *tx, const double *ty, const double *tz,
                                                          OutSoA outs, OutSoA outt, int do_src, int do_trg,
                                                          int want_fs, int want_ft, int want_ps, int want_pt)
{
    __shared__ float wp[kP2P32Warps][6][32];
    __shared__ float2 wq[kP2P32Warps][2][32];
    __shared__ float wv[kP2P32Warps][3][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int b = leaves[blockIdx.x];
    const double cx = tv.center[3L * b], cy = tv.center[3L * b + 1], cz = tv.center[3L * b + 2];
    const int s0 = tv.src0[b], nsb = tv.nsrc[b], ns = do_src ? nsb : 0;
    const int t0 = tv.trg0[b], nt = do_trg ? tv.ntrg[b] : 0;
    const int ne = ns + nt;
    const int l1a = tv.l1_start[b], nl = 1 + tv.l1_start[b + 1] - l1a;
    for (int e0 = w * 32 * kEPT; e0 < ne; e0 += kP2P32Threads * kEPT) {
        bool act[kEPT];
        int self[kEPT];
        double ed[kEPT][3];
        float eh[kEPT][3], el[kEPT][3];
        float hi[kEPT][8], lo[kEPT][8];
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
            for (int c = 0; c < 3; c++) split_df(ed[u][c], eh[u][c], el[u][c]);
#pragma unroll
            for (int c = 0; c < 8; c++) { hi[u][c] = 0.f; lo[u][c] = 0.f; }
        }
        // the box's own sources in FP64
        double a64[kEPT][8];
#pragma unroll
        for (int u = 0; u < kEPT; u++)
#pragma unroll
            for (int c = 0; c < 8; c++) a64[u][c] = 0.0;
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
        // list-1 sources in FP32, streamed per warp
        int j = 1, c0 = 0, js0 = 0, jn = 0;
        if (nl > 1) { int jb = tv.l1_idx[l1a]; js0 = tv.src0[jb]; jn = tv.nsrc[jb]; }
        auto advance = [&]() {
            while (j < nl && c0 >= jn) {
                j++;
                c0 = 0;
                if (j < nl) { int jb = tv.l1_idx[l1a + j - 1]; js0 = tv.src0[jb]; jn = tv.nsrc[jb]; }
            }
        };
        advance();
        double px = 0, py = 0, pz = 0, vxx = 0, vyy = 0, vzz = 0;
        double2 pq = cmk(0, 0), pd = cmk(0, 0);
        auto fetch = [&]() {
            int i = c0 + lane;
            if (j < nl && i < jn) {
                i += js0;
                px = src.x[i]; py = src.y[i]; pz = src.z[i];
                if (CHG) pq = src.q[i];
                if (DIP) { pd = src.dq[i]; vxx = src.vx[i]; vyy = src.vy[i]; vzz = src.vz[i]; }
            }
        };
        fetch();
        while (j < nl) {
            const int cn = min(32, jn - c0);
            __syncwarp();
            if (lane < cn) {
                split_df(px - cx, wp[w][0][lane], wp[w][3][lane]);
                split_df(py - cy, wp[w][1][lane], wp[w][4][lane]);
                split_df(pz - cz, wp[w][2][lane], wp[w][5][lane]);
                if (CHG) wq[w][0][lane] = make_float2((float)pq.x, (float)pq.y);
                if (DIP) {
                    wq[w][1][lane] = make_float2((float)pd.x, (float)pd.y);
                    wv[w][0][lane] = (float)vxx; wv[w][1][lane] = (float)vyy; wv[w][2][lane] = (float)vzz;
                }
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
                const float sxh = wp[w][0][k], syh = wp[w][1][k], szh = wp[w][2][k];
                const float sxl = wp[w][3][k], syl = wp[w][4][k], szl = wp[w][5][k];
                const float2 q = CHG ? wq[w][0][k] : make_float2(0.f, 0.f);
                const float2 d = DIP ? wq[w][1][k] : make_float2(0.f, 0.f);
                const float vx = DIP ? wv[w][0][k] : 0.f, vy = DIP ? wv[w][1][k] : 0.f, vz = DIP ? wv[w][2][k] : 0.f;
#pragma unroll
                for (int u = 0; u < kEPT; u++)
                    pair32<CHG, DIP>(eh[u][0], eh[u][1], eh[u][2], el[u][0], el[u][1], el[u][2], sxh, syh, szh,
                                     sxl, syl, szl, q, d, vx, vy, vz, a[u]);
            }
#pragma unroll
            for (int u = 0; u < kEPT; u++)
#pragma unroll
                for (int c = 0; c < 8; c++) two_sum_acc(hi[u][c], lo[u][c], a[u][c]);
        }
#pragma unroll
        for (int u = 0; u < kEPT; u++) {
            if (!act[u]) continue;
            const int e = e0 + lane + 32 * u;
            double r[8];
#pragma unroll
            for (int c = 0; c < 8; c++) r[c] = a64[u][c] + ((double)hi[u][c] + (double)lo[u][c]);
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
        }
    }
}

void launch_p2p32(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                  const double *ty, const double *tz, OutSoA outs, OutSoA outt, int ifcharge, int ifdipole,
                  int ifpot, int iffld, int ifpottarg, int iffldtarg, cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok()) return;
    int do_src = (ifpot == 1 || iffld == 1), do_trg = (ifpottarg == 1 || iffldtarg == 1);
    bool c = ifcharge == 1, d = ifdipole == 1;
    if (c && d) {
        k_p2p32<true, true><<<nleaves, kP2P32Threads, 0, s>>>(leaves, tv, src, tx, ty, tz, outs, outt, do_src,
                                                             do_trg, iffld == 1, iffldtarg == 1, ifpot == 1,
                                                             ifpottarg == 1); FMM_COUNT_LAUNCH();
    } else if (c) {
        k_p2p32<true, false><<<nleaves, kP2P32Threads, 0, s>>>(leaves, tv, src, tx, ty, tz, outs, outt, do_src,
                                                              do_trg, iffld == 1, iffldtarg == 1, ifpot == 1,
                                                              ifpottarg == 1); FMM_COUNT_LAUNCH();
    } else if (d) {
        k_p2p32<false, true><<<nleaves, kP2P32Threads, 0, s>>>(leaves, tv, src, tx, ty, tz, outs, outt, do_src,
                                                              do_trg, iffld == 1, iffldtarg == 1, ifpot == 1,
                                                              ifpottarg == 1); FMM_COUNT_LAUNCH();
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
