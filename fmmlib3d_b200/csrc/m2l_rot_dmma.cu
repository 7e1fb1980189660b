// FP64 rotate-shift-rotate M2L on the FP64 tensor cores (mma.sync m8n8k4 .f64).
//
// The same translation as the rotate-shift-rotate kernel (k_translate<1>,
// lap_kernels.cu) -- l3dmplocquad2_trunc0 (src/l3dtrans.f:1260-1387): per
// list-2 slot the source multipoles times e^{i m phi}, the rotation D(theta)
// degree by degree, the z-shift of l3dmploczshiftstab_fast (:1439-1534)
// order by order, D(theta)^T, times e^{-i m phi}, added into the target's
// local expansion -- with every product a small real GEMM on the tensor
// cores.  A CTA owns a tile of up to 8 target boxes, i.e. 16 real rows (the
// real parts of the 8 expansions, then their imaginary parts): the rows of
// the two 8 x 4 A fragments of every MMA.  Per slot:
//   forward rotation, degree n:  X1[r][n, m'] = sum_m  X0[r][n, m] D_n[m][m']
//   z-shift, order m:            X0[r][j, m]  = sum_l  X1[r][l, m] Z_m(j, l)
//   back rotation, degree n:     E[r][n, m]   = sum_m' X0[r][n, m'] D_n[m][m']
// (D, Z real: the real and imaginary rows share every B fragment.)  The work
// of each product is cut into tasks of one degree (order) and 8 output
// columns, dealt to the 16 warps round robin; the back rotation's tasks are
// dealt the same way for every slot, so each warp keeps the running sums of
// its tasks (8 targets x 8 coefficients) in registers across all slots and
// adds them into the local expansions once at the end.  A rotation task loads
// its B fragments (a column block of D_n, from L2) into registers before its
// MMAs; z-shift B fragments are formed from the binomial table (L1) and the
// powers of rt.  Orders up to kRdMaxP (28): two 16-row expansion buffers in
// shared memory, one CTA of 16 warps per SM.
#include "lap_kernels.cuh"

namespace fmm {

constexpr int kRdWarps = 16;
constexpr int kRdMaxP = 28;
constexpr int kRdMaxTasks = 8;      // back-rotation tasks per warp (orders <= 28: at most 120 tasks)
constexpr int kRdMaxKs = 15;        // K steps of one degree (2 * 28 + 1 = 57 columns: 15 steps of 4)

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Row stride of the expansion buffers: at least (p+1)^2 + 4 (the A fragments
// of a degree's last K step read up to 3 entries past the degree; those meet
// zero B entries and are finite, the buffers being cleared at the start) and
// = 4 (mod 16) doubles, so that the 8 rows x 4 doubles of an A fragment fall
// into two bank wavefronts.
__host__ __device__ inline int rd_ld(int p)
{
    const int nc = (p + 1) * (p + 1) + 4;
    return nc + ((4 - nc % 16) + 16) % 16;
}

// tasks (degree n, block of 8 columns) of the rotations, degree by degree
__host__ __device__ inline int rd_ntasks(int p)
{
    int t = 0;
    for (int n = 0; n <= p; n++) t += (2 * n + 8) / 8;
    return t;
}

// z-shift tasks (order m, block of 8 target degrees) of truncation p
__host__ __device__ inline int rd_nz(int p)
{
    int t = 0;
    for (int m = -p; m <= p; m++) t += (p + 1 - (m < 0 ? -m : m) + 7) / 8;
    return t;
}

// One rotation task: rows fr (real) and 8 + fr (imaginary) of X, degree n
// (columns e0 .. e0 + w - 1), times the column block `col` of the (2n+1)^2
// matrix Dn, read as Dn[k * w + col] (forward, TR = false) or Dn[col * w + k]
// (transposed, TR = true).  KS: K steps held in registers (>= nks); the A
// loads of the last step may run past the degree into finite entries that
// meet zero B entries.
template <int KS, bool TR>
__device__ __forceinline__ void rd_rot_task(const double *X, int LD, int fr, int fq, int w, int e0, int col,
                                            const double *Dn, double &c0r, double &c1r, double &c0i, double &c1i)
{
    const int nks = (w + 3) / 4;
    double bf[KS];
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
        const int kk = 4 * ks + fq;
        bf[ks] = (ks < nks && kk < w && col < w) ? (TR ? Dn[col * w + kk] : Dn[kk * w + col]) : 0.0;
    }
    const double *xr = X + fr * LD + e0 + fq, *xi = X + (8 + fr) * LD + e0 + fq;
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
        if (ks >= nks) break;
        dmma(c0r, c1r, xr[4 * ks], bf[ks]);
        dmma(c0i, c1i, xi[4 * ks], bf[ks]);
    }
}

template <bool TR>
__device__ __forceinline__ void rd_rot(const double *X, int LD, int fr, int fq, int n, int col, const double *Dn,
                                       double &c0r, double &c1r, double &c0i, double &c1i)
{
    const int w = 2 * n + 1, e0 = n * n;
    c0r = c1r = c0i = c1i = 0.0;
    if (w <= 16) rd_rot_task<4, TR>(X, LD, fr, fq, w, e0, col, Dn, c0r, c1r, c0i, c1i);
    else if (w <= 32) rd_rot_task<8, TR>(X, LD, fr, fq, w, e0, col, Dn, c0r, c1r, c0i, c1i);
    else if (w <= 48) rd_rot_task<12, TR>(X, LD, fr, fq, w, e0, col, Dn, c0r, c1r, c0i, c1i);
    else rd_rot_task<kRdMaxKs, TR>(X, LD, fr, fq, w, e0, col, Dn, c0r, c1r, c0i, c1i);
}

__global__ void __launch_bounds__(32 * kRdWarps, 1)
    k_m2l_rot_dmma(const Tile *tiles, const int *grouped, const Slot *slots, TreeView tv, int p, const double *rot,
                   const double *dc, int lddc, const double2 *in, double2 *out, int prune)
{
    extern __shared__ double rd_sm[];
    const int NC = (p + 1) * (p + 1), LD = rd_ld(p), NT = rd_ntasks(p);
    double *X0 = rd_sm, *X1 = X0 + 16 * LD;
    double2 *eph = (double2 *)(X1 + 16 * LD);      // e^{i m phi}, m = 0..p
    double *pw = (double *)(eph + (p + 1));          // rt^-(l+1), l = 0..2p+2
    short *tn = (short *)(pw + 2 * p + 3);           // task -> degree
    short *tb = tn + NT;                             // task -> column block
    short *em = tb + NT;                             // coefficient index -> m
    short *zt = em + NC;                             // z-shift tasks of the slot's truncation: (m + p) << 8 | block
    __shared__ int tg[8], sv[8];
    __shared__ int anyv, zpt, nzs;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int fr = lane >> 2, fq = lane & 3;          // fragment row (target) and quad index
    const Tile tile = tiles[blockIdx.x];
    if (tid < 8) tg[tid] = tid < tile.count ? grouped[tile.first + tid] : -1;
    for (int t = 0, n = 0; n <= p; n++)
        for (int b = 0; b < (2 * n + 8) / 8; b++, t++)
            if (t % (32 * kRdWarps) == tid) { tn[t] = (short)n; tb[t] = (short)b; }
    for (int e = tid; e < NC; e += 32 * kRdWarps) {
        int n = (int)sqrtf((float)e);
        while (n * n > e) n--;
        while ((n + 1) * (n + 1) <= e) n++;
        em[e] = (short)(e - n * n - n);
    }
    for (int i = tid; i < 32 * LD; i += 32 * kRdWarps) X0[i] = 0.0;   // X0 and X1
    if (tid == 0) zpt = -1;
    const size_t csz = rot_class_size(p);
    double acc[kRdMaxTasks][4];   // back-rotation running sums: (re, im) of columns oc, oc + 1
#pragma unroll
    for (int i = 0; i < kRdMaxTasks; i++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[i][c] = 0.0;

    for (int si = 0; si < tile.nslot; si++) {
        const Slot sl = slots[tile.slot0 + si];
        __syncthreads();
        if (tid == 0) anyv = 0;
        __syncthreads();
        if (tid < 8) {
            const int t = tg[tid];
            int sb = -1;
            if (t >= 0 && !(prune && tv.ntrg[t] == 0)) {
                const int P = tv.parent[t];
                const int C = P >= 0 ? tv.coll[27L * P + sl.coll] : -1;
                sb = C >= 0 ? tv.child[8L * C + sl.oct] : -1;
                if (sb >= 0 && tv.nsrc[sb] == 0) sb = -1;
            }
            sv[tid] = sb;
            if (sb >= 0) atomicOr(&anyv, 1);
        }
        if (tid == 32) {
            double2 e1 = cmk(sl.ex, sl.ey), e = cmk(1, 0);
            for (int m = 0; m <= p; m++) { eph[m] = e; e = cmul(e, e1); }
        }
        if (tid == 64) {
            const double ir = 1.0 / sl.rt;
            double x = ir;
            for (int l = 0; l <= 2 * p + 2; l++) { pw[l] = x; x *= ir; }
        }
        if (tid == 96 && zpt != sl.pt) {
            int t = 0;
            for (int m = -sl.pt; m <= sl.pt; m++) {
                const int L = sl.pt + 1 - (m < 0 ? -m : m);
                for (int b = 0; b < (L + 7) / 8; b++) zt[t++] = (short)(((m + p) << 8) | b);
            }
            nzs = t;
            zpt = sl.pt;
        }
        __syncthreads();
        if (!anyv) continue;
        const int pt = sl.pt, R = (pt + 1) * (pt + 1);
        // gather, times e^{i m phi}: real parts to rows 0..7, imaginary parts to rows 8..15
        for (int i = tid; i < 8 * R; i += 32 * kRdWarps) {
            const int k = i / R, e = i - k * R;
            const int sb = sv[k];
            double2 v = cmk(0, 0);
            if (sb >= 0) {
                const int m = em[e];
                const double2 ph = m >= 0 ? eph[m] : cconj(eph[-m]);
                v = cmul(in[(size_t)sb * NC + e], ph);
            }
            X0[k * LD + e] = v.x;
            X0[(8 + k) * LD + e] = v.y;
        }
        __syncthreads();
        const double *Rc = rot + csz * sl.cls;
        const int NTs = rd_ntasks(pt), nz = nzs;
        // forward rotation
        for (int t = warp; t < NTs; t += kRdWarps) {
            const int n = tn[t], b = tb[t], w = 2 * n + 1, e0 = n * n;
            const double *Dn = Rc + (size_t)n * (4 * n * n - 1) / 3;
            double c0r, c1r, c0i, c1i;
            rd_rot<false>(X0, LD, fr, fq, n, 8 * b + fr, Dn, c0r, c1r, c0i, c1i);
            const int oc = 8 * b + 2 * fq;
            if (oc < w) { X1[fr * LD + e0 + oc] = c0r; X1[(8 + fr) * LD + e0 + oc] = c0i; }
            if (oc + 1 < w) { X1[fr * LD + e0 + oc + 1] = c1r; X1[(8 + fr) * LD + e0 + oc + 1] = c1i; }
        }
        __syncthreads();
        // z-shift, order by order: out (j, m) = sum_l c(j, l, m) in (l, m), j, l in |m| .. pt,
        // c = (-1)^(j+|m|) sqrt(C(l+j, l-m) C(l+j, l+m)) / rt^(l+j+1)
        for (int t = warp; t < nz; t += kRdWarps) {
            const int m = (zt[t] >> 8) - p, b = zt[t] & 255;
            const int am = m < 0 ? -m : m, L = pt + 1 - am, nks = (L + 3) / 4;
            const int j = am + 8 * b + fr;   // this lane's B column (target degree)
            const double sg = ((j + am) & 1) ? -1.0 : 1.0;
            double c0r = 0, c1r = 0, c0i = 0, c1i = 0;
            for (int ks = 0; ks < nks; ks++) {
                const int l = am + 4 * ks + fq;   // this lane's K index (source degree)
                double bz = 0.0, ar = 0.0, ai = 0.0;
                if (l <= pt) {
                    const int ei = l * l + l + m;
                    ar = X1[fr * LD + ei];
                    ai = X1[(8 + fr) * LD + ei];
                    if (j <= pt) {
                        const int lj = l + j;
                        bz = sg * pw[lj] * dc[lj * lddc + (l - m)] * dc[lj * lddc + (l + m)];
                    }
                }
                dmma(c0r, c1r, ar, bz);
                dmma(c0i, c1i, ai, bz);
            }
            const int j0 = am + 8 * b + 2 * fq;
            if (j0 <= pt) {
                const int eo = j0 * j0 + j0 + m;
                X0[fr * LD + eo] = c0r;
                X0[(8 + fr) * LD + eo] = c0i;
            }
            if (j0 + 1 <= pt) {
                const int eo = (j0 + 1) * (j0 + 1) + (j0 + 1) + m;
                X0[fr * LD + eo] = c1r;
                X0[(8 + fr) * LD + eo] = c1i;
            }
        }
        __syncthreads();
        // back rotation, times e^{-i m phi}, into the running sums (tasks dealt as at the end)
        const bool live = sv[fr] >= 0;
#pragma unroll
        for (int lt = 0; lt < kRdMaxTasks; lt++) {
            const int t = kRdWarps * lt + warp;
            if (t >= NTs) break;
            const int n = tn[t], b = tb[t], w = 2 * n + 1;
            const double *Dn = Rc + (size_t)n * (4 * n * n - 1) / 3;
            double c0r, c1r, c0i, c1i;
            rd_rot<true>(X0, LD, fr, fq, n, 8 * b + fr, Dn, c0r, c1r, c0i, c1i);
            if (live) {
                const int oc = 8 * b + 2 * fq;
                const int m0 = oc - n, m1 = oc + 1 - n;
                if (oc < w) {
                    const double2 ph = m0 >= 0 ? cconj(eph[m0]) : eph[-m0];
                    const double2 z = cmul(cmk(c0r, c0i), ph);
                    acc[lt][0] += z.x;
                    acc[lt][1] += z.y;
                }
                if (oc + 1 < w) {
                    const double2 ph = m1 >= 0 ? cconj(eph[m1]) : eph[-m1];
                    const double2 z = cmul(cmk(c1r, c1i), ph);
                    acc[lt][2] += z.x;
                    acc[lt][3] += z.y;
                }
            }
        }
    }
    __syncthreads();
    // add the running sums into the local expansions
    const int t = tg[fr];
    if (t < 0) return;
#pragma unroll
    for (int lt = 0; lt < kRdMaxTasks; lt++) {
        const int ti = kRdWarps * lt + warp;
        if (ti >= NT) break;
        const int n = tn[ti], b = tb[ti], w = 2 * n + 1, oc = 8 * b + 2 * fq;
        double2 *o = out + (size_t)t * NC + n * n;
        if (oc < w) o[oc] = cadd(o[oc], cmk(acc[lt][0], acc[lt][1]));
        if (oc + 1 < w) o[oc + 1] = cadd(o[oc + 1], cmk(acc[lt][2], acc[lt][3]));
    }
}

bool m2l_rot_dmma_supported(int p) { return p >= 1 && p <= kRdMaxP && rd_ntasks(p) <= kRdWarps * kRdMaxTasks; }

void launch_m2l_rot_dmma(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots, const TreeView &tv,
                         int p, const double *rot, const double *dc, int lddc, const double2 *in, double2 *out,
                         int prune, cudaStream_t s, Status &st)
{
    if (ntiles == 0 || !st.ok()) return;
    const size_t sm = sizeof(double) * (32 * (size_t)rd_ld(p)) + sizeof(double2) * (p + 1) +
                      sizeof(double) * (2 * p + 3) +
                      sizeof(short) * (2 * rd_ntasks(p) + (p + 1) * (p + 1) + rd_nz(p));
    FMM_TRY(st, smem_allow(k_m2l_rot_dmma, (int)sm));
    if (!st.ok()) return;
    k_m2l_rot_dmma<<<ntiles, 32 * kRdWarps, sm, s>>>(tiles, grouped, slots, tv, p, rot, dc, lddc, in, out, prune);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

}  // namespace fmm
