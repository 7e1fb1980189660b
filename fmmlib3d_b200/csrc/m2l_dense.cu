// M2L as gathered dense GEMMs, one operator per translation offset (p <= 16).
//
// For a list-2 offset D (source box minus target box, in box units) the
// rotate-shift-rotate M2L of FMMLIB3D (l3dmplocquad2_trunc0,
// src/l3dtrans.f:1260-1387, truncated to nterms_trunc = pt) is a fixed
// linear map T_D from the (pt+1)^2 source coefficients to the (pt+1)^2
// target coefficients; with box-scaled coefficients it does not depend on
// the level.  k_build_m2l_ops composes T_D column by column on the GPU from
// the same rotation matrices and z-shift coefficients as the structured
// kernel:  T_D[(j,m)][(n,mc)] = e^{-i m phi} sum_k D^j[m][k] Z(j,k,n) D^n[mc][k] e^{i mc phi},
// Z(j,k,n) = (-1)^(j+k) sqrt(C(n+j,n-k) C(n+j,n+k)) / rt^(n+j+1).
// k_m2l_dense then computes, for the targets of one (level, octant) group,
//   L[:, t] += sum_slots T_{D(slot)} M[:, src(t, slot)]
// with a CTA owning a 64-row x 64-target tile of L and streaming the 189 slots
// (A = T tile, B = gathered source multipoles), so no output is shared
// between CTAs and no atomics are needed.
#include "lap_kernels.cuh"
#include "m2l_dense.cuh"

namespace fmm {

__global__ void k_build_m2l_ops(int p, const M2LOp *ops, const double *rot, const double *dc, int lddc,
                                double2 *T)
{
    const M2LOp op = ops[blockIdx.x];  // one unique offset per block row
    const int pt = op.pt, R = (pt + 1) * (pt + 1);
    const int col = blockIdx.y;
    if (col >= R) return;
    int nc = 0;
    while ((nc + 1) * (nc + 1) <= col) nc++;
    const int mc = col - nc * nc - nc;
    const size_t csz = rot_class_size(p);
    const double *Rm = rot + csz * op.cls;
    const double *Dn = Rm + (size_t)nc * (4 * nc * nc - 1) / 3 + (size_t)(mc + nc) * (2 * nc + 1);  // row mc
    // e^{i mc phi}
    double2 e1 = cmk(op.ex, op.ey), em = cmk(1, 0);
    for (int i = 0; i < (mc < 0 ? -mc : mc); i++) em = cmul(em, e1);
    if (mc < 0) em = cconj(em);
    for (int row = threadIdx.x; row < R; row += blockDim.x) {
        int j = 0;
        while ((j + 1) * (j + 1) <= row) j++;
        int m = row - j * j - j;
        const double *Dj = Rm + (size_t)j * (4 * j * j - 1) / 3 + (size_t)(m + j) * (2 * j + 1);
        int kmax = j < nc ? j : nc;
        double s = 0;
        double ir = 1.0 / op.rt, pw = 1;
        for (int i = 0; i < nc + j + 1; i++) pw *= ir;
        for (int k = -kmax; k <= kmax; k++) {
            double z = (((j + k) & 1) ? -1.0 : 1.0) * pw * dc[(nc + j) * lddc + (nc - k)] * dc[(nc + j) * lddc + (nc + k)];
            s += Dj[k + j] * z * Dn[k + nc];
        }
        // times e^{i mc phi} e^{-i m phi}
        double2 ph = em;
        double2 en = cmk(1, 0);
        for (int i = 0; i < (m < 0 ? -m : m); i++) en = cmul(en, e1);
        ph = m >= 0 ? cmulc(ph, en) : cmul(ph, en);
        T[op.toff + (size_t)col * R + row] = cscal(s, ph);  // column-major
    }
}

// ---------------------------------------------------------------- the GEMM
// kTN targets per tile: 64, or 16 when the problem is too small to fill the
// GPU with 64-target tiles; the small tiles take the operator in K blocks of
// 64 instead of 16 (fewer round trips to L2 per slot, which is what bounds a
// CTA that walks all 189 slots on a small problem).  The source boxes of the
// next slot are looked up while the current slot is multiplied.  Every
// target's sums are formed in the same order in all variants.
constexpr int kTM = 64, kDenseThreads = 256;

template <int kTN, int kTK>
__global__ void __launch_bounds__(kDenseThreads, 2) k_m2l_dense(const Tile *tiles, const int *grouped,
                                                             const Slot *slots, const long long *slot_toff,
                                                             const double2 *T, TreeView tv, int p,
                                                             const double2 *in, double2 *out, int prune)
{
    constexpr int NY = kTN / 16;                       // targets per thread
    constexpr int APT = kTM * kTK / kDenseThreads;     // A entries staged per thread
    constexpr int BPT = kTN * kTK / kDenseThreads;     // B entries staged per thread
    extern __shared__ double2 dsm[];
    double2(*As)[kTM] = reinterpret_cast<double2(*)[kTM]>(dsm);               // As[k][row]
    double2(*Bs)[kTN] = reinterpret_cast<double2(*)[kTN]>(dsm + kTK * kTM);   // Bs[k][target]
    __shared__ int tg[kTN], sv[kTN];
    const Tile tile = tiles[blockIdx.x];
    const int row0 = blockIdx.y * kTM;
    const int NC = (p + 1) * (p + 1);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads; rows ty+16x, targets tx+16y
    if (threadIdx.x < kTN) tg[threadIdx.x] = threadIdx.x < tile.count ? grouped[tile.first + threadIdx.x] : -1;
    double2 acc[4][NY];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < NY; b++) acc[a][b] = cmk(0, 0);
    __syncthreads();
    // source box of target threadIdx.x (< kTN) for slot si, -1 if none
    auto source_box = [&](int si) {
        const int t = tg[threadIdx.x];
        int sb = -1;
        if (t >= 0 && !(prune && tv.ntrg[t] == 0)) {
            const Slot sl = slots[tile.slot0 + si];
            const int P = tv.parent[t];
            const int C = P >= 0 ? tv.coll[27L * P + sl.coll] : -1;
            sb = C >= 0 ? tv.child[8L * C + sl.oct] : -1;
            if (sb >= 0 && tv.nsrc[sb] == 0) sb = -1;
        }
        return sb;
    };
    int next_sb = (threadIdx.x < kTN && tile.nslot > 0) ? source_box(0) : -1;
    for (int si = 0; si < tile.nslot; si++) {
        const int cur_sb = next_sb;
        if (threadIdx.x < kTN && si + 1 < tile.nslot) next_sb = source_box(si + 1);
        const Slot sl = slots[tile.slot0 + si];
        const int R = (sl.pt + 1) * (sl.pt + 1);
        if (row0 >= R) continue;  // uniform over the CTA
        __syncthreads();
        if (threadIdx.x < kTN) sv[threadIdx.x] = cur_sb;
        if (!__syncthreads_or(threadIdx.x < kTN && cur_sb >= 0)) continue;
        const double2 *Tu = T + slot_toff[tile.slot0 + si];
        for (int k0 = 0; k0 < R; k0 += kTK) {
            // A tile: rows row0.., cols k0..; consecutive threads take consecutive
            // rows of a column (the operators are column-major)
            {
                int r = threadIdx.x & 63, c = (threadIdx.x >> 6) * APT;
                int gr = row0 + r;
#pragma unroll
                for (int q = 0; q < APT; q++) {
                    int gc = k0 + c + q;
                    As[c + q][r] = (gr < R && gc < R) ? Tu[(size_t)gc * R + gr] : cmk(0, 0);
                }
            }
            // B tile: targets j, coefficients k0..; gathered source multipoles
            {
                int j = threadIdx.x % kTN, c = (threadIdx.x / kTN) * BPT;
                int sb = sv[j];
#pragma unroll
                for (int q = 0; q < BPT; q++) {
                    int gc = k0 + c + q;
                    Bs[c + q][j] = (sb >= 0 && gc < R) ? in[(size_t)sb * NC + gc] : cmk(0, 0);
                }
            }
            __syncthreads();
#pragma unroll 4
            for (int k = 0; k < kTK; k++) {
                double2 a[4], b[NY];
#pragma unroll
                for (int q = 0; q < 4; q++) a[q] = As[k][ty + 16 * q];
#pragma unroll
                for (int q = 0; q < NY; q++) b[q] = Bs[k][tx + 16 * q];
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < NY; y++) cfma(acc[x][y], a[x], b[y]);
            }
            __syncthreads();
        }
    }
    // epilogue: this CTA owns rows row0..row0+63 of its targets
#pragma unroll
    for (int y = 0; y < NY; y++) {
        int t = tg[tx + 16 * y];
        if (t < 0) continue;
#pragma unroll
        for (int x = 0; x < 4; x++) {
            int r = row0 + ty + 16 * x;
            if (r < NC) {
                double2 *o = out + (size_t)t * NC + r;
                *o = cadd(*o, acc[x][y]);
            }
        }
    }
}

void build_m2l_ops(int p, int nops, const M2LOp *d_ops, const double *rot, const double *dc, int lddc,
                   double2 *T, cudaStream_t s, Status &st)
{
    if (!st.ok() || nops == 0) return;
    dim3 g(nops, (p + 1) * (p + 1));
    k_build_m2l_ops<<<g, 128, 0, s>>>(p, d_ops, rot, dc, lddc, T); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

void launch_m2l_dense(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                      const long long *slot_toff, const double2 *T, const TreeView &tv, int p, const double2 *in,
                      double2 *out, int prune, int kt, cudaStream_t s, Status &st)
{
    if (!st.ok() || ntiles == 0) return;
    dim3 g(ntiles, div_up((p + 1) * (p + 1), kTM));
    if (kt <= 16) {
        constexpr size_t sm = sizeof(double2) * 64 * (kTM + 16);
        FMM_TRY(st, smem_allow(k_m2l_dense<16, 64>, (int)sm));
        k_m2l_dense<16, 64><<<g, kDenseThreads, sm, s>>>(tiles, grouped, slots, slot_toff, T, tv, p, in, out, prune); FMM_COUNT_LAUNCH();
    } else {
        constexpr size_t sm = sizeof(double2) * 16 * (kTM + 64);
        k_m2l_dense<64, 16><<<g, kDenseThreads, sm, s>>>(tiles, grouped, slots, slot_toff, T, tv, p, in, out, prune); FMM_COUNT_LAUNCH();
    }
    FMM_LAUNCH_CHECK(st);
}

}  // namespace fmm
