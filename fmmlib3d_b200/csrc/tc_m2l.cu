// M2L on the Blackwell tensor cores (mixed form, nterms <= 16).
//
// The dense per-offset operators T_D (m2l_dense.cu) applied to gathered source
// multipoles are products of complex matrices.  Here each CTA owns 64 complex
// rows of the local expansions of a tile of up to NMAX (128, or 256 as a
// tuning option) target boxes and streams the tile's 189 list-2 slots:
//   D[r, t] += sum_k A[r, k] B[t, k]
// with the complex product embedded in real arithmetic:
//   A rows 0..63   (real parts):      [Re T, -Im T] interleaved per column,
//   A rows 64..127 (imaginary parts): [Im T,  Re T],
//   B (per target): [Re M, Im M] interleaved per coefficient.
// A and B are rounded to FP32, split into TF32 pairs x = hi + lo (both
// rounded to nearest, so hi + lo is x to about 2^-24), and
// D += A_hi B_hi + A_hi B_lo + A_lo B_hi (+ A_lo B_lo with nprod 4) is issued
// as tcgen05.mma kind::tf32 (M = 128, N = targets, K = 8) by one thread, with D
// in TMEM (FP32).
// Operands are staged in shared memory by all threads (gather of the source
// multipoles, split, K-major no-swizzle layout) in a ring of S stages; each
// stage is released by a tcgen05.commit on its mbarrier.  The global loads of
// a stage are issued two stages ahead (a register ring), and the gather chain
// of the next slot (colleague, then child box) is loaded while the current
// slot's stages run.  The tensor cores accumulate a group of slots (TMEM
// columns 0..NMAX-1); the group's sum is then added by the CUDA cores, with
// round-to-nearest FP32 additions, into a running sum held in TMEM columns
// NMAX..2 NMAX-1: long tensor-core accumulations lose accuracy, groups of a
// few slots keep the FP32 CUDA-core form's error.
// At the end every warp reads its TMEM lane quarter of the running sum and
// adds the tile into the FP64 locals.
// Every wait is bounded: on expiry the kernel records an error, waits (again
// bounded) for its own MMAs, frees its TMEM and returns.
#include "lap_kernels.cuh"
#include "m2l_dense.cuh"
#include "tc_common.cuh"

namespace fmm {

constexpr int kTcThreads = 256;
constexpr uint32_t kTcLBO = 128 * 16 + 16;           // K-block stride (bytes): 128 rows + 16 B pad
constexpr long long kTcWaitCycles = 2000000000LL;    // ~1 s at 2 GHz

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *mbar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_wait(mbar, parity, 64))
        if (clock64() - t0 > kTcWaitCycles) return false;
    return true;
}

__device__ __forceinline__ void split4(float4 v, float4 &h, float4 &l)
{
    split_tf32(v.x, h.x, l.x);
    split_tf32(v.y, h.y, l.y);
    split_tf32(v.z, h.z, l.z);
    split_tf32(v.w, h.w, l.w);
}

// Issue the MMAs of one stage: K = KC in steps of 8; per step the product of
// the high parts and, for nprod >= 3, the two cross products, for nprod >= 4
// also the product of the low parts (then the sum is the exact product of
// hi + lo, i.e. of the operands to within about 2^-24 each).
// Stage layout: A_hi, A_lo (128 rows, K-block stride kTcLBO), then B_hi, B_lo
// (NMAX rows, K-block stride NMAX * 16 + 16).
template <int KC, int NMAX = 128>
__device__ __forceinline__ void issue_stage(uint32_t base, uint32_t tm, uint32_t idesc, bool first, int nprod)
{
    constexpr uint32_t LBOB = NMAX * 16 + 16;
    constexpr uint32_t OPA = (KC / 4) * kTcLBO, OPBB = (KC / 4) * LBOB;
#pragma unroll
    for (int s = 0; s < KC / 8; s++) {
        const uint32_t oa = 2 * s * kTcLBO, ob = 2 * s * LBOB;
        const uint64_t ah = tc_desc(base + oa, kTcLBO, 128), al = tc_desc(base + OPA + oa, kTcLBO, 128);
        const uint64_t bh = tc_desc(base + 2 * OPA + ob, LBOB, 128), bl = tc_desc(base + 2 * OPA + OPBB + ob, LBOB, 128);
        tc_mma_tf32(tm, ah, bh, idesc, (first && s == 0) ? 0u : 1u);
        if (nprod >= 3) {
            tc_mma_tf32(tm, ah, bl, idesc, 1u);
            tc_mma_tf32(tm, al, bh, idesc, 1u);
        }
        if (nprod >= 4) tc_mma_tf32(tm, al, bl, idesc, 1u);
    }
}

// NMAX: targets per tile at most (128: two CTAs per SM, 256 TMEM columns;
// 256: one CTA per SM, 512 TMEM columns, each staged operator serves twice
// the targets).
template <int KC, int S, int NMAX>
__global__ void __launch_bounds__(kTcThreads, NMAX == 128 ? 2 : 1)
    k_m2l_tc(const Tile *tiles, const int *grouped, const Slot *slots, const long long *slot_toff, const float2 *T,
             TreeView tv, int p, const float2 *mp, int ldm, double2 *out, int prune, int nprod, int group, int *err,
             int expire_stage_waits)
{
    constexpr int KB = KC / 4;                 // 16-byte K blocks per stage
    constexpr uint32_t OPB = KB * kTcLBO;      // one A buffer
    constexpr uint32_t LBOB = NMAX * 16 + 16;  // K-block stride of B
    constexpr uint32_t OPBB = KB * LBOB;       // one B buffer
    constexpr uint32_t STB = 2 * OPB + 2 * OPBB;   // A_hi, A_lo, B_hi, B_lo
    constexpr int TPP = kTcThreads / KB;       // targets staged per pass
    constexpr int NPASS = NMAX / TPP;
    constexpr int TCOLS = 2 * NMAX;            // TMEM columns: tensor-core sum, running sum
    constexpr int HC = NMAX / 2;               // columns per warp (two warps per lane quarter)
    constexpr int NA = 64 * KB / kTcThreads;   // operator pairs staged per thread
    static_assert(64 * KB % kTcThreads == 0, "stage tasks must divide evenly");
    extern __shared__ unsigned char tc_smraw[];
    unsigned char *sm = (unsigned char *)(((uintptr_t)tc_smraw + 127) & ~(uintptr_t)127);
    __shared__ uint64_t mbar[S];
    __shared__ uint32_t tbase;
    __shared__ int tg[NMAX];
    const Tile tile = tiles[blockIdx.x];
    const int row0 = 64 * blockIdx.y;          // first complex row of this CTA
    const int NC = (p + 1) * (p + 1);
    const int N = max(16, (tile.count + 15) & ~15);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int n = tid; n < NMAX; n += kTcThreads) tg[n] = n < tile.count ? grouped[tile.first + n] : -1;
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(&mbar[s], 1);
        mbar_fence_init();
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(&tbase, TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = tbase;
    const uint32_t idesc = tc_idesc_tf32(128, N);
    const uint32_t sbase = smem_u32(sm);
    const int q = warp & 3, h = warp >> 2;     // TMEM lane quarter and column half of this warp
    const uint32_t tD = tm + ((uint32_t)(32 * q) << 16) + (uint32_t)(HC * h);   // tensor-core sum (0 .. NMAX-1)
    const uint32_t tA = tD + NMAX;                                              // FP32 running sum (NMAX .. 2 NMAX-1)
    int it = 0;
    bool aborted = false, fresh = true;        // fresh: the next MMA starts a new TMEM sum
    bool have_acc = false;                     // the running sum holds flushed groups
    // Add the tensor-core sum of the group that ends with item it - 1 into the running sum.
    auto flush = [&]() {
        const int last = it - 1;
        const bool done = mbar_wait_bounded(&mbar[last % S], (last / S) & 1);
        if (__syncthreads_or(!done)) { aborted = true; return; }
        tc_fence_after();
        // 32 columns at a time, both loads under one wait, the stores completed once
        // (columns past N within a 32-column block hold unused values)
#pragma unroll
        for (int c0 = 0; c0 < HC; c0 += 32) {
            if (HC * h + c0 < N) {
                float v[32], a[32];
                tmem_ld32x2(tD + c0, tA + c0, v, a);
                if (have_acc) {
#pragma unroll
                    for (int u = 0; u < 32; u++) v[u] += a[u];
                }
                tmem_st32(tA + c0, v);
            }
        }
        tmem_wait_st();
        tc_fence_before();
        __syncthreads();
        fresh = true;
        have_acc = true;
    };
    // Source boxes of the staged targets for a slot: colleague of the target's
    // parent, then that colleague's child.  Empty source boxes are not skipped:
    // their multipoles are zero and add exact zeros.  The chain of the next slot
    // is loaded while the current slot's stages run (colleagues with the first
    // stage, children after it), so its dependent loads stay off the critical path.
    int par[NPASS], cnx[NPASS], sbn[NPASS];
#pragma unroll
    for (int j = 0; j < NPASS; j++) {
        const int n = tid / KB + TPP * j;
        const int t = n < tile.count ? tg[n] : -1;
        par[j] = (t >= 0 && !(prune && tv.ntrg[t] == 0)) ? tv.parent[t] : -1;
    }
    auto chain_coll = [&](const Slot &x) {
#pragma unroll
        for (int j = 0; j < NPASS; j++) cnx[j] = par[j] >= 0 ? tv.coll[27L * par[j] + x.coll] : -1;
    };
    auto chain_child = [&](const Slot &x) {
#pragma unroll
        for (int j = 0; j < NPASS; j++) sbn[j] = cnx[j] >= 0 ? tv.child[8L * cnx[j] + x.oct] : -1;
    };
    Slot sl_next = slots[tile.slot0];
    chain_coll(sl_next);
    chain_child(sl_next);
    for (int si = 0; si < tile.nslot && !aborted; si++) {
        const Slot sl = sl_next;
        int sbr[NPASS];
#pragma unroll
        for (int j = 0; j < NPASS; j++) sbr[j] = sbn[j];
        const bool has_next = si + 1 < tile.nslot;
        int chain = 0;   // next slot's chain: 0 not started, 1 colleagues loaded, 2 source boxes loaded
        if (has_next) sl_next = slots[tile.slot0 + si + 1];
        do {  // one slot; break = nothing to add for it
            const int R = (sl.pt + 1) * (sl.pt + 1);
            if (row0 >= R) break;
            int have = 0;
#pragma unroll
            for (int j = 0; j < NPASS; j++) have |= sbr[j] >= 0;
            if (!__syncthreads_or(have)) break;
            if (has_next) { chain_coll(sl_next); chain = 1; }
            const float2 *Tu = T + slot_toff[tile.slot0 + si];
            const int nk = (2 * R + KC - 1) / KC;
            // registers of two stages in flight: operator pairs (A) and multipole pairs (B)
            float2 ra0[2][NA], ra1[2][NA];
            float4 rb[2][NPASS];
            // A: operator rows row0 .. row0 + 63, columns jb .. jb + KC/2 - 1 (column-major T);
            // B: the gathered source multipoles, coefficients jb .. jb + KC/2 - 1
            auto load = [&](int kc, int set) {
                const int jb = kc * (KC / 2);
#pragma unroll
                for (int a = 0; a < NA; a++) {
                    const int task = tid + a * kTcThreads, i = task & 63, kb = task >> 6;
                    const int row = row0 + i, j0 = jb + 2 * kb;
                    ra0[set][a] = (row < R && j0 < R) ? Tu[(size_t)j0 * R + row] : make_float2(0.f, 0.f);
                    ra1[set][a] = (row < R && j0 + 1 < R) ? Tu[(size_t)(j0 + 1) * R + row] : make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int j = 0; j < NPASS; j++) {
                    const int n = tid / KB + TPP * j, kb = tid % KB, j0 = jb + 2 * kb;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (n < N && sbr[j] >= 0 && j0 < R) {
                        v = *(const float4 *)(mp + (size_t)sbr[j] * ldm + j0);
                        if (j0 + 1 >= R) { v.z = 0.f; v.w = 0.f; }
                    }
                    rb[set][j] = v;
                }
            };
            auto store = [&](unsigned char *base, int set) {
#pragma unroll
                for (int a = 0; a < NA; a++) {
                    const int task = tid + a * kTcThreads, i = task & 63, kb = task >> 6;
                    const float2 v0 = ra0[set][a], v1 = ra1[set][a];
                    float4 h, l;
                    unsigned char *ah = base + kb * kTcLBO, *al = base + OPB + kb * kTcLBO;
                    // one split serves both rows: rounding to nearest is odd, so the
                    // parts of -x are those of x negated
                    split4(make_float4(v0.x, v0.y, v1.x, v1.y), h, l);
                    *(float4 *)(ah + i * 16) = make_float4(h.x, -h.y, h.z, -h.w);
                    *(float4 *)(al + i * 16) = make_float4(l.x, -l.y, l.z, -l.w);
                    *(float4 *)(ah + (64 + i) * 16) = make_float4(h.y, h.x, h.w, h.z);
                    *(float4 *)(al + (64 + i) * 16) = make_float4(l.y, l.x, l.w, l.z);
                }
#pragma unroll
                for (int j = 0; j < NPASS; j++) {
                    const int n = tid / KB + TPP * j, kb = tid % KB;
                    if (n >= N) continue;
                    float4 h, l;
                    split4(rb[set][j], h, l);
                    *(float4 *)(base + 2 * OPB + kb * LBOB + n * 16) = h;
                    *(float4 *)(base + 2 * OPB + OPBB + kb * LBOB + n * 16) = l;
                }
            };
            // one stage: wait for its ring slot, stage it, start the loads two stages
            // ahead, then one thread issues its MMAs
            auto stage = [&](int kc, int set) {
                const int st = it % S;
                int late = 0;
                // (expire_stage_waits: the error-path test, every stage wait counts as expired)
                if (it >= S && (expire_stage_waits || !mbar_wait_bounded(&mbar[st], ((it - S) / S) & 1))) late = 1;
                store(sm + st * STB, set);
                if (kc + 2 < nk) load(kc + 2, set);
                fence_async_smem();
                if (__syncthreads_or(late)) { aborted = true; return false; }
                if (tid == 0) {
                    tc_fence_after();
                    issue_stage<KC, NMAX>(sbase + st * STB, tm, idesc, fresh && kc == 0, nprod);
                    tc_commit(&mbar[st]);
                }
                fresh = false;
                it++;
                if (chain == 1) { chain_child(sl_next); chain = 2; }
                return true;
            };
            load(0, 0);
            if (nk > 1) load(1, 1);
            for (int kc = 0; kc < nk; kc += 2) {
                if (!stage(kc, 0)) break;
                if (kc + 1 < nk && !stage(kc + 1, 1)) break;
            }
        } while (0);
        if (has_next && !aborted) {
            if (chain == 0) chain_coll(sl_next);
            if (chain <= 1) chain_child(sl_next);
        }
        // group boundaries at fixed slot indices, so a target's sums do not
        // depend on which other targets share its tile
        if (!aborted && group > 0 && (si + 1) % group == 0 && !fresh) flush();
    }
    if (!aborted && !fresh) flush();
    int bad = aborted ? 1 : 0;
    if (!bad && have_acc) {
        tc_fence_after();
        const int L = 32 * q + lane, ci = L & 63, part = L >> 6, row = row0 + ci;
#pragma unroll
        for (int c0 = 0; c0 < HC; c0 += 16) {
            if (HC * h + c0 < N) {
                float v[16];
                tmem_ld16(tA + c0, v);
                if (row < NC) {
#pragma unroll
                    for (int u = 0; u < 16; u++) {
                        const int n = HC * h + c0 + u;
                        const int t = n < tile.count ? tg[n] : -1;
                        if (t >= 0) {
                            double *o = (double *)(out + (size_t)t * NC + row) + part;
                            *o += (double)v[u];
                        }
                    }
                }
            }
        }
    }
    if (aborted && it > 0) {
        // let this CTA's own MMAs finish (bounded) before its TMEM is released
        const int last = it - 1;
        mbar_wait_bounded(&mbar[last % S], (last / S) & 1);
    }
    if (bad && tid == 0) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tm, TCOLS);
}

// Test hook (fmm3d_inject_tc_wait_expiry): the tensor-core M2L kernels this
// host thread launches treat every stage wait as expired.
static thread_local int g_tc_expire_waits = 0;

template <int KC, int S, int NMAX>
static void launch_tc_t(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                        const long long *slot_toff, const float2 *T, const TreeView &tv, int p, const float2 *mp,
                        int ldm, double2 *out, int prune, int nprod, int group, int *err, cudaStream_t s,
                        Status &st)
{
    const size_t sm = (size_t)S * 2 * (KC / 4) * (kTcLBO + NMAX * 16 + 16) + 128;
    FMM_TRY(st, smem_allow(k_m2l_tc<KC, S, NMAX>, (int)sm));
    dim3 g(ntiles, div_up((p + 1) * (p + 1), 64));
    k_m2l_tc<KC, S, NMAX><<<g, kTcThreads, sm, s>>>(tiles, grouped, slots, slot_toff, T, tv, p, mp, ldm, out, prune, nprod,
                                              group, err, g_tc_expire_waits); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

void launch_m2l_tc(int variant, const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                   const long long *slot_toff, const float2 *T, const TreeView &tv, int p, const float2 *mp,
                   int ldm, double2 *out, int prune, int nprod, int group, int *err, int max_tile, cudaStream_t s,
                   Status &st)
{
    if (!st.ok() || ntiles == 0) return;
    if (max_tile > 128)
        launch_tc_t<16, 3, 256>(tiles, ntiles, grouped, slots, slot_toff, T, tv, p, mp, ldm, out, prune, nprod, group, err, s, st);
    else if (variant == 1)
        launch_tc_t<32, 2, 128>(tiles, ntiles, grouped, slots, slot_toff, T, tv, p, mp, ldm, out, prune, nprod, group, err, s, st);
    else
        launch_tc_t<16, 3, 128>(tiles, ntiles, grouped, slots, slot_toff, T, tv, p, mp, ldm, out, prune, nprod, group, err, s, st);
}

// FP32 copy of the multipoles with an even row stride (16-byte aligned pairs).
__global__ void k_mp_f32(long long nb, int nc, int ldm, const double2 *in, float2 *out)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nb * ldm) return;
    long long b = i / ldm;
    int c = (int)(i - b * ldm);
    double2 v = c < nc ? in[b * nc + c] : make_double2(0.0, 0.0);
    out[i] = make_float2((float)v.x, (float)v.y);
}

void convert_mp_f32(long long nboxes, int nc, int ldm, const double2 *in, float2 *out, cudaStream_t s, Status &st)
{
    if (!st.ok() || nboxes == 0) return;
    long long n = nboxes * ldm;
    k_mp_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(nboxes, nc, ldm, in, out); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// ---------------------------------------------------------------- self-test
// D (128 x N) = A (128 x K) B^T (N x K), row-major FP32 inputs, through the
// same staging layout, descriptors, split products, commit/wait and TMEM
// loads as the M2L kernel (one CTA, K a multiple of 32; nprod 1, 3 or 4).
__global__ void __launch_bounds__(kTcThreads, 1) k_tc_selftest(int N, int K, const float *A, const float *B,
                                                               float *D, int nprod, int *err)
{
    constexpr int KC = 32, S = 2, KB = KC / 4;
    constexpr uint32_t OPB = KB * kTcLBO, STB = 4 * OPB;
    extern __shared__ unsigned char tc_smraw[];
    unsigned char *sm = (unsigned char *)(((uintptr_t)tc_smraw + 127) & ~(uintptr_t)127);
    __shared__ uint64_t mbar[S];
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(&mbar[s], 1);
        mbar_fence_init();
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(&tbase, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = tbase, idesc = tc_idesc_tf32(128, N), sbase = smem_u32(sm);
    int it = 0;
    bool aborted = false;
    for (int kc = 0; kc < K / KC; kc++, it++) {
        const int st = it % S;
        unsigned char *base = sm + st * STB;
        int late = 0;
        if (it >= S && !mbar_wait_bounded(&mbar[st], ((it - S) / S) & 1)) late = 1;
        for (int task = tid; task < 128 * KB; task += kTcThreads) {
            const int r = task & 127, kb = task >> 7;
            float4 h, l;
            split4(*(const float4 *)(A + (size_t)r * K + kc * KC + 4 * kb), h, l);
            *(float4 *)(base + kb * kTcLBO + r * 16) = h;
            *(float4 *)(base + OPB + kb * kTcLBO + r * 16) = l;
        }
        for (int task = tid; task < N * KB; task += kTcThreads) {
            const int n = task / KB, kb = task % KB;
            float4 h, l;
            split4(*(const float4 *)(B + (size_t)n * K + kc * KC + 4 * kb), h, l);
            *(float4 *)(base + 2 * OPB + kb * kTcLBO + n * 16) = h;
            *(float4 *)(base + 3 * OPB + kb * kTcLBO + n * 16) = l;
        }
        fence_async_smem();
        if (__syncthreads_or(late)) { aborted = true; break; }
        if (tid == 0) {
            tc_fence_after();
            issue_stage<KC>(sbase + st * STB, tm, idesc, it == 0, nprod);
            tc_commit(&mbar[st]);
        }
    }
    int bad = aborted ? 1 : 0;
    if (it > 0) {
        const int last = it - 1;
        const bool done = mbar_wait_bounded(&mbar[last % S], (last / S) & 1);
        if (__syncthreads_or(!done)) bad = 1;
        tc_fence_after();
        if (!bad) {
            const int q = warp & 3, h = warp >> 2, r = 32 * q + lane;
            for (int c0 = 0; c0 < 64; c0 += 16) {
                const int col = 64 * h + c0;
                if (col >= N) break;
                float v[16];
                tmem_ld16(tm + ((uint32_t)(32 * q) << 16) + (uint32_t)col, v);
#pragma unroll
                for (int u = 0; u < 16; u++) D[(size_t)r * N + col + u] = v[u];
            }
        }
    }
    if (bad && tid == 0) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tm, 128);
}

}  // namespace fmm

using namespace fmm;

// Error-path test of the tensor-core M2L: with on = 1 the kernels launched by
// later calls on this thread take their bounded-wait error path at the first
// stage wait (the wait counts as expired): every CTA that gets there stops
// issuing MMAs, waits (with the normal bound) for the MMAs it has issued,
// frees its TMEM and records the error, so the call returns ier 16 and the
// context stays usable.  0 turns it off.
extern "C" int fmm3d_inject_tc_wait_expiry(int on)
{
    fmm::g_tc_expire_waits = on ? 1 : 0;
    return 0;
}

// Runs the tensor-core self-test on the current device: D (128 x N) from
// A (128 x K) and B (N x K), host arrays.  N in 16..128 (multiple of 16), K a
// multiple of 32, nprod 1 (hi products only) or 3 (split products).
// Returns 0, 1 on a bad argument, 2 on a CUDA error, 3 on a wait that expired.
extern "C" int fmm3d_tc_selftest(int N, int K, const float *A, const float *B, float *D, int nprod)
{
    if (N < 16 || N > 128 || N % 16 || K < 32 || K % 32) return 1;
    float *dA = nullptr, *dB = nullptr, *dD = nullptr;
    int *derr = nullptr, herr = 0;
    cudaError_t e = cudaSuccess;
    const size_t sm = 2 * 4 * (32 / 4) * kTcLBO + 128;
    auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; return e == cudaSuccess; };
    if (ok(cudaMalloc(&dA, sizeof(float) * 128 * K)) && ok(cudaMalloc(&dB, sizeof(float) * N * K)) &&
        ok(cudaMalloc(&dD, sizeof(float) * 128 * N)) && ok(cudaMalloc(&derr, sizeof(int))) &&
        ok(cudaMemcpy(dA, A, sizeof(float) * 128 * K, cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(dB, B, sizeof(float) * N * K, cudaMemcpyHostToDevice)) && ok(cudaMemset(derr, 0, sizeof(int))) &&
        ok(cudaMemset(dD, 0, sizeof(float) * 128 * N)) &&
        ok(smem_allow(k_tc_selftest, (int)sm))) {
        k_tc_selftest<<<1, kTcThreads, sm>>>(N, K, dA, dB, dD, nprod, derr);
        if (ok(cudaGetLastError()) && ok(cudaDeviceSynchronize()))
            if (ok(cudaMemcpy(D, dD, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost)))
                ok(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(derr);
    if (e != cudaSuccess) return 2;
    return herr ? 3 : 0;
}
