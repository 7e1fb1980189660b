// Device-wide exclusive scan and a stable LSD radix sort (64-bit keys,
// 32-bit payload) used by the octree build.  Written for sm_100a: 256-thread
// CTAs, warp shuffles for intra-warp prefix, one read + one write per pass.
#include "fmm_common.cuh"

namespace fmm {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;  // items per thread per tile
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ int block_excl_scan(int v, int &excl)
{
    __shared__ int wsum[kScanThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = warp_incl_scan(v);
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        int t = lane < kScanThreads / 32 ? wsum[lane] : 0;
        int ti = warp_incl_scan(t);
        if (lane < kScanThreads / 32) wsum[lane] = ti - t;
    }
    __syncthreads();
    excl = inc - v + wsum[w];
    __shared__ int tot;
    if (threadIdx.x == kScanThreads - 1) tot = excl + v;
    __syncthreads();
    int total = tot;
    __syncthreads();
    return total;
}

__global__ void k_tile_sums(const int *in, int n, int *tile_sum)
{
    long base = (long)blockIdx.x * kScanTile;
    int s = 0;
    for (int i = 0; i < kScanItems; i++) {
        long j = base + (long)i * kScanThreads + threadIdx.x;
        if (j < n) s += in[j];
    }
    int ex;
    int tot = block_excl_scan(s, ex);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

// Single-CTA exclusive scan of the tile sums (ntiles small).
__global__ void k_scan_tiles(int *tile_sum, int ntiles, int *total)
{
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b = 0; b < ntiles; b += kScanThreads) {
        int j = b + threadIdx.x;
        int v = j < ntiles ? tile_sum[j] : 0;
        int ex;
        int tot = block_excl_scan(v, ex);
        if (j < ntiles) tile_sum[j] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_apply(const int *in, int *out, int n, const int *tile_off)
{
    long base = (long)blockIdx.x * kScanTile + (long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
    for (int i = 0; i < kScanItems; i++) {
        long j = base + i;
        v[i] = j < n ? in[j] : 0;
        s += v[i];
    }
    int ex;
    block_excl_scan(s, ex);
    int run = ex + tile_off[blockIdx.x];
    for (int i = 0; i < kScanItems; i++) {
        long j = base + i;
        if (j < n) out[j] = run;
        run += v[i];
    }
}

}  // namespace

void scan_exclusive_int(const int *d_in, int *d_out, int n, cudaStream_t s, Status &st, int *h_total)
{
    if (n <= 0) {
        if (h_total) *h_total = 0;
        return;
    }
    int ntiles = div_up(n, kScanTile);
    DBuf<int> tiles, tot;
    tiles.alloc(ntiles, s, st);
    tot.alloc(1, s, st);
    if (!st.ok()) return;
    k_tile_sums<<<ntiles, kScanThreads, 0, s>>>(d_in, n, tiles.p); FMM_COUNT_LAUNCH();
    k_scan_tiles<<<1, kScanThreads, 0, s>>>(tiles.p, ntiles, tot.p); FMM_COUNT_LAUNCH();
    k_scan_apply<<<ntiles, kScanThreads, 0, s>>>(d_in, d_out, n, tiles.p); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    if (h_total) {
        FMM_TRY(st, cudaMemcpyAsync(h_total, tot.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        FMM_TRY(st, cudaStreamSynchronize(s));
    }
}

// ---------------------------------------------------------------- radix sort
namespace {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 items per tile

// Per-tile digit histogram, written digit-major: hist[digit * ntiles + tile].
__global__ void k_radix_hist(const uint64_t *keys, int n, int shift, int *hist, int ntiles)
{
    __shared__ int h[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) h[i] = 0;
    __syncthreads();
    long base = (long)blockIdx.x * kSortTile;
    for (int i = 0; i < kSortItems; i++) {
        long j = base + (long)i * kSortThreads + threadIdx.x;
        if (j < n) atomicAdd(&h[(keys[j] >> shift) & (kRadix - 1)], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) hist[(long)i * ntiles + blockIdx.x] = h[i];
}

// Stable scatter.  Items of a tile are taken in tile order (item r of the
// tile is at base + r); the tile is processed in rounds of kSortThreads
// consecutive items, each warp ranks its 32 items with __match_any_sync and
// warps are ordered through a per-round shared prefix.
__global__ void k_radix_scatter(const uint64_t *kin, const int *vin, uint64_t *kout, int *vout, int n,
                                int shift, const int *offs, int ntiles)
{
    __shared__ int base_d[kRadix];       // running output position per digit
    __shared__ int wcnt[kSortThreads / 32][kRadix];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) base_d[i] = offs[(long)i * ntiles + blockIdx.x];
    long tbase = (long)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortItems; r++) {
        for (int i = threadIdx.x; i < (kSortThreads / 32) * kRadix; i += kSortThreads) (&wcnt[0][0])[i] = 0;
        __syncthreads();
        long j = tbase + (long)r * kSortThreads + threadIdx.x;
        bool valid = j < n;
        uint64_t k = valid ? kin[j] : 0;
        int v = valid ? vin[j] : 0;
        int d = valid ? (int)((k >> shift) & (kRadix - 1)) : -1;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int rank_in_warp = __popc(peers & ((1u << lane) - 1));
        int leader = __ffs(peers) - 1;
        if (valid && lane == leader) wcnt[w][d] = __popc(peers);
        __syncthreads();
        // exclusive prefix over warps for this digit
        int pre = 0;
        if (valid) {
            for (int ww = 0; ww < w; ww++) pre += wcnt[ww][d];
            int pos = base_d[d] + pre + rank_in_warp;
            kout[pos] = k;
            vout[pos] = v;
        }
        __syncthreads();
        // advance digit bases by this digit pass's totals
        for (int dd = threadIdx.x; dd < kRadix; dd += kSortThreads) {
            int t = 0;
            for (int ww = 0; ww < kSortThreads / 32; ww++) t += wcnt[ww][dd];
            base_d[dd] += t;
        }
        __syncthreads();
    }
}

}  // namespace

void radix_sort_u64(uint64_t *d_keys, int *d_vals, int n, int bits, cudaStream_t s, Status &st)
{
    if (n <= 1) return;
    int ntiles = div_up(n, kSortTile);
    DBuf<uint64_t> k2;
    DBuf<int> v2, hist;
    k2.alloc(n, s, st);
    v2.alloc(n, s, st);
    hist.alloc((size_t)kRadix * ntiles, s, st);
    if (!st.ok()) return;
    uint64_t *ka = d_keys, *kb = k2.p;
    int *va = d_vals, *vb = v2.p;
    int passes = 0;
    for (int shift = 0; shift < bits; shift += kRadixBits) {
        k_radix_hist<<<ntiles, kSortThreads, 0, s>>>(ka, n, shift, hist.p, ntiles); FMM_COUNT_LAUNCH();
        scan_exclusive_int(hist.p, hist.p, kRadix * ntiles, s, st, nullptr);
        if (!st.ok()) return;   // unscanned counts are not offsets: the scatter must not run
        k_radix_scatter<<<ntiles, kSortThreads, 0, s>>>(ka, va, kb, vb, n, shift, hist.p, ntiles); FMM_COUNT_LAUNCH();
        FMM_LAUNCH_CHECK(st);
        std::swap(ka, kb);
        std::swap(va, vb);
        passes++;
    }
    if (passes & 1) {
        FMM_TRY(st, cudaMemcpyAsync(d_keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        FMM_TRY(st, cudaMemcpyAsync(d_vals, va, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    }
}

}  // namespace fmm
