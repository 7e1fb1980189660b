// Shared definitions for the B200 particle-FMM library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <vector>

namespace fmm {

// ---------------------------------------------------------------- errors
// Library calls never abort the process: a failing CUDA call is recorded
// in the per-call status and surfaces as the Fortran `ier` code.
struct Status {
    cudaError_t err = cudaSuccess;
    const char *where = nullptr;
    bool ok() const { return err == cudaSuccess; }
};

#define FMM_TRY(st, call)                                                              \
    do {                                                                               \
        if ((st).ok()) {                                                               \
            cudaError_t e_ = (call);                                                   \
            if (e_ != cudaSuccess) { (st).err = e_; (st).where = #call; }              \
        }                                                                              \
    } while (0)

#define FMM_LAUNCH_CHECK(st) FMM_TRY(st, cudaGetLastError())

// Kernel launches issued by the current host thread (reported per call).
extern thread_local int g_launch_count;
#define FMM_COUNT_LAUNCH() (++::fmm::g_launch_count)

// ---------------------------------------------------------------- complex
__host__ __device__ __forceinline__ double2 cmk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// Products with the fused multiply-add written out: left to the compiler's
// contraction, a.x*b.x - a.y*b.y may fuse either product, and the choice can
// differ between instantiations of one kernel template (tile sizes), which
// would make results depend on launch shapes.
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b)  // a * conj(b)
{
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -(a.x * b.y)));
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscal(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
// acc += a * b
__host__ __device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
// acc += s * a  (s real)
__host__ __device__ __forceinline__ void crfma(double2 &acc, double s, double2 a)
{
    acc.x = fma(s, a.x, acc.x);
    acc.y = fma(s, a.y, acc.y);
}

// Compact index of expansion coefficient (n, m), |m| <= n.
__host__ __device__ __forceinline__ int eidx(int n, int m) { return n * n + n + m; }
// Triangular index of (n, m), 0 <= m <= n.
__host__ __device__ __forceinline__ int tidx(int n, int m) { return (n * (n + 1)) / 2 + m; }

constexpr int kMaxLevel = 21;  // 3 key bits per level in a 64-bit key
constexpr int kMaxP = 80;

// ---------------------------------------------------------------- dynamic shared memory
// Lets `func` take `bytes` of dynamic shared memory per block.  The limit is
// a process-wide attribute of the function: set per launch to that launch's
// size, a host thread could lower it just before another thread (a serving
// slot, a plan on its own stream) launches a larger problem, whose launch then
// fails.  So it is raised once per device to the most the device gives one
// block (less the function's static shared memory) and never lowered; the
// launch's own size still sets its occupancy.  Returns cudaErrorInvalidValue
// when `bytes` is beyond the device.
cudaError_t smem_allow_fn(const void *func, size_t bytes);
template <class T>
inline cudaError_t smem_allow(T *func, size_t bytes)
{
    return smem_allow_fn((const void *)func, bytes);
}

// ---------------------------------------------------------------- device buffers
// Test hook (fmm3d_inject_alloc_failure): when positive, counts this host
// thread's workspace allocations down and fails the one that reaches zero as
// if the device were out of memory.  Armed at the start of one allocation
// phase of a call by alloc_fail_point (the phases of the reference's error
// codes: 1 the host-array entry points' device copies, 2 the octree, 3 the
// per-point workspace, 4 the expansions).
extern thread_local int g_alloc_fail_countdown;
extern thread_local int g_alloc_fail_phase;
inline void alloc_fail_point(int phase)
{
    if (g_alloc_fail_phase == phase) {
        g_alloc_fail_phase = 0;
        g_alloc_fail_countdown = 1;
    }
}

// Stream-ordered allocations from the device's default memory pool, so that
// repeated calls reuse HBM without synchronising the device.
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    bool alloc(size_t count, cudaStream_t stream, Status &st)
    {
        release();
        s = stream;
        n = count;
        if (count == 0) return true;
        if (g_alloc_fail_countdown > 0 && st.ok() && --g_alloc_fail_countdown == 0) {
            st.err = cudaErrorMemoryAllocation;
            st.where = "injected allocation failure";
        }
        FMM_TRY(st, cudaMallocAsync((void **)&p, sizeof(T) * count, stream));
        if (!st.ok()) { p = nullptr; n = 0; return false; }
        return true;
    }
    bool zero(Status &st)
    {
        if (n) FMM_TRY(st, cudaMemsetAsync(p, 0, sizeof(T) * n, s));
        return st.ok();
    }
};

inline int div_up(long a, long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------- scan / sort utilities (scan_sort.cu)
// Exclusive prefix sum of n ints; out may alias in. Returns total (host) when
// want_total is set (one device->host read).
void scan_exclusive_int(const int *d_in, int *d_out, int n, cudaStream_t s, Status &st, int *h_total);
// Stable LSD radix sort of 64-bit keys with 32-bit payload over the low
// `bits` bits of the key.
void radix_sort_u64(uint64_t *d_keys, int *d_vals, int n, int bits, cudaStream_t s, Status &st);

}  // namespace fmm
