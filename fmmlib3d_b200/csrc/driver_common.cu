// Definitions for driver_common.cuh.
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <map>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <mutex>

#include "driver_common.cuh"

namespace fmm {

// ---------------------------------------------------------------- host copy threads
// A small pool of host threads for the pageable <-> pinned copies of the
// staging ring (a single memcpy thread reaches a fraction of the host's
// memory bandwidth).  Shared by all calling threads; jobs are independent
// ranges.  Created on first use and kept; a forked child (no pool threads)
// copies on the calling thread.
namespace {

class CopyPool {
public:
    explicit CopyPool(int n) : pid_(getpid())
    {
        for (int i = 0; i < n; i++) std::thread([this] { loop(); }).detach();
        nthreads_ = n;
    }
    int threads() const { return getpid() == pid_ ? nthreads_ : 0; }
    void submit(std::function<void()> f)
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(std::move(f));
        }
        cv_.notify_one();
    }

private:
    void loop()
    {
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return !q_.empty(); });
                f = std::move(q_.front());
                q_.pop_front();
            }
            f();
        }
    }
    pid_t pid_;
    int nthreads_ = 0;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> q_;
};

CopyPool &copy_pool()
{
    static CopyPool *pool = [] {
        int hw = (int)std::thread::hardware_concurrency();
        int n = std::max(0, std::min(7, hw / 2 - 1));
        if (const char *e = getenv("FMM3D_COPY_THREADS")) n = std::max(0, std::min(64, atoi(e) - 1));
        return new CopyPool(n);   // kept until exit (its threads are detached)
    }();
    return *pool;
}

// memcpy split over the pool's threads and the calling thread (pieces of at least 1 MB)
void parallel_memcpy(void *dst, const void *src, size_t n)
{
    CopyPool &pool = copy_pool();
    const size_t piece_min = 1u << 20;
    int parts = (int)std::min<size_t>((size_t)pool.threads() + 1, std::max<size_t>(1, n / piece_min));
    if (parts <= 1) {
        memcpy(dst, src, n);
        return;
    }
    const size_t piece = (n / parts + 4095) & ~(size_t)4095;
    std::mutex mu;
    std::condition_variable cv;
    int left = parts - 1;
    for (int i = 1; i < parts; i++) {
        const size_t a = std::min(n, i * piece), b = std::min(n, (i + 1) * piece);
        pool.submit([&, a, b] {
            if (b > a) memcpy((char *)dst + a, (const char *)src + a, b - a);
            std::lock_guard<std::mutex> lk(mu);
            if (--left == 0) cv.notify_one();
        });
    }
    memcpy(dst, src, std::min(n, piece));
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return left == 0; });
}

}  // namespace

StageRing *stage_ring()
{
    static thread_local StageRing ring;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    if (ring.buf && ring.dev == dev) return &ring;
    if (ring.buf) {   // another device: release the old ring after its copies
        for (int i = 0; i < kStageSlots; i++) {
            cudaEventSynchronize(ring.ev[i]);
            cudaEventDestroy(ring.ev[i]);
        }
        cudaFreeHost(ring.buf);
        ring.buf = nullptr;
    }
    if (cudaHostAlloc((void **)&ring.buf, kStageChunk * kStageSlots, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        ring.buf = nullptr;
        return nullptr;
    }
    for (int i = 0; i < kStageSlots; i++) cudaEventCreateWithFlags(&ring.ev[i], cudaEventDisableTiming);
    ring.next = 0;
    ring.dev = dev;
    return &ring;
}

bool host_pageable(const void *p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

void staged_h2d(StageRing &ring, void *dst, const void *src, size_t bytes, cudaStream_t s, Status &st)
{
    for (size_t off = 0; off < bytes && st.ok(); off += kStageChunk) {
        const size_t len = std::min(kStageChunk, bytes - off);
        const int slot = ring.next;
        ring.next = (ring.next + 1) % kStageSlots;
        char *buf = ring.buf + (size_t)slot * kStageChunk;
        FMM_TRY(st, cudaEventSynchronize(ring.ev[slot]));   // the slot's previous copy is done
        if (!st.ok()) return;
        parallel_memcpy(buf, (const char *)src + off, len);
        FMM_TRY(st, cudaMemcpyAsync((char *)dst + off, buf, len, cudaMemcpyHostToDevice, s));
        FMM_TRY(st, cudaEventRecord(ring.ev[slot], s));
    }
}

void staged_d2h(StageRing &ring, void *dst, const void *src, size_t bytes, cudaStream_t s, Status &st)
{
    const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
    int slot_of[kStageSlots];
    size_t issued = 0;
    for (size_t i = 0; i < nch && st.ok(); i++) {
        // keep up to kStageSlots chunks' DMAs in flight ahead of the host copies
        while (issued < nch && issued < i + kStageSlots && st.ok()) {
            const size_t off = issued * kStageChunk, len = std::min(kStageChunk, bytes - off);
            const int slot = ring.next;
            ring.next = (ring.next + 1) % kStageSlots;
            FMM_TRY(st, cudaEventSynchronize(ring.ev[slot]));
            FMM_TRY(st, cudaMemcpyAsync(ring.buf + (size_t)slot * kStageChunk, (const char *)src + off, len,
                                        cudaMemcpyDeviceToHost, s));
            FMM_TRY(st, cudaEventRecord(ring.ev[slot], s));
            slot_of[issued % kStageSlots] = slot;
            issued++;
        }
        if (!st.ok()) return;
        const int slot = slot_of[i % kStageSlots];
        FMM_TRY(st, cudaEventSynchronize(ring.ev[slot]));
        if (!st.ok()) return;
        const size_t off = i * kStageChunk, len = std::min(kStageChunk, bytes - off);
        parallel_memcpy((char *)dst + off, ring.buf + (size_t)slot * kStageChunk, len);
    }
}

thread_local ThreadInfo g_ti;
thread_local int g_alloc_fail_countdown = 0;
thread_local int g_alloc_fail_phase = 0;

cudaStream_t thread_stream()
{
    static thread_local cudaStream_t s = nullptr;
    static thread_local int sdev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!s || sdev != dev) {
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        sdev = dev;
    }
    return s;
}

SideStreams &side_streams()
{
    static thread_local SideStreams ss;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!ss.far || ss.dev != dev) {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        cudaStreamCreateWithPriority(&ss.far, cudaStreamNonBlocking, greatest);
        cudaStreamCreateWithFlags(&ss.copy, cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ss.copied, cudaEventDisableTiming);
        ss.dev = dev;
    }
    return ss;
}

// Keep freed workspace in the device's default memory pool across calls
// instead of returning it to the driver at every synchronisation.
void keep_pool_memory()
{
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[dev] = true;
}

__global__ void k_gather_src(int n, const int *perm, const double *src, const double *q, const double *dq,
                             const double *dv, int ifc, int ifd, PointsSoA o)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long j = perm[i];
    o.x[i] = src[3 * j];
    o.y[i] = src[3 * j + 1];
    o.z[i] = src[3 * j + 2];
    if (ifc) o.q[i] = make_double2(q[2 * j], q[2 * j + 1]);
    if (ifd) {
        o.dq[i] = make_double2(dq[2 * j], dq[2 * j + 1]);
        o.vx[i] = dv[3 * j];
        o.vy[i] = dv[3 * j + 1];
        o.vz[i] = dv[3 * j + 2];
    }
}

__global__ void k_gather_pts(int n, const int *perm, const double *p, double *x, double *y, double *z)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long j = perm[i];
    x[i] = p[3 * j];
    y[i] = p[3 * j + 1];
    z[i] = p[3 * j + 2];
}

// unsort: l3dpsort / l3dfsort (src/lfmm3drouts.f:583-615)
__global__ void k_scatter_out(int n, const int *perm, OutSoA o, double *pot, double *fld)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long j = perm ? perm[i] : i;
    if (pot) { pot[2 * j] = o.pot[i].x; pot[2 * j + 1] = o.pot[i].y; }
    if (fld) {
        double2 a = o.fx[i], b = o.fy[i], c = o.fz[i];
        fld[6 * j] = a.x; fld[6 * j + 1] = a.y;
        fld[6 * j + 2] = b.x; fld[6 * j + 3] = b.y;
        fld[6 * j + 4] = c.x; fld[6 * j + 5] = c.y;
    }
}

__global__ void k_split_aos(int n, const double *p, double *x, double *y, double *z)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = p[3L * i]; y[i] = p[3L * i + 1]; z[i] = p[3L * i + 2];
}

__global__ void k_split_c(int n, const double *c, double2 *o)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = make_double2(c[2L * i], c[2L * i + 1]);
}

cudaError_t smem_allow_fn(const void *func, size_t bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> cap_of;   // (function, device) -> limit set
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_pair(func, dev);
    auto it = cap_of.find(key);
    if (it == cap_of.end()) {
        int optin = 0;
        cudaFuncAttributes fa;
        if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess ||
            (e = cudaFuncGetAttributes(&fa, func)) != cudaSuccess)
            return e;
        const size_t cap = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
        if ((e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap)) != cudaSuccess)
            return e;
        it = cap_of.emplace(key, cap).first;
    }
    return bytes <= it->second ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace fmm

extern "C" int fmm3d_inject_alloc_failure(int phase)
{
    if (phase < 0 || phase > 4) return 1;
    fmm::g_alloc_fail_phase = phase;
    fmm::g_alloc_fail_countdown = 0;
    return 0;
}
