// Definitions for driver_common.cuh.
#include <mutex>

#include "driver_common.cuh"

namespace fmm {

thread_local ThreadInfo g_ti;

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

}  // namespace fmm
