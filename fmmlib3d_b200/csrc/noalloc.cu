// Direct sum without any device allocation (fmm3d_l3dpartdirect_noalloc).
//
// Some callers cannot let this library allocate device memory: a host
// application whose framework allocator has already reserved the GPU's
// memory, or a latency-bound service loop that forbids cudaMalloc/cudaFree
// after start-up because they synchronise the device.  For them the O(N^2)
// sum of l3dpartdirect is offered with its scratch (the structure-of-arrays
// copies of the inputs and of the outputs) in a fixed array declared at file
// scope below.  Every GPU that loads the library's device code holds that
// array (11 MB) until the process exits.  Under CUDA's default lazy module
// loading the array and the kernels used here are loaded on a device by the
// first call made there (which may allocate device memory for them); later
// calls allocate nothing.  The cached device address belongs to the device's
// current primary context: after cudaDeviceReset on that device, calls here
// are invalid until the process restarts.
#include <mutex>

#include "../../include/fmm3d_b200.h"
#include "lap_kernels.cuh"

namespace fmm {

// at most kNoAllocMaxPts sources and kNoAllocMaxPts evaluation points per call
constexpr int kNoAllocMaxPts = 65536;
// sources: x, y, z, vx, vy, vz (doubles) + charge, dipole strength (double2);
// evaluation points: x, y, z (doubles) + pot, fx, fy, fz (double2)
constexpr size_t kNoAllocBytes = (size_t)kNoAllocMaxPts * (6 * 8 + 2 * 16) + (size_t)kNoAllocMaxPts * (3 * 8 + 4 * 16);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_addr[64] = {nullptr};

// Device address of the scratch array on the current device.  In host code
// the symbol is only a host-side handle, so the address is looked up once per
// device (with that device current) and cached.
cudaError_t scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

__global__ void k_na_split3(int n, const double *a, double *x, double *y, double *z)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = a[3L * i]; y[i] = a[3L * i + 1]; z[i] = a[3L * i + 2];
}

__global__ void k_na_split2(int n, const double *a, double2 *o)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = make_double2(a[2L * i], a[2L * i + 1]);
}

__global__ void k_na_out(int n, OutSoA o, double *pot, double *fld)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (pot) { pot[2L * i] = o.pot[i].x; pot[2L * i + 1] = o.pot[i].y; }
    if (fld) {
        fld[6L * i] = o.fx[i].x; fld[6L * i + 1] = o.fx[i].y;
        fld[6L * i + 2] = o.fy[i].x; fld[6L * i + 3] = o.fy[i].y;
        fld[6L * i + 4] = o.fz[i].x; fld[6L * i + 5] = o.fz[i].y;
    }
}

}  // namespace

// per host thread, as fmm3d_last_error: calls on different GPUs may run
// concurrently from different threads
static thread_local const char *g_noalloc_msg = "";

static int noalloc_direct(int ns, const double *src, int ifc, const double *q, int ifd, const double *dq,
                          const double *dv, int ifpot, double *pot, int iffld, double *fld, int nt,
                          const double *trg, int ifpt, double *pt, int ifft, double *ft, cudaStream_t s)
{
    if (ns < 0 || nt < 0 || ns > kNoAllocMaxPts || nt > kNoAllocMaxPts) {
        g_noalloc_msg = "fmm3d_l3dpartdirect_noalloc: nsource and ntarget must each be in [0, 65536]";
        return 8;
    }
    void *base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) {
        g_noalloc_msg = "fmm3d_l3dpartdirect_noalloc: cudaGetSymbolAddress of the scratch array failed";
        return 16;
    }
    // carve the fixed array; every region is fully written before it is read,
    // so nothing needs clearing between calls
    char *c = (char *)base;
    const size_t N = kNoAllocMaxPts;
    double *sx = (double *)c, *sy = sx + N, *sz = sy + N, *vx = sz + N, *vy = vx + N, *vz = vy + N;
    double2 *sq = (double2 *)(vz + N), *sd = sq + N;
    double *ex = (double *)(sd + N), *ey = ex + N, *ez = ey + N;
    double2 *o0 = (double2 *)(ez + N), *o1 = o0 + N, *o2 = o1 + N, *o3 = o2 + N;
    Status st;
    auto grid = [](int n) { return (n + 255) / 256; };
    if (ns > 0) {
        k_na_split3<<<grid(ns), 256, 0, s>>>(ns, src, sx, sy, sz); FMM_COUNT_LAUNCH();
        if (ifc == 1) { k_na_split2<<<grid(ns), 256, 0, s>>>(ns, q, sq); FMM_COUNT_LAUNCH(); }
        if (ifd == 1) {
            k_na_split2<<<grid(ns), 256, 0, s>>>(ns, dq, sd); FMM_COUNT_LAUNCH();
            k_na_split3<<<grid(ns), 256, 0, s>>>(ns, dv, vx, vy, vz); FMM_COUNT_LAUNCH();
        }
    }
    OutSoA o;
    o.pot = o0; o.fx = o1; o.fy = o2; o.fz = o3;
    if (ns > 0 && (ifpot == 1 || iffld == 1)) {
        launch_direct(ns, sx, sy, sz, sq, sd, vx, vy, vz, ifc, ifd, ns, sx, sy, sz, nullptr, 1, o, s, st);
        k_na_out<<<grid(ns), 256, 0, s>>>(ns, o, ifpot == 1 ? pot : nullptr, iffld == 1 ? fld : nullptr);
        FMM_COUNT_LAUNCH();
    }
    if (nt > 0 && (ifpt == 1 || ifft == 1)) {
        k_na_split3<<<grid(nt), 256, 0, s>>>(nt, trg, ex, ey, ez); FMM_COUNT_LAUNCH();
        launch_direct(ns, sx, sy, sz, sq, sd, vx, vy, vz, ifc, ifd, nt, ex, ey, ez, nullptr, 0, o, s, st);
        k_na_out<<<grid(nt), 256, 0, s>>>(nt, o, ifpt == 1 ? pt : nullptr, ifft == 1 ? ft : nullptr);
        FMM_COUNT_LAUNCH();
    }
    FMM_LAUNCH_CHECK(st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) {
        g_noalloc_msg = "fmm3d_l3dpartdirect_noalloc: CUDA error";
        return 16;
    }
    g_noalloc_msg = "";
    return 0;
}

}  // namespace fmm

extern "C" int fmm3d_l3dpartdirect_noalloc(int nsource, const double *d_source, int ifcharge,
                                           const double *d_charge, int ifdipole, const double *d_dipstr,
                                           const double *d_dipvec, int ifpot, double *d_pot, int iffld,
                                           double *d_fld, int ntarget, const double *d_target, int ifpottarg,
                                           double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream)
{
    return fmm::noalloc_direct(nsource, d_source, ifcharge, d_charge, ifdipole, d_dipstr, d_dipvec, ifpot, d_pot,
                               iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg, iffldtarg, d_fldtarg,
                               (cudaStream_t)stream);
}

extern "C" const char *fmm3d_noalloc_last_error(void) { return fmm::g_noalloc_msg; }
