// Host-side plumbing shared by the Laplace and Helmholtz drivers: per-thread
// call state (timing, statistics, last error), the per-thread stream, the
// workspace pool policy, pass timers, the gather/scatter kernels between the
// caller's AoS arrays and the tree-ordered SoA arrays, and the host-array
// wrapper of the Fortran-named entry points.
#pragma once
#include <functional>
#include <string>
#include <thread>
#include <vector>

#include "lap_kernels.cuh"
#include "tree.cuh"

namespace fmm {

struct ThreadInfo {
    bool timing = false;
    bool want_stats = false;
    // set by the host-array entry points while charges are still being copied:
    // the charge-dependent passes wait for it
    cudaEvent_t inputs_ready = nullptr;
    // set with inputs_ready when a helper thread is still staging the charges
    // from pageable host memory: joined before the event is waited on
    std::function<void()> inputs_join;
    std::vector<double> ms;
    std::vector<long long> stats;
    std::string err;
    int launches = 0;
    int depth_capped = 0;   // Tree::capped of this thread's last tree
};
extern thread_local ThreadInfo g_ti;

cudaStream_t thread_stream();
void keep_pool_memory();

// The device routine's wait for charges still being copied from the host:
// joins the staging helper thread (if any), then orders `s` after the copies.
inline void wait_host_inputs(cudaStream_t s, Status &st)
{
    if (g_ti.inputs_join) {
        std::function<void()> f = std::move(g_ti.inputs_join);
        g_ti.inputs_join = nullptr;
        f();
    }
    if (g_ti.inputs_ready) {
        FMM_TRY(st, cudaStreamWaitEvent(s, g_ti.inputs_ready, 0));
        g_ti.inputs_ready = nullptr;
    }
}

// ---------------------------------------------------------------- pageable host memory
// A Fortran (or numpy) caller passes pageable arrays; cudaMemcpyAsync from
// pageable memory is staged by the driver through its own small pinned
// buffer by one host thread.  Large pageable transfers here go instead
// through a pinned ring of the calling host thread (kStageSlots chunks of
// kStageChunk bytes, allocated on first use and kept), the host-side copies
// split over the library's copy threads and each chunk's DMA overlapping the
// host copy of the next.
constexpr size_t kStageChunk = 16u << 20;
constexpr int kStageSlots = 6;
constexpr size_t kStageMin = 4u << 20;   // smaller transfers keep cudaMemcpyAsync

struct StageRing {
    char *buf = nullptr;
    cudaEvent_t ev[kStageSlots] = {};
    int next = 0;
    int dev = -1;
};
// The ring of the calling host thread on the current device (nullptr if
// pinned memory cannot be had: the caller then falls back to cudaMemcpyAsync).
StageRing *stage_ring();
// True for host memory that is neither pinned nor registered with CUDA.
bool host_pageable(const void *p);
// Stream-ordered copies between pageable host memory and the device through
// `ring`.  The host side is synchronous: staged_h2d returns once every chunk
// is in the ring and its DMA is enqueued on s (the source may then be
// reused); staged_d2h returns once dst holds the data.
void staged_h2d(StageRing &ring, void *dst, const void *src, size_t bytes, cudaStream_t s, Status &st);
void staged_d2h(StageRing &ring, void *dst, const void *src, size_t bytes, cudaStream_t s, Status &st);

struct Timer {
    cudaStream_t s;
    bool on;
    std::vector<cudaEvent_t> ev;
    std::function<void(std::vector<double> &)> fix;   // optional rewrite of the intervals
    Timer(cudaStream_t s_, bool on_) : s(s_), on(on_) {}
    void mark() { mark_on(s); }
    void mark_on(cudaStream_t st)
    {
        if (!on) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        ev.push_back(e);
    }
    void finish(std::vector<double> &ms)
    {
        ms.clear();
        if (!on || ev.size() < 2) return;
        cudaEventSynchronize(ev.back());
        for (size_t i = 1; i < ev.size(); i++) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[i - 1], ev[i]);
            ms.push_back(t);
        }
        float t = 0;
        cudaEventElapsedTime(&t, ev.front(), ev.back());
        ms.push_back(t);
        if (fix) fix(ms);
        for (auto e : ev) cudaEventDestroy(e);
        ev.clear();
    }
};

// Per-thread high-priority stream for the far-field passes of a call, and the
// fork / join events between it and the call's stream (made once per thread).
struct SideStreams {
    cudaStream_t far = nullptr, copy = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, copied = nullptr;
    int dev = -1;
};
SideStreams &side_streams();

// tree order <-> caller order (l3dreorder / l3dpsort / l3dfsort, src/lfmm3drouts.f:583-708)
__global__ void k_gather_src(int n, const int *perm, const double *src, const double *q, const double *dq,
                             const double *dv, int ifc, int ifd, PointsSoA o);
__global__ void k_gather_pts(int n, const int *perm, const double *p, double *x, double *y, double *z);
__global__ void k_scatter_out(int n, const int *perm, OutSoA o, double *pot, double *fld);
__global__ void k_split_aos(int n, const double *p, double *x, double *y, double *z);
__global__ void k_split_c(int n, const double *c, double2 *o);

inline TreeView make_treeview(const Tree &T)
{
    TreeView tv;
    tv.level = T.level.p; tv.parent = T.parent.p; tv.octant = T.octant.p; tv.nchild = T.nchild.p;
    tv.child = T.child.p; tv.coll = T.coll.p; tv.src0 = T.src0.p; tv.nsrc = T.nsrc.p; tv.trg0 = T.trg0.p;
    tv.ntrg = T.ntrg.p; tv.center = T.center.p; tv.l1_start = T.l1_start.p; tv.l1_idx = T.l1_idx.p;
    tv.l3_start = T.l3_start.p; tv.l3_idx = T.l3_idx.p; tv.l4_start = T.l4_start.p; tv.l4_idx = T.l4_idx.p;
    tv.size = T.size;
    if (T.ninst > 1) {
        tv.binst = T.binst.p;
        tv.inst_geom = T.inst_geom.p;
    }
    return tv;
}

// ---------------------------------------------------------------- host-array entry points
// Copies host inputs to the device, runs the device routine and copies the
// requested outputs back; unrequested outputs are left untouched.  The
// positions go first on the call's stream; the charges and dipoles follow on
// a copy stream, so that they travel while the tree is built: from pinned
// memory as DMA, from pageable memory (large arrays) staged by a helper host
// thread through the pinned ring.  With overlap_charges the device routine
// waits for them itself (wait_host_inputs) before its charge-dependent
// passes; otherwise the call's stream waits before the routine starts.
template <typename F>
inline int with_device_arrays(int ns, const double *source, int ifcharge, const double *charge, int ifdipole,
                              const double *dipstr, const double *dipvec, int ifpot, double *pot, int iffld,
                              double *fld, int nt, const double *target, int ifpottarg, double *pottarg,
                              int iffldtarg, double *fldtarg, F run, bool overlap_charges = false)
{
    cudaStream_t s = thread_stream();
    Status st;
    if (ns < 0) ns = 0;
    if (nt < 0) nt = 0;
    DBuf<double> dsrc, dq, ddq, ddv, dtrg, dpot, dfld, dpt, dft;
    alloc_fail_point(1);
    bool ok = dsrc.alloc(3L * std::max(ns, 1), s, st);
    if (ifcharge == 1) ok = ok && dq.alloc(2L * ns, s, st);
    if (ifdipole == 1) ok = ok && ddq.alloc(2L * ns, s, st) && ddv.alloc(3L * ns, s, st);
    if (nt) ok = ok && dtrg.alloc(3L * nt, s, st);
    if (ifpot == 1) ok = ok && dpot.alloc(2L * ns, s, st);
    if (iffld == 1) ok = ok && dfld.alloc(6L * ns, s, st);
    if (nt && ifpottarg == 1) ok = ok && dpt.alloc(2L * nt, s, st);
    if (nt && iffldtarg == 1) ok = ok && dft.alloc(6L * nt, s, st);
    if (!ok) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    // large transfers from / to pageable memory go through the pinned ring
    const size_t in_bytes = sizeof(double) * ((size_t)3 * ns + (ifcharge == 1 ? 2 * ns : 0) +
                                              (ifdipole == 1 ? 5 * ns : 0) + 3 * (size_t)nt);
    StageRing *ring = (in_bytes >= kStageMin && host_pageable(source)) ? stage_ring() : nullptr;
    auto h2d = [&](void *d, const void *h, size_t bytes, cudaStream_t stream) {
        if (ring && bytes >= kStageMin) staged_h2d(*ring, d, h, bytes, stream, st);
        else FMM_TRY(st, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, stream));
    };
    h2d(dsrc.p, source, sizeof(double) * 3 * ns, s);
    if (nt) h2d(dtrg.p, target, sizeof(double) * 3 * nt, s);
    SideStreams &ss = side_streams();
    // the charge buffers were allocated on s: the copy stream starts after that
    FMM_TRY(st, cudaEventRecord(ss.fork, s));
    FMM_TRY(st, cudaStreamWaitEvent(ss.copy, ss.fork, 0));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    Status cst;   // status of the charge copies (written by the helper thread when there is one)
    auto copy_charges = [&, ring]() {
        auto hc = [&](void *d, const void *h, size_t bytes) {
            if (ring && bytes >= kStageMin) staged_h2d(*ring, d, h, bytes, ss.copy, cst);
            else FMM_TRY(cst, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ss.copy));
        };
        if (ifcharge == 1) hc(dq.p, charge, sizeof(double) * 2 * ns);
        if (ifdipole == 1) {
            hc(ddq.p, dipstr, sizeof(double) * 2 * ns);
            hc(ddv.p, dipvec, sizeof(double) * 3 * ns);
        }
        FMM_TRY(cst, cudaEventRecord(ss.copied, ss.copy));
    };
    std::thread helper;
    if (ring && overlap_charges) {
        // pageable charges: a helper thread stages them while this thread builds the tree
        int dev = 0;
        cudaGetDevice(&dev);
        helper = std::thread([&, dev]() {
            cudaSetDevice(dev);
            copy_charges();
        });
        g_ti.inputs_join = [&helper]() { if (helper.joinable()) helper.join(); };
        g_ti.inputs_ready = ss.copied;
    } else {
        copy_charges();
        if (!cst.ok()) { g_ti.err = cudaGetErrorString(cst.err); return 8; }
        if (overlap_charges) g_ti.inputs_ready = ss.copied;
        else FMM_TRY(st, cudaStreamWaitEvent(s, ss.copied, 0));
    }
    int ier = run(dsrc.p, dq.p, ddq.p, ddv.p, dpot.p, dfld.p, dtrg.p, dpt.p, dft.p, s);
    if (g_ti.inputs_join || g_ti.inputs_ready) {
        // not consumed (an early error): order the stream after the copies anyway
        wait_host_inputs(s, st);
    }
    if (helper.joinable()) helper.join();
    if (!ier && !cst.ok()) { g_ti.err = cudaGetErrorString(cst.err); ier = 8; }
    if (ier) {
        cudaStreamSynchronize(s);
        return ier;
    }
    auto d2h = [&](void *h, const void *d, size_t bytes) {
        if (ring && bytes >= kStageMin && host_pageable(h)) staged_d2h(*ring, h, d, bytes, s, st);
        else FMM_TRY(st, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
    };
    if (ifpot == 1) d2h(pot, dpot.p, sizeof(double) * 2 * ns);
    if (iffld == 1) d2h(fld, dfld.p, sizeof(double) * 6 * ns);
    if (nt && ifpottarg == 1) d2h(pottarg, dpt.p, sizeof(double) * 2 * nt);
    if (nt && iffldtarg == 1) d2h(fldtarg, dft.p, sizeof(double) * 6 * nt);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    return 0;
}

// Host arrays in and out for the triangle entry points (pageable or pinned):
// device copies, the device call, copies back; a failed call leaves the
// outputs untouched.
template <class F>
inline int tri_host(int ns, const double *tri, const double *norm, const double *source, int ifcharge,
                    const double *charge, int ifdipole, const double *dipstr, int ifpot, double *pot, int iffld,
                    double *fld, int nt, const double *target, int ifpottarg, double *pottarg, int iffldtarg,
                    double *fldtarg, F run)
{
    ns = std::max(ns, 0);
    nt = std::max(nt, 0);
    cudaStream_t s = thread_stream();
    Status st;
    DBuf<double> dtri, dnorm, dsrc, dq, ddq, dtrg, po, fo, pt, ft;
    alloc_fail_point(1);
    bool ok = dtri.alloc(9L * std::max(ns, 1), s, st) && dsrc.alloc(3L * std::max(ns, 1), s, st);
    if (norm) ok = ok && dnorm.alloc(3L * std::max(ns, 1), s, st);
    if (ifcharge == 1) ok = ok && dq.alloc(2L * ns, s, st);
    if (ifdipole == 1) ok = ok && ddq.alloc(2L * ns, s, st);
    if (nt) ok = ok && dtrg.alloc(3L * nt, s, st);
    if (ifpot == 1) ok = ok && po.alloc(2L * ns, s, st);
    if (iffld == 1) ok = ok && fo.alloc(6L * ns, s, st);
    if (nt && ifpottarg == 1) ok = ok && pt.alloc(2L * nt, s, st);
    if (nt && iffldtarg == 1) ok = ok && ft.alloc(6L * nt, s, st);
    if (!ok) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    auto h2d = [&](DBuf<double> &d, const double *h, size_t n) {
        if (n) FMM_TRY(st, cudaMemcpyAsync(d.p, h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    };
    h2d(dtri, tri, 9L * ns);
    h2d(dsrc, source, 3L * ns);
    if (norm) h2d(dnorm, norm, 3L * ns);
    if (ifcharge == 1) h2d(dq, charge, 2L * ns);
    if (ifdipole == 1) h2d(ddq, dipstr, 2L * ns);
    if (nt) h2d(dtrg, target, 3L * nt);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    int e = run(dtri.p, dnorm.p, dsrc.p, dq.p, ddq.p, po.p, fo.p, nt, dtrg.p, nt ? ifpottarg : 0, pt.p,
                nt ? iffldtarg : 0, ft.p, s);
    if (e) return e;
    auto d2h = [&](double *h, DBuf<double> &d) {
        if (d.n) FMM_TRY(st, cudaMemcpyAsync(h, d.p, sizeof(double) * d.n, cudaMemcpyDeviceToHost, s));
    };
    if (ifpot == 1) d2h(pot, po);
    if (iffld == 1) d2h(fld, fo);
    if (nt && ifpottarg == 1) d2h(pottarg, pt);
    if (nt && iffldtarg == 1) d2h(fldtarg, ft);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    return 0;
}

}  // namespace fmm
