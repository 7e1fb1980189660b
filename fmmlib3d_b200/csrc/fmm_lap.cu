// Laplace particle FMM driver and the C ABI (include/fmm3d_b200.h).
//
// Host orchestration of lfmm3dparttarg (src/lfmm3dpart.f:138-522) and
// lfmm3dparttargmain (:528-1169) on one B200: the iprec tables, the octree,
// the expansion order, the eight passes and the unsort run as CUDA kernels on
// one stream; the host only sizes buffers and enqueues launches.
#include <math.h>
#include <string.h>

#include <map>
#include <memory>
#include <atomic>
#include <mutex>
#include <string>
#include <tuple>
#include <algorithm>
#include <vector>

#include "../../include/fmm3d_b200.h"
#include "lap_kernels.cuh"
#include "hess.cuh"
#include "tri.cuh"
#include "m2l_dense.cuh"
#include "tree.cuh"
#include "driver_common.cuh"
#include "tuning.cuh"

namespace fmm {

thread_local int g_launch_count = 0;

// ---------------------------------------------------------------- iprec tables
// src/lfmm3dpart.f:277-300
static bool lap_iprec(int iprec, int ns, int nt, double &eps, int &nbox)
{
    static const double e[] = {.5e0, .5e-1, .5e-2, .5e-3, .5e-6, .5e-9, .5e-12, .5e-15, 0.0};
    static const int nb[] = {40, 50, 80, 160, 400, 800, 1200, 1400};
    if (iprec < -2 || iprec > 6) return false;
    eps = e[iprec + 2];
    nbox = iprec == 6 ? ns + nt : nb[iprec + 2];
    return true;
}

// l3dterms, src/l3dterms.f:34-77
static int l3dterms(double eps)
{
    double z1 = 1.5, z2 = sqrt(3.0) / 2.0, jfun = z2, hfun = 1.0 / (z1 * z1);
    for (int j = 2; j <= 1000; j++) {
        hfun = hfun / z1;
        jfun = jfun * z2;
        if (jfun * hfun < eps) return j;
    }
    return 1;
}

// l3dterms_list2, src/l3dterms.f:136-248; itab[(i+3)*49+(j+3)*7+(k+3)]
static void l3dterms_list2(double eps, int *itab)
{
    int tab[2][4][4];
    for (int ii = 2; ii <= 3; ii++)
        for (int jj = 0; jj <= 3; jj++)
            for (int kk = 0; kk <= 3; kk++) {
                double dx = ii, dy = jj, dz = kk;
                if (dx > 0) dx -= .5;
                if (dy > 0) dy -= .5;
                if (dz > 0) dz -= .5;
                double rr = sqrt(dx * dx + dy * dy + dz * dz);
                double z2 = sqrt(3.0) / 2.0, jfun = z2, hfun = 1.0 / (rr * rr);
                int nt = 1;
                for (int j = 2; j <= 1000; j++) {
                    hfun = hfun / rr;
                    jfun = jfun * z2;
                    if (jfun * hfun < eps) { nt = j; break; }
                }
                tab[ii - 2][jj][kk] = nt;
            }
    for (int i = -3; i <= 3; i++)
        for (int j = -3; j <= 3; j++)
            for (int k = -3; k <= 3; k++) {
                int v = 0, ai = abs(i), aj = abs(j), ak = abs(k);
                if (ai > 1) v = tab[ai - 2][aj][ak];
                else if (aj > 1) v = tab[aj - 2][ai][ak];
                if (ai <= 1 && aj <= 1 && ak > 1) v = ai >= aj ? tab[ak - 2][ai][aj] : tab[ak - 2][aj][ai];
                itab[(i + 3) * 49 + (j + 3) * 7 + (k + 3)] = v;
            }
}

// ---------------------------------------------------------------- per-thread state
// ---------------------------------------------------------------- operator plan (per device, p, eps)
// Rotation matrices for every direction class, the slot tables of the three
// translation kinds and the sqrt-binomial table.  Built once on the device
// and kept for the life of the process.
struct LapPlan {
    int p = 0;
    int ncls = 0;
    int lddc = 0;
    DBuf<double> rot, dc;
    DBuf<Slot> slots;        // [0, 1512): M2L 8 octants x 189; [1512,1520): M2M; [1520,1528): L2L
    std::vector<Slot> hslots;
    int kt = 8;       // targets per tile of M2M / L2L
    int kt_m2l = 8;   // targets per tile of the rotate-shift-rotate M2L
    // dense M2L operators (p <= kDenseMaxP): one per list-2 offset, and the
    // operator offset of every M2L slot
    bool dense = false;
    DBuf<double2> T;
    DBuf<float2> T32;        // the same operators rounded to FP32 (mixed form)
    DBuf<long long> slot_toff;
};
// Switches of the Laplace calls: a process-wide value (fmm3d_set_m2l_mode,
// _precision, _tensor_m2l, _tensor_m2l_group, _overlap) and a per-host-thread
// override (fmm3d_set_switch_thread; -1 follows the process-wide value), read
// on the calling thread when a call or a plan execution starts, so that a
// thread (a serving worker) can set its own without touching other threads'
// calls.
enum Switch {
    kSwM2LMode = 0,    // 0 automatic, 1 rotate-shift-rotate, 2 dense operators, 3 rotate-shift-rotate
                       // on the CUDA cores (1 and 0 use the FP64 tensor cores up to order 28)
    kSwPrecision = 1,  // 0 FP64 throughout, 1 mixed (FP32 P2P and M2L) for iprec <= 1
    kSwTensorM2L = 2,  // mixed-form M2L: 0 FP32 CUDA cores, 1/2 tensor cores (stage variants 0/1)
    kSwTcGroup = 3,    // tensor-core M2L: slots per TMEM sum (0: one sum per tile)
    kSwOverlap = 4,    // near field concurrent with the far-field passes
    kNumSw = 5
};
static std::atomic<int> g_sw[kNumSw] = {{0}, {0}, {1}, {1}, {1}};
static thread_local int g_sw_thread[kNumSw] = {-1, -1, -1, -1, -1};
static inline int sw(int k) { return g_sw_thread[k] >= 0 ? g_sw_thread[k] : g_sw[k].load(std::memory_order_relaxed); }
static bool sw_valid(int k, int v)
{
    switch (k) {
    case kSwM2LMode: return v >= 0 && v <= 3;
    case kSwPrecision: return v == 0 || v == 1;
    case kSwTensorM2L: return v >= 0 && v <= 2;
    case kSwTcGroup: return v >= 0;
    case kSwOverlap: return v == 0 || v == 1;
    }
    return false;
}
constexpr int kSlotM2M = 8 * 189, kSlotL2L = 8 * 189 + 8;

static std::mutex g_plan_mu;
static std::map<std::tuple<int, int, long long>, std::shared_ptr<LapPlan>> g_plans;

static std::shared_ptr<LapPlan> get_plan(int p, double eps, cudaStream_t s, Status &st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    long long ekey;
    memcpy(&ekey, &eps, sizeof ekey);
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto key = std::make_tuple(dev, p, ekey);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) return it->second;
    auto P = std::make_shared<LapPlan>();
    P->p = p;
    // direction classes keyed by (rho^2, dz) of a doubled integer vector
    std::map<std::pair<int, int>, int> cls;
    std::vector<double> cs;
    auto class_of = [&](int dx, int dy, int dz) {
        auto k = std::make_pair(dx * dx + dy * dy, dz);
        auto f = cls.find(k);
        if (f != cls.end()) return f->second;
        double r = sqrt((double)(dx * dx + dy * dy + dz * dz));
        int id = (int)cls.size();
        cls[k] = id;
        cs.push_back(dz / r);
        cs.push_back(sqrt((double)(dx * dx + dy * dy)) / r);
        return id;
    };
    auto ephi = [](int dx, int dy, double &ex, double &ey) {
        double rho = sqrt((double)(dx * dx + dy * dy));
        if (rho == 0) { ex = 1; ey = 0; }
        else { ex = dx / rho; ey = dy / rho; }
    };
    int itab[343];
    l3dterms_list2(eps, itab);
    P->hslots.resize(8 * 189 + 16);
    for (int o = 0; o < 8; o++) {
        int ob[3] = {o & 1, (o >> 1) & 1, (o >> 2) & 1};
        int ns = 0;
        for (int c = 0; c < 27; c++) {
            int co[3] = {c / 9 - 1, (c / 3) % 3 - 1, c % 3 - 1};
            for (int d = 0; d < 8; d++) {
                int db[3] = {d & 1, (d >> 1) & 1, (d >> 2) & 1};
                int D[3];
                for (int e = 0; e < 3; e++) D[e] = 2 * co[e] + db[e] - ob[e];
                if (abs(D[0]) <= 1 && abs(D[1]) <= 1 && abs(D[2]) <= 1) continue;
                Slot &sl = P->hslots[o * 189 + ns++];
                sl.coll = c;
                sl.oct = d;
                // direction target - source = -D
                sl.cls = class_of(-2 * D[0], -2 * D[1], -2 * D[2]);
                ephi(-D[0], -D[1], sl.ex, sl.ey);
                sl.rt = sqrt((double)(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]));
                int nt = itab[(D[0] + 3) * 49 + (D[1] + 3) * 7 + (D[2] + 3)];
                sl.pt = nt < p ? nt : p;
            }
        }
    }
    for (int d = 0; d < 8; d++) {
        int b[3] = {d & 1, (d >> 1) & 1, (d >> 2) & 1};
        // M2M: parent - child = (0.5 - bits) -> doubled (1 - 2 bits)
        Slot &a = P->hslots[kSlotM2M + d];
        a.coll = -1; a.oct = d; a.pt = p; a.rt = sqrt(3.0) / 2;
        a.cls = class_of(1 - 2 * b[0], 1 - 2 * b[1], 1 - 2 * b[2]);
        ephi(1 - 2 * b[0], 1 - 2 * b[1], a.ex, a.ey);
        // L2L: child - parent = (bits - 0.5)
        Slot &l = P->hslots[kSlotL2L + d];
        l.coll = -1; l.oct = d; l.pt = p; l.rt = sqrt(3.0) / 2;
        l.cls = class_of(2 * b[0] - 1, 2 * b[1] - 1, 2 * b[2] - 1);
        ephi(2 * b[0] - 1, 2 * b[1] - 1, l.ex, l.ey);
    }
    P->ncls = (int)cls.size();
    // sqrt of binomial coefficients up to 2p+2
    P->lddc = 2 * p + 3;
    std::vector<double> car((size_t)P->lddc * P->lddc, 0.0), dch((size_t)P->lddc * P->lddc, 0.0);
    for (int n = 0; n < P->lddc; n++) {
        car[(size_t)n * P->lddc] = 1;
        for (int k = 1; k <= n; k++)
            car[(size_t)n * P->lddc + k] = car[(size_t)(n - 1) * P->lddc + k - 1] +
                                           (k <= n - 1 ? car[(size_t)(n - 1) * P->lddc + k] : 0.0);
        for (int k = 0; k <= n; k++) dch[(size_t)n * P->lddc + k] = sqrt(car[(size_t)n * P->lddc + k]);
    }
    DBuf<double> dcs;
    P->rot.alloc(rot_class_size(p) * P->ncls, s, st);
    P->dc.alloc(dch.size(), s, st);
    P->slots.alloc(P->hslots.size(), s, st);
    dcs.alloc(cs.size(), s, st);
    if (!st.ok()) return nullptr;
    FMM_TRY(st, cudaMemcpyAsync(P->dc.p, dch.data(), sizeof(double) * dch.size(), cudaMemcpyHostToDevice, s));
    FMM_TRY(st, cudaMemcpyAsync(P->slots.p, P->hslots.data(), sizeof(Slot) * P->hslots.size(),
                                cudaMemcpyHostToDevice, s));
    FMM_TRY(st, cudaMemcpyAsync(dcs.p, cs.data(), sizeof(double) * cs.size(), cudaMemcpyHostToDevice, s));
    build_rotations(p, P->ncls, dcs.p, P->rot.p, s, st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) return nullptr;
    // tile sizes: three KT x (p+1)^2 complex buffers.  M2M / L2L (8 slots per
    // tile) within ~50 KB of shared memory, so that several CTAs share an SM;
    // the rotate-shift-rotate M2L (189 slots, two rotation matrices read per
    // slot and tile) within ~200 KB, so that the matrices serve more targets.
    int NC = (p + 1) * (p + 1);
    P->kt = 8;
    while (P->kt > 1 && (size_t)3 * P->kt * NC * 16 > 50 * 1024) P->kt /= 2;
    // (up to order 26 the M2L kernel keeps its running sums in registers: two buffers)
    const int m2l_nbuf = NC <= 3 * 256 ? 2 : 3;
    P->kt_m2l = 8;
    while (P->kt_m2l > 1 && (size_t)m2l_nbuf * P->kt_m2l * NC * 16 > 200 * 1024) P->kt_m2l /= 2;
    if (p <= kDenseMaxP) {
        // unique list-2 offsets and their operators
        std::map<int, int> uidx;
        std::vector<M2LOp> uops;
        std::vector<long long> stoff(8 * 189);
        long long tot = 0;
        for (int o = 0; o < 8; o++) {
            int ob[3] = {o & 1, (o >> 1) & 1, (o >> 2) & 1};
            for (int si = 0; si < 189; si++) {
                const Slot &sl = P->hslots[o * 189 + si];
                int co[3] = {sl.coll / 9 - 1, (sl.coll / 3) % 3 - 1, sl.coll % 3 - 1};
                int db[3] = {sl.oct & 1, (sl.oct >> 1) & 1, (sl.oct >> 2) & 1};
                int key = 0;
                for (int e = 0; e < 3; e++) key = key * 16 + (2 * co[e] + db[e] - ob[e] + 8);
                auto f = uidx.find(key);
                if (f == uidx.end()) {
                    M2LOp op;
                    op.pt = sl.pt; op.cls = sl.cls; op.ex = sl.ex; op.ey = sl.ey; op.rt = sl.rt; op.toff = tot;
                    long long R = (long long)(sl.pt + 1) * (sl.pt + 1);
                    tot += R * R;
                    f = uidx.emplace(key, (int)uops.size()).first;
                    uops.push_back(op);
                }
                stoff[o * 189 + si] = uops[f->second].toff;
            }
        }
        DBuf<M2LOp> dops;
        if (dops.alloc(uops.size(), s, st) && P->T.alloc(tot, s, st) && P->slot_toff.alloc(stoff.size(), s, st)) {
            FMM_TRY(st, cudaMemcpyAsync(dops.p, uops.data(), sizeof(M2LOp) * uops.size(), cudaMemcpyHostToDevice, s));
            FMM_TRY(st, cudaMemcpyAsync(P->slot_toff.p, stoff.data(), sizeof(long long) * stoff.size(),
                                        cudaMemcpyHostToDevice, s));
            build_m2l_ops(p, (int)uops.size(), dops.p, P->rot.p, P->dc.p, P->lddc, P->T.p, s, st);
            if (P->T32.alloc(tot, s, st)) convert_f32(tot, P->T.p, P->T32.p, s, st);
            FMM_TRY(st, cudaStreamSynchronize(s));
        }
        if (!st.ok()) return nullptr;
        P->dense = true;
        P->T.s = nullptr;
        P->T32.s = nullptr;
        P->slot_toff.s = nullptr;
    }
    // buffers are process-lifetime: detach them from the stream they were made on
    P->rot.s = nullptr;
    P->dc.s = nullptr;
    P->slots.s = nullptr;
    g_plans[key] = P;
    return P;
}

// ---------------------------------------------------------------- small kernels
// statistics: near-field pairs and far-field pairs
__global__ void k_stats(int nleaves, const int *leaves, TreeView tv, int do_src, int do_trg,
                        unsigned long long *acc)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nleaves) return;
    int b = leaves[t];
    long ne = (do_src ? tv.nsrc[b] : 0) + (do_trg ? tv.ntrg[b] : 0);
    long ns = tv.nsrc[b];
    for (int k = tv.l1_start[b]; k < tv.l1_start[b + 1]; k++) ns += tv.nsrc[tv.l1_idx[k]];
    long self = do_src ? tv.nsrc[b] : 0;
    atomicAdd(acc, (unsigned long long)(ne * ns - self));
}

__global__ void k_m2l_count(int b0, int nb, TreeView tv, const Slot *slots, int prune, unsigned long long *hist)
{
    __shared__ unsigned int h[128];
    for (int i = threadIdx.x; i < 128; i += blockDim.x) h[i] = 0;
    __syncthreads();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int b = b0 + t;
    if (t < nb && !(prune && tv.ntrg[b] == 0) && tv.parent[b] >= 0) {
        int P = tv.parent[b];
        int o = tv.octant[b];
        for (int s = 0; s < 189; s++) {
            const Slot &sl = slots[o * 189 + s];
            int C = tv.coll[27L * P + sl.coll];
            if (C < 0) continue;
            int src = tv.child[8L * C + sl.oct];
            if (src < 0 || tv.nsrc[src] == 0) continue;
            atomicAdd(&h[sl.pt], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 128; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

static int device_sms()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

// ---------------------------------------------------------------- one evaluation geometry
// Device state of a Laplace evaluation for fixed sources and targets: tree and
// lists, tree-ordered coordinates, expansion and output workspace, translation
// tiles.  A single call builds it and runs the passes once; a plan
// (fmm3d_lfmm3d_plan_*) keeps it and runs the passes for new charges.
struct LapSetup {
    EvalItems ev;   // work items of the evaluation pass
    int iprec = 0, p = 0, K = 0, ns = 0, nt = 0, ldm = 0;
    int ifcharge = 0, ifdipole = 0, ifpot = 0, iffld = 0, ifpottarg = 0, iffldtarg = 0;
    int do_src = 0, do_trg = 0, prune = 0;
    bool mixed = false, dense = false, tcm2l = false;
    std::shared_ptr<LapPlan> plan;
    Tree T;
    TreeView tv;
    DBuf<double> sx, sy, sz, svx, svy, svz, tx, ty, tz;
    DBuf<double2> sq, sdq, opot, ofx, ofy, ofz, tpot, tfx, tfy, tfz, mpole, local;
    DBuf<float2> mp32;
    DBuf<int> tcerr;
    DBuf<Tile> dtiles;
    std::vector<std::pair<int, int>> m2m_rng, l2l_rng;  // per level: [first tile, count)
    int m2l_a = 0, m2l_n = 0, m2l_kt = 0, trans_kt = 0;
    // mixed form: list-3 boxes with few sources and the list-4 boxes of boxes with
    // few points are summed with the near field; tv_near is tv with list 1
    // replaced by the widened near list, tv_far with lists 3 and 4 by the rest
    DBuf<int> nl_start, nl_idx, fl_start, fl_idx, f4_start, f4_idx;
    TreeView tv_near, tv_far;
    int l3_direct = 0;        // source / point count up to which lists 3 / 4 go to the near field (0: none)
    TuneKnobs knobs;          // as requested (0 = automatic); m2l_kt / trans_kt hold the values in use
    bool knobs_from_cache = false;
    std::string signature;
    PointsSoA P;
    OutSoA os, ot;
    // Hessian outputs (dxx, dyy, dzz, dxy, dxz, dyz), set before lap_setup;
    // computed in FP64 with the near / far split of the potentials
    int ifhess = 0, ifhesstarg = 0;
    DBuf<double2> shess[6], thess[6];
    HessSoA hs, ht;
    double *hess_out = nullptr, *hesstarg_out = nullptr;
    // triangle FMM (lfmm3dtriatarg), set before lap_setup: the sources are
    // flat triangles, the tree's points their centroids; the far field runs
    // on the triangles' quadrature nodes (Pq, box ranges tv_quad), the near
    // field by exact integrals (ts).  Always FP64.
    bool tri = false;
    const double *tri_in = nullptr, *tri_norm = nullptr;
    TriRule rule;
    DBuf<double> tgeo, qx, qy, qz, qvx, qvy, qvz;
    DBuf<double2> tq, tdq, qq, qdq;
    DBuf<int> qsrc0, qnsrc;
    TriSoA ts;
    PointsSoA Pq;
    TreeView tv_quad;
};

// Problem signature of the tuning cache: the form, the flags that select
// kernel variants, and the sizes that set the launch shapes (log2 buckets).
static std::string lap_signature(const LapSetup &S)
{
    const char *form = S.tcm2l ? "mixed-tc" : S.mixed ? "mixed-cuda" : S.dense ? "fp64-dense" : "fp64-rotation";
    const char *kern = S.tri ? "laplace-triangles" : "laplace";
    char b[512];
    snprintf(b, sizeof b,
             "%s iprec=%d form=%s charge=%d dipole=%d out=%d%d%d%d inst=2^%d ns=2^%d nt=2^%d nlev=%d "
             "nboxes=2^%d dev=%s",
             kern, S.iprec, form, S.ifcharge == 1, S.ifdipole == 1, S.ifpot == 1, S.iffld == 1,
             S.do_trg && S.ifpottarg == 1, S.do_trg && S.iffldtarg == 1, log2_bucket(S.T.ninst),
             log2_bucket(S.ns), log2_bucket(S.do_trg ? S.nt : 0), S.T.nlev, log2_bucket(S.T.nboxes),
             device_tag().c_str());
    return b;
}

// form code reported with the knobs: 0 FP64 rotations, 1 FP64 dense, 2 mixed CUDA-core M2L, 3 mixed tensor-core M2L
static int lap_form(const LapSetup &S) { return S.tcm2l ? 3 : S.mixed ? 2 : S.dense ? 1 : 0; }

// Tiles of one (level, octant) group and translation kind: boxes [a, bnd) of
// the grouped box array in runs of kt, written from tile tile0 on.
struct TileSeg {
    int tile0, a, bnd, kt, slot0, nslot;
};

__global__ void k_make_tiles(const TileSeg *segs, Tile *tiles)
{
    const TileSeg g = segs[blockIdx.x];
    const int n = (g.bnd - g.a + g.kt - 1) / g.kt;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        Tile t;
        t.first = g.a + j * g.kt;
        t.count = min(g.kt, g.bnd - t.first);
        t.slot0 = g.slot0;
        t.nslot = g.nslot;
        tiles[g.tile0 + j] = t;
    }
}

// Translation tiles for the given knobs (0 = automatic): M2M / L2L tiles of
// trans_kt targets per (level, octant) group, M2L tiles of m2l_kt.  Returns 2
// for a knob this problem cannot take (tile size outside the kernel's range or
// its shared memory), with S unchanged.
static int lap_tiles(LapSetup &S, const TuneKnobs &k, cudaStream_t s, Status &st)
{
    Tree &T = S.T;
    auto &plan = S.plan;
    const int NC = S.K, p = S.p;
    const size_t smax = 226 * 1024;   // opt-in limit less room for the kernel's static shared memory
    auto trans_sm = [&](int nbuf, int kt) {
        return (size_t)nbuf * kt * NC * sizeof(double2) + (p + 1) * sizeof(double2) + (2 * p + 4) * sizeof(double);
    };
    auto pow2_le8 = [](int v) { return v == 1 || v == 2 || v == 4 || v == 8; };
    if (k.trans_kt && !(pow2_le8(k.trans_kt) && trans_sm(3, k.trans_kt) <= smax)) return 2;
    if (k.m2l_kt) {
        if (S.tcm2l) {
            if (k.m2l_kt % 16 || k.m2l_kt < 16 || k.m2l_kt > kTcTileTargetsMax) return 2;
        } else if (S.mixed) {
            if (k.m2l_kt != kDenseTileTargets) return 2;
        } else if (S.dense) {
            if (k.m2l_kt != 16 && k.m2l_kt != kDenseTileTargets) return 2;
        } else {
            const int nbuf = (k.m2l_kt == 8 && NC <= 3 * 256) ? 2 : 3;
            if (!pow2_le8(k.m2l_kt) || trans_sm(nbuf, k.m2l_kt) > smax) return 2;
        }
    }
    if (k.tc_variant < 0 || k.tc_variant > 2 || k.overlap < 0 || k.overlap > 2) return 2;
    if (!(k.p2p_ept == 0 || k.p2p_ept == 1 || k.p2p_ept == 2 || k.p2p_ept == 4)) return 2;

    // tile segments on the host (a few per level), the tiles themselves on the device
    std::vector<TileSeg> segs;
    int ntile = 0;
    auto make_tiles = [&](int lev, int kt, int slot0_base, int per_oct_stride, int nslot) {
        for (int o = 0; o < 8; o++) {
            int g = lev * 8 + o;
            int a = T.group_start[g], bnd = T.group_start[g + 1];
            if (bnd <= a) continue;
            segs.push_back({ntile, a, bnd, kt, slot0_base + o * per_oct_stride, nslot});
            ntile += div_up(bnd - a, kt);
        }
    };
    const int tkt = k.trans_kt ? k.trans_kt : plan->kt;
    std::vector<std::pair<int, int>> m2m, l2l;
    for (int l = T.nlev - 1; l >= 2; l--) {
        int a = ntile;
        make_tiles(l, tkt, kSlotM2M, 0, 8);
        m2m.push_back({a, ntile - a});
    }
    // M2L tile size (automatic): the largest whose tile count fills the GPU (two
    // CTAs per SM per 64-row block); smaller tiles only add CTAs, every target's
    // sums are unchanged
    int m2l_kt = S.tcm2l ? kTcTileTargets : S.dense ? kDenseTileTargets : plan->kt_m2l;
    if (k.m2l_kt) {
        m2l_kt = k.m2l_kt;
    } else if (S.dense && !(S.mixed && !S.tcm2l)) {
        const int rows = div_up(S.K, 64), want = 2 * device_sms();
        auto ntiles = [&](int kt) {
            long t = 0;
            for (int l = 2; l <= T.nlev; l++)
                for (int o = 0; o < 8; o++) t += div_up(T.group_start[l * 8 + o + 1] - T.group_start[l * 8 + o], kt);
            return t;
        };
        // (256-target tensor-core tiles run one CTA per SM and measured slower on every
        // workload tried; they are reached through the tuning knob only)
        while (m2l_kt > 16 && ntiles(m2l_kt) * rows < want) m2l_kt /= 2;
        if (!S.tcm2l && m2l_kt < kDenseTileTargets) m2l_kt = 16;   // FP64 dense kernel: 64 or 16
    }
    const int m2l_a = ntile;
    for (int l = 2; l <= T.nlev; l++) make_tiles(l, m2l_kt, 0, 189, 189);
    const int m2l_n = ntile - m2l_a;
    for (int l = 2; l <= T.nlev - 1; l++) {
        int a = ntile;
        make_tiles(l + 1, tkt, kSlotL2L, 1, 1);
        l2l.push_back({a, ntile - a});
    }
    if ((size_t)ntile != S.dtiles.n && !S.dtiles.alloc(ntile, s, st)) return 16;
    if (!segs.empty()) {
        DBuf<TileSeg> dsegs;
        if (!dsegs.alloc(segs.size(), s, st)) return 16;
        FMM_TRY(st, cudaMemcpyAsync(dsegs.p, segs.data(), sizeof(TileSeg) * segs.size(), cudaMemcpyHostToDevice, s));
        k_make_tiles<<<(unsigned)segs.size(), 256, 0, s>>>(dsegs.p, S.dtiles.p); FMM_COUNT_LAUNCH();
        FMM_LAUNCH_CHECK(st);
    }
    if (!st.ok()) return 16;
    S.m2m_rng = m2m;
    S.l2l_rng = l2l;
    S.m2l_a = m2l_a;
    S.m2l_n = m2l_n;
    S.m2l_kt = m2l_kt;
    S.trans_kt = tkt;
    S.knobs = k;
    return 0;
}

// Mixed form, near field widened by source or point count.  A list-3 box c of
// leaf b is a separated box whose multipole the reference evaluates at b's
// points (l3dmpeval_trunc0); a list-4 box c of box a is a separated leaf whose
// sources the reference expands about a (l3dformta_trunc0), the expansion
// then reaching every point below a.  When c holds at most `thr` sources
// (list 3), or a holds at most `thr` evaluation points (list 4), summing c's
// sources directly at the points is cheaper than the (p+2)^2 harmonics per
// point or per source, and exact.  Every box owns a contiguous range of the
// tree-ordered sources, so the near-field kernel takes such boxes as they are.
// Near list of leaf b: list 1, the small list-3 boxes, then the list-4 boxes of
// b and of each ancestor with few points; far lists 3 and 4: the others.
__device__ __forceinline__ bool l4_direct(const TreeView &tv, int a, int thr, int do_src, int do_trg)
{
    return (do_src ? tv.nsrc[a] : 0) + (do_trg ? tv.ntrg[a] : 0) <= thr;
}

__global__ void k_near_count(int nb, TreeView tv, int thr, int do_src, int do_trg, int *cn, int *c3, int *c4)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int near = 0, far3 = 0;
    for (int k = tv.l3_start[b]; k < tv.l3_start[b + 1]; k++) {
        if (tv.nsrc[tv.l3_idx[k]] <= thr) near++;
        else far3++;
    }
    if (tv.nchild[b] == 0) {
        near += tv.l1_start[b + 1] - tv.l1_start[b];
        for (int a = b; a >= 0; a = tv.parent[a])
            if (l4_direct(tv, a, thr, do_src, do_trg)) near += tv.l4_start[a + 1] - tv.l4_start[a];
    } else {
        near = 0;
    }
    cn[b] = near;
    c3[b] = far3;
    c4[b] = l4_direct(tv, b, thr, do_src, do_trg) ? 0 : tv.l4_start[b + 1] - tv.l4_start[b];
}

__global__ void k_near_fill(int nb, TreeView tv, int thr, int do_src, int do_trg, const int *n0, const int *f30,
                            const int *f40, int *nidx, int *f3idx, int *f4idx)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const bool leaf = tv.nchild[b] == 0;
    int o = n0[b], f = f30[b];
    if (leaf)
        for (int k = tv.l1_start[b]; k < tv.l1_start[b + 1]; k++) nidx[o++] = tv.l1_idx[k];
    for (int k = tv.l3_start[b]; k < tv.l3_start[b + 1]; k++) {
        const int c = tv.l3_idx[k];
        if (tv.nsrc[c] <= thr) { if (leaf) nidx[o++] = c; }
        else f3idx[f++] = c;
    }
    if (leaf)
        for (int a = b; a >= 0; a = tv.parent[a])
            if (l4_direct(tv, a, thr, do_src, do_trg))
                for (int k = tv.l4_start[a]; k < tv.l4_start[a + 1]; k++) nidx[o++] = tv.l4_idx[k];
    if (!l4_direct(tv, b, thr, do_src, do_trg)) {
        int g = f40[b];
        for (int k = tv.l4_start[b]; k < tv.l4_start[b + 1]; k++) f4idx[g++] = tv.l4_idx[k];
    }
}

static void lap_widen_near(LapSetup &S, int thr, cudaStream_t s, Status &st)
{
    Tree &T = S.T;
    const int nb = T.nboxes;
    S.tv_near = S.tv_far = S.tv;
    S.l3_direct = 0;
    if (thr <= 0 || nb == 0) return;
    DBuf<int> cn, c3, c4;
    if (!cn.alloc(nb + 1, s, st) || !c3.alloc(nb + 1, s, st) || !c4.alloc(nb + 1, s, st) ||
        !S.nl_start.alloc(nb + 1, s, st) || !S.fl_start.alloc(nb + 1, s, st) || !S.f4_start.alloc(nb + 1, s, st))
        return;
    cn.zero(st);
    c3.zero(st);
    c4.zero(st);
    k_near_count<<<div_up(nb, 256), 256, 0, s>>>(nb, S.tv, thr, S.do_src, S.do_trg, cn.p, c3.p, c4.p); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    int tn = 0, t3 = 0, t4 = 0;
    scan_exclusive_int(cn.p, S.nl_start.p, nb + 1, s, st, &tn);
    scan_exclusive_int(c3.p, S.fl_start.p, nb + 1, s, st, &t3);
    scan_exclusive_int(c4.p, S.f4_start.p, nb + 1, s, st, &t4);
    if (!st.ok() || !S.nl_idx.alloc(std::max(tn, 1), s, st) || !S.fl_idx.alloc(std::max(t3, 1), s, st) ||
        !S.f4_idx.alloc(std::max(t4, 1), s, st))
        return;
    k_near_fill<<<div_up(nb, 256), 256, 0, s>>>(nb, S.tv, thr, S.do_src, S.do_trg, S.nl_start.p, S.fl_start.p,
                                               S.f4_start.p, S.nl_idx.p, S.fl_idx.p, S.f4_idx.p); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    if (!st.ok()) return;
    S.tv_near.l1_start = S.nl_start.p;
    S.tv_near.l1_idx = S.nl_idx.p;
    S.tv_far.l3_start = S.fl_start.p;
    S.tv_far.l3_idx = S.fl_idx.p;
    S.tv_far.l4_start = S.f4_start.p;
    S.tv_far.l4_idx = S.f4_idx.p;
    S.l3_direct = thr;
}

// charges and dipoles into tree order (l3dreorder, src/lfmm3drouts.f:667-691)
__global__ void k_gather_q(int n, const int *perm, const double *q, const double *dq, const double *dv, int ifc,
                           int ifd, PointsSoA o)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long j = perm[i];
    if (ifc) o.q[i] = make_double2(q[2 * j], q[2 * j + 1]);
    if (ifd) {
        o.dq[i] = make_double2(dq[2 * j], dq[2 * j + 1]);
        o.vx[i] = dv[3 * j];
        o.vy[i] = dv[3 * j + 1];
        o.vz[i] = dv[3 * j + 2];
    }
}

// Geometry-dependent part: operator plan, tree and lists, sorted coordinates,
// workspace and tiles.  so / to (optional): instance offsets of a batch, each
// instance an independent FMM over its own sources and targets (a forest).
static int lap_setup(LapSetup &S, int iprec, int ns, const double *d_src, int ifcharge, int ifdipole, int ifpot,
                     int iffld, int nt, const double *d_trg, int ifpottarg, int iffldtarg, cudaStream_t s, Timer &tm,
                     const std::vector<int> *so = nullptr, const std::vector<int> *to = nullptr)
{
    Status st;
    double eps;
    int nbox;
    if (ns < 1 || !lap_iprec(iprec, ns, nt, eps, nbox)) return 4;
    if (S.tri) nbox = tri_nbox(iprec, ns, nt);
    if (nt < 0) nt = 0;
    lap_init_constants(st);
    keep_pool_memory();
    const int p = l3dterms(eps);
    if (p > 72) { g_ti.err = "expansion order " + std::to_string(p) + " above the supported 72"; return 16; }
    S.plan = get_plan(p, eps, s, st);
    if (!st.ok() || !S.plan) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    auto &plan = S.plan;
    S.iprec = iprec; S.p = p; S.K = (p + 1) * (p + 1); S.ns = ns; S.nt = nt;
    S.ifcharge = ifcharge; S.ifdipole = ifdipole; S.ifpot = ifpot; S.iffld = iffld;
    S.ifpottarg = ifpottarg; S.iffldtarg = iffldtarg;
    tm.mark();
    Tree &T = S.T;
    alloc_fail_point(2);
    if (so) build_forest(T, d_src, *so, d_trg, *to, nbox, s, st);
    else build_tree(T, d_src, ns, d_trg, nt, nbox, s, st);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 4; }
    g_ti.depth_capped = T.capped;
    tm.mark();
    const int K = S.K;
    alloc_fail_point(3);
    bool ok = S.sx.alloc(ns, s, st) && S.sy.alloc(ns, s, st) && S.sz.alloc(ns, s, st);
    if (ifcharge == 1) ok = ok && S.sq.alloc(ns, s, st);
    if (ifdipole == 1)
        ok = ok && S.sdq.alloc(ns, s, st) && S.svx.alloc(ns, s, st) && S.svy.alloc(ns, s, st) && S.svz.alloc(ns, s, st);
    if (nt) ok = ok && S.tx.alloc(nt, s, st) && S.ty.alloc(nt, s, st) && S.tz.alloc(nt, s, st);
    S.do_src = ifpot == 1 || iffld == 1 || S.ifhess == 1;
    S.do_trg = (ifpottarg == 1 || iffldtarg == 1 || S.ifhesstarg == 1) && nt > 0;
    if (S.ifhess == 1)
        for (int c = 0; c < 6; c++) ok = ok && S.shess[c].alloc(ns, s, st);
    if (S.do_trg && S.ifhesstarg == 1)
        for (int c = 0; c < 6; c++) ok = ok && S.thess[c].alloc(nt, s, st);
    if (ifpot == 1) ok = ok && S.opot.alloc(ns, s, st);
    if (iffld == 1) ok = ok && S.ofx.alloc(ns, s, st) && S.ofy.alloc(ns, s, st) && S.ofz.alloc(ns, s, st);
    if (S.do_trg && ifpottarg == 1) ok = ok && S.tpot.alloc(nt, s, st);
    if (S.do_trg && iffldtarg == 1) ok = ok && S.tfx.alloc(nt, s, st) && S.tfy.alloc(nt, s, st) && S.tfz.alloc(nt, s, st);
    if (!ok) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    alloc_fail_point(4);
    if (!S.mpole.alloc((size_t)T.nboxes * K, s, st) || !S.local.alloc((size_t)T.nboxes * K, s, st)) {
        g_ti.err = cudaGetErrorString(st.err);
        return 16;
    }
    PointsSoA &P = S.P;
    P.x = S.sx.p; P.y = S.sy.p; P.z = S.sz.p; P.q = S.sq.p; P.dq = S.sdq.p;
    P.vx = S.svx.p; P.vy = S.svy.p; P.vz = S.svz.p;
    k_gather_pts<<<div_up(ns, 256), 256, 0, s>>>(ns, T.perm_src.p, d_src, S.sx.p, S.sy.p, S.sz.p); FMM_COUNT_LAUNCH();
    if (nt) { k_gather_pts<<<div_up(nt, 256), 256, 0, s>>>(nt, T.perm_trg.p, d_trg, S.tx.p, S.ty.p, S.tz.p); FMM_COUNT_LAUNCH(); }
    FMM_LAUNCH_CHECK(st);
    S.tv = make_treeview(T);
    S.prune = !(ifpot == 1 || iffld == 1 || S.ifhess == 1);
    for (int c = 0; c < 6; c++) { S.hs.h[c] = S.shess[c].p; S.ht.h[c] = S.thess[c].p; }
    if (S.ifhess == 1 || S.ifhesstarg == 1) {
        hess_init_constants(st);
        if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    }
    S.os.pot = S.opot.p; S.os.fx = S.ofx.p; S.os.fy = S.ofy.p; S.os.fz = S.ofz.p;
    S.ot.pot = S.tpot.p; S.ot.fx = S.tfx.p; S.ot.fy = S.tfy.p; S.ot.fz = S.tfz.p;

    const int form = sw(kSwPrecision);
    S.mixed = !S.tri && form == 1 && iprec <= 1 && plan->dense;
    S.dense = (plan->dense && sw(kSwM2LMode) != 1 && sw(kSwM2LMode) != 3) || S.mixed;
    S.tcm2l = S.mixed && sw(kSwTensorM2L) > 0;
    // triangles in the mixed form: the M2L runs on the tensor cores (split TF32), the exact
    // near field and every other pass stay FP64
    if (S.tri && form == 1 && iprec <= 1 && plan->dense && sw(kSwTensorM2L) > 0) S.dense = S.tcm2l = true;
    // launch shapes: the autotuner's cached setting for this problem, else automatic
    S.signature = lap_signature(S);
    TuneKnobs kn;
    S.knobs_from_cache = tuning_lookup(S.signature, kn);
    int tier = S.knobs_from_cache ? lap_tiles(S, kn, s, st) : 2;
    if (tier == 2) {
        S.knobs_from_cache = false;
        tier = lap_tiles(S, TuneKnobs(), s, st);
    }
    if (tier) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    // mixed form: small list-3 / list-4 interactions join the near field (FP64 keeps the reference's lists)
    lap_widen_near(S, S.mixed ? (p + 2) * (p + 2) / 2 : 0, s, st);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    eval_items_prepare(T.leaves.p, T.nleaves, S.tv_far, S.do_src, S.do_trg, S.ev, s, st);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    if (S.tri) {
        // triangle data in tree order and the quadrature nodes (filled per call)
        const size_t nn = (size_t)ns * S.rule.n;
        bool okt = S.tgeo.alloc(30L * ns, s, st) && S.qx.alloc(nn, s, st) && S.qy.alloc(nn, s, st) &&
                   S.qz.alloc(nn, s, st) && S.qsrc0.alloc(T.nboxes, s, st) && S.qnsrc.alloc(T.nboxes, s, st);
        if (ifcharge == 1) okt = okt && S.tq.alloc(ns, s, st) && S.qq.alloc(nn, s, st);
        if (ifdipole == 1)
            okt = okt && S.tdq.alloc(ns, s, st) && S.qdq.alloc(nn, s, st) && S.qvx.alloc(nn, s, st) &&
                  S.qvy.alloc(nn, s, st) && S.qvz.alloc(nn, s, st);
        if (!okt) { g_ti.err = cudaGetErrorString(st.err); return 8; }
        S.ts.geo = S.tgeo.p; S.ts.q = S.tq.p; S.ts.dq = S.tdq.p;
        S.Pq.x = S.qx.p; S.Pq.y = S.qy.p; S.Pq.z = S.qz.p; S.Pq.q = S.qq.p; S.Pq.dq = S.qdq.p;
        S.Pq.vx = S.qvx.p; S.Pq.vy = S.qvy.p; S.Pq.vz = S.qvz.p;
        launch_scale_ranges(T.nboxes, S.tv.src0, S.tv.nsrc, S.rule.n, S.qsrc0.p, S.qnsrc.p, s, st);
        S.tv_quad = S.tv;
        S.tv_quad.src0 = S.qsrc0.p;
        S.tv_quad.nsrc = S.qnsrc.p;
    }
    S.ldm = K + (K & 1);
    if (S.tcm2l && (!S.mp32.alloc((size_t)T.nboxes * S.ldm, s, st) || !S.tcerr.alloc(1, s, st))) {
        g_ti.err = cudaGetErrorString(st.err);
        return 16;
    }
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    return 0;
}

// Charge-dependent part: charges into tree order, the eight passes of
// lfmm3dparttargmain (src/lfmm3dpart.f:528-1169) and the scatter back into the
// caller's order.  Stream work only (no host synchronisation, no allocation),
// so a plan captures it in a CUDA graph.
static void lap_passes(LapSetup &S, const double *d_q, const double *d_dq, const double *d_dv, double *d_pot,
                       double *d_fld, double *d_pottarg, double *d_fldtarg, cudaStream_t s, Timer &tm, Status &st)
{
    Tree &T = S.T;
    auto &plan = S.plan;
    const int p = S.p, K = S.K, ns = S.ns, nt = S.nt;
    const TreeView &tv = S.tv;
    const PointsSoA &P = S.P;
    const int prune = S.prune;
    wait_host_inputs(s, st);   // charges still in flight from the host
    if (S.tri) {
        launch_tri_gather(ns, T.perm_src.p, S.tri_in, S.tri_norm, d_q, d_dq, S.ifcharge, S.ifdipole, S.rule, S.ts,
                          S.Pq, s, st);
    } else if (S.ifcharge == 1 || S.ifdipole == 1) {
        k_gather_q<<<div_up(ns, 256), 256, 0, s>>>(ns, T.perm_src.p, d_q, d_dq, d_dv, S.ifcharge == 1,
                                                   S.ifdipole == 1, P); FMM_COUNT_LAUNCH();
    }
    FMM_TRY(st, cudaMemsetAsync(S.mpole.p, 0, sizeof(double2) * S.mpole.n, s));
    FMM_TRY(st, cudaMemsetAsync(S.local.p, 0, sizeof(double2) * S.local.n, s));
    // the outputs collect the near field and then the far field
    for (auto *o : {&S.opot, &S.ofx, &S.ofy, &S.ofz, &S.tpot, &S.tfx, &S.tfy, &S.tfz})
        if (o->n) FMM_TRY(st, cudaMemsetAsync(o->p, 0, sizeof(double2) * o->n, s));
    for (int c = 0; c < 6; c++) {
        if (S.shess[c].n) FMM_TRY(st, cudaMemsetAsync(S.shess[c].p, 0, sizeof(double2) * S.shess[c].n, s));
        if (S.thess[c].n) FMM_TRY(st, cudaMemsetAsync(S.thess[c].p, 0, sizeof(double2) * S.thess[c].n, s));
    }
    const int hsrc = S.ifhess == 1, htrg = S.do_trg && S.ifhesstarg == 1;
    FMM_LAUNCH_CHECK(st);
    tm.mark();
    // The near field (STEP 8) runs on the call's stream while the far-field
    // passes (STEPS 1-5) run on a high-priority side stream; they meet before
    // STEPS 6-7, which add the far field to the outputs.  In the mixed form the
    // two use different units (FP32 CUDA cores, tensor cores).  With the
    // overlap switched off (fmm3d_set_overlap(0)) everything runs on the call's
    // stream, far field first, with the same arithmetic.
    SideStreams &ss = side_streams();
    // fmm3d_set_overlap(0) forces the passes in order (per-pass timing); else the knob decides
    const bool overlap = sw(kSwOverlap) != 0 && S.knobs.overlap != 2;
    const cudaStream_t f = overlap ? ss.far : s;
    if (overlap) {
        FMM_TRY(st, cudaEventRecord(ss.fork, s));
        FMM_TRY(st, cudaStreamWaitEvent(f, ss.fork, 0));
    }
    cudaEvent_t p2p0 = nullptr, p2p1 = nullptr;
    if (tm.on) {
        cudaEventCreate(&p2p0);
        cudaEventCreate(&p2p1);
    }
    auto near_field = [&]() {
        if (tm.on) cudaEventRecord(p2p0, s);
        // STEP 8: P2P over self and list 1 (adds to the outputs)
        const int ppt = S.do_trg ? S.ifpottarg : 0, pft = S.do_trg ? S.iffldtarg : 0;
        if (S.tri)
            launch_p2p_tri(T.leaves.p, T.nleaves, tv, S.ts, S.sx.p, S.sy.p, S.sz.p, S.tx.p, S.ty.p, S.tz.p, S.os, S.ot,
                           S.ifcharge, S.ifdipole, S.do_src, S.do_trg, S.iffld == 1, pft == 1, s, st);
        else if (S.mixed)
            launch_p2p32(T.leaves.p, T.nleaves, S.tv_near, P, S.tx.p, S.ty.p, S.tz.p, S.os, S.ot, S.ifcharge,
                         S.ifdipole, S.ifpot, S.iffld, ppt, pft, S.knobs.p2p_ept, s, st);
        else
            launch_p2p(T.leaves.p, T.nleaves, tv, P, S.tx.p, S.ty.p, S.tz.p, S.os, S.ot, S.ifcharge, S.ifdipole,
                       S.ifpot, S.iffld, ppt, pft, s, st);
        // Hessians of the same near pairs (FP64 in every form)
        launch_p2p_hess(T.leaves.p, T.nleaves, S.mixed ? S.tv_near : tv, P, S.tx.p, S.ty.p, S.tz.p, S.hs, S.ht,
                        S.ifcharge, S.ifdipole, hsrc, htrg, s, st);
        if (tm.on) cudaEventRecord(p2p1, s);
    };
    if (overlap) near_field();
    // STEP 1: P2M at every childless box
    launch_p2m(T.leaves.p, T.nleaves, S.tri ? S.tv_quad : tv, S.tri ? S.Pq : P, S.ifcharge, S.ifdipole, p, S.mpole.p, f,
               st);
    tm.mark_on(f);
    // STEP 3: M2M, levels nlev-1 .. 2
    for (auto &r : S.m2m_rng)
        launch_translate(0, S.dtiles.p + r.first, r.second, T.grouped.p, plan->slots.p, tv, p, plan->rot.p,
                         plan->dc.p, plan->lddc, S.mpole.p, S.mpole.p, prune, S.trans_kt, f, st);
    tm.mark_on(f);
    // STEP 2: P2L from list 4 (every box; boxes with an empty list add nothing)
    launch_p2l(T.grouped.p, T.nboxes, S.tri ? S.tv_quad : S.tv_far, S.tri ? S.Pq : P, S.ifcharge, S.ifdipole, p,
               S.local.p, f, st);
    tm.mark_on(f);
    // STEP 4: M2L over list 2, all levels >= 2
    if (S.tcm2l) {
        FMM_TRY(st, cudaMemsetAsync(S.tcerr.p, 0, sizeof(int), f));
        convert_mp_f32(T.nboxes, K, S.ldm, S.mpole.p, S.mp32.p, f, st);
        const int tcv = S.knobs.tc_variant ? S.knobs.tc_variant - 1 : std::max(sw(kSwTensorM2L) - 1, 0);
        launch_m2l_tc(tcv, S.dtiles.p + S.m2l_a, S.m2l_n, T.grouped.p, plan->slots.p, plan->slot_toff.p,
                      plan->T32.p, tv, p, S.mp32.p, S.ldm, S.local.p, prune, 3, sw(kSwTcGroup), S.tcerr.p, S.m2l_kt, f,
                      st);
    } else if (S.mixed)
        launch_m2l_dense32(S.dtiles.p + S.m2l_a, S.m2l_n, T.grouped.p, plan->slots.p, plan->slot_toff.p,
                           plan->T32.p, tv, p, S.mpole.p, S.local.p, prune, f, st);
    else if (S.dense)
        launch_m2l_dense(S.dtiles.p + S.m2l_a, S.m2l_n, T.grouped.p, plan->slots.p, plan->slot_toff.p, plan->T.p,
                         tv, p, S.mpole.p, S.local.p, prune, S.m2l_kt, f, st);
    else if (sw(kSwM2LMode) != 3 && S.m2l_kt <= 8 && m2l_rot_dmma_supported(p))
        launch_m2l_rot_dmma(S.dtiles.p + S.m2l_a, S.m2l_n, T.grouped.p, plan->slots.p, tv, p, plan->rot.p,
                            plan->dc.p, plan->lddc, S.mpole.p, S.local.p, prune, f, st);
    else
        launch_translate(1, S.dtiles.p + S.m2l_a, S.m2l_n, T.grouped.p, plan->slots.p, tv, p, plan->rot.p,
                         plan->dc.p, plan->lddc, S.mpole.p, S.local.p, prune, S.m2l_kt, f, st);
    tm.mark_on(f);
    // STEP 5: L2L, levels 2 .. nlev-1
    for (auto &r : S.l2l_rng)
        launch_translate(2, S.dtiles.p + r.first, r.second, T.grouped.p, plan->slots.p, tv, p, plan->rot.p,
                         plan->dc.p, plan->lddc, S.local.p, S.local.p, prune, S.trans_kt, f, st);
    tm.mark_on(f);
    if (overlap) {
        FMM_TRY(st, cudaEventRecord(ss.join, f));
        FMM_TRY(st, cudaStreamWaitEvent(s, ss.join, 0));
    } else {
        near_field();
    }
    tm.mark();
    // STEPS 6, 7: M2P from list 3 and L2P (add the far field to the outputs)
    launch_eval(T.leaves.p, T.nleaves, S.ev, S.tv_far, S.sx.p, S.sy.p, S.sz.p, S.tx.p, S.ty.p, S.tz.p, p,
                S.mpole.p, S.local.p, S.os, S.ot, S.do_src, S.do_trg, s, st);
    launch_eval_hess(T.leaves.p, T.nleaves, S.tv_far, S.sx.p, S.sy.p, S.sz.p, S.tx.p, S.ty.p, S.tz.p, p, S.mpole.p,
                     S.local.p, S.hs, S.ht, hsrc, htrg, s, st);
    tm.mark();
    if (tm.on) {
        // intervals: ..., l2l, [wait for the near field], eval, scatter, total ->
        // ..., l2l, eval, p2p (its own events), scatter, total
        tm.fix = [p2p0, p2p1](std::vector<double> &ms) {
            float t = 0;
            cudaEventElapsedTime(&t, p2p0, p2p1);
            cudaEventDestroy(p2p0);
            cudaEventDestroy(p2p1);
            if (ms.size() == 11) ms = {ms[0], ms[1], ms[2], ms[3], ms[4], ms[5], ms[6], ms[8], (double)t, ms[9], ms[10]};
        };
    }
    // unsort into the caller's order
    if (S.do_src) {
        k_scatter_out<<<div_up(ns, 256), 256, 0, s>>>(ns, T.perm_src.p, S.os, S.ifpot == 1 ? d_pot : nullptr,
                                                      S.iffld == 1 ? d_fld : nullptr); FMM_COUNT_LAUNCH();
    }
    if (S.do_trg) {
        k_scatter_out<<<div_up(nt, 256), 256, 0, s>>>(nt, T.perm_trg.p, S.ot, S.ifpottarg == 1 ? d_pottarg : nullptr,
                                                      S.iffldtarg == 1 ? d_fldtarg : nullptr); FMM_COUNT_LAUNCH();
    }
    if (hsrc) launch_scatter_hess(ns, T.perm_src.p, S.hs, S.hess_out, s, st);
    if (htrg) launch_scatter_hess(nt, T.perm_trg.p, S.ht, S.hesstarg_out, s, st);
    FMM_LAUNCH_CHECK(st);
    tm.mark();
}

// tree and interaction statistics of the last call (on request: a few kernels and a device->host read)
static void lap_stats(LapSetup &S, cudaStream_t s, Status &st)
{
    Tree &T = S.T;
    DBuf<unsigned long long> acc;
    acc.alloc(1 + 128, s, st);
    acc.zero(st);
    if (!st.ok()) return;
    k_stats<<<div_up(std::max(T.nleaves, 1), 256), 256, 0, s>>>(T.nleaves, T.leaves.p, S.tv_near, S.do_src,
                                                                S.do_trg, acc.p); FMM_COUNT_LAUNCH();
    for (int l = 2; l <= T.nlev; l++) {
        k_m2l_count<<<div_up(T.lev_count[l], 128), 128, 0, s>>>(T.lev_start[l], T.lev_count[l], S.tv,
                                                               S.plan->slots.p, S.prune, acc.p + 1); FMM_COUNT_LAUNCH();
    }
    std::vector<unsigned long long> h(129);
    FMM_TRY(st, cudaMemcpyAsync(h.data(), acc.p, sizeof(unsigned long long) * 129, cudaMemcpyDeviceToHost, s));
    FMM_TRY(st, cudaStreamSynchronize(s));
    long long m2l = 0;
    for (int i = 0; i < 128; i++) m2l += (long long)h[1 + i];
    g_ti.stats.assign(9 + 128, 0);
    g_ti.stats[0] = T.nboxes; g_ti.stats[1] = T.nlev; g_ti.stats[2] = T.nleaves; g_ti.stats[3] = S.p;
    g_ti.stats[7] = (long long)h[0];
    g_ti.stats[8] = m2l;
    for (int i = 0; i < 128; i++) g_ti.stats[9 + i] = (long long)h[1 + i];
}

// Waits for the stream and turns launch errors and the tensor-core wait flag into ier.
static int lap_finish(LapSetup &S, cudaStream_t s, Status &st)
{
    int herr = 0;
    if (S.tcm2l) FMM_TRY(st, cudaMemcpyAsync(&herr, S.tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = std::string(st.where ? st.where : "") + ": " + cudaGetErrorString(st.err); return 16; }
    if (herr) { g_ti.err = "tensor-core M2L: a wait expired"; return 16; }
    return 0;
}

// ---------------------------------------------------------------- the FMM, one call
// knobs of the last single call on this thread (fmm3d_last_tuning)
thread_local std::string g_last_signature;
thread_local int g_last_knobs[kNumKnobs + 2] = {};

static void lap_effective_knobs(const LapSetup &S, int *out)
{
    out[0] = S.m2l_kt;
    out[1] = S.trans_kt;
    out[2] = S.tcm2l ? (S.knobs.tc_variant ? S.knobs.tc_variant : std::max(sw(kSwTensorM2L), 1)) : 0;
    out[3] = (sw(kSwOverlap) != 0 && S.knobs.overlap != 2) ? 1 : 2;
    out[4] = S.mixed ? (S.knobs.p2p_ept ? S.knobs.p2p_ept : 4) : 0;
    out[5] = lap_form(S);
    out[6] = S.knobs_from_cache ? 1 : 0;
}

static int lap_fmm_device(int iprec, int ns, const double *d_src, int ifcharge, const double *d_q, int ifdipole,
                          const double *d_dq, const double *d_dv, int ifpot, double *d_pot, int iffld,
                          double *d_fld, int nt, const double *d_trg, int ifpottarg, double *d_pottarg,
                          int iffldtarg, double *d_fldtarg, cudaStream_t s, const std::vector<int> *so = nullptr,
                          const std::vector<int> *to = nullptr, int ifhess = 0, double *d_hess = nullptr,
                          int ifhesstarg = 0, double *d_hesstarg = nullptr)
{
    g_launch_count = 0;
    Timer tm(s, g_ti.timing);
    LapSetup S;
    S.ifhess = ifhess == 1 ? 1 : 0;
    S.ifhesstarg = ifhesstarg == 1 ? 1 : 0;
    S.hess_out = d_hess;
    S.hesstarg_out = d_hesstarg;
    int ier = lap_setup(S, iprec, ns, d_src, ifcharge, ifdipole, ifpot, iffld, nt, d_trg, ifpottarg, iffldtarg, s, tm,
                        so, to);
    if (ier) return ier;
    g_last_signature = S.signature;
    lap_effective_knobs(S, g_last_knobs);
    Status st;
    lap_passes(S, d_q, d_dq, d_dv, d_pot, d_fld, d_pottarg, d_fldtarg, s, tm, st);
    tm.finish(g_ti.ms);
    if (g_ti.want_stats && st.ok()) lap_stats(S, s, st);
    return lap_finish(S, s, st);
}

// ---------------------------------------------------------------- triangles, one call
// lfmm3dtriatarg (src/lfmm3dtria.f:121-546): the tree on the centroids and
// targets with the triangle FMM's nbox, then the passes of
// lfmm3dtriatargmain (:547-1160) in the FP64 form.
static int tri_fmm_device(int iprec, int ns, const double *d_tri, const double *d_norm, const double *d_src,
                          int ifcharge, const double *d_q, int ifdipole, const double *d_dq, int ifpot, double *d_pot,
                          int iffld, double *d_fld, int nt, const double *d_trg, int ifpottarg, double *d_pottarg,
                          int iffldtarg, double *d_fldtarg, cudaStream_t s)
{
    g_launch_count = 0;
    Timer tm(s, g_ti.timing);
    LapSetup S;
    S.tri = true;
    S.tri_in = d_tri;
    S.tri_norm = d_norm;
    S.rule = tri_rule(iprec);
    int ier = lap_setup(S, iprec, ns, d_src, ifcharge, ifdipole, ifpot, iffld, nt, d_trg, ifpottarg, iffldtarg, s, tm);
    if (ier) return ier;
    g_last_signature = S.signature;
    lap_effective_knobs(S, g_last_knobs);
    Status st;
    lap_passes(S, d_q, d_dq, nullptr, d_pot, d_fld, d_pottarg, d_fldtarg, s, tm, st);
    tm.finish(g_ti.ms);
    if (g_ti.want_stats && st.ok()) lap_stats(S, s, st);
    return lap_finish(S, s, st);
}

// l3dtriadirect (src/lfmm3dtria.f:1385-1560): every triangle at every
// centroid (its own by the in-plane values) and target.
static int tri_direct_device(int ns, const double *d_tri, const double *d_src, int ifcharge, const double *d_q,
                             int ifdipole, const double *d_dq, int ifpot, double *d_pot, int iffld, double *d_fld,
                             int nt, const double *d_trg, int ifpottarg, double *d_pottarg, int iffldtarg,
                             double *d_fldtarg, cudaStream_t s)
{
    g_launch_count = 0;
    Status st;
    if (ns < 0 || nt < 0) return 4;
    DBuf<double> geo;
    DBuf<double2> q, dq;
    TriRule none;   // no quadrature nodes: the direct sum uses the exact integrals only
    bool ok = geo.alloc(30L * std::max(ns, 1), s, st);
    if (ifcharge == 1) ok = ok && q.alloc(std::max(ns, 1), s, st);
    if (ifdipole == 1) ok = ok && dq.alloc(std::max(ns, 1), s, st);
    if (!ok) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    TriSoA t;
    t.geo = geo.p; t.q = q.p; t.dq = dq.p;
    launch_tri_gather(ns, nullptr, d_tri, nullptr, d_q, d_dq, ifcharge, ifdipole, none, t, PointsSoA(), s, st);
    auto run = [&](int npts, const double *pts, int centroids, int wp, double *op, int wf, double *of) {
        if (!(wp == 1 || wf == 1) || npts <= 0) return;
        launch_tri_direct(ns, t, ifcharge, ifdipole, npts, pts, centroids, nullptr, wp == 1 ? op : nullptr,
                          wf == 1 ? of : nullptr, s, st);
    };
    run(ns, d_src, 1, ifpot, d_pot, iffld, d_fld);
    run(nt, d_trg, 0, ifpottarg, d_pottarg, iffldtarg, d_fldtarg);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = std::string(st.where ? st.where : "") + ": " + cudaGetErrorString(st.err); return 16; }
    return 0;
}

// ---------------------------------------------------------------- plans: fixed geometry, new charges
// A plan keeps one evaluation geometry on the device (tree, lists, sorted
// coordinates, workspace) and runs the charge-dependent passes for any number
// of charge vectors.  The passes are captured once per set of caller pointers
// and stream into a CUDA graph and replayed (one launch instead of ~150).
// Tree queries mirror d3tgetb / d3tgetl (src/d3tstrcr.f:576-665).
struct LapPlanExec {
    LapSetup S;
    std::mutex mu;
    cudaStream_t made_on = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void *key[8] = {};
    int key_cfg = -1;          // the overlap and tensor-core switches when the graph was captured
    int graph_launches = 0;
    std::vector<cudaStream_t> used;
    // host copy of the tree for the queries (filled on first use)
    bool host = false;
    std::vector<int> level, ijk, parent, child, src0, nsrc, trg0, ntrg, coll;
    std::vector<int> lst[6], lidx[6];   // CSR of lists 1, 3, 4 (index = list type)
    std::vector<double> center, geom;   // geom: 4 per instance (centre, side)
    std::vector<int> binst;
};

static void plan_host_tree(LapPlanExec &E, Status &st)
{
    if (E.host) return;
    Tree &T = E.S.T;
    const int nb = T.nboxes;
    auto get = [&](std::vector<int> &h, const DBuf<int> &d, size_t n) {
        h.resize(n);
        if (n) FMM_TRY(st, cudaMemcpy(h.data(), d.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    };
    get(E.level, T.level, nb); get(E.ijk, T.ijk, 3L * nb); get(E.parent, T.parent, nb); get(E.child, T.child, 8L * nb);
    get(E.src0, T.src0, nb); get(E.nsrc, T.nsrc, nb); get(E.trg0, T.trg0, nb); get(E.ntrg, T.ntrg, nb);
    get(E.coll, T.coll, 27L * nb);
    const DBuf<int> *cs[6] = {nullptr, &T.l1_start, nullptr, &T.l3_start, &T.l4_start, nullptr};
    const DBuf<int> *ci[6] = {nullptr, &T.l1_idx, nullptr, &T.l3_idx, &T.l4_idx, nullptr};
    for (int ty : {1, 3, 4}) {
        get(E.lst[ty], *cs[ty], nb + 1);
        get(E.lidx[ty], *ci[ty], st.ok() && nb ? (size_t)E.lst[ty][nb] : 0);
    }
    E.center.resize(3L * nb);
    if (nb) FMM_TRY(st, cudaMemcpy(E.center.data(), T.center.p, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost));
    if (T.ninst > 1) {
        get(E.binst, T.binst, nb);
        E.geom.resize(4L * T.ninst);
        FMM_TRY(st, cudaMemcpy(E.geom.data(), T.inst_geom.p, sizeof(double) * 4 * T.ninst, cudaMemcpyDeviceToHost));
    }
    E.host = st.ok();
}

}  // namespace fmm

using namespace fmm;

extern "C" {

int fmm3d_lfmm3d_plan_create(int iprec, int nsource, const double *d_source, int ifcharge, int ifdipole, int ifpot,
                             int iffld, int ntarget, const double *d_target, int ifpottarg, int iffldtarg,
                             void *stream, void **plan)
{
    if (!plan) return 1;
    *plan = nullptr;
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    g_launch_count = 0;
    auto *E = new LapPlanExec;
    Timer tm(s, false);
    int ier = lap_setup(E->S, iprec, nsource, d_source, ifcharge, ifdipole, ifpot, iffld, ntarget, d_target,
                        ifpottarg, iffldtarg, s, tm);
    Status st;
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!ier && !st.ok()) { g_ti.err = cudaGetErrorString(st.err); ier = 16; }
    if (ier) {
        delete E;
        return ier;
    }
    E->made_on = s;
    E->used.push_back(s);
    *plan = E;
    return 0;
}

// d3tstrcrem (src/d3tstrcr.f:264-460): the tree alone, for the tree queries
// (fmm3d_lfmm3d_plan_getb / _getl / _info; _destroy frees it).  Device arrays
// as for fmm3d_lfmm3d_plan_create.  ier 128 when nsource < 1 (as the
// reference); levels are capped at 21.  ier 4 for nbox < 1, and for box counts
// beyond 32-bit indexing: empty boxes kept above minlevel make 8^minlevel
// boxes (minlevel <= 7 then), and every level down to minlevel holds up to
// one box per point.
int fmm3d_d3tstrcrem(int nsource, const double *d_source, int nbox, int ntarget, const double *d_target,
                     int ifempty, int minlevel, int maxlevel, void *stream, void **tree)
{
    if (!tree) return 1;
    *tree = nullptr;
    if (nsource < 1) return 128;
    const int lmin = std::max(0, std::min(minlevel, maxlevel));
    if (nbox < 1 || ntarget < 0) return 4;
    if (ifempty == 1 && lmin > 7) return 4;
    if (((long)nsource + ntarget) * (std::min(lmin, kMaxLevel) + 1) > (1L << 30)) return 4;
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    g_launch_count = 0;
    keep_pool_memory();
    auto *E = new LapPlanExec;
    E->S.ns = nsource;
    E->S.nt = ntarget;
    TreeOptions opt;
    opt.ifempty = ifempty;
    opt.minlevel = minlevel;
    opt.maxlevel = maxlevel;
    Status st;
    build_tree(E->S.T, d_source, nsource, d_target, ntarget, nbox, s, st, opt);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) {
        g_ti.err = cudaGetErrorString(st.err);
        delete E;
        return 16;
    }
    E->made_on = s;
    E->used.push_back(s);
    *tree = E;
    return 0;
}

int fmm3d_lfmm3d_plan_create_batched(int iprec, int ninst, const int *src_offsets, const double *d_source,
                                     int ifcharge, int ifdipole, int ifpot, int iffld, const int *trg_offsets,
                                     const double *d_target, int ifpottarg, int iffldtarg, void *stream, void **plan)
{
    if (!plan) return 1;
    *plan = nullptr;
    if (ninst < 1 || !src_offsets || src_offsets[0] != 0) return 4;
    std::vector<int> so(src_offsets, src_offsets + ninst + 1), to(ninst + 1, 0);
    if (trg_offsets) to.assign(trg_offsets, trg_offsets + ninst + 1);
    for (int i = 0; i < ninst; i++)
        if (so[i + 1] < so[i] || to[i + 1] < to[i] || to[0] != 0) return 4;
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    g_launch_count = 0;
    auto *E = new LapPlanExec;
    Timer tm(s, false);
    int ier = lap_setup(E->S, iprec, so[ninst], d_source, ifcharge, ifdipole, ifpot, iffld, to[ninst], d_target,
                        ifpottarg, iffldtarg, s, tm, &so, &to);
    Status st;
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!ier && !st.ok()) { g_ti.err = cudaGetErrorString(st.err); ier = 16; }
    if (ier) {
        delete E;
        return ier;
    }
    E->made_on = s;
    E->used.push_back(s);
    *plan = E;
    return 0;
}

int fmm3d_lfmm3d_plan_execute(void *plan, const double *d_charge, const double *d_dipstr, const double *d_dipvec,
                              double *d_pot, double *d_fld, double *d_pottarg, double *d_fldtarg, int use_graph,
                              void *stream)
{
    if (!plan) return 1;
    auto *E = (LapPlanExec *)plan;
    if (!E->S.plan) return 4;   // a tree from fmm3d_d3tstrcrem: no FMM on it
    std::lock_guard<std::mutex> lk(E->mu);
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    if (std::find(E->used.begin(), E->used.end(), s) == E->used.end()) {
        // the plan's buffers were made on another stream: order this one after it
        cudaStreamSynchronize(E->made_on);
        E->used.push_back(s);
    }
    Status st;
    g_launch_count = 0;
    if (use_graph) {
        const void *key[8] = {d_charge, d_dipstr, d_dipvec, d_pot, d_fld, d_pottarg, d_fldtarg, (const void *)s};
        const int cfg = sw(kSwOverlap) * 16 + sw(kSwTensorM2L);
        if (!E->exec || memcmp(key, E->key, sizeof key) != 0 || E->key_cfg != cfg) {
            if (E->exec) cudaGraphExecDestroy(E->exec);
            E->exec = nullptr;
            cudaGraph_t g = nullptr;
            Timer off(s, false);
            FMM_TRY(st, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            if (st.ok()) lap_passes(E->S, d_charge, d_dipstr, d_dipvec, d_pot, d_fld, d_pottarg, d_fldtarg, s, off, st);
            cudaError_t ce = cudaStreamEndCapture(s, &g);
            if (st.ok() && ce != cudaSuccess) { st.err = ce; st.where = "cudaStreamEndCapture"; }
            if (st.ok()) FMM_TRY(st, cudaGraphInstantiate(&E->exec, g, 0));
            if (g) cudaGraphDestroy(g);
            if (!st.ok()) {
                E->exec = nullptr;
                g_ti.err = std::string("graph capture: ") + cudaGetErrorString(st.err);
                return 16;
            }
            memcpy(E->key, key, sizeof key);
            E->key_cfg = cfg;
            E->graph_launches = g_launch_count;
        }
        FMM_TRY(st, cudaGraphLaunch(E->exec, s));
        g_launch_count = E->graph_launches;
        g_ti.ms.clear();
    } else {
        Timer tm(s, g_ti.timing);
        tm.mark();
        tm.mark();   // no tree work in an execute: the "tree" interval is empty
        lap_passes(E->S, d_charge, d_dipstr, d_dipvec, d_pot, d_fld, d_pottarg, d_fldtarg, s, tm, st);
        tm.finish(g_ti.ms);
    }
    return lap_finish(E->S, s, st);
}

int fmm3d_lfmm3d_plan_destroy(void *plan)
{
    if (!plan) return 0;
    auto *E = (LapPlanExec *)plan;
    {
        std::lock_guard<std::mutex> lk(E->mu);
        for (auto s : E->used) cudaStreamSynchronize(s);
        if (E->exec) cudaGraphExecDestroy(E->exec);
        E->exec = nullptr;
    }
    delete E;
    return 0;
}

int fmm3d_lfmm3d_plan_set_tuning(void *plan, const int *knobs, int n)
{
    if (!plan || !knobs || n < kNumKnobs) return 1;
    auto *E = (LapPlanExec *)plan;
    if (!E->S.plan) return 4;   // a tree from fmm3d_d3tstrcrem: no FMM on it
    std::lock_guard<std::mutex> lk(E->mu);
    for (int i = 0; i < kNumKnobs; i++)
        if (knobs[i] < 0) return 2;
    // the tiles may be in use by work in flight, and a captured graph holds them
    for (auto s : E->used) cudaStreamSynchronize(s);
    if (E->exec) cudaGraphExecDestroy(E->exec);
    E->exec = nullptr;
    Status st;
    const TuneKnobs old = E->S.knobs;
    int ier = lap_tiles(E->S, knobs_from_array(knobs), E->made_on, st);
    if (ier == 0) E->S.knobs_from_cache = false;
    else if (ier == 2) lap_tiles(E->S, old, E->made_on, st);
    FMM_TRY(st, cudaStreamSynchronize(E->made_on));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    return ier;
}

// out[0..4] = knobs in use (m2l_kt, trans_kt, tc_variant, overlap, p2p_ept; 0 = not
// applicable to this form), out[5] = form, out[6] = 1 if they came from the cache
int fmm3d_lfmm3d_plan_get_tuning(void *plan, int *out, int n)
{
    if (!plan || !out || n < kNumKnobs + 2) return 1;
    auto *E = (LapPlanExec *)plan;
    if (!E->S.plan) return 4;   // a tree from fmm3d_d3tstrcrem: no FMM on it
    std::lock_guard<std::mutex> lk(E->mu);
    lap_effective_knobs(E->S, out);
    return 0;
}

int fmm3d_lfmm3d_plan_signature(void *plan, char *buf, int n)
{
    if (!plan) return -1;
    auto *E = (LapPlanExec *)plan;
    if (!E->S.plan) return 4;   // a tree from fmm3d_d3tstrcrem: no FMM on it
    std::lock_guard<std::mutex> lk(E->mu);
    const std::string &sg = E->S.signature;
    if (!buf || n <= 0) return (int)sg.size() + 1;
    snprintf(buf, (size_t)n, "%s", sg.c_str());
    return (int)sg.size() + 1 <= n ? 0 : (int)sg.size() + 1;
}

// the knobs (as fmm3d_lfmm3d_plan_get_tuning) and signature of this thread's last single Laplace call
int fmm3d_last_tuning(int *out, int n, char *sig, int nsig)
{
    if (out && n >= kNumKnobs + 2) memcpy(out, g_last_knobs, sizeof(int) * (kNumKnobs + 2));
    if (sig && nsig > 0) snprintf(sig, (size_t)nsig, "%s", g_last_signature.c_str());
    return (int)g_last_signature.size() + 1;
}

// out[0..9] = nboxes, nlev, nleaves, nterms, nsource, ntarget, centre x, y, z, side of the root cube
// (of the first instance for a batch)
int fmm3d_lfmm3d_plan_info(void *plan, double *out, int n)
{
    if (!plan || !out) return 1;
    auto *E = (LapPlanExec *)plan;
    Tree &T = E->S.T;
    const double v[10] = {(double)T.nboxes, (double)T.nlev, (double)T.nleaves, (double)E->S.p, (double)E->S.ns,
                          (double)E->S.nt, T.center0[0], T.center0[1], T.center0[2], T.size};
    for (int i = 0; i < n && i < 10; i++) out[i] = v[i];
    return 0;
}

// d3tgetb: box(20), centre(3) and corners(3,8) of box ibox (1-based).  ier 2 for a bad ibox.
int fmm3d_lfmm3d_plan_getb(void *plan, int ibox, int *box, double *center, double *corners)
{
    if (!plan) return 1;
    auto *E = (LapPlanExec *)plan;
    std::lock_guard<std::mutex> lk(E->mu);
    Status st;
    plan_host_tree(*E, st);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    const int nb = E->S.T.nboxes;
    if (ibox < 1 || ibox > nb) return 2;
    const int b = ibox - 1;
    if (box) {
        int nk = 0;
        box[0] = E->level[b];
        for (int k = 0; k < 3; k++) box[1 + k] = E->ijk[3L * b + k] + 1;
        box[4] = E->parent[b] + 1;
        for (int k = 0; k < 8; k++) box[5 + k] = 0;
        for (int k = 0; k < 8; k++)
            if (E->child[8L * b + k] >= 0) box[5 + nk++] = E->child[8L * b + k] + 1;
        box[13] = E->src0[b] + 1;
        box[14] = E->nsrc[b];
        box[15] = E->trg0[b] + 1;
        box[16] = E->ntrg[b];
        // type 2 only for a box split because it held more than nbox points
        // (a box split to reach minlevel stays 1, src/d3tstrcr.f:1490-1498)
        const bool over = nk > 0 && (E->nsrc[b] > E->S.T.nbox || E->ntrg[b] > E->S.T.nbox);
        box[17] = E->nsrc[b] == 0 ? 0 : (over ? 2 : 1);
        box[18] = E->ntrg[b] == 0 ? 0 : (over ? 2 : 1);
        box[19] = 0;
    }
    const double side = (E->binst.empty() ? E->S.T.size : E->geom[4L * E->binst[b] + 3]) / (double)(1L << E->level[b]);
    const double *c = &E->center[3L * b];
    if (center)
        for (int k = 0; k < 3; k++) center[k] = c[k];
    if (corners)
        for (int q = 0; q < 8; q++) {
            corners[3 * q] = c[0] + ((q >> 2) ? 0.5 : -0.5) * side;
            corners[3 * q + 1] = c[1] + (((q >> 1) & 1) ? 0.5 : -0.5) * side;
            corners[3 * q + 2] = c[2] + ((q & 1) ? 0.5 : -0.5) * side;
        }
    return 0;
}

// d3tgetl: list itype (1..5) of box ibox (1-based boxes in list[]); ier 4 when
// the list is empty, 2 for a bad ibox or itype.  list must hold the list
// (lists 2 and 5 at most 189 and 26 boxes; fmm3d_lfmm3d_plan_getl with
// list = NULL returns the length in *nlist).
int fmm3d_lfmm3d_plan_getl(void *plan, int ibox, int itype, int *list, int *nlist)
{
    if (!plan || !nlist) return 1;
    auto *E = (LapPlanExec *)plan;
    std::lock_guard<std::mutex> lk(E->mu);
    Status st;
    plan_host_tree(*E, st);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    const int nb = E->S.T.nboxes;
    *nlist = 0;
    if (ibox < 1 || ibox > nb || itype < 1 || itype > 5) return 2;
    const int b = ibox - 1;
    std::vector<int> out;
    if (itype == 1 || itype == 3 || itype == 4) {
        for (int k = E->lst[itype][b]; k < E->lst[itype][b + 1]; k++) out.push_back(E->lidx[itype][k]);
    } else if (itype == 5) {
        for (int k = 0; k < 27; k++)
            if (k != 13 && E->coll[27L * b + k] >= 0) out.push_back(E->coll[27L * b + k]);
    } else {
        // list 2: children of the parent's colleagues that do not touch b
        const int P = E->parent[b];
        if (P >= 0)
            for (int k = 0; k < 27; k++) {
                const int C = E->coll[27L * P + k];
                if (C < 0) continue;
                for (int o = 0; o < 8; o++) {
                    const int c = E->child[8L * C + o];
                    if (c < 0 || c == b) continue;
                    bool touch = true;
                    for (int d = 0; d < 3; d++) touch = touch && std::abs(E->ijk[3L * c + d] - E->ijk[3L * b + d]) <= 1;
                    if (!touch) out.push_back(c);
                }
            }
    }
    *nlist = (int)out.size();
    if (list)
        for (size_t i = 0; i < out.size(); i++) list[i] = out[i] + 1;
    return out.empty() ? 4 : 0;
}

}  // extern "C"

namespace fmm {

static int lap_direct_device(int ns, const double *d_src, int ifcharge, const double *d_q, int ifdipole,
                             const double *d_dq, const double *d_dv, int ifpot, double *d_pot, int iffld,
                             double *d_fld, int nt, const double *d_trg, int ifpottarg, double *d_pottarg,
                             int iffldtarg, double *d_fldtarg, cudaStream_t s)
{
    Status st;
    DBuf<double> sx, sy, sz, vx, vy, vz, tx, ty, tz;
    DBuf<double2> q, dq, o0, o1, o2, o3;
    bool ok = sx.alloc(ns, s, st) && sy.alloc(ns, s, st) && sz.alloc(ns, s, st);
    if (ifcharge == 1) ok = ok && q.alloc(ns, s, st);
    if (ifdipole == 1) ok = ok && dq.alloc(ns, s, st) && vx.alloc(ns, s, st) && vy.alloc(ns, s, st) && vz.alloc(ns, s, st);
    int ne = std::max(ns, nt);
    ok = ok && o0.alloc(ne, s, st) && o1.alloc(ne, s, st) && o2.alloc(ne, s, st) && o3.alloc(ne, s, st);
    if (nt > 0) ok = ok && tx.alloc(nt, s, st) && ty.alloc(nt, s, st) && tz.alloc(nt, s, st);
    if (!ok) return 8;
    k_split_aos<<<div_up(ns, 256), 256, 0, s>>>(ns, d_src, sx.p, sy.p, sz.p); FMM_COUNT_LAUNCH();
    if (ifcharge == 1) { k_split_c<<<div_up(ns, 256), 256, 0, s>>>(ns, d_q, q.p); FMM_COUNT_LAUNCH(); }
    if (ifdipole == 1) {
        k_split_c<<<div_up(ns, 256), 256, 0, s>>>(ns, d_dq, dq.p); FMM_COUNT_LAUNCH();
        k_split_aos<<<div_up(ns, 256), 256, 0, s>>>(ns, d_dv, vx.p, vy.p, vz.p); FMM_COUNT_LAUNCH();
    }
    OutSoA o;
    o.pot = o0.p; o.fx = o1.p; o.fy = o2.p; o.fz = o3.p;
    if (ifpot == 1 || iffld == 1) {
        launch_direct(ns, sx.p, sy.p, sz.p, q.p, dq.p, vx.p, vy.p, vz.p, ifcharge, ifdipole, ns, sx.p, sy.p, sz.p,
                      nullptr, 1, o, s, st);
        k_scatter_out<<<div_up(ns, 256), 256, 0, s>>>(ns, nullptr, o, ifpot == 1 ? d_pot : nullptr,
                                                      iffld == 1 ? d_fld : nullptr); FMM_COUNT_LAUNCH();
    }
    if (nt > 0 && (ifpottarg == 1 || iffldtarg == 1)) {
        k_split_aos<<<div_up(nt, 256), 256, 0, s>>>(nt, d_trg, tx.p, ty.p, tz.p); FMM_COUNT_LAUNCH();
        launch_direct(ns, sx.p, sy.p, sz.p, q.p, dq.p, vx.p, vy.p, vz.p, ifcharge, ifdipole, nt, tx.p, ty.p, tz.p,
                      nullptr, 0, o, s, st);
        k_scatter_out<<<div_up(nt, 256), 256, 0, s>>>(nt, nullptr, o, ifpottarg == 1 ? d_pottarg : nullptr,
                                                      iffldtarg == 1 ? d_fldtarg : nullptr); FMM_COUNT_LAUNCH();
    }
    FMM_LAUNCH_CHECK(st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    return 0;
}

}  // namespace fmm

using namespace fmm;

extern "C" {

int fmm3d_lfmm3dparttarg_device(int iprec, int nsource, const double *d_source, int ifcharge, const double *d_charge,
                                int ifdipole, const double *d_dipstr, const double *d_dipvec, int ifpot,
                                double *d_pot, int iffld, double *d_fld, int ntarget, const double *d_target,
                                int ifpottarg, double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return lap_fmm_device(iprec, nsource, d_source, ifcharge, d_charge, ifdipole, d_dipstr, d_dipvec, ifpot, d_pot,
                          iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg, iffldtarg, d_fldtarg, s);
}

int fmm3d_lfmm3dparttarg_hess_device(int iprec, int nsource, const double *d_source, int ifcharge,
                                     const double *d_charge, int ifdipole, const double *d_dipstr,
                                     const double *d_dipvec, int ifpot, double *d_pot, int iffld, double *d_fld,
                                     int ifhess, double *d_hess, int ntarget, const double *d_target, int ifpottarg,
                                     double *d_pottarg, int iffldtarg, double *d_fldtarg, int ifhesstarg,
                                     double *d_hesstarg, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return lap_fmm_device(iprec, nsource, d_source, ifcharge, d_charge, ifdipole, d_dipstr, d_dipvec, ifpot, d_pot,
                          iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg, iffldtarg, d_fldtarg, s, nullptr,
                          nullptr, ifhess, d_hess, ifhesstarg, d_hesstarg);
}

int fmm3d_l3dtaevalhess_device(double rscale, const double *center, const double *d_local, int nterms, int npts,
                               const double *d_targ, double *d_pot, int iffld, double *d_fld, int ifhess,
                               double *d_hess, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    Status st;
    g_launch_count = 0;
    launch_expeval_hess(true, rscale, center, d_local, nterms, npts, d_targ, d_pot, iffld, d_fld, ifhess, d_hess, s,
                        st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = std::string(st.where ? st.where : "") + ": " + cudaGetErrorString(st.err); return 16; }
    return 0;
}

int fmm3d_l3dmpevalhess_device(double rscale, const double *center, const double *d_mpole, int nterms, int npts,
                               const double *d_targ, double *d_pot, int iffld, double *d_fld, int ifhess,
                               double *d_hess, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    Status st;
    g_launch_count = 0;
    launch_expeval_hess(false, rscale, center, d_mpole, nterms, npts, d_targ, d_pot, iffld, d_fld, ifhess, d_hess, s,
                        st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = std::string(st.where ? st.where : "") + ": " + cudaGetErrorString(st.err); return 16; }
    return 0;
}

int fmm3d_lfmm3dtriatarg_device(int iprec, int nsource, const double *d_triaflat, const double *d_trianorm,
                                const double *d_source, int ifcharge, const double *d_charge, int ifdipole,
                                const double *d_dipstr, const double *d_dipvec, int ifpot, double *d_pot, int iffld,
                                double *d_fld, int ntarget, const double *d_target, int ifpottarg, double *d_pottarg,
                                int iffldtarg, double *d_fldtarg, void *stream)
{
    (void)d_dipvec;   // as in the reference, the dipoles are oriented by the triangles' normals
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return tri_fmm_device(iprec, nsource, d_triaflat, d_trianorm, d_source, ifcharge, d_charge, ifdipole, d_dipstr,
                          ifpot, d_pot, iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg, iffldtarg, d_fldtarg, s);
}

int fmm3d_l3dtriadirect_device(int nsource, const double *d_triaflat, const double *d_trianorm,
                               const double *d_source, int ifcharge, const double *d_charge, int ifdipole,
                               const double *d_dipstr, const double *d_dipvec, int ifpot, double *d_pot, int iffld,
                               double *d_fld, int ntarget, const double *d_target, int ifpottarg, double *d_pottarg,
                               int iffldtarg, double *d_fldtarg, void *stream)
{
    (void)d_trianorm;
    (void)d_dipvec;
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return tri_direct_device(nsource, d_triaflat, d_source, ifcharge, d_charge, ifdipole, d_dipstr, ifpot, d_pot,
                             iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg, iffldtarg, d_fldtarg, s);
}

int fmm3d_l3dtriadirect_points_device(int nsource, const double *d_triaflat, int ifcharge, const double *d_charge,
                                      int ifdipole, const double *d_dipstr, int npts, const double *d_pts,
                                      const int *d_self, double *d_pot, double *d_fld, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    g_launch_count = 0;
    Status st;
    DBuf<double> geo;
    DBuf<double2> q, dq;
    TriRule none;
    bool ok = geo.alloc(30L * std::max(nsource, 1), s, st);
    if (ifcharge == 1) ok = ok && q.alloc(std::max(nsource, 1), s, st);
    if (ifdipole == 1) ok = ok && dq.alloc(std::max(nsource, 1), s, st);
    if (!ok) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    TriSoA t;
    t.geo = geo.p; t.q = q.p; t.dq = dq.p;
    launch_tri_gather(nsource, nullptr, d_triaflat, nullptr, d_charge, d_dipstr, ifcharge, ifdipole, none, t,
                      PointsSoA(), s, st);
    launch_tri_direct(nsource, t, ifcharge, ifdipole, npts, d_pts, 0, d_self, d_pot, d_fld, s, st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = std::string(st.where ? st.where : "") + ": " + cudaGetErrorString(st.err); return 16; }
    return 0;
}

int fmm3d_l3dpartdirect_device(int nsource, const double *d_source, int ifcharge, const double *d_charge,
                               int ifdipole, const double *d_dipstr, const double *d_dipvec, int ifpot,
                               double *d_pot, int iffld, double *d_fld, int ntarget, const double *d_target,
                               int ifpottarg, double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return lap_direct_device(nsource, d_source, ifcharge, d_charge, ifdipole, d_dipstr, d_dipvec, ifpot, d_pot,
                             iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg, iffldtarg, d_fldtarg, s);
}

int fmm3d_l3ddirect_points_device(int nsource, const double *d_source, int ifcharge, const double *d_charge,
                                  int ifdipole, const double *d_dipstr, const double *d_dipvec, int npts,
                                  const double *d_pts, const int *d_skip, double *d_pot, double *d_fld,
                                  void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    Status st;
    int ns = nsource;
    DBuf<double> sx, sy, sz, vx, vy, vz, px, py, pz;
    DBuf<double2> q, dq, o0, o1, o2, o3;
    bool ok = sx.alloc(ns, s, st) && sy.alloc(ns, s, st) && sz.alloc(ns, s, st) && px.alloc(npts, s, st) &&
              py.alloc(npts, s, st) && pz.alloc(npts, s, st) && o0.alloc(npts, s, st) && o1.alloc(npts, s, st) &&
              o2.alloc(npts, s, st) && o3.alloc(npts, s, st);
    if (ifcharge == 1) ok = ok && q.alloc(ns, s, st);
    if (ifdipole == 1) ok = ok && dq.alloc(ns, s, st) && vx.alloc(ns, s, st) && vy.alloc(ns, s, st) && vz.alloc(ns, s, st);
    if (!ok) return 8;
    k_split_aos<<<div_up(ns, 256), 256, 0, s>>>(ns, d_source, sx.p, sy.p, sz.p); FMM_COUNT_LAUNCH();
    k_split_aos<<<div_up(npts, 256), 256, 0, s>>>(npts, d_pts, px.p, py.p, pz.p); FMM_COUNT_LAUNCH();
    if (ifcharge == 1) { k_split_c<<<div_up(ns, 256), 256, 0, s>>>(ns, d_charge, q.p); FMM_COUNT_LAUNCH(); }
    if (ifdipole == 1) {
        k_split_c<<<div_up(ns, 256), 256, 0, s>>>(ns, d_dipstr, dq.p); FMM_COUNT_LAUNCH();
        k_split_aos<<<div_up(ns, 256), 256, 0, s>>>(ns, d_dipvec, vx.p, vy.p, vz.p); FMM_COUNT_LAUNCH();
    }
    OutSoA o;
    o.pot = o0.p; o.fx = o1.p; o.fy = o2.p; o.fz = o3.p;
    launch_direct_split(ns, sx.p, sy.p, sz.p, q.p, dq.p, vx.p, vy.p, vz.p, ifcharge, ifdipole, npts, px.p, py.p,
                        pz.p, d_skip, o, s, st);
    k_scatter_out<<<div_up(npts, 256), 256, 0, s>>>(npts, nullptr, o, d_pot, d_fld); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    return 0;
}

int fmm3d_lfmm3dparttarg_batched_device(int iprec, int ninst, const int *src_offsets, const double *d_source,
                                        int ifcharge, const double *d_charge, int ifdipole, const double *d_dipstr,
                                        const double *d_dipvec, int ifpot, double *d_pot, int iffld, double *d_fld,
                                        const int *trg_offsets, const double *d_target, int ifpottarg,
                                        double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream)
{
    if (ninst < 1 || !src_offsets) return 4;
    std::vector<int> so(src_offsets, src_offsets + ninst + 1), to(ninst + 1, 0);
    if (trg_offsets) to.assign(trg_offsets, trg_offsets + ninst + 1);
    for (int i = 0; i < ninst; i++)
        if (so[i + 1] < so[i] || to[i + 1] < to[i] || so[i] < 0 || to[i] < 0) return 4;
    if (so[0] != 0 || to[0] != 0) return 4;
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return lap_fmm_device(iprec, so[ninst], d_source, ifcharge, d_charge, ifdipole, d_dipstr, d_dipvec, ifpot, d_pot,
                          iffld, d_fld, to[ninst], d_target, ifpottarg, d_pottarg, iffldtarg, d_fldtarg, s, &so, &to);
}

void lfmm3dparttarg_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                     const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                     const int *ifpot, double *pot, const int *iffld, double *fld, const int *ntarget,
                     const double *target, const int *ifpottarg, double *pottarg, const int *iffldtarg,
                     double *fldtarg)
{
    int ns = *nsource, nt = *ntarget, ip = *iprec;
    *ier = with_device_arrays(
        ns, source, *ifcharge, charge, *ifdipole, dipstr, dipvec, *ifpot, pot, *iffld, fld, nt, target, *ifpottarg,
        pottarg, *iffldtarg, fldtarg,
        [&](const double *s_, const double *q, const double *dq, const double *dv, double *po, double *fo,
            const double *t_, double *pt, double *ft, cudaStream_t s) {
            return lap_fmm_device(ip, ns, s_, *ifcharge, q, *ifdipole, dq, dv, *ifpot, po, *iffld, fo, nt, t_,
                                  *ifpottarg, pt, *iffldtarg, ft, s);
        },
        true);
}

void lfmm3dtriatarg_(int *ier, const int *iprec, const int *nsource, const double *triaflat, const double *trianorm,
                     const double *source, const int *ifcharge, const double *charge, const int *ifdipole,
                     const double *dipstr, const double *dipvec, const int *ifpot, double *pot, const int *iffld,
                     double *fld, const int *ntarget, const double *target, const int *ifpottarg, double *pottarg,
                     const int *iffldtarg, double *fldtarg)
{
    (void)dipvec;
    const int ip = *iprec, ns = *nsource, ifc = *ifcharge, ifd = *ifdipole, ifp = *ifpot, iff = *iffld;
    *ier = tri_host(ns, triaflat, trianorm, source, ifc, charge, ifd, dipstr, ifp, pot, iff, fld, *ntarget, target,
                    *ifpottarg, pottarg, *iffldtarg, fldtarg,
                    [&](const double *t_, const double *n_, const double *s_, const double *q, const double *dq,
                        double *po, double *fo, int nt, const double *tg, int ipt, double *pt, int ift, double *ft,
                        cudaStream_t s) {
                        return tri_fmm_device(ip, ns, t_, n_, s_, ifc, q, ifd, dq, ifp, po, iff, fo, nt, tg, ipt, pt,
                                              ift, ft, s);
                    });
}

void lfmm3dtriaself_(int *ier, const int *iprec, const int *nsource, const double *triaflat, const double *trianorm,
                     const double *source, const int *ifcharge, const double *charge, const int *ifdipole,
                     const double *dipstr, const double *dipvec, const int *ifpot, double *pot, const int *iffld,
                     double *fld)
{
    int zero = 0;
    lfmm3dtriatarg_(ier, iprec, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot,
                    pot, iffld, fld, &zero, source, &zero, nullptr, &zero, nullptr);
}

void lfmm3dtria_(int *ier, const int *iprec, const int *nsource, const double *triaflat, const double *trianorm,
                 const double *source, const int *ifcharge, const double *charge, const int *ifdipole,
                 const double *dipstr, const double *dipvec, const int *ifpot, double *pot, const int *iffld,
                 double *fld)
{
    lfmm3dtriaself_(ier, iprec, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot,
                    pot, iffld, fld);
}

void l3dtriadirect_(const int *nsource, const double *triaflat, const double *trianorm, const double *source,
                    const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                    const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld,
                    const int *ntarget, const double *target, const int *ifpottarg, double *pottarg,
                    const int *iffldtarg, double *fldtarg)
{
    (void)trianorm;
    (void)dipvec;
    const int ns = *nsource, ifc = *ifcharge, ifd = *ifdipole, ifp = *ifpot, iff = *iffld;
    tri_host(ns, triaflat, nullptr, source, ifc, charge, ifd, dipstr, ifp, pot, iff, fld, *ntarget, target, *ifpottarg,
             pottarg, *iffldtarg, fldtarg,
             [&](const double *t_, const double *, const double *s_, const double *q, const double *dq, double *po,
                 double *fo, int nt, const double *tg, int ipt, double *pt, int ift, double *ft, cudaStream_t s) {
                 return tri_direct_device(ns, t_, s_, ifc, q, ifd, dq, ifp, po, iff, fo, nt, tg, ipt, pt, ift, ft, s);
             });
}

// Host arrays in and out, as lfmm3dparttarg_, plus the Hessians.  The
// outputs of a failed call are left untouched.
void lfmm3dparttarghess_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                         const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                         const int *ifpot, double *pot, const int *iffld, double *fld, const int *ifhess,
                         double *hess, const int *ntarget, const double *target, const int *ifpottarg,
                         double *pottarg, const int *iffldtarg, double *fldtarg, const int *ifhesstarg,
                         double *hesstarg)
{
    const int ns = std::max(*nsource, 0), nt = std::max(*ntarget, 0);
    cudaStream_t s = thread_stream();
    Status st;
    DBuf<double> src, q, dq, dv, trg, po, fo, ho, pt, ft, ht;
    alloc_fail_point(1);
    bool ok = src.alloc(3L * std::max(ns, 1), s, st);
    if (*ifcharge == 1) ok = ok && q.alloc(2L * ns, s, st);
    if (*ifdipole == 1) ok = ok && dq.alloc(2L * ns, s, st) && dv.alloc(3L * ns, s, st);
    if (nt) ok = ok && trg.alloc(3L * nt, s, st);
    if (*ifpot == 1) ok = ok && po.alloc(2L * ns, s, st);
    if (*iffld == 1) ok = ok && fo.alloc(6L * ns, s, st);
    if (*ifhess == 1) ok = ok && ho.alloc(12L * ns, s, st);
    if (nt && *ifpottarg == 1) ok = ok && pt.alloc(2L * nt, s, st);
    if (nt && *iffldtarg == 1) ok = ok && ft.alloc(6L * nt, s, st);
    if (nt && *ifhesstarg == 1) ok = ok && ht.alloc(12L * nt, s, st);
    if (!ok) { g_ti.err = cudaGetErrorString(st.err); *ier = 8; return; }
    auto h2d = [&](DBuf<double> &d, const double *h, size_t n) {
        if (n) FMM_TRY(st, cudaMemcpyAsync(d.p, h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    };
    h2d(src, source, 3L * ns);
    if (*ifcharge == 1) h2d(q, charge, 2L * ns);
    if (*ifdipole == 1) { h2d(dq, dipstr, 2L * ns); h2d(dv, dipvec, 3L * ns); }
    if (nt) h2d(trg, target, 3L * nt);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); *ier = 8; return; }
    int e = lap_fmm_device(*iprec, ns, src.p, *ifcharge, q.p, *ifdipole, dq.p, dv.p, *ifpot, po.p, *iffld, fo.p, nt,
                           trg.p, nt ? *ifpottarg : 0, pt.p, nt ? *iffldtarg : 0, ft.p, s, nullptr, nullptr, *ifhess,
                           ho.p, nt ? *ifhesstarg : 0, ht.p);
    if (e) { *ier = e; return; }
    auto d2h = [&](double *h, DBuf<double> &d) {
        if (d.n) FMM_TRY(st, cudaMemcpyAsync(h, d.p, sizeof(double) * d.n, cudaMemcpyDeviceToHost, s));
    };
    if (*ifpot == 1) d2h(pot, po);
    if (*iffld == 1) d2h(fld, fo);
    if (*ifhess == 1) d2h(hess, ho);
    if (nt && *ifpottarg == 1) d2h(pottarg, pt);
    if (nt && *iffldtarg == 1) d2h(fldtarg, ft);
    if (nt && *ifhesstarg == 1) d2h(hesstarg, ht);
    FMM_TRY(st, cudaStreamSynchronize(s));
    *ier = st.ok() ? 0 : 16;
    if (!st.ok()) g_ti.err = cudaGetErrorString(st.err);
}

// One expansion at one point, with the calling sequence of l3dtaevalhess /
// l3dmpevalhess (src/laprouts3d.f:5297, 5229): rscale, center(3),
// expansion(0:nterms, -nterms:nterms), nterms, ztarg(3), pot, iffld, fld(3),
// ifhess, hess(6), ier.  For many points use fmm3d_l3dtaevalhess_device.
static void expeval_hess_host(bool loc, const double *rscale, const double *center, const double *coef,
                              const int *nterms, const double *ztarg, double *pot, const int *iffld, double *fld,
                              const int *ifhess, double *hess, int *ier)
{
    const int p = *nterms;
    cudaStream_t s = thread_stream();
    Status st;
    DBuf<double> c, t, out;
    const size_t nc = 2L * (p + 1) * (2 * p + 1);
    if (p < 0 || !c.alloc(nc, s, st) || !t.alloc(3, s, st) || !out.alloc(2 + 6 + 12, s, st)) {
        *ier = p < 0 ? 16 : 8;
        return;
    }
    FMM_TRY(st, cudaMemcpyAsync(c.p, coef, sizeof(double) * nc, cudaMemcpyHostToDevice, s));
    FMM_TRY(st, cudaMemcpyAsync(t.p, ztarg, sizeof(double) * 3, cudaMemcpyHostToDevice, s));
    launch_expeval_hess(loc, *rscale, center, c.p, p, 1, t.p, out.p, *iffld, out.p + 2, *ifhess, out.p + 8, s, st);
    double h[20];
    FMM_TRY(st, cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); *ier = 16; return; }
    pot[0] = h[0]; pot[1] = h[1];
    if (*iffld == 1) memcpy(fld, h + 2, 6 * sizeof(double));
    if (*ifhess == 1) memcpy(hess, h + 8, 12 * sizeof(double));
    *ier = 0;
}

void l3dtaevalhess_(const double *rscale, const double *center, const double *local, const int *nterms,
                    const double *ztarg, double *pot, const int *iffld, double *fld, const int *ifhess, double *hess,
                    int *ier)
{
    expeval_hess_host(true, rscale, center, local, nterms, ztarg, pot, iffld, fld, ifhess, hess, ier);
}

void l3dmpevalhess_(const double *rscale, const double *center, const double *mpole, const int *nterms,
                    const double *ztarg, double *pot, const int *iffld, double *fld, const int *ifhess, double *hess,
                    int *ier)
{
    expeval_hess_host(false, rscale, center, mpole, nterms, ztarg, pot, iffld, fld, ifhess, hess, ier);
}

void lfmm3dpartself_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                     const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                     const int *ifpot, double *pot, const int *iffld, double *fld)
{
    int zero = 0;
    lfmm3dparttarg_(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, pot, iffld, fld,
                    &zero, source, &zero, nullptr, &zero, nullptr);
}

void lfmm3dpart_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                 const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                 const int *ifpot, double *pot, const int *iffld, double *fld)
{
    lfmm3dpartself_(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, pot, iffld, fld);
}

void l3dpartdirect_(const int *nsource, const double *source, const int *ifcharge, const double *charge,
                    const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                    const int *iffld, double *fld, const int *ntarget, const double *target,
                    const int *ifpottarg, double *pottarg, const int *iffldtarg, double *fldtarg)
{
    int ns = *nsource, nt = *ntarget;
    with_device_arrays(ns, source, *ifcharge, charge, *ifdipole, dipstr, dipvec, *ifpot, pot, *iffld, fld, nt, target,
                       *ifpottarg, pottarg, *iffldtarg, fldtarg,
                       [&](const double *s_, const double *q, const double *dq, const double *dv, double *po,
                           double *fo, const double *t_, double *pt, double *ft, cudaStream_t s) {
                           return lap_direct_device(ns, s_, *ifcharge, q, *ifdipole, dq, dv, *ifpot, po, *iffld,
                                                    fo, nt, t_, *ifpottarg, pt, *iffldtarg, ft, s);
                       });
}

int fmm3d_set_timing(int on)
{
    g_ti.timing = on != 0;
    return 0;
}

int fmm3d_set_precision(int mode)
{
    g_sw[kSwPrecision] = mode;
    return 0;
}

int fmm3d_set_precision_thread(int mode)
{
    if (mode < -1 || mode > 1) return 1;
    g_sw_thread[kSwPrecision] = mode;
    return 0;
}

int fmm3d_set_tensor_m2l(int mode)
{
    if (mode < 0 || mode > 2) return 1;
    g_sw[kSwTensorM2L] = mode;
    return 0;
}

int fmm3d_set_overlap(int on)
{
    g_sw[kSwOverlap] = on ? 1 : 0;
    return 0;
}

int fmm3d_set_tensor_m2l_group(int slots)
{
    if (slots < 0) return 1;
    g_sw[kSwTcGroup] = slots;
    return 0;
}

int fmm3d_set_m2l_mode(int mode)
{
    g_sw[kSwM2LMode] = mode;
    return 0;
}

int fmm3d_set_switch_thread(int which, int value)
{
    if (which < 0 || which >= kNumSw) return 1;
    if (value == -1) {
        g_sw_thread[which] = -1;
        return 0;
    }
    if (!sw_valid(which, value)) return 1;
    g_sw_thread[which] = value;
    return 0;
}

int fmm3d_set_stats(int on)
{
    g_ti.want_stats = on != 0;
    return 0;
}

int fmm3d_last_timing(double *ms, int n)
{
    int k = std::min(n, (int)g_ti.ms.size());
    for (int i = 0; i < k; i++) ms[i] = g_ti.ms[i];
    return k;
}

int fmm3d_last_stats(long long *out, int n)
{
    int k = std::min(n, (int)g_ti.stats.size());
    for (int i = 0; i < k; i++) out[i] = g_ti.stats[i];
    return k;
}

const char *fmm3d_last_error(void) { return g_ti.err.c_str(); }

int fmm3d_last_launches(void) { return g_launch_count; }

int fmm3d_last_depth_capped(void) { return g_ti.depth_capped; }

}  // extern "C"
