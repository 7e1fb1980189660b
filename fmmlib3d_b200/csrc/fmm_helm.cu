// Helmholtz particle FMM driver and its C ABI (include/fmm3d_b200.h).
//
// Host orchestration of hfmm3dparttarg (src/hfmm3dpart.f:141-539),
// hfmm3dparttargmain (:545-1086) and hfmm3d_list2 (src/hfmm3drouts.f:153-564)
// on one B200: iprec tables, the octree (the Laplace tree: same d3tstrcr
// semantics), the per-level expansion orders and scales, the z-shift
// operators of every level (built on the GPU), the eight passes and the
// unsort.  All arithmetic is FP64.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <complex>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/fmm3d_b200.h"
#include "driver_common.cuh"
#include "helm_kernels.cuh"
#include "tri.cuh"

namespace fmm {

using cplx = std::complex<double>;

// ---------------------------------------------------------------- expansion orders (host)
// h3dall (src/helmrouts3d.f:709-809), values only.
static void h3dall_host(int nt, cplx z, double scale, std::vector<cplx> &h)
{
    h.assign(nt + 2, cplx(0, 0));
    if (std::abs(z) < 1.0e-15) return;
    cplx iz = cplx(0, 1) * z;
    cplx h0 = std::exp(iz) / iz;
    h[0] = h0;
    h[1] = h0 * (1.0 / z - cplx(0, 1)) * scale;
    double s2 = scale * scale;
    cplx zinv = scale / z;
    for (int i = 1; i <= nt - 1; i++) h[i + 1] = (zinv * (2 * i + 1.0)) * h[i] - s2 * h[i - 1];
}

// jfuns3d (src/cdjseval3d.f:15-197), values only; returns the reference's ier.
static int jfuns3d_host(int nt, cplx z, double scale, std::vector<cplx> &f, int lw)
{
    f.assign(lw + 2, cplx(0, 0));
    if (std::abs(z) < 1.0e-200) { f[0] = 1; return 0; }
    std::vector<char> isc(lw + 2, 0);
    cplx zinv = 1.0 / z;
    f[nt] = 1;
    f[nt - 1] = 0;
    int ntop = 0;
    for (int i = nt; i <= lw; i++) {
        cplx t = (2 * i + 1.0) * zinv * f[i] - f[i - 1];
        f[i + 1] = t;
        if (std::norm(t) > 1.0e40) { ntop = i + 1; break; }
    }
    if (ntop == 0) return 8;
    f[ntop] = 0;
    f[ntop - 1] = 1;
    for (int i = ntop - 1; i >= 1; i--) {
        cplx t = (2 * i + 1.0) * zinv * f[i] - f[i + 1];
        f[i - 1] = t;
        if (std::norm(t) > 1.0e40) { f[i] *= 1.0e-40; f[i - 1] *= 1.0e-40; isc[i] = 1; }
    }
    double sct = 1;
    for (int i = 1; i <= ntop; i++) {
        sct /= scale;
        if (isc[i - 1]) sct *= 1.0e-40;
        f[i] *= sct;
    }
    cplx j0 = std::sin(z) * zinv, j1 = j0 * zinv - std::cos(z) * zinv;
    cplx zs = std::abs(j1) > std::abs(j0) ? j1 / (f[1] * scale) : j0 / f[0];
    for (int i = 0; i <= nt; i++) f[i] *= zs;
    return 0;
}

// h3dterms (src/h3dterms.f:28-102) with the Hankel argument factor fh (1.5,
// or a list-2 separation as in h3dterms_list2 :192-344); the Bessel values
// j (at |zk| size sqrt(3)/2) are passed in when already known.
static int hterms(double size, cplx zk, double eps, double fh, int *ier, const std::vector<cplx> *jv = nullptr)
{
    const int NT = 1000;
    std::vector<cplx> h, jl;
    double rs = std::abs(zk * size) < 1.0 ? std::abs(zk * size) : 1.0;
    h3dall_host(NT, (zk * size) * fh, rs, h);
    *ier = 0;
    if (!jv) {
        if (jfuns3d_host(NT, (zk * size) * (sqrt(3.0) / 2.0), rs, jl, 2000) == 8) { *ier = 11; return 0; }
        jv = &jl;
    }
    const std::vector<cplx> &j = *jv;
    double x0 = std::abs(j[0] * h[0]) + std::abs(j[1] * h[1]);
    for (int k = 2; k <= NT; k++) {
        double x = std::abs(j[k] * h[k]) + std::abs(j[k - 1] * h[k - 1]);
        if (x < eps * x0) return k + 1;
    }
    *ier = 13;
    return 1000;
}

// h3dterms_list2 (src/h3dterms.f:192-344); itab[(i+3)*49+(j+3)*7+(k+3)]
static void hterms_list2(double size, cplx zk, double eps, int *itab)
{
    int tab[2][4][4], e;
    std::vector<cplx> j;
    double rs = std::abs(zk * size) < 1.0 ? std::abs(zk * size) : 1.0;
    bool jok = jfuns3d_host(1000, (zk * size) * (sqrt(3.0) / 2.0), rs, j, 2000) == 0;
    for (int ii = 2; ii <= 3; ii++)
        for (int jj = 0; jj <= 3; jj++)
            for (int kk = 0; kk <= 3; kk++) {
                double dx = ii, dy = jj, dz = kk;
                if (dx > 0) dx -= .5;
                if (dy > 0) dy -= .5;
                if (dz > 0) dz -= .5;
                tab[ii - 2][jj][kk] =
                    jok ? hterms(size, zk, eps, sqrt(dx * dx + dy * dy + dz * dz), &e, &j) : 0;
            }
    for (int i = -3; i <= 3; i++)
        for (int jx = -3; jx <= 3; jx++)
            for (int k = -3; k <= 3; k++) {
                int v = 0, ai = abs(i), aj = abs(jx), ak = abs(k);
                if (ai > 1) v = tab[ai - 2][aj][ak];
                else if (aj > 1) v = tab[aj - 2][ai][ak];
                if (ai <= 1 && aj <= 1 && ak > 1) v = ai >= aj ? tab[ak - 2][ai][aj] : tab[ak - 2][aj][ai];
                itab[(i + 3) * 49 + (jx + 3) * 7 + (k + 3)] = v;
            }
}

// ---------------------------------------------------------------- rotation plan (per device, pmax)
// Rotation matrices of every direction a translation uses (the list-2
// offsets and the 8 parent/child diagonals), keyed by (rho^2, dz) of the
// doubled integer vector; built once per (device, pmax).
struct HRotPlan {
    int pmax = 0, ncls = 0;
    std::map<std::pair<int, int>, int> cls;
    DBuf<double> rot;
};
static std::mutex g_hrot_mu;
static std::map<std::pair<int, int>, std::shared_ptr<HRotPlan>> g_hrot;

static int class_key(std::map<std::pair<int, int>, int> &cls, std::vector<double> *cs, int dx, int dy, int dz)
{
    auto k = std::make_pair(dx * dx + dy * dy, dz);
    auto f = cls.find(k);
    if (f != cls.end()) return f->second;
    int id = (int)cls.size();
    cls[k] = id;
    if (cs) {
        double r = sqrt((double)(dx * dx + dy * dy + dz * dz));
        cs->push_back(dz / r);
        cs->push_back(sqrt((double)(dx * dx + dy * dy)) / r);
    }
    return id;
}

static std::shared_ptr<HRotPlan> get_hrot(int pmax, cudaStream_t s, Status &st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_hrot_mu);
    auto key = std::make_pair(dev, pmax);
    auto it = g_hrot.find(key);
    if (it != g_hrot.end()) return it->second;
    auto P = std::make_shared<HRotPlan>();
    P->pmax = pmax;
    std::vector<double> cs;
    for (int i = -3; i <= 3; i++)
        for (int j = -3; j <= 3; j++)
            for (int k = -3; k <= 3; k++)
                if (i || j || k) class_key(P->cls, &cs, 2 * i, 2 * j, 2 * k);
    for (int d = 0; d < 8; d++) {
        int b[3] = {d & 1, (d >> 1) & 1, (d >> 2) & 1};
        class_key(P->cls, &cs, 1 - 2 * b[0], 1 - 2 * b[1], 1 - 2 * b[2]);
        class_key(P->cls, &cs, 2 * b[0] - 1, 2 * b[1] - 1, 2 * b[2] - 1);
    }
    P->ncls = (int)P->cls.size();
    DBuf<double> dcs;
    if (!P->rot.alloc(rot_class_size(pmax) * P->ncls, s, st) || !dcs.alloc(cs.size(), s, st)) return nullptr;
    FMM_TRY(st, cudaMemcpyAsync(dcs.p, cs.data(), sizeof(double) * cs.size(), cudaMemcpyHostToDevice, s));
    build_rotations(pmax, P->ncls, dcs.p, P->rot.p, s, st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) return nullptr;
    P->rot.s = nullptr;  // process lifetime
    g_hrot[key] = P;
    return P;
}

static void ephi_of(int dx, int dy, double &ex, double &ey)
{
    double rho = sqrt((double)(dx * dx + dy * dy));
    if (rho == 0) { ex = 1; ey = 0; }
    else { ex = dx / rho; ey = dy / rho; }
}

// iprec tables of hfmm3dparttarg (src/hfmm3dpart.f:277-300): the Laplace ones.
static bool helm_iprec(int iprec, int ns, int nt, double &eps, int &nbox)
{
    static const double e[] = {.5e0, .5e-1, .5e-2, .5e-3, .5e-6, .5e-9, .5e-12, .5e-15, 0.0};
    static const int nb[] = {40, 50, 80, 160, 400, 800, 1200, 1400};
    if (iprec < -2 || iprec > 6) return false;
    eps = e[iprec + 2];
    nbox = iprec == 6 ? ns + nt : nb[iprec + 2];
    return true;
}

__global__ void k_hstats(int nleaves, const int *leaves, TreeView tv, int do_src, int do_trg, unsigned long long *acc)
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

// M2L pair count of one level (targets b0..b0+nb-1), by truncation order.
__global__ void k_hm2l_count(int b0, int nb, TreeView tv, const HSlot *slots, int prune, unsigned long long *hist)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int b = b0 + t;
    if (t >= nb || (prune && tv.ntrg[b] == 0) || tv.parent[b] < 0) return;
    int P = tv.parent[b], o = tv.octant[b];
    for (int s = 0; s < 189; s++) {
        const HSlot &sl = slots[o * 189 + s];
        int C = tv.coll[27L * P + sl.coll];
        if (C < 0) continue;
        int src = tv.child[8L * C + sl.oct];
        if (src < 0 || tv.nsrc[src] == 0) continue;
        atomicAdd(&hist[sl.nin], 1ull);
    }
}

// Triangle mode (hfmm3dtriatarg, src/hfmm3dtria.f:133-1215): the sources
// are flat triangles tri (3,3,n) with unit normals norm, d_src their
// centroids; the far field runs on the far rule's nodes, the near field
// integrates each triangle with the near rule (degrees norder / nqtri of
// :730-751).
struct HTriIn {
    const double *tri = nullptr, *norm = nullptr;
    TriRule far, near_;
};

static int helm_fmm_device(int iprec, double2 zk, int ns, const double *d_src, int ifcharge, const double *d_q,
                           int ifdipole, const double *d_dq, const double *d_dv, int ifpot, double *d_pot, int iffld,
                           double *d_fld, int nt, const double *d_trg, int ifpottarg, double *d_pottarg,
                           int iffldtarg, double *d_fldtarg, cudaStream_t s, const HTriIn *tri = nullptr)
{
    Status st;
    g_launch_count = 0;
    double eps;
    int nbox;
    if (ns < 1 || !helm_iprec(iprec, ns, nt, eps, nbox)) return 4;
    if (tri) nbox = tri_nbox(iprec, ns, nt);
    if (nt < 0) nt = 0;
    keep_pool_memory();
    Timer tm(s, g_ti.timing);
    tm.mark();
    Tree T;
    alloc_fail_point(2);
    build_tree(T, d_src, ns, d_trg, nt, nbox, s, st);
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 4; }
    g_ti.depth_capped = T.capped;
    tm.mark();
    // per-level orders and scales (src/hfmm3dpart.f:336-340, 398-405).  In
    // hfmm3dparttarg zk is not declared complex, so under its implicit real*8
    // typing the scale rule sees only the real part (the first of zk's two
    // doubles): scale = min(1, |Re(zk)| * size / 2^l).  The orders (h3dterms)
    // and every operator receive the complex zk.
    const cplx zkc(zk.x, zk.y);
    const int nlev = T.nlev;
    HLevels lv;
    memset(&lv, 0, sizeof lv);
    std::vector<double> bsize(nlev + 1);
    int pmax = 1;
    for (int l = 0; l <= nlev; l++) {
        bsize[l] = T.size / pow(2.0, l);
        // hfmm3dtriatarg declares zk complex*16: its rule sees |zk| (src/hfmm3dtria.f:248, 350-355)
        double bs = tri ? std::abs(bsize[l] * zkc) : std::abs(bsize[l] * zk.x);
        lv.sc[l] = bs < 1 ? bs : 1.0;
        if (l >= 2) {
            int e;
            lv.p[l] = hterms(bsize[l], zkc, eps, 1.5, &e);
            pmax = std::max(pmax, lv.p[l]);
        }
    }
    if (nlev >= 2 && pmax > kHelmMaxP) {
        g_ti.err = "expansion order " + std::to_string(pmax) + " above the supported " + std::to_string(kHelmMaxP) +
                   " (|zk| times the box size too large for this iprec)";
        return 16;
    }
    const int NC = (pmax + 1) * (pmax + 1);
    DBuf<double> sx, sy, sz, svx, svy, svz, tx, ty, tz;
    DBuf<double2> sq, sdq, opot, ofx, ofy, ofz, tpot, tfx, tfy, tfz, mpole, local;
    alloc_fail_point(3);
    bool ok = sx.alloc(ns, s, st) && sy.alloc(ns, s, st) && sz.alloc(ns, s, st);
    if (ifcharge == 1) ok = ok && sq.alloc(ns, s, st);
    if (ifdipole == 1) ok = ok && sdq.alloc(ns, s, st) && svx.alloc(ns, s, st) && svy.alloc(ns, s, st) && svz.alloc(ns, s, st);
    if (nt) ok = ok && tx.alloc(nt, s, st) && ty.alloc(nt, s, st) && tz.alloc(nt, s, st);
    const int do_src = ifpot == 1 || iffld == 1, do_trg = (ifpottarg == 1 || iffldtarg == 1) && nt > 0;
    if (ifpot == 1) ok = ok && opot.alloc(ns, s, st) && opot.zero(st);
    if (iffld == 1) ok = ok && ofx.alloc(ns, s, st) && ofy.alloc(ns, s, st) && ofz.alloc(ns, s, st) && ofx.zero(st) &&
                         ofy.zero(st) && ofz.zero(st);
    if (do_trg && ifpottarg == 1) ok = ok && tpot.alloc(nt, s, st) && tpot.zero(st);
    if (do_trg && iffldtarg == 1) ok = ok && tfx.alloc(nt, s, st) && tfy.alloc(nt, s, st) && tfz.alloc(nt, s, st) &&
                                      tfx.zero(st) && tfy.zero(st) && tfz.zero(st);
    if (!ok) { g_ti.err = cudaGetErrorString(st.err); return 8; }
    const bool far = nlev >= 2;
    if (far) {
        alloc_fail_point(4);
        if (!mpole.alloc((size_t)T.nboxes * NC, s, st) || !local.alloc((size_t)T.nboxes * NC, s, st)) {
            g_ti.err = cudaGetErrorString(st.err);
            return 16;
        }
        mpole.zero(st);
        local.zero(st);
    }
    PointsSoA P;
    P.x = sx.p; P.y = sy.p; P.z = sz.p; P.q = sq.p; P.dq = sdq.p; P.vx = svx.p; P.vy = svy.p; P.vz = svz.p;
    wait_host_inputs(s, st);   // charges still in flight from the host
    k_gather_src<<<div_up(ns, 256), 256, 0, s>>>(ns, T.perm_src.p, d_src, d_q, d_dq, d_dv, ifcharge == 1,
                                                 ifdipole == 1, P); FMM_COUNT_LAUNCH();
    if (nt) { k_gather_pts<<<div_up(nt, 256), 256, 0, s>>>(nt, T.perm_trg.p, d_trg, tx.p, ty.p, tz.p); FMM_COUNT_LAUNCH(); }
    FMM_LAUNCH_CHECK(st);
    TreeView tv = make_treeview(T);
    // triangles: tree-ordered geometry and densities, the far rule's nodes, box ranges in nodes
    DBuf<double> tgeo, qx, qy, qz, qvx, qvy, qvz;
    DBuf<double2> tq, tdq, qq, qdq;
    DBuf<int> qsrc0, qnsrc;
    TriSoA ts;
    PointsSoA Pq;
    TreeView tv_quad = tv;
    if (tri) {
        const size_t nn = (size_t)ns * tri->far.n;
        bool okt = tgeo.alloc(30L * ns, s, st) && qx.alloc(nn, s, st) && qy.alloc(nn, s, st) && qz.alloc(nn, s, st) &&
                   qsrc0.alloc(T.nboxes, s, st) && qnsrc.alloc(T.nboxes, s, st);
        if (ifcharge == 1) okt = okt && tq.alloc(ns, s, st) && qq.alloc(nn, s, st);
        if (ifdipole == 1)
            okt = okt && tdq.alloc(ns, s, st) && qdq.alloc(nn, s, st) && qvx.alloc(nn, s, st) && qvy.alloc(nn, s, st) &&
                  qvz.alloc(nn, s, st);
        if (!okt) { g_ti.err = cudaGetErrorString(st.err); return 8; }
        ts.geo = tgeo.p; ts.q = tq.p; ts.dq = tdq.p;
        Pq.x = qx.p; Pq.y = qy.p; Pq.z = qz.p; Pq.q = qq.p; Pq.dq = qdq.p; Pq.vx = qvx.p; Pq.vy = qvy.p; Pq.vz = qvz.p;
        launch_tri_gather(ns, T.perm_src.p, tri->tri, tri->norm, d_q, d_dq, ifcharge, ifdipole, tri->far, ts, Pq, s, st);
        launch_scale_ranges(T.nboxes, tv.src0, tv.nsrc, tri->far.n, qsrc0.p, qnsrc.p, s, st);
        tv_quad.src0 = qsrc0.p;
        tv_quad.nsrc = qnsrc.p;
    }
    const int prune = !(ifpot == 1 || iffld == 1);
    OutSoA os, ot;
    os.pot = opot.p; os.fx = ofx.p; os.fy = ofy.p; os.fz = ofz.p;
    ot.pot = tpot.p; ot.fx = tfx.p; ot.fy = tfy.p; ot.fz = tfz.p;

    std::shared_ptr<HRotPlan> rp;
    std::vector<HSlot> hs;
    std::vector<HZBlock> hb;
    std::vector<double> xw;
    std::vector<int> m2m_base(nlev + 1, -1), l2l_base(nlev + 1, -1), m2l_base(nlev + 1, -1);
    DBuf<HSlot> dslots;
    DBuf<HZBlock> dblk;
    DBuf<double> dxw;
    DBuf<double2> Z, rad;
    DBuf<Tile> dtiles;
    std::vector<Tile> htiles;
    std::vector<std::pair<int, int>> m2m_rng, l2l_rng;
    int m2l_a = 0, m2l_n = 0, kt = 1;
    if (far) {
        rp = get_hrot(pmax, s, st);
        if (!st.ok() || !rp) { g_ti.err = cudaGetErrorString(st.err); return 16; }
        // z-shift operator blocks, shared by slots with the same (kind, level, distance, degrees)
        std::map<std::tuple<int, int, int, int>, int> bidx;
        long long ztot = 0, rtot = 0;
        auto block = [&](int kind, int lev, int dkey, int nin, int nout, int nq, double zs, double radius, double sc1,
                         double sc2) {
            auto key = std::make_tuple(kind, lev, dkey, nin);
            auto f = bidx.find(key);
            if (f != bidx.end()) return f->second;
            HZBlock B;
            B.kind = kind; B.nin = nin; B.nout = nout; B.nq = nq;
            B.qoff = (int)(xw.size() / 2);
            B.zshift = zs; B.radius = radius; B.sc1 = sc1; B.sc2 = sc2;
            B.zoff = ztot;
            B.roff = rtot;
            ztot += hz_block_size(nin, nout);
            rtot += 2LL * (nq + 1) * (pmax + 2);
            std::vector<double> gx, gw;
            gauss_legendre(nq, gx, gw);
            for (int i = 0; i < nq; i++) { xw.push_back(gx[i]); xw.push_back(gw[i]); }
            int id = (int)hb.size();
            hb.push_back(B);
            bidx[key] = id;
            return id;
        };
        const double r3 = sqrt(3.0) / 2.0;
        for (int l = 2; l <= nlev; l++) {
            int itab[343];
            hterms_list2(bsize[l], zkc, eps, itab);
            int nq = std::max(6, (int)((float)lv.p[l] * 1.2f));  // a default-real product in the reference
            m2l_base[l] = (int)hs.size();
            for (int o = 0; o < 8; o++) {
                int ob[3] = {o & 1, (o >> 1) & 1, (o >> 2) & 1};
                for (int c = 0; c < 27; c++) {
                    int co[3] = {c / 9 - 1, (c / 3) % 3 - 1, c % 3 - 1};
                    for (int d = 0; d < 8; d++) {
                        int db[3] = {d & 1, (d >> 1) & 1, (d >> 2) & 1};
                        int D[3];
                        for (int e = 0; e < 3; e++) D[e] = 2 * co[e] + db[e] - ob[e];
                        if (abs(D[0]) <= 1 && abs(D[1]) <= 1 && abs(D[2]) <= 1) continue;
                        HSlot sl;
                        sl.coll = c; sl.oct = d;
                        sl.cls = class_key(rp->cls, nullptr, -2 * D[0], -2 * D[1], -2 * D[2]);
                        ephi_of(-D[0], -D[1], sl.ex, sl.ey);
                        int pt = std::min(itab[(D[0] + 3) * 49 + (D[1] + 3) * 7 + (D[2] + 3)], lv.p[l]);
                        int d2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
                        int bi = block(1, l, d2, pt, pt, nq, sqrt((double)d2) * bsize[l], r3 * bsize[l], lv.sc[l],
                                       lv.sc[l]);
                        sl.nin = pt; sl.nout = pt; sl.mmax = pt; sl.zoff = hb[bi].zoff;
                        hs.push_back(sl);
                    }
                }
            }
        }
        for (int l = 2; l <= nlev - 1; l++) {
            int bm = block(0, l, 3, lv.p[l + 1], lv.p[l], std::max(6, (int)(lv.p[l] * 2.5)), r3 * bsize[l + 1],
                           r3 * bsize[l], lv.sc[l + 1], lv.sc[l]);
            int bl = block(2, l, 3, lv.p[l], lv.p[l + 1], std::max(6, 2 * lv.p[l]), r3 * bsize[l + 1],
                           r3 * bsize[l + 1], lv.sc[l], lv.sc[l + 1]);
            m2m_base[l] = (int)hs.size();
            for (int d = 0; d < 8; d++) {
                int b[3] = {d & 1, (d >> 1) & 1, (d >> 2) & 1};
                HSlot a;
                a.coll = -1; a.oct = d;
                a.cls = class_key(rp->cls, nullptr, 1 - 2 * b[0], 1 - 2 * b[1], 1 - 2 * b[2]);
                ephi_of(1 - 2 * b[0], 1 - 2 * b[1], a.ex, a.ey);
                a.nin = lv.p[l + 1]; a.nout = lv.p[l]; a.mmax = std::min(a.nin, a.nout); a.zoff = hb[bm].zoff;
                hs.push_back(a);
            }
            l2l_base[l] = (int)hs.size();
            for (int d = 0; d < 8; d++) {
                int b[3] = {d & 1, (d >> 1) & 1, (d >> 2) & 1};
                HSlot a;
                a.coll = -1; a.oct = d;
                a.cls = class_key(rp->cls, nullptr, 2 * b[0] - 1, 2 * b[1] - 1, 2 * b[2] - 1);
                ephi_of(2 * b[0] - 1, 2 * b[1] - 1, a.ex, a.ey);
                a.nin = lv.p[l]; a.nout = lv.p[l + 1]; a.mmax = std::min(a.nin, a.nout); a.zoff = hb[bl].zoff;
                hs.push_back(a);
            }
        }
        if ((int)rp->cls.size() != rp->ncls) { g_ti.err = "internal: rotation class missing"; return 16; }
        ok = dslots.alloc(hs.size(), s, st) && dblk.alloc(hb.size(), s, st) && dxw.alloc(xw.size(), s, st) &&
             Z.alloc(ztot, s, st) && rad.alloc(rtot, s, st);
        if (!ok) { g_ti.err = cudaGetErrorString(st.err); return 16; }
        FMM_TRY(st, cudaMemcpyAsync(dslots.p, hs.data(), sizeof(HSlot) * hs.size(), cudaMemcpyHostToDevice, s));
        FMM_TRY(st, cudaMemcpyAsync(dblk.p, hb.data(), sizeof(HZBlock) * hb.size(), cudaMemcpyHostToDevice, s));
        FMM_TRY(st, cudaMemcpyAsync(dxw.p, xw.data(), sizeof(double) * xw.size(), cudaMemcpyHostToDevice, s));
        build_hz((int)hb.size(), dblk.p, hb.data(), dxw.p, zk, pmax, rad.p, Z.p, s, st);
        // translation tiles per (level, octant) group
        // targets per translation tile: buffers of at most ~50 KB, so that several
        // CTAs share an SM (the passes are bound by L2 latency, not by reuse)
        kt = 8;
        while (kt > 1 && (size_t)3 * kt * NC * 16 > 50 * 1024) kt /= 2;
        auto make_tiles = [&](int lev, int base, int per_oct, int nslot) {
            for (int o = 0; o < 8; o++) {
                int g = lev * 8 + o;
                int a = T.group_start[g], bnd = T.group_start[g + 1];
                for (int i = a; i < bnd; i += kt) {
                    Tile t;
                    t.first = i; t.count = std::min(kt, bnd - i); t.slot0 = base + o * per_oct; t.nslot = nslot;
                    htiles.push_back(t);
                }
            }
        };
        for (int l = nlev - 1; l >= 2; l--) {
            int a = (int)htiles.size();
            make_tiles(l, m2m_base[l], 0, 8);
            m2m_rng.push_back({a, (int)htiles.size() - a});
        }
        m2l_a = (int)htiles.size();
        for (int l = 2; l <= nlev; l++) make_tiles(l, m2l_base[l], 189, 189);
        m2l_n = (int)htiles.size() - m2l_a;
        for (int l = 2; l <= nlev - 1; l++) {
            int a = (int)htiles.size();
            make_tiles(l + 1, l2l_base[l], 1, 1);
            l2l_rng.push_back({a, (int)htiles.size() - a});
        }
        if (!htiles.empty() && dtiles.alloc(htiles.size(), s, st))
            FMM_TRY(st, cudaMemcpyAsync(dtiles.p, htiles.data(), sizeof(Tile) * htiles.size(), cudaMemcpyHostToDevice, s));
    }
    tm.mark();
    if (far) {
        // STEP 1: P2M at leaves of level >= 2 (src/hfmm3dpart.f:696-760)
        launch_hform(false, T.leaves.p, T.nleaves, tri ? tv_quad : tv, tri ? Pq : P, ifcharge, ifdipole, lv, NC, zk,
                     mpole.p, s, st);
        tm.mark();
        // STEP 3: M2M, levels nlev-1 .. 2
        for (auto &r : m2m_rng)
            launch_htranslate(0, dtiles.p + r.first, r.second, T.grouped.p, dslots.p, tv, pmax, rp->rot.p, Z.p,
                              mpole.p, mpole.p, prune, kt, s, st);
        tm.mark();
        // STEP 2: P2L into boxes with a list 4 (src/hfmm3dpart.f:775-846)
        launch_hform(true, T.grouped.p, T.nboxes, tri ? tv_quad : tv, tri ? Pq : P, ifcharge, ifdipole, lv, NC, zk,
                     local.p, s, st);
        tm.mark();
        // STEP 4: M2L over list 2
        launch_htranslate(1, dtiles.p + m2l_a, m2l_n, T.grouped.p, dslots.p, tv, pmax, rp->rot.p, Z.p, mpole.p,
                          local.p, prune, kt, s, st);
        tm.mark();
        // STEP 5: L2L, levels 2 .. nlev-1
        for (auto &r : l2l_rng)
            launch_htranslate(2, dtiles.p + r.first, r.second, T.grouped.p, dslots.p, tv, pmax, rp->rot.p, Z.p,
                              local.p, local.p, prune, kt, s, st);
        tm.mark();
        // STEPS 6, 7: M2P from list 3 and L2P
        launch_heval(T.leaves.p, T.nleaves, tv, sx.p, sy.p, sz.p, tx.p, ty.p, tz.p, lv, NC, zk, mpole.p, local.p,
                     os, ot, do_src, do_trg, s, st);
        tm.mark();
    } else {
        for (int i = 0; i < 6; i++) tm.mark();
    }
    // STEP 8: P2P over self and list 1
    if (tri)
        launch_hp2p_tri(T.leaves.p, T.nleaves, tv, ts, sx.p, sy.p, sz.p, tx.p, ty.p, tz.p, zk, tri->near_, os, ot,
                        ifcharge, ifdipole, do_src, do_trg, iffld == 1, do_trg && iffldtarg == 1, s, st);
    else
        launch_hp2p(T.leaves.p, T.nleaves, tv, P, tx.p, ty.p, tz.p, zk, os, ot, ifcharge, ifdipole, ifpot, iffld,
                    do_trg ? ifpottarg : 0, do_trg ? iffldtarg : 0, s, st);
    tm.mark();
    if (do_src) {
        k_scatter_out<<<div_up(ns, 256), 256, 0, s>>>(ns, T.perm_src.p, os, ifpot == 1 ? d_pot : nullptr,
                                                      iffld == 1 ? d_fld : nullptr); FMM_COUNT_LAUNCH();
    }
    if (do_trg) {
        k_scatter_out<<<div_up(nt, 256), 256, 0, s>>>(nt, T.perm_trg.p, ot, ifpottarg == 1 ? d_pottarg : nullptr,
                                                      iffldtarg == 1 ? d_fldtarg : nullptr); FMM_COUNT_LAUNCH();
    }
    FMM_LAUNCH_CHECK(st);
    tm.mark();
    tm.finish(g_ti.ms);
    if (g_ti.want_stats) {
        DBuf<unsigned long long> acc;
        acc.alloc(1 + 128, s, st);
        acc.zero(st);
        if (st.ok()) {
            k_hstats<<<div_up(std::max(T.nleaves, 1), 256), 256, 0, s>>>(T.nleaves, T.leaves.p, tv, do_src, do_trg,
                                                                         acc.p); FMM_COUNT_LAUNCH();
            if (far)
                for (int l = 2; l <= nlev; l++) {
                    k_hm2l_count<<<div_up(std::max(T.lev_count[l], 1), 128), 128, 0, s>>>(
                        T.lev_start[l], T.lev_count[l], tv, dslots.p + m2l_base[l], prune, acc.p + 1); FMM_COUNT_LAUNCH();
                }
            std::vector<unsigned long long> h(129);
            FMM_TRY(st, cudaMemcpyAsync(h.data(), acc.p, sizeof(unsigned long long) * 129, cudaMemcpyDeviceToHost, s));
            FMM_TRY(st, cudaStreamSynchronize(s));
            long long m2l = 0;
            for (int i = 0; i < 128; i++) m2l += (long long)h[1 + i];
            g_ti.stats.assign(9 + 128 + kMaxLevel + 1, 0);
            g_ti.stats[0] = T.nboxes; g_ti.stats[1] = nlev; g_ti.stats[2] = T.nleaves; g_ti.stats[3] = pmax;
            g_ti.stats[7] = (long long)h[0];
            g_ti.stats[8] = m2l;
            for (int i = 0; i < 128; i++) g_ti.stats[9 + i] = (long long)h[1 + i];
            for (int l = 0; l <= kMaxLevel; l++) g_ti.stats[9 + 128 + l] = lv.p[l];
        }
    }
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = std::string(st.where ? st.where : "") + ": " + cudaGetErrorString(st.err); return 16; }
    return 0;
}

static void split_points(int n, const double *d_src, const double *d_q, const double *d_dq, const double *d_dv,
                         int ifc, int ifd, DBuf<double> &x, DBuf<double> &y, DBuf<double> &z, DBuf<double2> &q,
                         DBuf<double2> &dq, DBuf<double> &vx, DBuf<double> &vy, DBuf<double> &vz, PointsSoA &P,
                         cudaStream_t s, Status &st)
{
    bool ok = x.alloc(n, s, st) && y.alloc(n, s, st) && z.alloc(n, s, st);
    if (ifc == 1) ok = ok && q.alloc(n, s, st);
    if (ifd == 1) ok = ok && dq.alloc(n, s, st) && vx.alloc(n, s, st) && vy.alloc(n, s, st) && vz.alloc(n, s, st);
    if (!ok || n == 0) return;
    k_split_aos<<<div_up(n, 256), 256, 0, s>>>(n, d_src, x.p, y.p, z.p); FMM_COUNT_LAUNCH();
    if (ifc == 1) { k_split_c<<<div_up(n, 256), 256, 0, s>>>(n, d_q, q.p); FMM_COUNT_LAUNCH(); }
    if (ifd == 1) {
        k_split_c<<<div_up(n, 256), 256, 0, s>>>(n, d_dq, dq.p); FMM_COUNT_LAUNCH();
        k_split_aos<<<div_up(n, 256), 256, 0, s>>>(n, d_dv, vx.p, vy.p, vz.p); FMM_COUNT_LAUNCH();
    }
    P.x = x.p; P.y = y.p; P.z = z.p; P.q = q.p; P.dq = dq.p; P.vx = vx.p; P.vy = vy.p; P.vz = vz.p;
}

// h3dpartdirect (src/hfmm3dpart.f:1268-1401) on device arrays.
static int helm_direct_device(double2 zk, int ns, const double *d_src, int ifcharge, const double *d_q, int ifdipole,
                              const double *d_dq, const double *d_dv, int ifpot, double *d_pot, int iffld,
                              double *d_fld, int nt, const double *d_trg, int ifpottarg, double *d_pottarg,
                              int iffldtarg, double *d_fldtarg, cudaStream_t s)
{
    Status st;
    g_launch_count = 0;
    if (ns < 0) ns = 0;
    if (nt < 0) nt = 0;
    DBuf<double> sx, sy, sz, vx, vy, vz, tx, ty, tz;
    DBuf<double2> q, dq, o0, o1, o2, o3;
    PointsSoA P;
    split_points(ns, d_src, d_q, d_dq, d_dv, ifcharge, ifdipole, sx, sy, sz, q, dq, vx, vy, vz, P, s, st);
    int ne = std::max(std::max(ns, nt), 1);
    if (!(st.ok() && o0.alloc(ne, s, st) && o1.alloc(ne, s, st) && o2.alloc(ne, s, st) && o3.alloc(ne, s, st))) return 8;
    OutSoA o;
    o.pot = o0.p; o.fx = o1.p; o.fy = o2.p; o.fz = o3.p;
    if (ns > 0 && (ifpot == 1 || iffld == 1)) {
        launch_hdirect(ns, P, ifcharge, ifdipole, ns, sx.p, sy.p, sz.p, nullptr, 1, zk, o, s, st);
        k_scatter_out<<<div_up(ns, 256), 256, 0, s>>>(ns, nullptr, o, ifpot == 1 ? d_pot : nullptr,
                                                      iffld == 1 ? d_fld : nullptr); FMM_COUNT_LAUNCH();
    }
    if (nt > 0 && (ifpottarg == 1 || iffldtarg == 1)) {
        if (!(tx.alloc(nt, s, st) && ty.alloc(nt, s, st) && tz.alloc(nt, s, st))) return 8;
        k_split_aos<<<div_up(nt, 256), 256, 0, s>>>(nt, d_trg, tx.p, ty.p, tz.p); FMM_COUNT_LAUNCH();
        launch_hdirect(ns, P, ifcharge, ifdipole, nt, tx.p, ty.p, tz.p, nullptr, 0, zk, o, s, st);
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

int fmm3d_hfmm3dparttarg_device(int iprec, const double *zk, int nsource, const double *d_source, int ifcharge,
                                const double *d_charge, int ifdipole, const double *d_dipstr, const double *d_dipvec,
                                int ifpot, double *d_pot, int iffld, double *d_fld, int ntarget,
                                const double *d_target, int ifpottarg, double *d_pottarg, int iffldtarg,
                                double *d_fldtarg, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return helm_fmm_device(iprec, make_double2(zk[0], zk[1]), nsource, d_source, ifcharge, d_charge, ifdipole,
                           d_dipstr, d_dipvec, ifpot, d_pot, iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg,
                           iffldtarg, d_fldtarg, s);
}

int fmm3d_h3dpartdirect_device(const double *zk, int nsource, const double *d_source, int ifcharge,
                               const double *d_charge, int ifdipole, const double *d_dipstr, const double *d_dipvec,
                               int ifpot, double *d_pot, int iffld, double *d_fld, int ntarget,
                               const double *d_target, int ifpottarg, double *d_pottarg, int iffldtarg,
                               double *d_fldtarg, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    return helm_direct_device(make_double2(zk[0], zk[1]), nsource, d_source, ifcharge, d_charge, ifdipole, d_dipstr,
                              d_dipvec, ifpot, d_pot, iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg,
                              iffldtarg, d_fldtarg, s);
}

int fmm3d_h3ddirect_points_device(const double *zk, int nsource, const double *d_source, int ifcharge,
                                  const double *d_charge, int ifdipole, const double *d_dipstr,
                                  const double *d_dipvec, int npts, const double *d_pts, const int *d_skip,
                                  double *d_pot, double *d_fld, void *stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    Status st;
    g_launch_count = 0;
    DBuf<double> sx, sy, sz, vx, vy, vz, px, py, pz;
    DBuf<double2> q, dq, o0, o1, o2, o3;
    PointsSoA P;
    split_points(nsource, d_source, d_charge, d_dipstr, d_dipvec, ifcharge, ifdipole, sx, sy, sz, q, dq, vx, vy, vz,
                 P, s, st);
    bool ok = st.ok() && px.alloc(npts, s, st) && py.alloc(npts, s, st) && pz.alloc(npts, s, st) &&
              o0.alloc(npts, s, st) && o1.alloc(npts, s, st) && o2.alloc(npts, s, st) && o3.alloc(npts, s, st);
    if (!ok) return 8;
    if (npts == 0) return 0;
    k_split_aos<<<div_up(npts, 256), 256, 0, s>>>(npts, d_pts, px.p, py.p, pz.p); FMM_COUNT_LAUNCH();
    OutSoA o;
    o.pot = o0.p; o.fx = o1.p; o.fy = o2.p; o.fz = o3.p;
    launch_hdirect(nsource, P, ifcharge, ifdipole, npts, px.p, py.p, pz.p, d_skip, 0, make_double2(zk[0], zk[1]), o,
                   s, st);
    k_scatter_out<<<div_up(npts, 256), 256, 0, s>>>(npts, nullptr, o, d_pot, d_fld); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = cudaGetErrorString(st.err); return 16; }
    return 0;
}

static HTriIn htri_in(int iprec, const double *tri, const double *norm)
{
    HTriIn t;
    t.tri = tri;
    t.norm = norm;
    // norder / nqtri of hfmm3dtriatarg (src/hfmm3dtria.f:730-751)
    const int norder = (iprec == -2 || iprec == -1) ? 2 : iprec >= 0 ? 4 : 1;
    const int nqtri = (iprec == -2 || iprec == -1) ? 2 : iprec == 0 ? 4 : iprec >= 1 ? 6 : 1;
    t.far = tri_rule_degree(norder);
    t.near_ = tri_rule_degree(nqtri);
    return t;
}

int fmm3d_hfmm3dtriatarg_device(int iprec, const double *zk, int nsource, const double *d_triaflat,
                                const double *d_trianorm, const double *d_source, int ifcharge, const double *d_charge,
                                int ifdipole, const double *d_dipstr, const double *d_dipvec, int ifpot, double *d_pot,
                                int iffld, double *d_fld, int ntarget, const double *d_target, int ifpottarg,
                                double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream)
{
    (void)d_dipvec;   // the dipoles are oriented by the triangles' normals, as in the reference
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream();
    HTriIn t = htri_in(iprec, d_triaflat, d_trianorm);
    return helm_fmm_device(iprec, make_double2(zk[0], zk[1]), nsource, d_source, ifcharge, d_charge, ifdipole,
                           d_dipstr, d_trianorm, ifpot, d_pot, iffld, d_fld, ntarget, d_target, ifpottarg, d_pottarg,
                           iffldtarg, d_fldtarg, s, &t);
}

int fmm3d_h3dtriadirect_points_device(int nqtri, const double *zk, int nsource, const double *d_triaflat,
                                      int ifcharge, const double *d_charge, int ifdipole, const double *d_dipstr,
                                      int npts, const double *d_pts, const int *d_self, int centroids, double *d_pot,
                                      double *d_fld, void *stream)
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
    launch_htri_direct(nsource, t, ifcharge, ifdipole, npts, d_pts, centroids, d_self, make_double2(zk[0], zk[1]),
                       tri_rule_degree(nqtri), d_pot, d_fld, s, st);
    FMM_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok()) { g_ti.err = std::string(st.where ? st.where : "") + ": " + cudaGetErrorString(st.err); return 16; }
    return 0;
}

void hfmm3dtriatarg_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *triaflat,
                     const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                     const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                     const int *iffld, double *fld, const int *ntarget, const double *target, const int *ifpottarg,
                     double *pottarg, const int *iffldtarg, double *fldtarg)
{
    (void)dipvec;
    const int ip = *iprec, ns = *nsource, ifc = *ifcharge, ifd = *ifdipole, ifp = *ifpot, iff = *iffld;
    const double2 k = make_double2(zk[0], zk[1]);
    *ier = tri_host(ns, triaflat, trianorm, source, ifc, charge, ifd, dipstr, ifp, pot, iff, fld, *ntarget, target,
                    *ifpottarg, pottarg, *iffldtarg, fldtarg,
                    [&](const double *t_, const double *n_, const double *s_, const double *q, const double *dq,
                        double *po, double *fo, int nt, const double *tg, int ipt, double *pt, int ift, double *ft,
                        cudaStream_t s) {
                        HTriIn t = htri_in(ip, t_, n_);
                        return helm_fmm_device(ip, k, ns, s_, ifc, q, ifd, dq, n_, ifp, po, iff, fo, nt, tg, ipt, pt,
                                               ift, ft, s, &t);
                    });
}

void hfmm3dtriaself_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *triaflat,
                     const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                     const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                     const int *iffld, double *fld)
{
    int zero = 0;
    hfmm3dtriatarg_(ier, iprec, zk, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, dipvec,
                    ifpot, pot, iffld, fld, &zero, source, &zero, nullptr, &zero, nullptr);
}

void hfmm3dtria_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *triaflat,
                 const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                 const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                 const int *iffld, double *fld)
{
    hfmm3dtriaself_(ier, iprec, zk, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, dipvec,
                    ifpot, pot, iffld, fld);
}

void h3dtriadirect_(const int *nqtri, const double *zk, const int *nsource, const double *triaflat,
                    const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                    const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                    const int *iffld, double *fld, const int *ntarget, const double *target, const int *ifpottarg,
                    double *pottarg, const int *iffldtarg, double *fldtarg)
{
    (void)trianorm;
    (void)dipvec;
    const int ns = *nsource, ifc = *ifcharge, ifd = *ifdipole, ifp = *ifpot, iff = *iffld, nq = *nqtri;
    tri_host(ns, triaflat, nullptr, source, ifc, charge, ifd, dipstr, ifp, pot, iff, fld, *ntarget, target, *ifpottarg,
             pottarg, *iffldtarg, fldtarg,
             [&](const double *t_, const double *, const double *s_, const double *q, const double *dq, double *po,
                 double *fo, int nt, const double *tg, int ipt, double *pt, int ift, double *ft, cudaStream_t s) {
                 int e = 0;
                 if (ifp == 1 || iff == 1)
                     e = fmm3d_h3dtriadirect_points_device(nq, zk, ns, t_, ifc, q, ifd, dq, ns, s_, nullptr, 1,
                                                           ifp == 1 ? po : nullptr, iff == 1 ? fo : nullptr, s);
                 if (!e && nt && (ipt == 1 || ift == 1))
                     e = fmm3d_h3dtriadirect_points_device(nq, zk, ns, t_, ifc, q, ifd, dq, nt, tg, nullptr, 0,
                                                           ipt == 1 ? pt : nullptr, ift == 1 ? ft : nullptr, s);
                 return e;
             });
}

void hfmm3dparttarg_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *source,
                     const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                     const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld,
                     const int *ntarget, const double *target, const int *ifpottarg, double *pottarg,
                     const int *iffldtarg, double *fldtarg)
{
    int ns = *nsource, nt = *ntarget, ip = *iprec;
    double2 k = make_double2(zk[0], zk[1]);
    *ier = with_device_arrays(
        ns, source, *ifcharge, charge, *ifdipole, dipstr, dipvec, *ifpot, pot, *iffld, fld, nt, target, *ifpottarg,
        pottarg, *iffldtarg, fldtarg,
        [&](const double *s_, const double *q, const double *dq, const double *dv, double *po, double *fo,
            const double *t_, double *pt, double *ft, cudaStream_t s) {
            return helm_fmm_device(ip, k, ns, s_, *ifcharge, q, *ifdipole, dq, dv, *ifpot, po, *iffld, fo, nt, t_,
                                   *ifpottarg, pt, *iffldtarg, ft, s);
        },
        true);
}

void hfmm3dpartself_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *source,
                     const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                     const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld)
{
    int zero = 0;
    hfmm3dparttarg_(ier, iprec, zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, pot, iffld,
                    fld, &zero, source, &zero, nullptr, &zero, nullptr);
}

void hfmm3dpart_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *source,
                 const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                 const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld)
{
    hfmm3dpartself_(ier, iprec, zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, pot, iffld,
                    fld);
}

void h3dpartdirect_(const double *zk, const int *nsource, const double *source, const int *ifcharge,
                    const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                    const int *ifpot, double *pot, const int *iffld, double *fld, const int *ntarget,
                    const double *target, const int *ifpottarg, double *pottarg, const int *iffldtarg,
                    double *fldtarg)
{
    int ns = *nsource, nt = *ntarget;
    double2 k = make_double2(zk[0], zk[1]);
    with_device_arrays(ns, source, *ifcharge, charge, *ifdipole, dipstr, dipvec, *ifpot, pot, *iffld, fld, nt, target,
                       *ifpottarg, pottarg, *iffldtarg, fldtarg,
                       [&](const double *s_, const double *q, const double *dq, const double *dv, double *po,
                           double *fo, const double *t_, double *pt, double *ft, cudaStream_t s) {
                           return helm_direct_device(k, ns, s_, *ifcharge, q, *ifdipole, dq, dv, *ifpot, po, *iffld,
                                                     fo, nt, t_, *ifpottarg, pt, *iffldtarg, ft, s);
                       });
}

}  // extern "C"
