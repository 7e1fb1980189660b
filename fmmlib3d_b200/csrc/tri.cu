// Laplace layer potentials on flat triangles: the kernels particular to the
// triangle FMM (the far-field passes are the particle FMM's, run on the
// triangles' quadrature nodes).
//
// Near field (direct3dtritarglaps2 / direct3dtritarglapd2 and the self terms
// direct3dtrilaps2 / direct3dtrilapd2, src/triquadflatlib.f:147-818): for a
// triangle with unit density, at x,
//   S = int 1/|x-y| dS,   D = int n.(x-y)/|x-y|^3 dS   (n: vertex-order normal),
// and their gradients, in closed form: with h = n.(x - v1), D the signed
// solid angle the triangle subtends at x, and per edge a -> b (unit tangent
// t, outward in-plane normal m = t x n), s- = (a-x).t, s+ = (b-x).t,
// p = (a-x).m, R- = |a-x|, R+ = |b-x|, f = log((R+ + s+)/(R- + s-)):
//   S = sum p f - h D,   grad S = -sum m f - n D,
//   grad D = -sum (u x w)(|u|+|w|)/(|u||w|(|u||w|+u.w)),   u = x - a, w = x - b.  At a triangle's own centroid h is taken as 0, as the
// reference does (iquad = 0): the jumps of grad S . n and of D across the
// triangle are split evenly (both vanish), grad D is continuous there.
// Fields are -grad.
#include "tri.cuh"

#include <cmath>

namespace fmm {

constexpr int kTriGeo = 30;

TriRule tri_rule(int iprec)
{
    // nqtri of lfmm3dtriatarg: 2 for iprec -2 / -1, 4 for 0, 6 for >= 1, else 1
    int norder = (iprec == -2 || iprec == -1) ? 2 : iprec == 0 ? 4 : iprec >= 1 ? 6 : 1;
    TriRule r;
    if (norder <= 1) {
        r.n = 1;
        r.xi[0] = r.eta[0] = 1.0 / 3.0;
        r.w[0] = 1.0;
        return r;
    }
    const int k = norder / 2 + 1;   // exact to degree 2k - 2 = norder
    std::vector<double> x, w;
    gauss_legendre(k, x, w);
    r.n = 0;
    for (int i = 0; i < k; i++)
        for (int j = 0; j < k; j++) {
            const double u = 0.5 * (x[i] + 1), v = 0.5 * (x[j] + 1);
            r.xi[r.n] = u;
            r.eta[r.n] = (1 - u) * v;
            r.w[r.n] = 2 * (0.5 * w[i]) * (0.5 * w[j]) * (1 - u);   // the reference triangle's area is 1/2
            r.n++;
        }
    return r;
}

int tri_nbox(int iprec, int ns, int nt)
{
    switch (iprec) {
    case -2: return 8 / 3;
    case -1: return 15 / 3;
    case 0: return 30 / 3;
    case 1: return 60 / 3;
    case 2: return 120 / 3;
    case 3: return 240 / 3;
    case 4: return 480 / 3;
    case 5: return 700 / 3;
    case 6: return ns + nt;
    }
    return -1;
}

__global__ void k_tri_gather(int n, const int *perm, const double *tri, const double *norm, const double *q,
                             const double *dq, int ifcharge, int ifdipole, TriRule rule, TriSoA t, PointsSoA nodes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long j = perm ? perm[i] : i;
    double v[9];
    for (int c = 0; c < 9; c++) v[c] = tri[9 * j + c];
    const double e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]}, e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
    double nr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double len = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]), area = 0.5 * len;
    for (int c = 0; c < 3; c++) nr[c] /= len;
    double *g = t.geo + (size_t)kTriGeo * i;
    for (int c = 0; c < 9; c++) g[c] = v[c];
    for (int c = 0; c < 3; c++) g[9 + c] = nr[c];
    for (int k = 0; k < 3; k++) {
        const int a = k, b = (k + 1) % 3;
        double tv[3] = {v[3 * b] - v[3 * a], v[3 * b + 1] - v[3 * a + 1], v[3 * b + 2] - v[3 * a + 2]};
        const double L = sqrt(tv[0] * tv[0] + tv[1] * tv[1] + tv[2] * tv[2]);
        for (int c = 0; c < 3; c++) tv[c] /= L;
        g[12 + 3 * k] = tv[0]; g[13 + 3 * k] = tv[1]; g[14 + 3 * k] = tv[2];
        g[21 + 3 * k] = tv[1] * nr[2] - tv[2] * nr[1];
        g[22 + 3 * k] = tv[2] * nr[0] - tv[0] * nr[2];
        g[23 + 3 * k] = tv[0] * nr[1] - tv[1] * nr[0];
    }
    double2 qi = cmk(0, 0), di = cmk(0, 0);
    if (ifcharge) { qi = cmk(q[2 * j], q[2 * j + 1]); t.q[i] = qi; }
    if (ifdipole) { di = cmk(dq[2 * j], dq[2 * j + 1]); t.dq[i] = di; }
    for (int k = 0; k < rule.n; k++) {
        const long o = (long)i * rule.n + k;
        nodes.x[o] = v[0] + rule.xi[k] * e1[0] + rule.eta[k] * e2[0];
        nodes.y[o] = v[1] + rule.xi[k] * e1[1] + rule.eta[k] * e2[1];
        nodes.z[o] = v[2] + rule.xi[k] * e1[2] + rule.eta[k] * e2[2];
        const double wa = rule.w[k] * area;
        if (ifcharge) nodes.q[o] = cscal(wa, qi);
        if (ifdipole) {
            nodes.dq[o] = cscal(wa, di);
            // the far field orients the dipoles by trianorm, as l3dformmptrid2_add does
            nodes.vx[o] = norm[3 * j]; nodes.vy[o] = norm[3 * j + 1]; nodes.vz[o] = norm[3 * j + 2];
        }
    }
}

void launch_tri_gather(int n, const int *perm, const double *tri, const double *norm, const double *q,
                       const double *dq, int ifcharge, int ifdipole, const TriRule &rule, TriSoA t, PointsSoA nodes,
                       cudaStream_t s, Status &st)
{
    if (n <= 0 || !st.ok()) return;
    k_tri_gather<<<(n + 127) / 128, 128, 0, s>>>(n, perm, tri, norm, q, dq, ifcharge == 1, ifdipole == 1, rule, t,
                                                 nodes);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

__global__ void k_scale_ranges(int nb, const int *src0, const int *nsrc, int k, int *qs0, int *qns)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    qs0[b] = src0[b] * k;
    qns[b] = nsrc[b] * k;
}

void launch_scale_ranges(int nboxes, const int *src0, const int *nsrc, int k, int *qsrc0, int *qnsrc, cudaStream_t s,
                         Status &st)
{
    if (nboxes <= 0 || !st.ok()) return;
    k_scale_ranges<<<(nboxes + 255) / 256, 256, 0, s>>>(nboxes, src0, nsrc, k, qsrc0, qnsrc);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// One triangle (geometry g, 30 doubles) at x: S, grad S (CHG), D, grad D (DIP).
// The sum of the edge angles beta is the solid angle the triangle subtends,
// taken in one atan2 (Van Oosterom and Strackee, IEEE Trans. Biomed. Eng. 30,
// 1983): D = 2 atan2(-a.(b x c), |a||b||c| + (a.b)|c| + (a.c)|b| + (b.c)|a|)
// with a, b, c = v1 - x, v2 - x, v3 - x; then S = sum p f - h D and
// grad S = -sum m f - n D.
template <bool CHG, bool DIP>
__device__ __forceinline__ void tri_pair(const double *g, double x0, double x1, double x2, bool self, bool fld,
                                         double &S, double (&gS)[3], double &D, double (&gD)[3])
{
    double d[3][3], R[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        d[k][0] = g[3 * k] - x0;
        d[k][1] = g[3 * k + 1] - x1;
        d[k][2] = g[3 * k + 2] - x2;
        R[k] = sqrt(d[k][0] * d[k][0] + d[k][1] * d[k][1] + d[k][2] * d[k][2]);
    }
    const double *n = g + 9;
    const double h = self ? 0.0 : -(n[0] * d[0][0] + n[1] * d[0][1] + n[2] * d[0][2]);
    double om = 0;
    if (!self) {
        const double bc0 = d[1][1] * d[2][2] - d[1][2] * d[2][1], bc1 = d[1][2] * d[2][0] - d[1][0] * d[2][2],
                     bc2 = d[1][0] * d[2][1] - d[1][1] * d[2][0];
        const double num = d[0][0] * bc0 + d[0][1] * bc1 + d[0][2] * bc2;
        const double ab = d[0][0] * d[1][0] + d[0][1] * d[1][1] + d[0][2] * d[1][2];
        const double ac = d[0][0] * d[2][0] + d[0][1] * d[2][1] + d[0][2] * d[2][2];
        const double bcd = d[1][0] * d[2][0] + d[1][1] * d[2][1] + d[1][2] * d[2][2];
        const double den = R[0] * R[1] * R[2] + ab * R[2] + ac * R[1] + bcd * R[0];
        om = 2.0 * atan2(-num, den);
    }
    double spf = 0, gm[3] = {0, 0, 0}, bs[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int a = i, b = (i + 1) % 3;
        if (CHG) {
            const double *t = g + 12 + 3 * i, *m = g + 21 + 3 * i;
            const double sm = d[a][0] * t[0] + d[a][1] * t[1] + d[a][2] * t[2];
            const double sp = d[b][0] * t[0] + d[b][1] * t[1] + d[b][2] * t[2];
            const double pd = d[a][0] * m[0] + d[a][1] * m[1] + d[a][2] * m[2];
            const double f = (sp + sm >= 0) ? log((R[b] + sp) / (R[a] + sm)) : log((R[a] - sm) / (R[b] - sp));
            spf += pd * f;
            if (fld) { gm[0] += m[0] * f; gm[1] += m[1] * f; gm[2] += m[2] * f; }
        }
        if (DIP && fld) {
            const double co = (R[a] + R[b]) /
                              (R[a] * R[b] * (R[a] * R[b] + d[a][0] * d[b][0] + d[a][1] * d[b][1] + d[a][2] * d[b][2]));
            bs[0] += (d[a][1] * d[b][2] - d[a][2] * d[b][1]) * co;
            bs[1] += (d[a][2] * d[b][0] - d[a][0] * d[b][2]) * co;
            bs[2] += (d[a][0] * d[b][1] - d[a][1] * d[b][0]) * co;
        }
    }
    if (CHG) {
        S = spf - h * om;
        gS[0] = -gm[0] - n[0] * om;
        gS[1] = -gm[1] - n[1] * om;
        gS[2] = -gm[2] - n[2] * om;
    }
    if (DIP) {
        D = om;
        gD[0] = -bs[0]; gD[1] = -bs[1]; gD[2] = -bs[2];
    }
}

constexpr int kTriThreads = 128;

// Adds triangle j's contribution (charge q, dipstr dq) at one point to pot / fld sums.
template <bool CHG, bool DIP>
__device__ __forceinline__ void tri_accum(const double *g, double2 q, double2 dq, double x0, double x1, double x2,
                                          bool self, bool fld, double (&acc)[8])
{
    double S = 0, D = 0, gS[3] = {0, 0, 0}, gD[3] = {0, 0, 0};
    tri_pair<CHG, DIP>(g, x0, x1, x2, self, fld, S, gS, D, gD);
    if (CHG) {
        acc[0] = fma(q.x, S, acc[0]);
        acc[1] = fma(q.y, S, acc[1]);
        if (fld)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                acc[2 + 2 * c] = fma(-q.x, gS[c], acc[2 + 2 * c]);
                acc[3 + 2 * c] = fma(-q.y, gS[c], acc[3 + 2 * c]);
            }
    }
    if (DIP) {
        acc[0] = fma(dq.x, D, acc[0]);
        acc[1] = fma(dq.y, D, acc[1]);
        if (fld)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                acc[2 + 2 * c] = fma(-dq.x, gD[c], acc[2 + 2 * c]);
                acc[3 + 2 * c] = fma(-dq.y, gD[c], acc[3 + 2 * c]);
            }
    }
}

// A leaf holds at most nbox (<= 233 below iprec 6) triangles, usually ~10-20:
// one thread per evaluation point would leave most of a CTA idle.  So the
// CTA's threads are split into G groups of np threads, np = min(points left,
// 128): thread (group g, lane e) evaluates point e against every G-th staged
// triangle from g on, and the groups' partial sums are added in shared memory
// in group order (a fixed order for a given leaf).
template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kTriThreads) k_p2p_tri(const int *leaves, TreeView tv, TriSoA t, const double *sx,
                                                         const double *sy, const double *sz, const double *tx,
                                                         const double *ty, const double *tz, OutSoA outs,
                                                         OutSoA outt, int do_src, int do_trg, int want_fs,
                                                         int want_ft)
{
    __shared__ double sg[kTriThreads * kTriGeo];
    __shared__ double2 sq[kTriThreads], sd[kTriThreads];
    __shared__ double red[8][kTriThreads];
    const int b = leaves[blockIdx.x];
    const int s0 = tv.src0[b], ns = do_src ? tv.nsrc[b] : 0;
    const int t0 = tv.trg0[b], nt = do_trg ? tv.ntrg[b] : 0;
    const int ne = ns + nt;
    const int l1a = tv.l1_start[b], nl = 1 + tv.l1_start[b + 1] - l1a;
    for (int e0 = 0; e0 < ne; e0 += kTriThreads) {
        const int np = min(kTriThreads, ne - e0);
        const int G = kTriThreads / np;
        const int lane = threadIdx.x % np, grp = threadIdx.x / np;
        const int e = e0 + lane;
        const bool act = grp < G;
        const bool is_src = e < ns;
        double x0 = 0, x1 = 0, x2 = 0;
        int self = -1;
        if (act) {
            if (is_src) { const int i = s0 + e; x0 = sx[i]; x1 = sy[i]; x2 = sz[i]; self = i; }
            else { const int i = t0 + e - ns; x0 = tx[i]; x1 = ty[i]; x2 = tz[i]; }
        }
        const bool fld = is_src ? want_fs != 0 : want_ft != 0;
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < nl; j++) {
            const int jb = j == 0 ? b : tv.l1_idx[l1a + j - 1];
            const int js0 = tv.src0[jb], jn = tv.nsrc[jb];
            for (int c0 = 0; c0 < jn; c0 += kTriThreads) {
                const int cn = min(kTriThreads, jn - c0);
                __syncthreads();
                const double *gsrc = t.geo + (size_t)kTriGeo * (js0 + c0);
                for (int k = threadIdx.x; k < cn * kTriGeo; k += kTriThreads) sg[k] = gsrc[k];
                if (threadIdx.x < cn) {
                    if (CHG) sq[threadIdx.x] = t.q[js0 + c0 + threadIdx.x];
                    if (DIP) sd[threadIdx.x] = t.dq[js0 + c0 + threadIdx.x];
                }
                __syncthreads();
                if (!act) continue;
                const int selfk = self - (js0 + c0);
                for (int k = grp; k < cn; k += G)
                    tri_accum<CHG, DIP>(sg + kTriGeo * k, CHG ? sq[k] : cmk(0, 0), DIP ? sd[k] : cmk(0, 0), x0, x1,
                                        x2, k == selfk, fld, acc);
            }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < 8; c++) red[c][threadIdx.x] = act ? acc[c] : 0.0;
        __syncthreads();
        if (threadIdx.x < np) {
            double sum[8];
#pragma unroll
            for (int c = 0; c < 8; c++) {
                sum[c] = red[c][threadIdx.x];
                for (int g = 1; g < G; g++) sum[c] += red[c][threadIdx.x + g * np];
            }
            const OutSoA &o = is_src ? outs : outt;
            const int i = is_src ? s0 + e : t0 + e - ns;
            if (o.pot) o.pot[i] = cadd(o.pot[i], cmk(sum[0], sum[1]));
            if (fld && o.fx) {
                o.fx[i] = cadd(o.fx[i], cmk(sum[2], sum[3]));
                o.fy[i] = cadd(o.fy[i], cmk(sum[4], sum[5]));
                o.fz[i] = cadd(o.fz[i], cmk(sum[6], sum[7]));
            }
        }
    }
}

void launch_p2p_tri(const int *leaves, int nleaves, const TreeView &tv, const TriSoA &t, const double *sx,
                    const double *sy, const double *sz, const double *tx, const double *ty, const double *tz,
                    OutSoA outs, OutSoA outt, int ifcharge, int ifdipole, int do_src, int do_trg, int want_fs,
                    int want_ft, cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok() || !(do_src || do_trg)) return;
    const bool c = ifcharge == 1, d = ifdipole == 1;
    if (c && d)
        k_p2p_tri<true, true><<<nleaves, kTriThreads, 0, s>>>(leaves, tv, t, sx, sy, sz, tx, ty, tz, outs, outt,
                                                              do_src, do_trg, want_fs, want_ft);
    else if (c)
        k_p2p_tri<true, false><<<nleaves, kTriThreads, 0, s>>>(leaves, tv, t, sx, sy, sz, tx, ty, tz, outs, outt,
                                                               do_src, do_trg, want_fs, want_ft);
    else if (d)
        k_p2p_tri<false, true><<<nleaves, kTriThreads, 0, s>>>(leaves, tv, t, sx, sy, sz, tx, ty, tz, outs, outt,
                                                               do_src, do_trg, want_fs, want_ft);
    else
        return;
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// l3dtriadirect: one point per thread against every triangle, staged in chunks.
template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kTriThreads) k_tri_direct(int ntri, TriSoA t, int npts, const double *pts,
                                                            int centroids, const int *self_idx, int want_f,
                                                            double *pot, double *fld)
{
    __shared__ double sg[kTriThreads * kTriGeo];
    __shared__ double2 sq[kTriThreads], sd[kTriThreads];
    const int i = blockIdx.x * kTriThreads + threadIdx.x;
    const bool act = i < npts;
    double x0 = 0, x1 = 0, x2 = 0;
    int self = -1;
    if (act) {
        x0 = pts[3L * i]; x1 = pts[3L * i + 1]; x2 = pts[3L * i + 2];
        if (self_idx) self = self_idx[i];
        else if (centroids) self = i;
    }
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c0 = 0; c0 < ntri; c0 += kTriThreads) {
        const int cn = min(kTriThreads, ntri - c0);
        __syncthreads();
        const double *gsrc = t.geo + (size_t)kTriGeo * c0;
        for (int k = threadIdx.x; k < cn * kTriGeo; k += kTriThreads) sg[k] = gsrc[k];
        if (threadIdx.x < cn) {
            if (CHG) sq[threadIdx.x] = t.q[c0 + threadIdx.x];
            if (DIP) sd[threadIdx.x] = t.dq[c0 + threadIdx.x];
        }
        __syncthreads();
        if (!act) continue;
        for (int k = 0; k < cn; k++)
            tri_accum<CHG, DIP>(sg + kTriGeo * k, CHG ? sq[k] : cmk(0, 0), DIP ? sd[k] : cmk(0, 0), x0, x1, x2,
                                c0 + k == self, want_f != 0, acc);
    }
    if (!act) return;
    if (pot) { pot[2L * i] = acc[0]; pot[2L * i + 1] = acc[1]; }
    if (fld)
        for (int c = 0; c < 6; c++) fld[6L * i + c] = acc[2 + c];
}

void launch_tri_direct(int ntri, const TriSoA &t, int ifcharge, int ifdipole, int npts, const double *pts,
                       int centroids, const int *self_idx, double *pot, double *fld, cudaStream_t s, Status &st)
{
    if (npts <= 0 || !st.ok()) return;
    const bool c = ifcharge == 1, d = ifdipole == 1;
    const int grid = (npts + kTriThreads - 1) / kTriThreads;
    if (!c && !d) {
        if (pot) FMM_TRY(st, cudaMemsetAsync(pot, 0, sizeof(double) * 2 * npts, s));
        if (fld) FMM_TRY(st, cudaMemsetAsync(fld, 0, sizeof(double) * 6 * npts, s));
        return;
    }
    if (c && d) k_tri_direct<true, true><<<grid, kTriThreads, 0, s>>>(ntri, t, npts, pts, centroids, self_idx, fld != nullptr, pot, fld);
    else if (c) k_tri_direct<true, false><<<grid, kTriThreads, 0, s>>>(ntri, t, npts, pts, centroids, self_idx, fld != nullptr, pot, fld);
    else k_tri_direct<false, true><<<grid, kTriThreads, 0, s>>>(ntri, t, npts, pts, centroids, self_idx, fld != nullptr, pot, fld);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// ================================================================ Helmholtz triangles
// Near field of hfmm3dtriatarg (direct3dtritarghelms3, direct3dtrihelms2,
// direct3dtritarghelmd3, direct3dtrihelmd2 with triquadhelm2 / triquadselfhelm
// / triquadhelmd2 / triquadselfhelmd, src/triquadflatlib.f:819-2356): the
// Laplace part of e^{ikr}/r integrated exactly (tri_pair), the difference by
// the near rule on the triangle (series when |kr| < 0.01).  With z = ikr,
// d = x - y, h = n.(x - v1), F = e^z (z-1) + 1:
//   single layer: (e^z - 1)/r, gradient (d/r) F/r^2;
//   double layer: h f2, gradient n f2 + h f2' d/r, f2 = -F/r^3,
//   f2' = k^2 e^z/r^2 + 3F/r^4.
// At the triangle's own centroid (h = 0): the single layer's gradient rule
// takes (d/r)(F/r^2 - (ik)^2/2) and adds (ik)^2/2 int d/r = -(ik)^2/2 sum_e
// m_e int_e r dl (closed form); the double layer's value and in-plane
// gradient vanish, its normal gradient is int (f2 - k^2/(2r)) + (k^2/2) S.
__device__ __forceinline__ double2 cexp2(double2 z)
{
    double sn, cs;
    sincos(z.y, &sn, &cs);
    const double e = exp(z.x);
    return cmk(e * cs, e * sn);
}

template <bool CHG, bool DIP>
__device__ __forceinline__ void htri_pair(const double *g, double x0, double x1, double x2, bool self, bool fld,
                                          double2 ik, const TriRule &rule, double2 &S, double2 (&gS)[3], double2 &D,
                                          double2 (&gD)[3])
{
    double Sl = 0, Dl = 0, gSl[3] = {0, 0, 0}, gDl[3] = {0, 0, 0};
    tri_pair<true, DIP>(g, x0, x1, x2, self, true, Sl, gSl, Dl, gDl);   // S is needed by the double layer's self term
    const double *n = g + 9;
    const double e1[3] = {g[3] - g[0], g[4] - g[1], g[5] - g[2]}, e2[3] = {g[6] - g[0], g[7] - g[1], g[8] - g[2]};
    const double c0 = e1[1] * e2[2] - e1[2] * e2[1], c1 = e1[2] * e2[0] - e1[0] * e2[2], c2 = e1[0] * e2[1] - e1[1] * e2[0];
    const double area = 0.5 * sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    const double h = self ? 0.0 : n[0] * (x0 - g[0]) + n[1] * (x1 - g[1]) + n[2] * (x2 - g[2]);
    const double2 ik2 = cmul(ik, ik);
    const double2 hik2 = cscal(0.5, ik2);
    double2 sp = cmk(0, 0), dp = cmk(0, 0), dn = cmk(0, 0);
    double2 sg[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)}, dg[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    for (int q = 0; q < rule.n; q++) {
        const double d[3] = {x0 - (g[0] + rule.xi[q] * e1[0] + rule.eta[q] * e2[0]),
                             x1 - (g[1] + rule.xi[q] * e1[1] + rule.eta[q] * e2[1]),
                             x2 - (g[2] + rule.xi[q] * e1[2] + rule.eta[q] * e2[2])};
        // a node on x itself (the one-node rule at a triangle's own centroid) adds the limit of the
        // bounded difference kernel: its value ik, a zero gradient
        const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], rr = sqrt(r2), ir = rr > 0 ? 1.0 / rr : 0.0;
        const double w = rule.w[q] * area;
        const double2 z = cscal(rr, ik);
        double2 gv, Fr2, f2, f2p, f2s;
        if (z.x * z.x + z.y * z.y < 1e-4) {
            const double2 ik3 = cmul(ik2, ik), ik4 = cmul(ik3, ik), ik5 = cmul(ik4, ik), ik6 = cmul(ik5, ik);
            const double2 z2 = cmul(z, z), z3 = cmul(z2, z), z4 = cmul(z3, z);
            double2 ser = cmk(1.0 + z.x / 2 + z2.x / 6 + z3.x / 24 + z4.x / 120, z.y / 2 + z2.y / 6 + z3.y / 24 + z4.y / 120);
            gv = cmul(ik, ser);
            Fr2 = cadd(cadd(hik2, cscal(rr / 3.0, ik3)), cadd(cscal(r2 / 8.0, ik4), cscal(r2 * rr / 30.0, ik5)));
            f2s = cscal(-1.0, cadd(cadd(cscal(1.0 / 3.0, ik3), cscal(rr / 8.0, ik4)),
                                   cadd(cscal(r2 / 30.0, ik5), cscal(r2 * rr / 144.0, ik6))));
            f2 = csub(f2s, cscal(ir, hik2));
            f2p = csub(csub(cscal(ir * ir, hik2), cscal(1.0 / 8.0, ik4)),
                       cadd(cscal(2.0 * rr / 30.0, ik5), cscal(3.0 * r2 / 144.0, ik6)));
        } else {
            const double2 E = cexp2(z);
            const double2 F = cadd(cmul(E, cmk(z.x - 1.0, z.y)), cmk(1.0, 0.0));
            gv = cscal(ir, cmk(E.x - 1.0, E.y));
            Fr2 = cscal(ir * ir, F);
            f2 = cscal(-ir * ir * ir, F);
            f2s = cadd(f2, cscal(ir, hik2));
            f2p = cadd(cscal(-ir * ir, cmul(ik2, E)), cscal(3.0 * ir * ir * ir * ir, F));
        }
        if (CHG) {
            sp = cadd(sp, cscal(w, gv));
            if (fld) {
                const double2 t = self ? csub(Fr2, hik2) : Fr2;
#pragma unroll
                for (int c = 0; c < 3; c++) sg[c] = cadd(sg[c], cscal(w * d[c] * ir, t));
            }
        }
        if (DIP) {
            if (self) {
                if (fld) dn = cadd(dn, cscal(w, f2s));
            } else {
                dp = cadd(dp, cscal(w * h, f2));
                if (fld)
#pragma unroll
                    for (int c = 0; c < 3; c++)
                        dg[c] = cadd(dg[c], cadd(cscal(w * n[c], f2), cscal(w * h * d[c] * ir, f2p)));
            }
        }
    }
    if (CHG) {
        S = cadd(cmk(Sl, 0), sp);
#pragma unroll
        for (int c = 0; c < 3; c++) gS[c] = cadd(cmk(gSl[c], 0), sg[c]);
        if (self && fld) {
            // (ik)^2/2 int d/r dS = -(ik)^2/2 sum_e m_e int_e r dl (the triangle's plane)
            double dv[3][3], R[3], J[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                dv[k][0] = g[3 * k] - x0; dv[k][1] = g[3 * k + 1] - x1; dv[k][2] = g[3 * k + 2] - x2;
                R[k] = sqrt(dv[k][0] * dv[k][0] + dv[k][1] * dv[k][1] + dv[k][2] * dv[k][2]);
            }
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const int a = i, b = (i + 1) % 3;
                const double *t = g + 12 + 3 * i, *m = g + 21 + 3 * i;
                const double sm = dv[a][0] * t[0] + dv[a][1] * t[1] + dv[a][2] * t[2];
                const double spp = dv[b][0] * t[0] + dv[b][1] * t[1] + dv[b][2] * t[2];
                const double pd = dv[a][0] * m[0] + dv[a][1] * m[1] + dv[a][2] * m[2];
                const double f = (spp + sm >= 0) ? log((R[b] + spp) / (R[a] + sm)) : log((R[a] - sm) / (R[b] - spp));
                const double line = 0.5 * (spp * R[b] - sm * R[a] + pd * pd * f);
                J[0] -= m[0] * line; J[1] -= m[1] * line; J[2] -= m[2] * line;
            }
#pragma unroll
            for (int c = 0; c < 3; c++) gS[c] = cadd(gS[c], cscal(J[c], hik2));
        }
    }
    if (DIP) {
        if (self) {
            D = cmk(0, 0);
            const double2 nrm = csub(dn, cscal(Sl, hik2));
#pragma unroll
            for (int c = 0; c < 3; c++) gD[c] = cadd(cmk(gDl[c], 0), cscal(n[c], nrm));
        } else {
            D = cadd(cmk(Dl, 0), dp);
#pragma unroll
            for (int c = 0; c < 3; c++) gD[c] = cadd(cmk(gDl[c], 0), dg[c]);
        }
    }
}

template <bool CHG, bool DIP>
__device__ __forceinline__ void htri_accum(const double *g, double2 q, double2 dq, double x0, double x1, double x2,
                                           bool self, bool fld, double2 ik, const TriRule &rule, double2 (&acc)[4])
{
    double2 S = cmk(0, 0), D = cmk(0, 0), gS[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)}, gD[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    htri_pair<CHG, DIP>(g, x0, x1, x2, self, fld, ik, rule, S, gS, D, gD);
    if (CHG) {
        cfma(acc[0], q, S);
        if (fld)
#pragma unroll
            for (int c = 0; c < 3; c++) cfma(acc[1 + c], cmk(-q.x, -q.y), gS[c]);
    }
    if (DIP) {
        cfma(acc[0], dq, D);
        if (fld)
#pragma unroll
            for (int c = 0; c < 3; c++) cfma(acc[1 + c], cmk(-dq.x, -dq.y), gD[c]);
    }
}

// As k_p2p_tri, with complex sums.
template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kTriThreads) k_hp2p_tri(const int *leaves, TreeView tv, TriSoA t, const double *sx,
                                                          const double *sy, const double *sz, const double *tx,
                                                          const double *ty, const double *tz, double2 zk, TriRule rule,
                                                          OutSoA outs, OutSoA outt, int do_src, int do_trg,
                                                          int want_fs, int want_ft)
{
    __shared__ double sg[kTriThreads * kTriGeo];
    __shared__ double2 sq[kTriThreads], sd[kTriThreads];
    __shared__ double2 red[4][kTriThreads];
    const double2 ik = cmk(-zk.y, zk.x);
    const int b = leaves[blockIdx.x];
    const int s0 = tv.src0[b], ns = do_src ? tv.nsrc[b] : 0;
    const int t0 = tv.trg0[b], nt = do_trg ? tv.ntrg[b] : 0;
    const int ne = ns + nt;
    const int l1a = tv.l1_start[b], nl = 1 + tv.l1_start[b + 1] - l1a;
    for (int e0 = 0; e0 < ne; e0 += kTriThreads) {
        const int np = min(kTriThreads, ne - e0);
        const int G = kTriThreads / np;
        const int lane = threadIdx.x % np, grp = threadIdx.x / np;
        const int e = e0 + lane;
        const bool act = grp < G;
        const bool is_src = e < ns;
        double x0 = 0, x1 = 0, x2 = 0;
        int self = -1;
        if (act) {
            if (is_src) { const int i = s0 + e; x0 = sx[i]; x1 = sy[i]; x2 = sz[i]; self = i; }
            else { const int i = t0 + e - ns; x0 = tx[i]; x1 = ty[i]; x2 = tz[i]; }
        }
        const bool fld = is_src ? want_fs != 0 : want_ft != 0;
        double2 acc[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
        for (int j = 0; j < nl; j++) {
            const int jb = j == 0 ? b : tv.l1_idx[l1a + j - 1];
            const int js0 = tv.src0[jb], jn = tv.nsrc[jb];
            for (int c0 = 0; c0 < jn; c0 += kTriThreads) {
                const int cn = min(kTriThreads, jn - c0);
                __syncthreads();
                const double *gsrc = t.geo + (size_t)kTriGeo * (js0 + c0);
                for (int k = threadIdx.x; k < cn * kTriGeo; k += kTriThreads) sg[k] = gsrc[k];
                if (threadIdx.x < cn) {
                    if (CHG) sq[threadIdx.x] = t.q[js0 + c0 + threadIdx.x];
                    if (DIP) sd[threadIdx.x] = t.dq[js0 + c0 + threadIdx.x];
                }
                __syncthreads();
                if (!act) continue;
                const int selfk = self - (js0 + c0);
                for (int k = grp; k < cn; k += G)
                    htri_accum<CHG, DIP>(sg + kTriGeo * k, CHG ? sq[k] : cmk(0, 0), DIP ? sd[k] : cmk(0, 0), x0, x1,
                                         x2, k == selfk, fld, ik, rule, acc);
            }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < 4; c++) red[c][threadIdx.x] = act ? acc[c] : cmk(0, 0);
        __syncthreads();
        if (threadIdx.x < np) {
            double2 sum[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                sum[c] = red[c][threadIdx.x];
                for (int gi = 1; gi < G; gi++) sum[c] = cadd(sum[c], red[c][threadIdx.x + gi * np]);
            }
            const OutSoA &o = is_src ? outs : outt;
            const int i = is_src ? s0 + e : t0 + e - ns;
            if (o.pot) o.pot[i] = cadd(o.pot[i], sum[0]);
            if (fld && o.fx) {
                o.fx[i] = cadd(o.fx[i], sum[1]);
                o.fy[i] = cadd(o.fy[i], sum[2]);
                o.fz[i] = cadd(o.fz[i], sum[3]);
            }
        }
    }
}

void launch_hp2p_tri(const int *leaves, int nleaves, const TreeView &tv, const TriSoA &t, const double *sx,
                     const double *sy, const double *sz, const double *tx, const double *ty, const double *tz,
                     double2 zk, const TriRule &rule, OutSoA outs, OutSoA outt, int ifcharge, int ifdipole,
                     int do_src, int do_trg, int want_fs, int want_ft, cudaStream_t s, Status &st)
{
    if (nleaves == 0 || !st.ok() || !(do_src || do_trg)) return;
    const bool c = ifcharge == 1, d = ifdipole == 1;
    if (c && d)
        k_hp2p_tri<true, true><<<nleaves, kTriThreads, 0, s>>>(leaves, tv, t, sx, sy, sz, tx, ty, tz, zk, rule, outs,
                                                               outt, do_src, do_trg, want_fs, want_ft);
    else if (c)
        k_hp2p_tri<true, false><<<nleaves, kTriThreads, 0, s>>>(leaves, tv, t, sx, sy, sz, tx, ty, tz, zk, rule, outs,
                                                                outt, do_src, do_trg, want_fs, want_ft);
    else if (d)
        k_hp2p_tri<false, true><<<nleaves, kTriThreads, 0, s>>>(leaves, tv, t, sx, sy, sz, tx, ty, tz, zk, rule, outs,
                                                                outt, do_src, do_trg, want_fs, want_ft);
    else
        return;
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

// h3dtriadirect at npts points (self_idx / centroids as in launch_tri_direct).
template <bool CHG, bool DIP>
__global__ void __launch_bounds__(kTriThreads) k_htri_direct(int ntri, TriSoA t, int npts, const double *pts,
                                                             int centroids, const int *self_idx, double2 zk,
                                                             TriRule rule, int want_f, double *pot, double *fld)
{
    __shared__ double sg[kTriThreads * kTriGeo];
    __shared__ double2 sq[kTriThreads], sd[kTriThreads];
    const double2 ik = cmk(-zk.y, zk.x);
    const int i = blockIdx.x * kTriThreads + threadIdx.x;
    const bool act = i < npts;
    double x0 = 0, x1 = 0, x2 = 0;
    int self = -1;
    if (act) {
        x0 = pts[3L * i]; x1 = pts[3L * i + 1]; x2 = pts[3L * i + 2];
        if (self_idx) self = self_idx[i];
        else if (centroids) self = i;
    }
    double2 acc[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    for (int c0 = 0; c0 < ntri; c0 += kTriThreads) {
        const int cn = min(kTriThreads, ntri - c0);
        __syncthreads();
        const double *gsrc = t.geo + (size_t)kTriGeo * c0;
        for (int k = threadIdx.x; k < cn * kTriGeo; k += kTriThreads) sg[k] = gsrc[k];
        if (threadIdx.x < cn) {
            if (CHG) sq[threadIdx.x] = t.q[c0 + threadIdx.x];
            if (DIP) sd[threadIdx.x] = t.dq[c0 + threadIdx.x];
        }
        __syncthreads();
        if (!act) continue;
        for (int k = 0; k < cn; k++)
            htri_accum<CHG, DIP>(sg + kTriGeo * k, CHG ? sq[k] : cmk(0, 0), DIP ? sd[k] : cmk(0, 0), x0, x1, x2,
                                 c0 + k == self, want_f != 0, ik, rule, acc);
    }
    if (!act) return;
    if (pot) { pot[2L * i] = acc[0].x; pot[2L * i + 1] = acc[0].y; }
    if (fld)
        for (int c = 0; c < 3; c++) { fld[6L * i + 2 * c] = acc[1 + c].x; fld[6L * i + 2 * c + 1] = acc[1 + c].y; }
}

void launch_htri_direct(int ntri, const TriSoA &t, int ifcharge, int ifdipole, int npts, const double *pts,
                        int centroids, const int *self_idx, double2 zk, const TriRule &rule, double *pot, double *fld,
                        cudaStream_t s, Status &st)
{
    if (npts <= 0 || !st.ok()) return;
    const bool c = ifcharge == 1, d = ifdipole == 1;
    const int grid = (npts + kTriThreads - 1) / kTriThreads;
    if (!c && !d) {
        if (pot) FMM_TRY(st, cudaMemsetAsync(pot, 0, sizeof(double) * 2 * npts, s));
        if (fld) FMM_TRY(st, cudaMemsetAsync(fld, 0, sizeof(double) * 6 * npts, s));
        return;
    }
    if (c && d)
        k_htri_direct<true, true><<<grid, kTriThreads, 0, s>>>(ntri, t, npts, pts, centroids, self_idx, zk, rule,
                                                               fld != nullptr, pot, fld);
    else if (c)
        k_htri_direct<true, false><<<grid, kTriThreads, 0, s>>>(ntri, t, npts, pts, centroids, self_idx, zk, rule,
                                                                fld != nullptr, pot, fld);
    else
        k_htri_direct<false, true><<<grid, kTriThreads, 0, s>>>(ntri, t, npts, pts, centroids, self_idx, zk, rule,
                                                                fld != nullptr, pot, fld);
    FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
}

TriRule tri_rule_degree(int norder)
{
    // the rule of tri_rule for an iprec whose degree is norder
    return tri_rule(norder <= 1 ? -3 : norder == 2 ? -1 : norder == 4 ? 0 : 1);
}

}  // namespace fmm
