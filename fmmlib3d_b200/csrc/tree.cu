// Device octree build and interaction lists (see tree.cuh).
#include <algorithm>

#include "tree.cuh"

namespace fmm {

namespace {

// ---------------------------------------------------------------- bounding cube
// d3tallbem (src/d3tstrcr.f:1357-1395): min/max over sources and targets,
// size = largest extent, center = midpoints.
__global__ void k_bbox_partial(const double *src, int n, const double *trg, int m, double *part)
{
    double mn[3] = {1e308, 1e308, 1e308}, mx[3] = {-1e308, -1e308, -1e308};
    long tot = (long)n + m;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
        const double *p = i < n ? src + 3 * i : trg + 3 * (i - n);
        for (int d = 0; d < 3; d++) {
            double v = p[d];
            mn[d] = fmin(mn[d], v);
            mx[d] = fmax(mx[d], v);
        }
    }
    for (int d = 0; d < 3; d++) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    }
    __shared__ double s[32][6];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int d = 0; d < 3; d++) { s[w][d] = mn[d]; s[w][3 + d] = mx[d]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ww++)
            for (int d = 0; d < 3; d++) {
                s[0][d] = fmin(s[0][d], s[ww][d]);
                s[0][3 + d] = fmax(s[0][3 + d], s[ww][3 + d]);
            }
        for (int d = 0; d < 6; d++) part[6 * blockIdx.x + d] = s[0][d];
    }
}

// Reduces the per-block partials with one CTA (min / max are exact in any order).
__global__ void k_bbox_final(const double *part, int nb, double *geom /* c0x c0y c0z size */)
{
    double mn[3] = {1e308, 1e308, 1e308}, mx[3] = {-1e308, -1e308, -1e308};
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
        for (int d = 0; d < 3; d++) {
            mn[d] = fmin(mn[d], part[6 * b + d]);
            mx[d] = fmax(mx[d], part[6 * b + 3 + d]);
        }
    for (int d = 0; d < 3; d++)
        for (int o = 16; o > 0; o >>= 1) {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    __shared__ double sh[32][6];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int d = 0; d < 3; d++) { sh[w][d] = mn[d]; sh[w][3 + d] = mx[d]; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ww++)
        for (int d = 0; d < 3; d++) {
            sh[0][d] = fmin(sh[0][d], sh[ww][d]);
            sh[0][3 + d] = fmax(sh[0][3 + d], sh[ww][3 + d]);
        }
    for (int d = 0; d < 3; d++) { mn[d] = sh[0][d]; mx[d] = sh[0][3 + d]; }
    double size = __dsub_rn(mx[0], mn[0]);
    double sy = __dsub_rn(mx[1], mn[1]), sz = __dsub_rn(mx[2], mn[2]);
    if (sy > size) size = sy;
    if (sz > size) size = sz;
    for (int d = 0; d < 3; d++) geom[d] = __dadd_rn(mn[d], mx[d]) / 2;
    geom[3] = size;
}

// Bounding cube of every instance of a forest: CTA per instance over its
// source range [so[i], so[i+1]) and target range [to[i], to[i+1]).
__global__ void k_bbox_inst(const double *src, const int *so, const double *trg, const int *to, double *geom)
{
    const int inst = blockIdx.x;
    double mn[3] = {1e308, 1e308, 1e308}, mx[3] = {-1e308, -1e308, -1e308};
    const long a = so[inst], ns = so[inst + 1] - a, b = to[inst], nt = to[inst + 1] - b;
    for (long i = threadIdx.x; i < ns + nt; i += blockDim.x) {
        const double *p = i < ns ? src + 3 * (a + i) : trg + 3 * (b + i - ns);
        for (int d = 0; d < 3; d++) {
            mn[d] = fmin(mn[d], p[d]);
            mx[d] = fmax(mx[d], p[d]);
        }
    }
    for (int d = 0; d < 3; d++)
        for (int o = 16; o > 0; o >>= 1) {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    __shared__ double sh[32][6];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int d = 0; d < 3; d++) { sh[w][d] = mn[d]; sh[w][3 + d] = mx[d]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ww++)
            for (int d = 0; d < 3; d++) {
                sh[0][d] = fmin(sh[0][d], sh[ww][d]);
                sh[0][3 + d] = fmax(sh[0][3 + d], sh[ww][3 + d]);
            }
        double size = __dsub_rn(sh[0][3], sh[0][0]);
        double sy = __dsub_rn(sh[0][4], sh[0][1]), sz = __dsub_rn(sh[0][5], sh[0][2]);
        if (sy > size) size = sy;
        if (sz > size) size = sz;
        for (int d = 0; d < 3; d++) geom[4 * inst + d] = __dadd_rn(sh[0][d], sh[0][3 + d]) / 2;
        geom[4 * inst + 3] = size;
    }
}

// instance id of every point of the concatenated arrays
__global__ void k_point_inst(const int *off, int *pinst)
{
    for (int i = off[blockIdx.x] + threadIdx.x; i < off[blockIdx.x + 1]; i += blockDim.x) pinst[i] = blockIdx.x;
}

// ---------------------------------------------------------------- keys
// Path key of a point: for every level the octant (z,y,x bits) it falls in,
// decided exactly as d3tsepa0 does (upper half iff coordinate > center) with
// the center computed as in d3tcentf (src/d3tstrcr.f:1671-1700):
// x0 + (i-1)*side + side/2, evaluated without contraction.
__global__ void k_keys(const double *pts, int n, const double *geom_all, const int *pinst, uint64_t *keys, int *idx)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *geom = geom_all + (pinst ? 4 * pinst[i] : 0);
    double size = geom[3];
    double h = size / 2;
    double x0[3] = {__dsub_rn(geom[0], h), __dsub_rn(geom[1], h), __dsub_rn(geom[2], h)};
    double p[3] = {pts[3L * i], pts[3L * i + 1], pts[3L * i + 2]};
    int c[3] = {0, 0, 0};
    uint64_t key = 0;
    for (int l = 0; l < kMaxLevel; l++) {
        // size / 2^l and side / 2 by exact power-of-two scaling (bitwise the same values)
        double side = ldexp(size, -l);
        double side2 = ldexp(side, -1);
        int oct = 0;
        for (int d = 0; d < 3; d++) {
            double ce = __dadd_rn(__dadd_rn(x0[d], __dmul_rn((double)c[d], side)), side2);
            int bit = p[d] > ce;
            c[d] = 2 * c[d] + bit;
            oct |= bit << d;
        }
        key = (key << 3) | (uint64_t)oct;
    }
    keys[i] = key;
    idx[i] = i;
}

__device__ __forceinline__ int key_digit(uint64_t key, int child_level)
{
    return (int)((key >> (3 * (kMaxLevel - child_level))) & 7);
}

// first index in [lo, hi) whose digit at child_level is >= d
__device__ int lower_digit(const uint64_t *keys, int lo, int hi, int child_level, int d)
{
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (key_digit(keys[mid], child_level) < d) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Split decision and child ranges for the boxes of one level
// (d3tallbem, src/d3tstrcr.f:1458-1578).  Sixteen threads per box: the
// fourteen digit boundaries (7 source, 7 target) are independent binary
// searches over the box's sorted range, done in parallel.
constexpr int kSplitLanes = 16;

__global__ void k_split(int b0, int nb, int level, int nbox, TreeOptions opt, const int *src0, const int *nsrc,
                        const int *trg0, const int *ntrg, const uint64_t *ksrc, const uint64_t *ktrg, int *nkids,
                        int *cs0, int *cns, int *ct0, int *cnt)
{
    __shared__ int bound[128 / kSplitLanes][16];
    const int g = threadIdx.x / kSplitLanes, j = threadIdx.x % kSplitLanes;
    const int t = blockIdx.x * (blockDim.x / kSplitLanes) + g;
    const bool live = t < nb;
    int s0 = 0, ns = 0, q0 = 0, nq = 0;
    bool split = false;
    if (live) {
        const int b = b0 + t;
        s0 = src0[b]; ns = nsrc[b]; q0 = trg0[b]; nq = ntrg[b];
        split = level < opt.maxlevel && (ns > nbox || nq > nbox || level < opt.minlevel);
        const int cl = level + 1;
        if (split && j >= 1 && j <= 7) bound[g][j] = lower_digit(ksrc, s0, s0 + ns, cl, j);
        if (split && j >= 9 && j <= 15) bound[g][j] = lower_digit(ktrg, q0, q0 + nq, cl, j - 8);
    }
    __syncthreads();
    if (!live || j != 0) return;
    int k = 0;
    if (split) {
        int sb[9], tb[9];
        sb[0] = s0; sb[8] = s0 + ns;
        tb[0] = q0; tb[8] = q0 + nq;
        for (int d = 1; d < 8; d++) {
            sb[d] = bound[g][d];
            tb[d] = bound[g][8 + d];
        }
        for (int d = 0; d < 8; d++) {
            cs0[8 * t + d] = sb[d];
            cns[8 * t + d] = sb[d + 1] - sb[d];
            ct0[8 * t + d] = tb[d];
            cnt[8 * t + d] = tb[d + 1] - tb[d];
            k += opt.ifempty == 1 || (sb[d + 1] > sb[d]) || (tb[d + 1] > tb[d]);
        }
    }
    nkids[t] = k;
}

__global__ void k_make_children(int b0, int nb, int level, int next0, int keep_empty, const int *kbase,
                                const int *nkids, const int *cs0, const int *cns, const int *ct0, const int *cnt,
                                const double *geom_all, int *ijk, int *lev, int *par, int *oct, int *nch,
                                int *child, int *src0, int *nsrc, int *trg0, int *ntrg, double *center, int *binst)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    int b = b0 + t;
    int id = next0 + kbase[t];
    nch[b] = nkids[t];
    if (nkids[t] == 0) return;
    const int inst = binst[b];
    const double *geom = geom_all + 4 * inst;
    double size = geom[3], h = size / 2;
    double side = size / (double)(1 << (level + 1)), side2 = side / 2;
    for (int d = 0; d < 8; d++) {
        int ns = cns[8 * t + d], nq = cnt[8 * t + d];
        if (ns == 0 && nq == 0 && !keep_empty) continue;
        int c[3] = {2 * ijk[3 * b] + (d & 1), 2 * ijk[3 * b + 1] + ((d >> 1) & 1), 2 * ijk[3 * b + 2] + ((d >> 2) & 1)};
        for (int e = 0; e < 3; e++) {
            ijk[3L * id + e] = c[e];
            // d3tcentc, src/d3tstrcr.f:1589-1669
            double x00 = __dsub_rn(geom[e], h);
            center[3L * id + e] = __dadd_rn(__dadd_rn(x00, __dmul_rn((double)c[e], side)), side2);
        }
        lev[id] = level + 1;
        binst[id] = inst;
        par[id] = b;
        oct[id] = d;
        nch[id] = 0;
        for (int e = 0; e < 8; e++) child[8L * id + e] = -1;
        src0[id] = cs0[8 * t + d];
        nsrc[id] = ns;
        trg0[id] = ct0[8 * t + d];
        ntrg[id] = nq;
        child[8L * b + d] = id;
        id++;
    }
}

// Root box of every instance (box id = instance id).
__global__ void k_root(int ninst, const int *so, const int *to, const double *geom, int *ijk, int *lev, int *par,
                       int *oct, int *nch, int *child, int *src0, int *nsrc, int *trg0, int *ntrg, double *center,
                       int *binst)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= ninst) return;
    for (int e = 0; e < 3; e++) { ijk[3 * r + e] = 0; center[3 * r + e] = geom[4 * r + e]; }
    lev[r] = 0; par[r] = -1; oct[r] = 0; nch[r] = 0; binst[r] = r;
    for (int e = 0; e < 8; e++) child[8 * r + e] = -1;
    src0[r] = so[r]; nsrc[r] = so[r + 1] - so[r]; trg0[r] = to[r]; ntrg[r] = to[r + 1] - to[r];
}

// ---------------------------------------------------------------- colleagues (list 5 plus self)
__global__ void k_colleagues(int b0, int nb, const int *ijk, const int *par, const int *child, int *coll)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    int b = b0 + t;
    int out[27];
    for (int s = 0; s < 27; s++) out[s] = -1;
    int P = par[b];
    if (P < 0) {
        out[13] = b;
    } else {
        for (int s = 0; s < 27; s++) {
            int C = coll[27L * P + s];
            if (C < 0) continue;
            for (int d = 0; d < 8; d++) {
                int ch = child[8L * C + d];
                if (ch < 0) continue;
                int dx = ijk[3L * ch] - ijk[3L * b], dy = ijk[3L * ch + 1] - ijk[3L * b + 1],
                    dz = ijk[3L * ch + 2] - ijk[3L * b + 2];
                if (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1) out[coll_slot(dx, dy, dz)] = ch;
            }
        }
    }
    for (int s = 0; s < 27; s++) coll[27L * b + s] = out[s];
}

// Closed boxes on (possibly different) levels intersect or touch: the
// integer form of d3tifint (src/d3tstrcr.f:1075-1172).
__device__ __forceinline__ bool touch(const int *ijk, const int *lev, int a, int b)
{
    int la = lev[a], lb = lev[b];
    if (la > lb) { int t = a; a = b; b = t; t = la; la = lb; lb = t; }
    long sc = 1L << (lb - la);
    for (int e = 0; e < 3; e++) {
        long ia = ijk[3L * a + e], ib = ijk[3L * b + e];
        if (ia * sc > ib + 1 || ib > (ia + 1) * sc) return false;
    }
    return true;
}

// Lists 1 and 3 of a childless non-root box b (d3tlsts/d3tlst31,
// src/d3tstrcr.f:827-851 and :912-1069).  List 1 = childless boxes that
// touch b (any level); list 3 = boxes on finer levels that do not touch b
// but whose parents do.  mode 0 counts, mode 1 writes.
__global__ void k_lists13(const int *leaves, int nleaves, const int *ijk, const int *lev, const int *par,
                          const int *nch, const int *child, const int *coll, int mode, int *n1, int *n3,
                          const int *s1, int *i1, const int *s3, int *i3)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nleaves) return;
    int b = leaves[t];
    if (lev[b] == 0) {
        if (mode == 0) { n1[b] = 0; n3[b] = 0; }
        return;
    }
    int c1 = 0, c3 = 0;
    int o1 = mode ? s1[b] : 0, o3 = mode ? s3[b] : 0;
    int stk[8 * kMaxLevel + 8];
    for (int s = 0; s < 27; s++) {
        if (s == 13) continue;
        int C = coll[27L * b + s];
        if (C < 0) continue;
        if (nch[C] == 0) {
            if (mode) i1[o1 + c1] = C;
            c1++;
            continue;
        }
        int top = 0;
        for (int d = 7; d >= 0; d--)
            if (child[8L * C + d] >= 0) stk[top++] = child[8L * C + d];
        while (top) {
            int x = stk[--top];
            if (!touch(ijk, lev, b, x)) {
                if (mode) i3[o3 + c3] = x;
                c3++;
            } else if (nch[x] == 0) {
                if (mode) i1[o1 + c1] = x;
                c1++;
            } else {
                for (int d = 7; d >= 0; d--)
                    if (child[8L * x + d] >= 0) stk[top++] = child[8L * x + d];
            }
        }
    }
    // childless boxes on coarser levels are colleagues of an ancestor of b
    for (int A = par[b]; A >= 0 && lev[A] >= 1; A = par[A]) {
        for (int s = 0; s < 27; s++) {
            if (s == 13) continue;
            int C = coll[27L * A + s];
            if (C < 0 || nch[C] != 0) continue;
            if (touch(ijk, lev, b, C)) {
                if (mode) i1[o1 + c1] = C;
                c1++;
            }
        }
    }
    if (mode == 0) { n1[b] = c1; n3[b] = c3; }
}

__global__ void k_list4_count(const int *leaves, int nleaves, const int *s3, const int *i3, int *n4)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nleaves) return;
    int b = leaves[t];
    for (int k = s3[b]; k < s3[b + 1]; k++) atomicAdd(&n4[i3[k]], 1);
}

__global__ void k_list4_fill(const int *leaves, int nleaves, const int *s3, const int *i3, int *cursor, int *i4)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nleaves) return;
    int b = leaves[t];
    for (int k = s3[b]; k < s3[b + 1]; k++) i4[atomicAdd(&cursor[i3[k]], 1)] = b;
}

// deterministic order inside each list-4 row
__global__ void k_sort_rows(int nb, const int *st, int *idx)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int lo = st[b], hi = st[b + 1];
    for (int i = lo + 1; i < hi; i++) {
        int v = idx[i], j = i - 1;
        while (j >= lo && idx[j] > v) { idx[j + 1] = idx[j]; j--; }
        idx[j + 1] = v;
    }
}

__global__ void k_flag_leaves(int nb, const int *nch, int *flag)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb) flag[b] = nch[b] == 0;
}

__global__ void k_compact(int nb, const int *flag, const int *pos, int *out)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb && flag[b]) out[pos[b]] = b;
}

__global__ void k_group_keys(int nb, const int *lev, const int *oct, uint64_t *keys, int *vals)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    keys[b] = (uint64_t)(lev[b] * 8 + oct[b]);
    vals[b] = b;
}

__global__ void k_group_bounds(int nb, const uint64_t *keys, int ngroups, int *gstart)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nb) return;
    int g0 = i == 0 ? 0 : (int)keys[i - 1] + 1;
    int g1 = i == nb ? ngroups : (int)keys[i];
    for (int g = g0; g <= g1 && g <= ngroups; g++) gstart[g] = i;
}

template <typename T>
bool grow(DBuf<T> &b, size_t need, size_t copy, cudaStream_t s, Status &st)
{
    if (b.n >= need) return true;
    DBuf<T> nb;
    if (!nb.alloc(need, s, st)) return false;
    if (copy) FMM_TRY(st, cudaMemcpyAsync(nb.p, b.p, sizeof(T) * copy, cudaMemcpyDeviceToDevice, s));
    std::swap(b.p, nb.p);
    std::swap(b.n, nb.n);
    std::swap(b.s, nb.s);
    return st.ok();
}

// Stable reorder of (key, perm) into instance-major order: sort by the
// instance of each point (gathered through perm), carrying the position,
// then gather keys and perm by the resulting order.
__global__ void k_gather_inst(int n, const int *perm, const int *pinst, uint64_t *ikey, int *pos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ikey[i] = (uint64_t)pinst[perm[i]];
    pos[i] = i;
}

__global__ void k_apply_pos(int n, const int *pos, const uint64_t *kin, const int *pin, uint64_t *kout, int *pout)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    kout[i] = kin[pos[i]];
    pout[i] = pin[pos[i]];
}

void instance_major(DBuf<uint64_t> &keys, DBuf<int> &perm, const DBuf<int> &pinst, int n, int ibits,
                    cudaStream_t s, Status &st)
{
    if (n == 0 || !st.ok()) return;
    DBuf<uint64_t> ik, k2;
    DBuf<int> pos, p2;
    if (!ik.alloc(n, s, st) || !pos.alloc(n, s, st) || !k2.alloc(n, s, st) || !p2.alloc(n, s, st)) return;
    k_gather_inst<<<div_up(n, 256), 256, 0, s>>>(n, perm.p, pinst.p, ik.p, pos.p); FMM_COUNT_LAUNCH();
    radix_sort_u64(ik.p, pos.p, n, ibits, s, st);
    k_apply_pos<<<div_up(n, 256), 256, 0, s>>>(n, pos.p, keys.p, perm.p, k2.p, p2.p); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);
    std::swap(keys.p, k2.p);
    std::swap(keys.n, k2.n);
    std::swap(perm.p, p2.p);
    std::swap(perm.n, p2.n);
}

}  // namespace

void build_tree(Tree &T, const double *d_src, int n, const double *d_trg, int m, int nbox, cudaStream_t s,
                Status &st, const TreeOptions &opt)
{
    std::vector<int> so = {0, n}, to = {0, m};
    build_forest(T, d_src, so, d_trg, to, nbox, s, st, opt);
}

void build_forest(Tree &T, const double *d_src, const std::vector<int> &so, const double *d_trg,
                  const std::vector<int> &to, int nbox, cudaStream_t s, Status &st, const TreeOptions &opt_in)
{
    TreeOptions opt = opt_in;
    opt.ifempty = opt.ifempty == 1;
    opt.minlevel = std::max(0, std::min(opt.minlevel, kMaxLevel));
    opt.maxlevel = std::max(0, std::min(opt.maxlevel, kMaxLevel));
    T.nbox = nbox;
    const int ninst = (int)so.size() - 1;
    const int n = so[ninst], m = to[ninst];
    T.n = n;
    T.m = m;
    T.ninst = ninst;
    // bounding cube of every instance
    DBuf<double> part, &geom = T.inst_geom;
    DBuf<int> dso, dto, pis, pit;
    geom.alloc(4L * ninst, s, st);
    if (!st.ok()) return;
    if (ninst == 1) {
        int nbb = std::max(1, std::min(1184, div_up((long)n + m, 256)));
        part.alloc(6 * nbb, s, st);
        if (!st.ok()) return;
        k_bbox_partial<<<nbb, 256, 0, s>>>(d_src, n, d_trg, m, part.p); FMM_COUNT_LAUNCH();
        k_bbox_final<<<1, 256, 0, s>>>(part.p, nbb, geom.p); FMM_COUNT_LAUNCH();
    } else {
        if (!dso.alloc(ninst + 1, s, st) || !dto.alloc(ninst + 1, s, st) || !pis.alloc(std::max(n, 1), s, st) ||
            !pit.alloc(std::max(m, 1), s, st))
            return;
        FMM_TRY(st, cudaMemcpyAsync(dso.p, so.data(), sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice, s));
        FMM_TRY(st, cudaMemcpyAsync(dto.p, to.data(), sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice, s));
        k_bbox_inst<<<ninst, 256, 0, s>>>(d_src, dso.p, d_trg, dto.p, geom.p); FMM_COUNT_LAUNCH();
        k_point_inst<<<ninst, 256, 0, s>>>(dso.p, pis.p); FMM_COUNT_LAUNCH();
        k_point_inst<<<ninst, 256, 0, s>>>(dto.p, pit.p); FMM_COUNT_LAUNCH();
    }
    // keys and sort: by path key, then (forests) stably by instance
    DBuf<uint64_t> ks, kt;
    ks.alloc(std::max(n, 1), s, st);
    kt.alloc(std::max(m, 1), s, st);
    T.perm_src.alloc(std::max(n, 1), s, st);
    T.perm_trg.alloc(std::max(m, 1), s, st);
    if (!st.ok()) return;
    if (n) { k_keys<<<div_up(n, 256), 256, 0, s>>>(d_src, n, geom.p, ninst > 1 ? pis.p : nullptr, ks.p, T.perm_src.p); FMM_COUNT_LAUNCH(); }
    if (m) { k_keys<<<div_up(m, 256), 256, 0, s>>>(d_trg, m, geom.p, ninst > 1 ? pit.p : nullptr, kt.p, T.perm_trg.p); FMM_COUNT_LAUNCH(); }
    FMM_LAUNCH_CHECK(st);
    radix_sort_u64(ks.p, T.perm_src.p, n, 3 * kMaxLevel, s, st);
    radix_sort_u64(kt.p, T.perm_trg.p, m, 3 * kMaxLevel, s, st);
    if (ninst > 1) {
        int ibits = 8;
        while ((1L << ibits) < ninst) ibits += 8;
        instance_major(ks, T.perm_src, pis, n, ibits, s, st);
        instance_major(kt, T.perm_trg, pit, m, ibits, s, st);
    }
    double hgeom[4];
    FMM_TRY(st, cudaMemcpyAsync(hgeom, geom.p, sizeof(hgeom), cudaMemcpyDeviceToHost, s));
    // boxes
    int cap = std::max(1024, 2 * (int)(((long)n + m) / std::max(nbox, 1)) + 64 + 2 * ninst);
    auto ensure = [&](int need, int used) {
        if (need <= T.cap) return st.ok();
        int nc = std::max(need, 2 * T.cap);
        grow(T.ijk, 3L * nc, 3L * used, s, st);
        grow(T.level, nc, used, s, st);
        grow(T.parent, nc, used, s, st);
        grow(T.octant, nc, used, s, st);
        grow(T.nchild, nc, used, s, st);
        grow(T.child, 8L * nc, 8L * used, s, st);
        grow(T.src0, nc, used, s, st);
        grow(T.nsrc, nc, used, s, st);
        grow(T.trg0, nc, used, s, st);
        grow(T.ntrg, nc, used, s, st);
        grow(T.center, 3L * nc, 3L * used, s, st);
        grow(T.binst, nc, used, s, st);
        T.cap = nc;
        return st.ok();
    };
    T.cap = 0;
    if (!ensure(cap, 0)) return;
    {
        DBuf<int> rso, rto;
        if (!rso.alloc(ninst + 1, s, st) || !rto.alloc(ninst + 1, s, st)) return;
        // root ranges in sorted order: instances are contiguous and in order
        FMM_TRY(st, cudaMemcpyAsync(rso.p, so.data(), sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice, s));
        FMM_TRY(st, cudaMemcpyAsync(rto.p, to.data(), sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice, s));
        k_root<<<div_up(ninst, 128), 128, 0, s>>>(ninst, rso.p, rto.p, geom.p, T.ijk.p, T.level.p, T.parent.p,
                                                  T.octant.p, T.nchild.p, T.child.p, T.src0.p, T.nsrc.p, T.trg0.p,
                                                  T.ntrg.p, T.center.p, T.binst.p); FMM_COUNT_LAUNCH();
        FMM_TRY(st, cudaStreamSynchronize(s));  // the host range vectors are read by the copies above
    }
    T.lev_start.assign(1, 0);
    T.lev_count.assign(1, ninst);
    int nboxes = ninst;
    DBuf<int> nk, kb, cs0, cns, ct0, cnt;
    for (int level = 0; level < kMaxLevel; level++) {
        int b0 = T.lev_start[level], nb = T.lev_count[level];
        if (!nk.alloc(nb, s, st) || !kb.alloc(nb, s, st) || !cs0.alloc(8L * nb, s, st) ||
            !cns.alloc(8L * nb, s, st) || !ct0.alloc(8L * nb, s, st) || !cnt.alloc(8L * nb, s, st))
            return;
        k_split<<<div_up(nb, 128 / kSplitLanes), 128, 0, s>>>(b0, nb, level, nbox, opt, T.src0.p, T.nsrc.p,
                                                               T.trg0.p, T.ntrg.p, ks.p, kt.p, nk.p, cs0.p, cns.p,
                                                               ct0.p, cnt.p); FMM_COUNT_LAUNCH();
        FMM_LAUNCH_CHECK(st);
        int total = 0;
        scan_exclusive_int(nk.p, kb.p, nb, s, st, &total);
        if (!st.ok()) return;
        if (total > 0 && !ensure(nboxes + total, nboxes)) return;
        k_make_children<<<div_up(nb, 128), 128, 0, s>>>(b0, nb, level, nboxes, opt.ifempty, kb.p, nk.p, cs0.p, cns.p, ct0.p,
                                                         cnt.p, geom.p, T.ijk.p, T.level.p, T.parent.p,
                                                         T.octant.p, T.nchild.p, T.child.p, T.src0.p, T.nsrc.p,
                                                         T.trg0.p, T.ntrg.p, T.center.p, T.binst.p); FMM_COUNT_LAUNCH();
        FMM_LAUNCH_CHECK(st);
        if (total == 0) break;
        T.lev_start.push_back(nboxes);
        T.lev_count.push_back(total);
        nboxes += total;
    }
    T.nboxes = nboxes;
    T.nlev = (int)T.lev_start.size() - 1;
    T.capped = 0;
    if (opt_in.maxlevel > kMaxLevel && T.nlev == kMaxLevel && st.ok()) {
        const int b0 = T.lev_start[kMaxLevel], nb = T.lev_count[kMaxLevel];
        std::vector<int> hs(nb), ht(nb);
        FMM_TRY(st, cudaMemcpyAsync(hs.data(), T.nsrc.p + b0, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
        FMM_TRY(st, cudaMemcpyAsync(ht.data(), T.ntrg.p + b0, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
        FMM_TRY(st, cudaStreamSynchronize(s));
        for (int i = 0; i < nb && st.ok(); i++) T.capped += (hs[i] > nbox || ht[i] > nbox) ? 1 : 0;
    }
    for (int d = 0; d < 3; d++) T.center0[d] = hgeom[d];
    T.size = hgeom[3];

    // colleagues, level by level
    T.coll.alloc(27L * nboxes, s, st);
    if (!st.ok()) return;
    for (int l = 0; l <= T.nlev; l++) {
        k_colleagues<<<div_up(T.lev_count[l], 128), 128, 0, s>>>(T.lev_start[l], T.lev_count[l], T.ijk.p,
                                                                  T.parent.p, T.child.p, T.coll.p); FMM_COUNT_LAUNCH();
    }
    FMM_LAUNCH_CHECK(st);

    // leaves
    DBuf<int> flag, pos;
    flag.alloc(nboxes, s, st);
    pos.alloc(nboxes, s, st);
    if (!st.ok()) return;
    k_flag_leaves<<<div_up(nboxes, 256), 256, 0, s>>>(nboxes, T.nchild.p, flag.p); FMM_COUNT_LAUNCH();
    int nleaves = 0;
    scan_exclusive_int(flag.p, pos.p, nboxes, s, st, &nleaves);
    T.nleaves = nleaves;
    T.leaves.alloc(std::max(nleaves, 1), s, st);
    if (!st.ok()) return;
    k_compact<<<div_up(nboxes, 256), 256, 0, s>>>(nboxes, flag.p, pos.p, T.leaves.p); FMM_COUNT_LAUNCH();

    // lists 1 and 3 (count, scan, fill), list 4 as the dual of list 3
    DBuf<int> n1, n3;
    n1.alloc(nboxes + 1, s, st);
    n3.alloc(nboxes + 1, s, st);
    T.l1_start.alloc(nboxes + 1, s, st);
    T.l3_start.alloc(nboxes + 1, s, st);
    T.l4_start.alloc(nboxes + 1, s, st);
    if (!st.ok()) return;
    n1.zero(st);
    n3.zero(st);
    int lb = std::max(nleaves, 1);
    k_lists13<<<div_up(lb, 128), 128, 0, s>>>(T.leaves.p, nleaves, T.ijk.p, T.level.p, T.parent.p, T.nchild.p,
                                              T.child.p, T.coll.p, 0, n1.p, n3.p, nullptr, nullptr, nullptr,
                                              nullptr); FMM_COUNT_LAUNCH();
    int tot1 = 0, tot3 = 0;
    scan_exclusive_int(n1.p, T.l1_start.p, nboxes + 1, s, st, &tot1);
    scan_exclusive_int(n3.p, T.l3_start.p, nboxes + 1, s, st, &tot3);
    T.l1_idx.alloc(std::max(tot1, 1), s, st);
    T.l3_idx.alloc(std::max(tot3, 1), s, st);
    if (!st.ok()) return;
    k_lists13<<<div_up(lb, 128), 128, 0, s>>>(T.leaves.p, nleaves, T.ijk.p, T.level.p, T.parent.p, T.nchild.p,
                                              T.child.p, T.coll.p, 1, nullptr, nullptr, T.l1_start.p,
                                              T.l1_idx.p, T.l3_start.p, T.l3_idx.p); FMM_COUNT_LAUNCH();
    DBuf<int> n4, cur;
    n4.alloc(nboxes + 1, s, st);
    cur.alloc(nboxes + 1, s, st);
    if (!st.ok()) return;
    n4.zero(st);
    k_list4_count<<<div_up(lb, 128), 128, 0, s>>>(T.leaves.p, nleaves, T.l3_start.p, T.l3_idx.p, n4.p); FMM_COUNT_LAUNCH();
    int tot4 = 0;
    scan_exclusive_int(n4.p, T.l4_start.p, nboxes + 1, s, st, &tot4);
    T.l4_idx.alloc(std::max(tot4, 1), s, st);
    if (!st.ok()) return;
    FMM_TRY(st, cudaMemcpyAsync(cur.p, T.l4_start.p, sizeof(int) * (nboxes + 1), cudaMemcpyDeviceToDevice, s));
    k_list4_fill<<<div_up(lb, 128), 128, 0, s>>>(T.leaves.p, nleaves, T.l3_start.p, T.l3_idx.p, cur.p,
                                                 T.l4_idx.p); FMM_COUNT_LAUNCH();
    k_sort_rows<<<div_up(nboxes, 128), 128, 0, s>>>(nboxes, T.l4_start.p, T.l4_idx.p); FMM_COUNT_LAUNCH();
    FMM_LAUNCH_CHECK(st);

    // boxes grouped by (level, octant)
    int ngroups = (T.nlev + 1) * 8;
    DBuf<uint64_t> gk;
    DBuf<int> gs;
    gk.alloc(nboxes, s, st);
    T.grouped.alloc(nboxes, s, st);
    gs.alloc(ngroups + 1, s, st);
    if (!st.ok()) return;
    k_group_keys<<<div_up(nboxes, 256), 256, 0, s>>>(nboxes, T.level.p, T.octant.p, gk.p, T.grouped.p); FMM_COUNT_LAUNCH();
    int gbits = 8;
    while ((1 << gbits) < ngroups + 1) gbits += 8;
    radix_sort_u64(gk.p, T.grouped.p, nboxes, gbits, s, st);
    if (!st.ok()) return;
    k_group_bounds<<<div_up(nboxes + 1, 256), 256, 0, s>>>(nboxes, gk.p, ngroups, gs.p); FMM_COUNT_LAUNCH();
    T.group_start.assign(ngroups + 1, 0);
    FMM_TRY(st, cudaMemcpyAsync(T.group_start.data(), gs.p, sizeof(int) * (ngroups + 1), cudaMemcpyDeviceToHost, s));
    FMM_TRY(st, cudaStreamSynchronize(s));
}

}  // namespace fmm
