// Laplace FMM kernels (FP64 plain form).  Expansions are stored per box in
// the normalization of FMMLIB3D (Y_n^m = sqrt((n-m)!/(n+m)!) P_n^m with the
// Condon-Shortley phase, src/yrecursion.f:386-430), with coefficient (n,m) at
// index n*n+n+m and rescaled by the box side s of the box's level:
// multipoles hold M_n^m / s^n and locals hold L_n^m * s^(n+1), so that every
// translation operator is independent of the level.
#pragma once
#include "fmm_common.cuh"

namespace fmm {

// Points in tree order, structure of arrays.
struct PointsSoA {
    double *x = nullptr, *y = nullptr, *z = nullptr;
    double2 *q = nullptr;    // charge
    double2 *dq = nullptr;   // dipole strength
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;  // dipole direction
};

struct OutSoA {
    double2 *pot = nullptr;
    double2 *fx = nullptr, *fy = nullptr, *fz = nullptr;
};

struct TreeView {
    const int *level, *parent, *octant, *nchild, *child, *coll;
    const int *src0, *nsrc, *trg0, *ntrg;
    const double *center;
    const int *l1_start, *l1_idx, *l3_start, *l3_idx, *l4_start, *l4_idx;
    double size;  // side of the level-0 box
    // forests (several instances): the instance of every box and, per
    // instance, its bounding cube (center x, y, z, side); null for one tree
    const int *binst = nullptr;
    const double *inst_geom = nullptr;
};

// One source slot of a translation: where the source box is relative to the
// target and the geometry of the shift.
struct Slot {
    int coll;      // colleague slot of the target's parent (M2L), or -1
    int oct;       // child octant of that colleague (M2L, M2M)
    int cls;       // rotation class
    int pt;        // truncation order of this translation
    double ex, ey; // e^{i phi} of the direction target - source
    double rt;     // distance in units of the source box side
};

struct Tile {
    int first;     // index into the grouped box array
    int count;     // number of targets (<= KT)
    int slot0;     // first slot of this tile's slot table
    int nslot;
};

void lap_init_constants(Status &st);

void launch_p2p(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                const double *ty, const double *tz, OutSoA outs, OutSoA outt, int ifcharge, int ifdipole,
                int ifpot, int iffld, int ifpottarg, int iffldtarg, cudaStream_t s, Status &st);

void launch_p2m(const int *boxes, int nboxes, const TreeView &tv, const PointsSoA &src, int ifcharge,
                int ifdipole, int p, double2 *mpole, cudaStream_t s, Status &st);

void launch_p2l(const int *boxes, int nboxes, const TreeView &tv, const PointsSoA &src, int ifcharge,
                int ifdipole, int p, double2 *local, cudaStream_t s, Status &st);

// Work items of the evaluation pass (L2P + M2P): item offsets per leaf, scratch
// offsets of the leaves with more than one group of source expansions, and the
// scratch.  Built with the tree (host-synchronising); the launch then only
// enqueues kernels (graph-capturable).
struct EvalItems {
    DBuf<int> off, soff;
    DBuf<double> part;
    int nitems = 0, nscratch = 0;
};
int eval_items_prepare(const int *leaves, int nleaves, const TreeView &tv, int do_src, int do_trg, EvalItems &E,
                       cudaStream_t s, Status &st);
void launch_eval(const int *leaves, int nleaves, const EvalItems &E, const TreeView &tv, const double *sx,
                 const double *sy, const double *sz, const double *tx, const double *ty, const double *tz, int p,
                 const double2 *mpole, const double2 *local, OutSoA outs, OutSoA outt, int do_src, int do_trg,
                 cudaStream_t s, Status &st);

// kind 0 = M2M, 1 = M2L, 2 = L2L
void launch_translate(int kind, const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                      const TreeView &tv, int p, const double *rot, const double *dc, int lddc,
                      const double2 *in, double2 *out, int prune, int kt, cudaStream_t s, Status &st);

// Gauss-Legendre nodes and weights on [-1, 1] (host).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w);

// Rotation matrices about the y axis for each class (cos, sin of theta).
void build_rotations(int p, int ncls, const double *d_cs, double *d_rot, cudaStream_t s, Status &st);

// Largest order of the rotation matrices (build_rotations): the length of its
// recurrence tables.
constexpr int kRotTabP = 130;

__host__ __device__ inline size_t rot_class_size(int p) { return (size_t)(p + 1) * (2 * p + 1) * (2 * p + 3) / 3; }

// FP64 rotate-shift-rotate M2L with its products on the FP64 tensor cores
// (m2l_rot_dmma.cu), tiles of up to 8 targets, orders up to 28.
bool m2l_rot_dmma_supported(int p);
void launch_m2l_rot_dmma(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots, const TreeView &tv,
                         int p, const double *rot, const double *dc, int lddc, const double2 *in, double2 *out,
                         int prune, cudaStream_t s, Status &st);

void launch_direct(int nsrc, const double *sx, const double *sy, const double *sz, const double2 *q,
                   const double2 *dq, const double *vx, const double *vy, const double *vz, int ifcharge,
                   int ifdipole, int neval, const double *ex, const double *ey, const double *ez, const int *skip, int self,
                   OutSoA out, cudaStream_t s, Status &st);

void launch_direct_split(int nsrc, const double *sx, const double *sy, const double *sz, const double2 *q,
                         const double2 *dq, const double *vx, const double *vy, const double *vz, int ifcharge,
                         int ifdipole, int neval, const double *ex, const double *ey, const double *ez,
                         const int *skip, OutSoA out, cudaStream_t s, Status &st);

}  // namespace fmm
