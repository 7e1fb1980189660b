// Helmholtz FMM kernels (FP64).  Expansions follow FMMLIB3D's Helmholtz
// conventions (src/helmrouts3d.f): Y_n^m = sqrt(2n+1) sqrt((n-m)!/(n+m)!)
// P_n^m with the Condon-Shortley phase, coefficient (n,m) at index n*n+n+m,
// multipoles scaled as M_n^m / s^n and locals as L_n^m * s^n with the level's
// scale s = min(1, |zk| * box side) (src/hfmm3dpart.f:336-340), so the stored
// numbers are the reference's.  Every expansion has the stride (pmax+1)^2 of
// the largest order used; level l uses degrees 0..p(l).
#pragma once
#include "lap_kernels.cuh"

namespace fmm {

// Largest Helmholtz expansion order: the evaluation kernel keeps a box's
// (p+1)^2 coefficients and 32 points' radial columns in shared memory.
constexpr int kHelmMaxP = 104;
static_assert(kHelmMaxP <= kRotTabP, "rotation tables shorter than the Helmholtz orders");

// Expansion order and scale of every level.
struct HLevels {
    int p[kMaxLevel + 1];
    double sc[kMaxLevel + 1];
};

// One source slot of a Helmholtz translation.
struct HSlot {
    int coll, oct;   // as Slot: colleague slot of the target's parent (M2L), child octant
    int cls;         // rotation class of the direction target - source
    int nin, nout;   // source and target degrees
    int mmax;        // largest |m| the z-shift produces (min(nin, nout))
    long long zoff;  // offset of the z-shift operator in the operator table
    double ex, ey;   // e^{i phi} of the direction target - source
};

// One z-shift operator: the linear map of h3dmpmpzshift_fast,
// h3dmploczshiftstab_fast or h3dlocloczshiftstab_fast (src/h3dtrans.f)
// for one (kind, level, distance, degrees), stored per |m| as a row-major
// (nout+1-m) x (nin+1-m) block, rows = target degree.
struct HZBlock {
    int kind;        // 0 M2M, 1 M2L, 2 L2L
    int nin, nout, nq;
    int qoff;        // first node of its Gauss-Legendre rule in the node table
    double zshift, radius, sc1, sc2;
    long long zoff;  // operator offset
    long long roff;  // radial scratch offset (complex entries)
};

__host__ __device__ inline long long hz_block_size(int nin, int nout)
{
    long long t = 0;
    int mm = nin < nout ? nin : nout;
    for (int m = 0; m <= mm; m++) t += (long long)(nout + 1 - m) * (nin + 1 - m);
    return t;
}

// z-shift operators for all blocks (two launches: node radial functions,
// then one CTA per block and |m|).  `rad` is scratch of
// sum over blocks of 2 (nq+1)(pmax+2) complex entries.
void build_hz(int nblk, const HZBlock *d_blk, const HZBlock *h_blk, const double *d_xw, double2 zk, int pmax,
              double2 *rad, double2 *Z, cudaStream_t s, Status &st);

// P2M (irreg=false: leaves, their own sources) and P2L (irreg=true: every
// box of level >= 2, the sources of its list-4 boxes) with charges and/or
// dipoles.
void launch_hform(bool irreg, const int *boxes, int nboxes, const TreeView &tv, const PointsSoA &src,
                  int ifcharge, int ifdipole, HLevels lv, int NC, double2 zk, double2 *exps, cudaStream_t s,
                  Status &st);

// L2P at leaves of level >= 2 and M2P from list-3 boxes, at sources and targets.
void launch_heval(const int *leaves, int nleaves, const TreeView &tv, const double *sx, const double *sy,
                  const double *sz, const double *tx, const double *ty, const double *tz, HLevels lv, int NC,
                  double2 zk, const double2 *mpole, const double2 *local, OutSoA outs, OutSoA outt, int do_src,
                  int do_trg, cudaStream_t s, Status &st);

// kind 0 = M2M, 1 = M2L, 2 = L2L by rotation, z-shift operator, rotation.
void launch_htranslate(int kind, const Tile *tiles, int ntiles, const int *grouped, const HSlot *slots,
                       const TreeView &tv, int pmax, const double *rot, const double2 *Z, const double2 *in,
                       double2 *out, int prune, int kt, cudaStream_t s, Status &st);

// P2P over self and list 1.
void launch_hp2p(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                 const double *ty, const double *tz, double2 zk, OutSoA outs, OutSoA outt, int ifcharge,
                 int ifdipole, int ifpot, int iffld, int ifpottarg, int iffldtarg, cudaStream_t s, Status &st);

// Direct sum at neval points over all sources, split over source chunks and
// reduced in a fixed order; skip[k] is the source excluded at point k (or
// null, and `self` excludes index k at point k).
void launch_hdirect(int nsrc, const PointsSoA &src, int ifcharge, int ifdipole, int neval, const double *ex,
                    const double *ey, const double *ez, const int *skip, int self, double2 zk, OutSoA out,
                    cudaStream_t s, Status &st);

}  // namespace fmm
