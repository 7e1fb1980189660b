// Adaptive octree on the device, with the logical structure of FMMLIB3D's
// d3tstrcr (src/d3tstrcr.f:24-259): the bounding cube of sources and
// targets, level-by-level refinement of every box that holds more than
// `nbox` sources or more than `nbox` targets, empty children dropped, boxes
// of one level contiguous and ordered by (parent, child octant z-y-x), and
// lists 1-5 with the reference's semantics (src/d3tstrcr.f:695-1069).
#pragma once
#include "fmm_common.cuh"

namespace fmm {

struct Tree {
    int n = 0, m = 0;        // sources, targets
    int ninst = 1;           // instances of a forest (one root each, boxes 0..ninst-1)
    DBuf<double> inst_geom;  // 4 per instance: center of the bounding cube, side
    int nboxes = 0, nlev = 0;
    int nleaves = 0;
    // boxes of level kMaxLevel that the reference would split further (it refines to
    // maxlevel 100; the keys here hold 21 levels): they stay leaves with more than nbox
    // points, summed directly, so results keep their accuracy and only cost more
    int capped = 0;
    double center0[3] = {0, 0, 0}, size = 0;
    std::vector<int> lev_start, lev_count;  // host copies, per level 0..nlev

    // per box (device)
    DBuf<int> ijk;      // 3 per box, 0-based integer coordinates on its level
    DBuf<int> level, parent, octant, nchild;
    DBuf<int> child;    // 8 per box, indexed by octant (bit0 x, bit1 y, bit2 z), -1 if absent
    DBuf<int> src0, nsrc, trg0, ntrg;
    DBuf<double> center;  // 3 per box
    DBuf<int> binst;      // instance of every box
    DBuf<int> coll;     // 27 per box: same-level boxes at offsets in [-1,1]^3 (self at 13), -1 if absent
    DBuf<int> leaves;   // ids of childless boxes
    // lists in CSR form
    DBuf<int> l1_start, l1_idx, l3_start, l3_idx, l4_start, l4_idx;
    // sorted position -> original index
    DBuf<int> perm_src, perm_trg;
    // boxes grouped by (level, octant), for the translation passes
    DBuf<int> grouped;                       // box ids
    std::vector<int> group_start;            // host, (nlev+1)*8 + 1 entries
    int cap = 0;
    int nbox = 0;                            // refinement threshold the tree was built with
};

// Refinement options of d3tstrcrem (src/d3tstrcr.f:264-460; applied in
// d3tallbem, :1450-1451, 1490-1498, 1529-1530): a box splits while it holds more than nbox sources
// or targets or lies above minlevel, never at or below maxlevel (capped at
// kMaxLevel here), and with ifempty = 1 its empty children are kept.  The
// defaults are those d3tstrcr uses.
struct TreeOptions {
    int ifempty = 0, minlevel = 0, maxlevel = 100;   // 100: d3tstrcr's (src/d3tstrcr.f:181-182)
};

// Builds the tree for device arrays src (n x 3, AoS) and trg (m x 3).
void build_tree(Tree &T, const double *d_src, int n, const double *d_trg, int m, int nbox, cudaStream_t s,
                Status &st, const TreeOptions &opt = TreeOptions());

// A forest of independent trees, one per instance: instance i owns sources
// so[i]..so[i+1]-1 and targets to[i]..to[i+1]-1 of the concatenated arrays
// (host offsets).  Every instance gets its own bounding cube and the same
// refinement rule; points are sorted instance-major, boxes of one level of all
// instances are contiguous, and lists never cross instances.
void build_forest(Tree &T, const double *d_src, const std::vector<int> &so, const double *d_trg,
                  const std::vector<int> &to, int nbox, cudaStream_t s, Status &st,
                  const TreeOptions &opt = TreeOptions());

__host__ __device__ __forceinline__ int coll_slot(int dx, int dy, int dz) { return (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1); }

}  // namespace fmm
