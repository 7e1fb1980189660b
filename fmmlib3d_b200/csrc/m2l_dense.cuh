// M2L as gathered dense GEMMs per translation offset (see m2l_dense.cu).
#pragma once
#include "lap_kernels.cuh"

namespace fmm {

constexpr int kDenseMaxP = 16;   // largest expansion order served by the dense M2L
constexpr int kDenseTileTargets = 64;

// One list-2 translation offset: truncation, rotation class, e^{i phi} and
// distance of the direction target - source, and where its operator starts.
struct M2LOp {
    int pt, cls;
    double ex, ey, rt;
    long long toff;
};

void build_m2l_ops(int p, int nops, const M2LOp *d_ops, const double *rot, const double *dc, int lddc,
                   double2 *T, cudaStream_t s, Status &st);

void launch_m2l_dense(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                      const long long *slot_toff, const double2 *T, const TreeView &tv, int p, const double2 *in,
                      double2 *out, int prune, cudaStream_t s, Status &st);

}  // namespace fmm
