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

// kt: targets per tile (64, or 16 for problems too small to fill the GPU)
void launch_m2l_dense(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                      const long long *slot_toff, const double2 *T, const TreeView &tv, int p, const double2 *in,
                      double2 *out, int prune, int kt, cudaStream_t s, Status &st);

}  // namespace fmm

namespace fmm {

// Mixed-precision form (mixed.cu): FP32 P2P with compensated accumulation
// (max_ept: at most 1, 2 or 4 evaluation points per lane) and FP32 dense M2L.
void launch_p2p32(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                  const double *ty, const double *tz, OutSoA outs, OutSoA outt, int ifcharge, int ifdipole,
                  int ifpot, int iffld, int ifpottarg, int iffldtarg, int max_ept, cudaStream_t s, Status &st);
void convert_f32(long long n, const double2 *in, float2 *out, cudaStream_t s, Status &st);
// Tensor-core (tcgen05, split TF32) form of the FP32 dense M2L (tc_m2l.cu):
// tiles of up to max_tile (<= 256) targets, FP32 multipoles with an even row
// stride ldm; the TMEM sum is added into an FP32 running sum every `group`
// slots (0: once, at the end); *err is set on an expired wait.  Tiles of up
// to 128 targets: variant 0: K stage 16, 3 stages; 1: K stage 32, 2 stages
// (two CTAs per SM); larger tiles: K stage 16, 3 stages, one CTA per SM.
void launch_m2l_tc(int variant, const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                   const long long *slot_toff, const float2 *T, const TreeView &tv, int p, const float2 *mp,
                   int ldm, double2 *out, int prune, int nprod, int group, int *err, int max_tile, cudaStream_t s,
                   Status &st);
void convert_mp_f32(long long nboxes, int nc, int ldm, const double2 *in, float2 *out, cudaStream_t s, Status &st);
constexpr int kTcTileTargets = 128;      // largest tile of the two-CTA-per-SM kernel
constexpr int kTcTileTargetsMax = 256;   // largest tile of all

void launch_m2l_dense32(const Tile *tiles, int ntiles, const int *grouped, const Slot *slots,
                        const long long *slot_toff, const float2 *T, const TreeView &tv, int p, const double2 *in,
                        double2 *out, int prune, cudaStream_t s, Status &st);

}  // namespace fmm
