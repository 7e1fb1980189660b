// Laplace Hessians: the second derivatives of the potential (dxx, dyy, dzz,
// dxy, dxz, dyz, the order of l3dmpevalhessd / l3dtaevalhessd,
// src/laprouts3d.f:6945, 7384) at the evaluation points of the FMM, and the
// evaluation of one multipole or local expansion with its potential,
// -gradient and Hessian at many points.
#pragma once
#include "lap_kernels.cuh"

namespace fmm {

// Hessians in tree order: h[0..5] = dxx, dyy, dzz, dxy, dxz, dyz (complex).
struct HessSoA {
    double2 *h[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

// Largest expansion order the Hessian kernels take (their recurrence tables
// run to degree kHessMaxP + 2).
constexpr int kHessMaxP = 74;

void hess_init_constants(Status &st);

// Near field: the Hessians of the pairs of self and list 1 (lpotfld3dhess,
// lpotfld3dhess_dp, src/laprouts3d.f:5442, 5619), added to hs / ht.
void launch_p2p_hess(const int *leaves, int nleaves, const TreeView &tv, const PointsSoA &src, const double *tx,
                     const double *ty, const double *tz, HessSoA hs, HessSoA ht, int ifcharge, int ifdipole,
                     int do_src, int do_trg, cudaStream_t s, Status &st);

// Far field: the Hessians of the leaf's local expansion and of its list-3
// multipoles, added to hs / ht.
void launch_eval_hess(const int *leaves, int nleaves, const TreeView &tv, const double *sx, const double *sy,
                      const double *sz, const double *tx, const double *ty, const double *tz, int p,
                      const double2 *mpole, const double2 *local, HessSoA hs, HessSoA ht, int do_src, int do_trg,
                      cudaStream_t s, Status &st);

// Tree order -> the caller's hess(6, n) (complex, interleaved).
void launch_scatter_hess(int n, const int *perm, HessSoA h, double *out, cudaStream_t s, Status &st);

// One expansion (the caller's layout: coefficient (n, m) at n + (m + nterms)
// (nterms + 1), complex interleaved, rscale as in FMMLIB3D) at npts points:
// pot, fld = -gradient (iffld) and hess (ifhess).  loc: local (true) or
// multipole (false).
void launch_expeval_hess(bool loc, double rscale, const double *center, const double *coef, int nterms, int npts,
                         const double *pts, double *pot, int iffld, double *fld, int ifhess, double *hess,
                         cudaStream_t s, Status &st);

}  // namespace fmm
