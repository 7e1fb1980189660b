// Laplace layer potentials on flat triangles (lfmm3dtriatarg,
// src/lfmm3dtria.f:121-1160): piecewise-constant single-layer (charge) and
// double-layer (dipstr, oriented by the triangle's normal) densities on a
// triangulation, evaluated at the triangles' centroids and at targets.  The
// far field is the particle FMM with each triangle's density placed at
// quadrature nodes; the near field (the leaf itself and list 1) integrates
// 1/r and its derivatives exactly over each triangle.
#pragma once
#include "lap_kernels.cuh"

namespace fmm {

constexpr int kTriMaxNodes = 16;

// Quadrature on the reference triangle (0,0), (1,0), (0,1): y = v1 + xi (v2 -
// v1) + eta (v3 - v1), weights summing to 1 (times the area).
struct TriRule {
    int n = 0;
    double xi[kTriMaxNodes], eta[kTriMaxNodes], w[kTriMaxNodes];
};

// The rule of polynomial degree >= the reference's nqtri for this iprec
// (src/lfmm3dtria.f:679-701): nqtri 1 -> the centroid, 2k -> the collapsed
// Gauss-Legendre product rule of (k+1) x (k+1) nodes.
TriRule tri_rule(int iprec);
// nbox of lfmm3dtriatarg (src/lfmm3dtria.f:290-300), -1 for an unknown iprec.
int tri_nbox(int iprec, int ns, int nt);

// Triangles in tree order.  geo: 30 doubles per triangle: vertices v1, v2,
// v3 (9), the unit normal n = (v2-v1)x(v3-v1)/|.| (3), per edge k (v_k ->
// v_k+1) the unit tangent t_k (9) and the outward in-plane normal m_k = t_k x
// n (9).
struct TriSoA {
    double *geo = nullptr;
    double2 *q = nullptr, *dq = nullptr;
};

// Gathers the caller's triangles (triaflat(3,3,n), trianorm(3,n), charge,
// dipstr) into tree order and places each triangle's density at the rule's
// nodes: node k of sorted triangle i is point i * rule.n + k of `nodes`, a
// charge q w_k A (or a dipole dipstr w_k A along trianorm, as
// l3dformmptrid2_add does).
void launch_tri_gather(int n, const int *perm, const double *tri, const double *norm, const double *q,
                       const double *dq, int ifcharge, int ifdipole, const TriRule &rule, TriSoA t, PointsSoA nodes,
                       cudaStream_t s, Status &st);

// Box source ranges in nodes: src0 * k, nsrc * k.
void launch_scale_ranges(int nboxes, const int *src0, const int *nsrc, int k, int *qsrc0, int *qnsrc, cudaStream_t s,
                         Status &st);

// Near field: every evaluation point of a leaf (its centroids, then its
// targets) against the triangles of the leaf and of its list 1, by the
// exact integrals; adds to the outputs.
void launch_p2p_tri(const int *leaves, int nleaves, const TreeView &tv, const TriSoA &t, const double *sx,
                    const double *sy, const double *sz, const double *tx, const double *ty, const double *tz,
                    OutSoA outs, OutSoA outt, int ifcharge, int ifdipole, int do_src, int do_trg, int want_fs,
                    int want_ft, cudaStream_t s, Status &st);

// O(N^2) l3dtriadirect at npts points, triangles in the caller's order;
// point k is the centroid of triangle self_idx[k] (-1: none) when self_idx is
// given, else of triangle k when centroids = 1 (that triangle then takes the
// in-plane values).  pot (2 doubles) / fld (6) per point written.
void launch_tri_direct(int ntri, const TriSoA &t, int ifcharge, int ifdipole, int npts, const double *pts,
                       int centroids, const int *self_idx, double *pot, double *fld, cudaStream_t s, Status &st);

// The collapsed Gauss-Legendre rule of polynomial degree norder (1, 2, 4, 6).
TriRule tri_rule_degree(int norder);

// Helmholtz triangles (hfmm3dtriatarg): the near field with zk and the near
// rule (degree nqtri), and the direct sum h3dtriadirect.
void launch_hp2p_tri(const int *leaves, int nleaves, const TreeView &tv, const TriSoA &t, const double *sx,
                     const double *sy, const double *sz, const double *tx, const double *ty, const double *tz,
                     double2 zk, const TriRule &rule, OutSoA outs, OutSoA outt, int ifcharge, int ifdipole,
                     int do_src, int do_trg, int want_fs, int want_ft, cudaStream_t s, Status &st);
void launch_htri_direct(int ntri, const TriSoA &t, int ifcharge, int ifdipole, int npts, const double *pts,
                        int centroids, const int *self_idx, double2 zk, const TriRule &rule, double *pot, double *fld,
                        cudaStream_t s, Status &st);

}  // namespace fmm
