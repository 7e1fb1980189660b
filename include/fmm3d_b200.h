/*
 * fmm3d_b200.h -- C ABI of libfmm3d_b200.so, the B200 (sm_100a) particle FMM.
 *
 * The Fortran-callable entry points below have exactly the calling sequences
 * of FMMLIB3D's particle FMM (all arguments by reference, gfortran name
 * mangling with one trailing underscore, complex*16 passed as interleaved
 * (re, im) doubles, source(3,n) as xyz-interleaved doubles, default 32-bit
 * integers).  A Fortran program linked against this library instead of the
 * reference's objects runs on the GPU with no source change.
 *
 * Ownership and flags follow the reference: the caller allocates every input
 * and output; the library allocates its own device workspace; an output is
 * written iff its flag equals 1; inputs are never modified.  ier = 0 on
 * success, 4 / 8 / 16 when workspace cannot be allocated (here: device
 * memory), as in src/lfmm3dpart.f:192-197.
 */
#ifndef FMM3D_B200_H
#define FMM3D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces lfmm3dpart (src/lfmm3dpart.f:36-80): sources only. */
void lfmm3dpart_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                 const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                 const int *ifpot, double *pot, const int *iffld, double *fld);

/* Replaces lfmm3dpartself (src/lfmm3dpart.f:87-131). */
void lfmm3dpartself_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                     const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                     const int *ifpot, double *pot, const int *iffld, double *fld);

/* Replaces lfmm3dparttarg (src/lfmm3dpart.f:138-522). */
void lfmm3dparttarg_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                     const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                     const int *ifpot, double *pot, const int *iffld, double *fld, const int *ntarget,
                     const double *target, const int *ifpottarg, double *pottarg, const int *iffldtarg,
                     double *fldtarg);

/* Replaces l3dpartdirect (src/lfmm3dpart.f:1391-1523), the O(N^2) sum. */
void l3dpartdirect_(const int *nsource, const double *source, const int *ifcharge, const double *charge,
                    const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                    const int *iffld, double *fld, const int *ntarget, const double *target,
                    const int *ifpottarg, double *pottarg, const int *iffldtarg, double *fldtarg);

/* Replaces hfmm3dparttarg (src/hfmm3dpart.f:141-539): Helmholtz potential
 * e^{ik r}/r and field at sources and targets.  zk is complex*16 (two
 * doubles, re and im) passed after iprec; every other argument as for
 * lfmm3dparttarg_. */
void hfmm3dparttarg_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *source,
                     const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                     const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld,
                     const int *ntarget, const double *target, const int *ifpottarg, double *pottarg,
                     const int *iffldtarg, double *fldtarg);

/* Replaces hfmm3dpartself (src/hfmm3dpart.f:90-131): sources only. */
void hfmm3dpartself_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *source,
                     const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                     const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld);

/* Replaces hfmm3dpart (src/hfmm3dpart.f:39-84), the older name of hfmm3dpartself. */
void hfmm3dpart_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *source,
                 const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                 const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld);

/* Replaces h3dpartdirect (src/hfmm3dpart.f:1268-1401), the O(N^2) Helmholtz sum. */
void h3dpartdirect_(const double *zk, const int *nsource, const double *source, const int *ifcharge,
                    const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                    const int *ifpot, double *pot, const int *iffld, double *fld, const int *ntarget,
                    const double *target, const int *ifpottarg, double *pottarg, const int *iffldtarg,
                    double *fldtarg);

/* Replaces lfmm3dtriatarg (src/lfmm3dtria.f:121-546): Laplace layer
 * potentials of flat triangles triaflat(3,3,nsource) (vertices), with
 * piecewise-constant single-layer density charge and double-layer density
 * dipstr, at the triangles' centroids source(3,nsource) and at targets.
 * pot = sum int charge/|x-y| + dipstr n.(x-y)/|x-y|^3 dS_y, fld = -grad pot.
 * As in the reference, the double layer is oriented by the triangle's
 * vertex-order normal (v2-v1)x(v3-v1) in the near field and by trianorm in
 * the far field (trianorm must equal that unit normal), and dipvec is not
 * used.  nbox per iprec and the near field by exact integrals follow the
 * reference; the far-field quadrature is a collapsed Gauss-Legendre rule of
 * the reference's polynomial degree (the reference's triasymq tables are not
 * used).  Always FP64.  ier as lfmm3dparttarg_. */
void lfmm3dtriatarg_(int *ier, const int *iprec, const int *nsource, const double *triaflat, const double *trianorm,
                     const double *source, const int *ifcharge, const double *charge, const int *ifdipole,
                     const double *dipstr, const double *dipvec, const int *ifpot, double *pot, const int *iffld,
                     double *fld, const int *ntarget, const double *target, const int *ifpottarg, double *pottarg,
                     const int *iffldtarg, double *fldtarg);

/* Replaces lfmm3dtriaself (src/lfmm3dtria.f:80-114) and lfmm3dtria (:39-73): no targets. */
void lfmm3dtriaself_(int *ier, const int *iprec, const int *nsource, const double *triaflat, const double *trianorm,
                     const double *source, const int *ifcharge, const double *charge, const int *ifdipole,
                     const double *dipstr, const double *dipvec, const int *ifpot, double *pot, const int *iffld,
                     double *fld);
void lfmm3dtria_(int *ier, const int *iprec, const int *nsource, const double *triaflat, const double *trianorm,
                 const double *source, const int *ifcharge, const double *charge, const int *ifdipole,
                 const double *dipstr, const double *dipvec, const int *ifpot, double *pot, const int *iffld,
                 double *fld);

/* Replaces l3dtriadirect (src/lfmm3dtria.f:1385-1560): the O(N^2) sum of the
 * exact triangle integrals (each centroid takes its own triangle's in-plane
 * values). */
void l3dtriadirect_(const int *nsource, const double *triaflat, const double *trianorm, const double *source,
                    const int *ifcharge, const double *charge, const int *ifdipole, const double *dipstr,
                    const double *dipvec, const int *ifpot, double *pot, const int *iffld, double *fld,
                    const int *ntarget, const double *target, const int *ifpottarg, double *pottarg,
                    const int *iffldtarg, double *fldtarg);

/* Replaces hfmm3dtriatarg (src/hfmm3dtria.f:133-560): Helmholtz layer
 * potentials e^{ikr}/r of flat triangles, arguments as lfmm3dtriatarg_ with
 * zk (complex*16) after iprec.  The near field integrates the Laplace part
 * exactly and the difference e^{ikr}/r - 1/r (and its derivatives) with a
 * quadrature rule of the reference's degree (nqtri), the far field runs on
 * quadrature nodes of degree norder (src/hfmm3dtria.f:730-751); the rules
 * are collapsed Gauss-Legendre rules, not the reference's triasymq tables.
 * FP64.  The box scale uses |zk| here (zk is complex in this driver). */
void hfmm3dtriatarg_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *triaflat,
                     const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                     const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                     const int *iffld, double *fld, const int *ntarget, const double *target, const int *ifpottarg,
                     double *pottarg, const int *iffldtarg, double *fldtarg);

/* Replaces hfmm3dtriaself (src/hfmm3dtria.f:92-126) and hfmm3dtria (:51-85). */
void hfmm3dtriaself_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *triaflat,
                     const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                     const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                     const int *iffld, double *fld);
void hfmm3dtria_(int *ier, const int *iprec, const double *zk, const int *nsource, const double *triaflat,
                 const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                 const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                 const int *iffld, double *fld);

/* Replaces h3dtriadirect (src/hfmm3dtria.f:1456): the O(N^2) sum with the
 * near-field integrals of quadrature degree nqtri (1, 2, 4 or 6). */
void h3dtriadirect_(const int *nqtri, const double *zk, const int *nsource, const double *triaflat,
                    const double *trianorm, const double *source, const int *ifcharge, const double *charge,
                    const int *ifdipole, const double *dipstr, const double *dipvec, const int *ifpot, double *pot,
                    const int *iffld, double *fld, const int *ntarget, const double *target, const int *ifpottarg,
                    double *pottarg, const int *iffldtarg, double *fldtarg);

/* Replaces l3dtaevalhess (src/laprouts3d.f:5297-5363; it calls
 * l3dtaevalhessdini + l3dtaevalhessd, :7613, :7384) and l3dmpevalhess
 * (:5229-5295; l3dmpevalhessdini + l3dmpevalhessd, :7129, :6945): potential,
 * field = -gradient (iffld = 1) and Hessian hess(6) = dxx, dyy, dzz, dxy, dxz,
 * dyz (ifhess = 1) of one local / multipole expansion
 * expansion(0:nterms, -nterms:nterms) with scaling rscale about center, at
 * ztarg.  ier = 0, or 8 / 16 (device memory, nterms outside 0..74).  One point
 * per call; fmm3d_l3dtaevalhess_device evaluates many points in one call. */
void l3dtaevalhess_(const double *rscale, const double *center, const double *local, const int *nterms,
                    const double *ztarg, double *pot, const int *iffld, double *fld, const int *ifhess, double *hess,
                    int *ier);
void l3dmpevalhess_(const double *rscale, const double *center, const double *mpole, const int *nterms,
                    const double *ztarg, double *pot, const int *iffld, double *fld, const int *ifhess, double *hess,
                    int *ier);

/* ---- extensions (no counterpart in the reference) ---------------------- */

/* lfmm3dparttarg_ with Hessians: ifhess / ifhesstarg = 1 also return
 * hess(6, nsource) / hesstarg(6, ntarget), complex*16, ordered dxx, dyy, dzz,
 * dxy, dxz, dyz (the order of l3dmpevalhessd / l3dtaevalhessd and of the
 * sort l3dhsort, src/lfmm3drouts.f:621).  The reference has the evaluators
 * (l3dmpevalhessd_trunc :7194, l3dtaevalhessd_trunc :7682, lpotfld3dhess
 * :5442, lpotfld3dhess_dp :5619) but no particle driver that calls them; this
 * one runs the FMM of lfmm3dparttarg and adds, at every evaluation point, the
 * Hessians of its near pairs, its list-3 multipoles and its leaf's local
 * expansion.  Potentials and fields are those of lfmm3dparttarg_ bit for bit
 * (same form, same kernels); the Hessians are computed in FP64 in every form. */
void lfmm3dparttarghess_(int *ier, const int *iprec, const int *nsource, const double *source, const int *ifcharge,
                         const double *charge, const int *ifdipole, const double *dipstr, const double *dipvec,
                         const int *ifpot, double *pot, const int *iffld, double *fld, const int *ifhess,
                         double *hess, const int *ntarget, const double *target, const int *ifpottarg,
                         double *pottarg, const int *iffldtarg, double *fldtarg, const int *ifhesstarg,
                         double *hesstarg);

/* lfmm3dtriatarg_ and l3dtriadirect_ on device-resident arrays (same
 * layouts), enqueued on `stream`; the direct sum waits for its stream. */
int fmm3d_lfmm3dtriatarg_device(int iprec, int nsource, const double *d_triaflat, const double *d_trianorm,
                                const double *d_source, int ifcharge, const double *d_charge, int ifdipole,
                                const double *d_dipstr, const double *d_dipvec, int ifpot, double *d_pot, int iffld,
                                double *d_fld, int ntarget, const double *d_target, int ifpottarg, double *d_pottarg,
                                int iffldtarg, double *d_fldtarg, void *stream);
int fmm3d_l3dtriadirect_device(int nsource, const double *d_triaflat, const double *d_trianorm,
                               const double *d_source, int ifcharge, const double *d_charge, int ifdipole,
                               const double *d_dipstr, const double *d_dipvec, int ifpot, double *d_pot, int iffld,
                               double *d_fld, int ntarget, const double *d_target, int ifpottarg, double *d_pottarg,
                               int iffldtarg, double *d_fldtarg, void *stream);

/* The triangle direct sum at npts arbitrary device points pts(3,npts): point k
 * is the centroid of triangle self[k] (0-based; -1 or self NULL: none), which
 * then takes its own triangle's in-plane values.  pot(npts), fld(3,npts)
 * complex*16 written.  The sampled form of l3dtriadirect. */
int fmm3d_l3dtriadirect_points_device(int nsource, const double *d_triaflat, int ifcharge, const double *d_charge,
                                      int ifdipole, const double *d_dipstr, int npts, const double *d_pts,
                                      const int *d_self, double *d_pot, double *d_fld, void *stream);

/* hfmm3dtriatarg_ on device-resident arrays (zk: two host doubles), and the
 * Helmholtz triangle direct sum at npts device points (point k is the
 * centroid of triangle self[k] when self is given, of triangle k when
 * centroids = 1; pot / fld written; synchronous). */
int fmm3d_hfmm3dtriatarg_device(int iprec, const double *zk, int nsource, const double *d_triaflat,
                                const double *d_trianorm, const double *d_source, int ifcharge, const double *d_charge,
                                int ifdipole, const double *d_dipstr, const double *d_dipvec, int ifpot, double *d_pot,
                                int iffld, double *d_fld, int ntarget, const double *d_target, int ifpottarg,
                                double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream);
int fmm3d_h3dtriadirect_points_device(int nqtri, const double *zk, int nsource, const double *d_triaflat,
                                      int ifcharge, const double *d_charge, int ifdipole, const double *d_dipstr,
                                      int npts, const double *d_pts, const int *d_self, int centroids, double *d_pot,
                                      double *d_fld, void *stream);

/* The same on device-resident arrays, enqueued on `stream`. */
int fmm3d_lfmm3dparttarg_hess_device(int iprec, int nsource, const double *d_source, int ifcharge,
                                     const double *d_charge, int ifdipole, const double *d_dipstr,
                                     const double *d_dipvec, int ifpot, double *d_pot, int iffld, double *d_fld,
                                     int ifhess, double *d_hess, int ntarget, const double *d_target, int ifpottarg,
                                     double *d_pottarg, int iffldtarg, double *d_fldtarg, int ifhesstarg,
                                     double *d_hesstarg, void *stream);

/* l3dtaevalhess / l3dmpevalhess at npts device-resident points targ(3, npts):
 * pot(npts), fld(3, npts) (iffld = 1), hess(6, npts) (ifhess = 1), complex*16,
 * in device memory; the expansion (reference layout) in device memory, rscale
 * and center(3) on the host.  Synchronous; returns ier. */
int fmm3d_l3dtaevalhess_device(double rscale, const double *center, const double *d_local, int nterms, int npts,
                               const double *d_targ, double *d_pot, int iffld, double *d_fld, int ifhess,
                               double *d_hess, void *stream);
int fmm3d_l3dmpevalhess_device(double rscale, const double *center, const double *d_mpole, int nterms, int npts,
                               const double *d_targ, double *d_pot, int iffld, double *d_fld, int ifhess,
                               double *d_hess, void *stream);

/* lfmm3dparttarg on arrays already resident in device memory (same layouts),
 * enqueued on `stream` (a cudaStream_t, or NULL for the library's own
 * stream).  Returns ier.  Used by services that keep inputs in HBM. */
int fmm3d_lfmm3dparttarg_device(int iprec, int nsource, const double *d_source, int ifcharge,
                                const double *d_charge, int ifdipole, const double *d_dipstr,
                                const double *d_dipvec, int ifpot, double *d_pot, int iffld, double *d_fld,
                                int ntarget, const double *d_target, int ifpottarg, double *d_pottarg,
                                int iffldtarg, double *d_fldtarg, void *stream);

/* l3dpartdirect on device-resident arrays (same layouts). */
int fmm3d_l3dpartdirect_device(int nsource, const double *d_source, int ifcharge, const double *d_charge,
                               int ifdipole, const double *d_dipstr, const double *d_dipvec, int ifpot,
                               double *d_pot, int iffld, double *d_fld, int ntarget, const double *d_target,
                               int ifpottarg, double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream);

/* Direct sum at npts arbitrary device-resident points pts(3,npts); skip[k]
 * (0-based source index, or -1; the array may be NULL) is left out of point
 * k's sum, which gives the self-excluded values at source points.  Outputs
 * pot(npts) and fld(3,npts) as complex*16.  The sampled form of
 * l3dpartdirecttime (src/lfmm3dpart.f:1529-1661). */
int fmm3d_l3ddirect_points_device(int nsource, const double *d_source, int ifcharge, const double *d_charge,
                                  int ifdipole, const double *d_dipstr, const double *d_dipvec, int npts,
                                  const double *d_pts, const int *d_skip, double *d_pot, double *d_fld,
                                  void *stream);

/* Batched lfmm3dparttarg on device arrays: ninst independent FMMs in one
 * call.  No counterpart in the reference (it has one FMM per call).  Instance
 * i owns sources src_offsets[i]..src_offsets[i+1]-1 and targets
 * trg_offsets[i]..trg_offsets[i+1]-1 of the concatenated arrays (host offset
 * arrays of ninst+1 entries starting at 0; trg_offsets may be NULL for no
 * targets); outputs are written in the same concatenated order.  Each
 * instance gets its own octree (bounding cube, lists, expansions) exactly as a
 * single call would build it, so its results equal those of a single call; all
 * instances share every pass (one kernel launch per pass for the batch). */
int fmm3d_lfmm3dparttarg_batched_device(int iprec, int ninst, const int *src_offsets, const double *d_source,
                                        int ifcharge, const double *d_charge, int ifdipole, const double *d_dipstr,
                                        const double *d_dipvec, int ifpot, double *d_pot, int iffld, double *d_fld,
                                        const int *trg_offsets, const double *d_target, int ifpottarg,
                                        double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream);

/* hfmm3dparttarg, h3dpartdirect and the sampled Helmholtz direct sum on
 * device-resident arrays (layouts as above; zk = two doubles on the host). */
int fmm3d_hfmm3dparttarg_device(int iprec, const double *zk, int nsource, const double *d_source, int ifcharge,
                                const double *d_charge, int ifdipole, const double *d_dipstr, const double *d_dipvec,
                                int ifpot, double *d_pot, int iffld, double *d_fld, int ntarget,
                                const double *d_target, int ifpottarg, double *d_pottarg, int iffldtarg,
                                double *d_fldtarg, void *stream);
int fmm3d_h3dpartdirect_device(const double *zk, int nsource, const double *d_source, int ifcharge,
                               const double *d_charge, int ifdipole, const double *d_dipstr, const double *d_dipvec,
                               int ifpot, double *d_pot, int iffld, double *d_fld, int ntarget,
                               const double *d_target, int ifpottarg, double *d_pottarg, int iffldtarg,
                               double *d_fldtarg, void *stream);
int fmm3d_h3ddirect_points_device(const double *zk, int nsource, const double *d_source, int ifcharge,
                                  const double *d_charge, int ifdipole, const double *d_dipstr,
                                  const double *d_dipvec, int npts, const double *d_pts, const int *d_skip,
                                  double *d_pot, double *d_fld, void *stream);

/* l3dpartdirect on device-resident arrays WITHOUT any device allocation.
 * No counterpart in the reference.  For callers that cannot let the library
 * allocate: an application whose framework allocator already holds the
 * GPU's memory, or a latency-bound service loop that forbids cudaMalloc and
 * cudaFree (which synchronise the device) after start-up.  Scratch lives in
 * a fixed 11 MB array in the library's device image, present on every GPU
 * that loads the library until the process exits.  Limit: nsource and
 * ntarget each at most 65536 (larger sizes return 8 without touching the
 * GPU).  The first call on a device is the set-up: it looks up the array's
 * device address and, under CUDA's default lazy module loading, loads the
 * array and the kernels used here, which can allocate device memory once.
 * Make that first call at start-up, before the caller's allocator takes the
 * GPU's memory and before any stream capture (or run with
 * CUDA_MODULE_LOADING=EAGER); later calls allocate nothing.  The address is
 * cached per device: after cudaDeviceReset, calls are invalid.  Calls share
 * the array: calls whose GPU work overlaps (other streams, other host
 * threads) race; serialise them.  stream NULL = the legacy default stream.
 * Returns ier (0 ok, 8 size limit, 16 CUDA error);
 * fmm3d_noalloc_last_error() describes this thread's last failure. */
int fmm3d_l3dpartdirect_noalloc(int nsource, const double *d_source, int ifcharge, const double *d_charge,
                                int ifdipole, const double *d_dipstr, const double *d_dipvec, int ifpot,
                                double *d_pot, int iffld, double *d_fld, int ntarget, const double *d_target,
                                int ifpottarg, double *d_pottarg, int iffldtarg, double *d_fldtarg, void *stream);
const char *fmm3d_noalloc_last_error(void);

/* Per-pass device times (ms) of the last FMM call made by this host thread
 * when timing is on: [tree, sort+gather, P2M, M2M, P2L, M2L, L2L, L2P+M2P,
 * P2P, scatter, total].  Returns the number of entries written. */
int fmm3d_set_timing(int on);
int fmm3d_last_timing(double *ms, int n);

/* Tree statistics of the last call on this thread, gathered only while
 * fmm3d_set_stats(1) is in effect:
 * [nboxes, nlev, nleaves, nterms, list1 entries, list3 entries,
 *  list4 entries, p2p pairs (sum over leaves), m2l pairs, then 128 counts of
 *  M2L pairs by truncation order]; Helmholtz calls append the expansion
 *  order of levels 0..21 (0 where a level carries no expansions) and report
 *  the largest order as nterms.  For Helmholtz the "sort+gather" timing entry
 *  also holds the construction of that call's z-shift operators. */
int fmm3d_set_stats(int on);

/* M2L form: 0 automatic (dense per-offset operators for nterms <= 16,
 * rotate-shift-rotate otherwise), 1 always rotate-shift-rotate, 2 dense
 * where available, 3 rotate-shift-rotate on the CUDA cores (modes 0 and 1
 * run the rotations and z-shifts as FP64 tensor-core products up to order
 * 28).  All give the same results to rounding; the switch exists for testing
 * and measurement. */
int fmm3d_set_m2l_mode(int mode);

/* Arithmetic form of later calls (process-wide): 0 = FP64 throughout (the
 * default: the reference's arithmetic), 1 = mixed precision for iprec <= 1:
 * P2P in FP32 with TwoSum-compensated accumulation and M2L with FP32
 * operators, FP64 for the tree, geometry, recurrences, rotations and the
 * other passes.  iprec >= 2 always runs FP64. */
int fmm3d_set_precision(int mode);
/* The same for the calling host thread only: 0 or 1 override the process-wide
 * setting for later calls made on this thread, -1 (the default) follows it.
 * Lets a multi-threaded caller (a serving loop) choose the form per request.
 * Returns 1 for an unknown mode. */
int fmm3d_set_precision_thread(int mode);

/* Per-host-thread override of one of the switches above (no counterpart in
 * the reference): which = 0 M2L form (fmm3d_set_m2l_mode), 1 arithmetic form
 * (fmm3d_set_precision), 2 tensor-core M2L (fmm3d_set_tensor_m2l), 3 slots per
 * tensor-core sum (fmm3d_set_tensor_m2l_group), 4 near/far overlap
 * (fmm3d_set_overlap); value -1 follows the process-wide setting again.  Later
 * calls made on this thread use the override; other threads' calls are not
 * affected.  Returns 1 for an unknown switch or value. */
int fmm3d_set_switch_thread(int which, int value);

/* Error-path tests (no counterpart in the reference, whose error codes come
 * from failed allocations: ier 4 tree, 8 per-point workspace, 16 expansions,
 * src/lfmm3dpart.f:309-330, 424-466).
 * fmm3d_inject_alloc_failure(phase): the next FMM call made on this host
 * thread that reaches the phase fails its first device allocation there as
 * if the device were out of memory: phase 1 the host-array entry points'
 * device copies of the caller's arrays (ier 8), 2 the octree (ier 4), 3 the
 * per-point workspace (ier 8), 4 the expansions (ier 16); 0 cancels.  One
 * call only; the caller's host outputs are left untouched.
 * fmm3d_inject_tc_wait_expiry(on): the tensor-core M2L kernels launched by
 * later calls on this thread treat their first stage wait as expired and
 * take their error path (drain their issued MMAs, free TMEM, flag the error):
 * the call returns 16.  Both return 1 for an unknown phase. */
int fmm3d_inject_alloc_failure(int nth);
int fmm3d_inject_tc_wait_expiry(int on);

/* M2L of the mixed form (iprec <= 1, nterms <= 16) on the tensor cores:
 * 0 = FP32 CUDA cores, 1 or 2 = tcgen05 kind::tf32 with operands split into
 * TF32 pairs (three products per step, FP32 accumulation in TMEM; the
 * default is 1); 1 and 2 differ only in the shared-memory staging (K stage
 * 16 with three stages, K stage 32 with two).  No counterpart in the reference.  Returns 1 for an
 * unknown mode. */
int fmm3d_set_tensor_m2l(int mode);

/* Laplace passes: 1 (default) runs the near field (P2P) concurrently with the
 * far-field passes on a second stream; 0 runs all passes one after the other on
 * the call's stream (same results bitwise; per-pass timings then show each
 * kernel alone).  No counterpart in the reference. */
int fmm3d_set_overlap(int on);

/* Tensor-core M2L: number of list-2 slots summed in the tensor-core (TMEM)
 * accumulator before the sum is added, with round-to-nearest FP32 additions,
 * into the tile's running sum (default 1; 0 = one tensor-core sum per tile).
 * Smaller groups bound the accumulation error of the tensor cores: on
 * adaptive trees one slot per group is more accurate than the FP32 CUDA-core
 * form, four per group is not.  No counterpart in the reference.  Returns 1 if negative. */
int fmm3d_set_tensor_m2l_group(int slots);

/* Self-test of the tensor-core path on the current device: D (128 x N, row
 * major) = A (128 x K) B^T (B is N x K), FP32 host arrays, through the same
 * staging, descriptors and TMEM reads as the M2L kernel.  N in 16..128 (a
 * multiple of 16), K a multiple of 32; nprod 1 = TF32 high parts only,
 * 3 = high and cross products, 4 = all four split products.  Returns 0, 1 on a bad argument, 2 on a CUDA error,
 * 3 when a bounded wait expired.  No counterpart in the reference. */
int fmm3d_tc_selftest(int N, int K, const float *A, const float *B, float *D, int nprod);
int fmm3d_last_stats(long long *out, int n);

/* ---- Plans: one geometry, many charge vectors (no counterpart in the reference's
 * particle API; the tree queries mirror d3tgetb / d3tgetl, src/d3tstrcr.f:576-665).
 * fmm3d_lfmm3d_plan_create builds the tree, lists, tree-ordered coordinates and
 * all workspace for device arrays source(3,nsource) and target(3,ntarget) and the
 * given output flags (the arithmetic form, fmm3d_set_precision, is fixed at
 * creation).  fmm3d_lfmm3d_plan_execute runs the passes for device charge /
 * dipole arrays (NULL where the plan's flag is off) and writes the requested
 * outputs; with use_graph = 1 the passes are captured into a CUDA graph once
 * per set of pointers and stream and replayed.  Results equal those of
 * lfmm3dparttarg on the same inputs bitwise.  Calls on one plan are serialised.
 * Returns ier as lfmm3dparttarg (1: NULL plan). */
int fmm3d_lfmm3d_plan_create(int iprec, int nsource, const double *d_source, int ifcharge, int ifdipole, int ifpot,
                             int iffld, int ntarget, const double *d_target, int ifpottarg, int iffldtarg,
                             void *stream, void **plan);
/* The same for a batch of independent instances (offsets as in
 * fmm3d_lfmm3dparttarg_batched_device; trg_offsets may be NULL). */
int fmm3d_lfmm3d_plan_create_batched(int iprec, int ninst, const int *src_offsets, const double *d_source,
                                     int ifcharge, int ifdipole, int ifpot, int iffld, const int *trg_offsets,
                                     const double *d_target, int ifpottarg, int iffldtarg, void *stream, void **plan);
int fmm3d_lfmm3d_plan_execute(void *plan, const double *d_charge, const double *d_dipstr, const double *d_dipvec,
                              double *d_pot, double *d_fld, double *d_pottarg, double *d_fldtarg, int use_graph,
                              void *stream);
int fmm3d_lfmm3d_plan_destroy(void *plan);
/* out[0..9]: nboxes, nlev, nleaves, nterms, nsource, ntarget, root centre (3), root side. */
int fmm3d_lfmm3d_plan_info(void *plan, double *out, int n);
/* d3tgetb: box(20) (level; i, j, k; parent; children; first source (1-based in tree
 * order), count; first target, count; source and target type 0 empty / 1 leaf /
 * 2 subdivided for holding more than nbox points; 0), centre(3) and corners(3,8)
 * of box ibox (1-based); ier 2 for a bad ibox. */
int fmm3d_lfmm3d_plan_getb(void *plan, int ibox, int *box, double *center, double *corners);
/* d3tgetl: list itype (1..5) of box ibox as 1-based box numbers; ier 4 when empty,
 * 2 for a bad ibox or itype; list = NULL returns only the length in *nlist. */
int fmm3d_lfmm3d_plan_getl(void *plan, int ibox, int itype, int *list, int *nlist);
/* d3tstrcrem (src/d3tstrcr.f:264-460): the adaptive octree of device arrays
 * d_source (nsource x 3) and d_target (ntarget x 3) alone, with the reference's
 * refinement options: a box splits while it holds more than nbox sources or
 * targets or its level is below minlevel, never at maxlevel or deeper (capped at
 * 21 levels), and ifempty = 1 keeps empty children.  The handle answers
 * fmm3d_lfmm3d_plan_info / _getb / _getl (box types: 2 only for a box split for
 * its point count) and is freed by fmm3d_lfmm3d_plan_destroy; _execute and the
 * tuning calls return 4 on it.  ier 128 when nsource < 1 (as the reference); 4
 * for nbox < 1, for ifempty = 1 with minlevel above 7 (8^minlevel boxes), and
 * when (nsource + ntarget) x (minlevel + 1) exceeds 2^30. */
int fmm3d_d3tstrcrem(int nsource, const double *d_source, int nbox, int ntarget, const double *d_target,
                     int ifempty, int minlevel, int maxlevel, void *stream, void **tree);

/* ---- Launch-shape tuning (no counterpart in the reference, whose only
 * tuning input is iprec).  Five knobs, 0 = automatic:
 *   [0] M2L targets per tile (tensor-core form 16..256 in steps of 16; FP64
 *       dense operators 16 or 64; FP32 CUDA-core form 64; rotations 1, 2, 4, 8),
 *   [1] M2M / L2L targets per tile (1, 2, 4, 8),
 *   [2] tensor-core M2L staging variant (1 or 2, as fmm3d_set_tensor_m2l),
 *   [3] 1 = near field concurrent with the far field, 2 = passes in order
 *       (fmm3d_set_overlap(0) forces the passes in order whatever the knob),
 *   [4] mixed-form P2P: at most 1, 2 or 4 evaluation points per lane.
 * No knob changes the arithmetic: every setting gives the same outputs bitwise.
 * Single calls and new plans take their knobs from the autotuner's JSON cache
 * (fmmlib3d_b200/autotune.py) when it holds the problem's signature, else
 * automatic values.  Cache file: the path set here (NULL: back to the default;
 * "" or "none": no cache), else $FMM3D_TUNING_CACHE, else tuning_cache.json
 * beside libfmm3d_b200.so. */
int fmm3d_set_tuning_cache(const char *path);
/* Re-read the cache file; returns the number of entries. */
int fmm3d_tuning_reload(void);
/* The cache path in use (returns 0, or the buffer size needed). */
int fmm3d_tuning_cache_path(char *buf, int n);
/* Set a plan's knobs (n >= 5).  Returns 0, 2 for a value this problem cannot
 * take (the plan keeps its previous knobs), 16 on a CUDA error. */
int fmm3d_lfmm3d_plan_set_tuning(void *plan, const int *knobs, int n);
/* out (n >= 7): the five knobs in use (0 where the form has no such knob), the
 * form (0 FP64 rotations, 1 FP64 dense operators, 2 mixed with CUDA-core M2L,
 * 3 mixed with tensor-core M2L) and 1 if the knobs came from the cache. */
int fmm3d_lfmm3d_plan_get_tuning(void *plan, int *out, int n);
/* The plan's problem signature (the cache key); returns 0 or the buffer size needed. */
int fmm3d_lfmm3d_plan_signature(void *plan, char *buf, int n);
/* Knobs (as fmm3d_lfmm3d_plan_get_tuning) and signature of this thread's last
 * single Laplace call; returns the signature's buffer size. */
int fmm3d_last_tuning(int *out, int n, char *sig, int nsig);

/* Human-readable description of the last CUDA error on this thread. */
const char *fmm3d_last_error(void);

/* Number of CUDA kernels launched by the last call on this thread. */
int fmm3d_last_launches(void);

/* Depth cap: the reference refines its octree to 100 levels (src/d3tstrcr.f:181-182); the
 * GPU tree's 64-bit keys hold 21.  Returns how many boxes of level 21 in this host thread's
 * last tree still held more than nbox sources or targets, which the reference would split
 * further (0 for any input whose points are not clustered below 2^-21 of the bounding cube).
 * Such boxes stay leaves and their points are summed directly, so results keep the iprec
 * accuracy and only the cost grows (quadratically in the box's point count). */
int fmm3d_last_depth_capped(void);

#ifdef __cplusplus
}
#endif

#endif /* FMM3D_B200_H */
