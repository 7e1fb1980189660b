"""fmmlib3d_b200 -- FMMLIB3D's particle FMM on one NVIDIA B200 (sm_100a).

Python mirror of the reference calling sequences (the ``cf2py`` interfaces of
src/lfmm3dpart.f:205-226 and src/hfmm3dpart.f:206-227): ``lfmm3dpartself``,
``lfmm3dparttarg``, ``lfmm3dpart``, ``l3dpartdirect`` and the Helmholtz
``hfmm3dpartself``, ``hfmm3dparttarg``, ``hfmm3dpart``, ``h3dpartdirect``
(with ``zk`` after ``iprec``) return ``ier`` and the requested outputs.  Every call goes through the C ABI of ``libfmm3d_b200.so``
(include/fmm3d_b200.h); there is no CPU path.  Importing this package on a
machine without the built library raises immediately.

Array conventions follow the Fortran layouts: ``source`` is (N, 3) C-order
(= ``source(3, N)`` in Fortran), complex strengths are complex128, ``fld`` is
(N, 3) complex128.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libfmm3d_b200.so")

if not os.path.exists(LIBPATH):
    raise ImportError(
        "fmmlib3d_b200: %s is missing; build it with `python fmmlib3d_b200/build.py`" % LIBPATH)

_lib = ctypes.CDLL(LIBPATH)
_P = ctypes.c_void_p
_I = ctypes.c_int
_IP = ctypes.POINTER(ctypes.c_int)

for _name in ("lfmm3dpart_", "lfmm3dpartself_"):
    getattr(_lib, _name).restype = None
_lib.lfmm3dparttarg_.restype = None
_lib.l3dpartdirect_.restype = None
_lib.fmm3d_lfmm3dparttarg_device.restype = _I
_lib.fmm3d_lfmm3dparttarg_device.argtypes = [_I, _I, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I, _P,
                                             _I, _P, _P]
_lib.fmm3d_l3dpartdirect_device.restype = _I
_lib.fmm3d_l3dpartdirect_device.argtypes = [_I, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P]
_lib.fmm3d_l3ddirect_points_device.restype = _I
_lib.fmm3d_l3ddirect_points_device.argtypes = [_I, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P, _P]
for _name in ("hfmm3dpart_", "hfmm3dpartself_", "hfmm3dparttarg_", "h3dpartdirect_"):
    getattr(_lib, _name).restype = None
_lib.fmm3d_hfmm3dparttarg_device.restype = _I
_lib.fmm3d_hfmm3dparttarg_device.argtypes = [_I, _P, _I, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I, _P,
                                             _I, _P, _P]
_lib.fmm3d_h3dpartdirect_device.restype = _I
_lib.fmm3d_h3dpartdirect_device.argtypes = [_P, _I, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P,
                                            _P]
_lib.fmm3d_h3ddirect_points_device.restype = _I
_lib.fmm3d_h3ddirect_points_device.argtypes = [_P, _I, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P, _P]
_lib.fmm3d_lfmm3dparttarg_batched_device.restype = _I
_lib.fmm3d_lfmm3dparttarg_batched_device.argtypes = [_I, _I, _P, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _P, _P, _I,
                                                     _P, _I, _P, _P]
_lib.fmm3d_last_launches.restype = _I
_lib.fmm3d_last_depth_capped.restype = _I
_lib.lfmm3dparttarghess_.restype = None
for _name in ("lfmm3dtriatarg_", "lfmm3dtriaself_", "lfmm3dtria_", "l3dtriadirect_", "hfmm3dtriatarg_",
              "hfmm3dtriaself_", "hfmm3dtria_", "h3dtriadirect_"):
    getattr(_lib, _name).restype = None
_lib.fmm3d_lfmm3dtriatarg_device.restype = _I
_lib.fmm3d_lfmm3dtriatarg_device.argtypes = [_I, _I, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I, _P,
                                             _I, _P, _P]
_lib.fmm3d_hfmm3dtriatarg_device.restype = _I
_lib.fmm3d_hfmm3dtriatarg_device.argtypes = [_I, _P, _I, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I,
                                             _P, _I, _P, _P]
_lib.fmm3d_h3dtriadirect_points_device.restype = _I
_lib.fmm3d_h3dtriadirect_points_device.argtypes = [_I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P]
_lib.fmm3d_l3dtriadirect_points_device.restype = _I
_lib.fmm3d_l3dtriadirect_points_device.argtypes = [_I, _P, _I, _P, _I, _P, _I, _P, _P, _P, _P, _P]
_lib.fmm3d_l3dtriadirect_device.restype = _I
_lib.fmm3d_l3dtriadirect_device.argtypes = [_I, _P, _P, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I,
                                            _P, _P]
_lib.l3dtaevalhess_.restype = None
_lib.l3dmpevalhess_.restype = None
_lib.fmm3d_lfmm3dparttarg_hess_device.restype = _I
_lib.fmm3d_lfmm3dparttarg_hess_device.argtypes = [_I, _I, _P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _I, _P,
                                                  _I, _P, _I, _P, _I, _P, _P]
for _name in ("fmm3d_l3dtaevalhess_device", "fmm3d_l3dmpevalhess_device"):
    getattr(_lib, _name).restype = _I
    getattr(_lib, _name).argtypes = [ctypes.c_double, _P, _P, _I, _I, _P, _P, _I, _P, _I, _P, _P]
_lib.fmm3d_set_timing.argtypes = [_I]
_lib.fmm3d_set_stats.argtypes = [_I]
_lib.fmm3d_set_m2l_mode.argtypes = [_I]
_lib.fmm3d_set_precision.argtypes = [_I]
_lib.fmm3d_set_precision_thread.argtypes = [_I]
_lib.fmm3d_set_precision_thread.restype = _I
_lib.fmm3d_set_tensor_m2l.argtypes = [_I]
_lib.fmm3d_set_tensor_m2l.restype = _I
_lib.fmm3d_set_overlap.argtypes = [_I]
_lib.fmm3d_set_tensor_m2l_group.argtypes = [_I]
_lib.fmm3d_set_tensor_m2l_group.restype = _I
_lib.fmm3d_tc_selftest.argtypes = [_I, _I, _P, _P, _P, _I]
_lib.fmm3d_tc_selftest.restype = _I
_lib.fmm3d_lfmm3d_plan_create.argtypes = [_I, _I, _P, _I, _I, _I, _I, _I, _P, _I, _I, _P, ctypes.POINTER(_P)]
_lib.fmm3d_lfmm3d_plan_create.restype = _I
_lib.fmm3d_lfmm3d_plan_create_batched.argtypes = [_I, _I, _P, _P, _I, _I, _I, _I, _P, _P, _I, _I, _P,
                                                  ctypes.POINTER(_P)]
_lib.fmm3d_lfmm3d_plan_create_batched.restype = _I
_lib.fmm3d_lfmm3d_plan_execute.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P, _I, _P]
_lib.fmm3d_lfmm3d_plan_execute.restype = _I
_lib.fmm3d_lfmm3d_plan_destroy.argtypes = [_P]
_lib.fmm3d_lfmm3d_plan_destroy.restype = _I
_lib.fmm3d_lfmm3d_plan_info.argtypes = [_P, _P, _I]
_lib.fmm3d_lfmm3d_plan_info.restype = _I
_lib.fmm3d_lfmm3d_plan_getb.argtypes = [_P, _I, _P, _P, _P]
_lib.fmm3d_d3tstrcrem.argtypes = [_I, _P, _I, _I, _P, _I, _I, _I, _P, ctypes.POINTER(_P)]
_lib.fmm3d_d3tstrcrem.restype = _I
_lib.fmm3d_lfmm3d_plan_getb.restype = _I
_lib.fmm3d_lfmm3d_plan_getl.argtypes = [_P, _I, _I, _P, ctypes.POINTER(_I)]
_lib.fmm3d_lfmm3d_plan_getl.restype = _I
_lib.fmm3d_last_timing.argtypes = [_P, _I]
_lib.fmm3d_last_timing.restype = _I
_lib.fmm3d_last_stats.argtypes = [_P, _I]
_lib.fmm3d_last_stats.restype = _I
_lib.fmm3d_last_error.restype = ctypes.c_char_p
_lib.fmm3d_set_tuning_cache.argtypes = [ctypes.c_char_p]
_lib.fmm3d_set_tuning_cache.restype = _I
_lib.fmm3d_tuning_reload.restype = _I
_lib.fmm3d_tuning_cache_path.argtypes = [ctypes.c_char_p, _I]
_lib.fmm3d_tuning_cache_path.restype = _I
_lib.fmm3d_lfmm3d_plan_set_tuning.argtypes = [_P, _P, _I]
_lib.fmm3d_lfmm3d_plan_set_tuning.restype = _I
_lib.fmm3d_lfmm3d_plan_get_tuning.argtypes = [_P, _P, _I]
_lib.fmm3d_lfmm3d_plan_get_tuning.restype = _I
_lib.fmm3d_lfmm3d_plan_signature.argtypes = [_P, ctypes.c_char_p, _I]
_lib.fmm3d_lfmm3d_plan_signature.restype = _I
_lib.fmm3d_last_tuning.argtypes = [_P, _I, ctypes.c_char_p, _I]
_lib.fmm3d_last_tuning.restype = _I

PASSES = ["tree", "sort", "p2m", "m2m", "p2l", "m2l", "l2l", "eval", "p2p", "scatter", "total"]


def lib():
    return _lib


def _iref(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _ptr(a):
    return a.ctypes.data_as(_P)


def _pts(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim == 2 and a.shape[0] == 3 and a.shape[1] != 3:
        a = np.ascontiguousarray(a.T)
    return a.reshape(-1, 3) if a.size else np.zeros((0, 3))


def _cplx(a, n):
    if a is None:
        return np.zeros(max(n, 1), np.complex128)
    return np.ascontiguousarray(a, dtype=np.complex128).reshape(-1)


def lfmm3dparttarg(iprec, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, iffld,
                   target=None, ifpottarg=0, iffldtarg=0):
    """Laplace FMM over sources and targets; returns (ier, pot, fld, pottarg, fldtarg).

    Same arguments and outputs as lfmm3dparttarg (src/lfmm3dpart.f:138-522);
    unrequested outputs are returned as zero arrays.
    """
    src = _pts(source)
    n = src.shape[0]
    trg = _pts(target) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _cplx(charge, n)
    ds = _cplx(dipstr, n)
    dv = _pts(dipvec) if (ifdipole == 1 and dipvec is not None) else np.zeros((max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = ctypes.c_int(0)
    _lib.lfmm3dparttarg_(ctypes.byref(ier), _iref(iprec), _iref(n), _ptr(src), _iref(ifcharge), _ptr(q),
                         _iref(ifdipole), _ptr(ds), _ptr(dv), _iref(ifpot), _ptr(pot), _iref(iffld), _ptr(fld),
                         _iref(m), _ptr(trg if m else src), _iref(ifpottarg), _ptr(pt), _iref(iffldtarg),
                         _ptr(ft))
    return ier.value, pot[:n], fld[:n], pt[:m], ft[:m]


def lfmm3dparttarghess(iprec, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, iffld, ifhess,
                       target=None, ifpottarg=0, iffldtarg=0, ifhesstarg=0):
    """lfmm3dparttarg with Hessians; returns (ier, pot, fld, hess, pottarg, fldtarg, hesstarg).

    hess / hesstarg: (N, 6) complex, ordered dxx, dyy, dzz, dxy, dxz, dyz.
    """
    src = _pts(source)
    n = src.shape[0]
    trg = _pts(target) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _cplx(charge, n)
    ds = _cplx(dipstr, n)
    dv = _pts(dipvec) if (ifdipole == 1 and dipvec is not None) else np.zeros((max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    hs = np.zeros((max(n, 1), 6), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    ht = np.zeros((max(m, 1), 6), np.complex128)
    ier = ctypes.c_int(0)
    _lib.lfmm3dparttarghess_(ctypes.byref(ier), _iref(iprec), _iref(n), _ptr(src), _iref(ifcharge), _ptr(q),
                             _iref(ifdipole), _ptr(ds), _ptr(dv), _iref(ifpot), _ptr(pot), _iref(iffld), _ptr(fld),
                             _iref(ifhess), _ptr(hs), _iref(m), _ptr(trg if m else src), _iref(ifpottarg), _ptr(pt),
                             _iref(iffldtarg), _ptr(ft), _iref(ifhesstarg), _ptr(ht))
    return ier.value, pot[:n], fld[:n], hs[:n], pt[:m], ft[:m], ht[:m]


def _expansion_layout(coef, nterms):
    """Compact expansion (index n*n+n+m) -> the reference's (0:nterms, -nterms:nterms) column-major array."""
    out = np.zeros((2 * nterms + 1, nterms + 1), np.complex128)
    for n in range(nterms + 1):
        for m in range(-n, n + 1):
            out[m + nterms, n] = coef[n * n + n + m]
    return out


def _evalhess(fn, rscale, center, coef, nterms, ztarg, iffld=1, ifhess=1):
    c = np.ascontiguousarray(coef, np.complex128)
    if c.ndim == 1:
        c = _expansion_layout(c, nterms)
    ctr = np.ascontiguousarray(center, np.float64)
    z = np.ascontiguousarray(ztarg, np.float64)
    pot = np.zeros(1, np.complex128)
    fld = np.zeros(3, np.complex128)
    hess = np.zeros(6, np.complex128)
    ier = ctypes.c_int(0)
    fn(ctypes.byref(ctypes.c_double(rscale)), _ptr(ctr), _ptr(c), _iref(nterms), _ptr(z), _ptr(pot), _iref(iffld),
       _ptr(fld), _iref(ifhess), _ptr(hess), ctypes.byref(ier))
    return ier.value, pot[0], fld, hess


def l3dtaevalhess(rscale, center, local, nterms, ztarg, iffld=1, ifhess=1):
    """l3dtaevalhess at one point; ``local``: compact (index n*n+n+m) or (2p+1, p+1) reference layout.
    Returns (ier, pot, fld(3), hess(6))."""
    return _evalhess(_lib.l3dtaevalhess_, rscale, center, local, nterms, ztarg, iffld, ifhess)


def l3dmpevalhess(rscale, center, mpole, nterms, ztarg, iffld=1, ifhess=1):
    """l3dmpevalhess at one point (layouts as l3dtaevalhess)."""
    return _evalhess(_lib.l3dmpevalhess_, rscale, center, mpole, nterms, ztarg, iffld, ifhess)


def evalhess_device(kind, rscale, center, coef, nterms, targ, pot, fld=None, hess=None, stream=0):
    """One expansion at many device points.  kind "local" or "mpole"; ``coef``: device float64 tensor in
    the reference layout ((2p+1)*(p+1)*2 doubles); ``targ`` (M,3); outputs ``pot`` (M,2), ``fld`` (M,6),
    ``hess`` (M,12) float64 or None.  Returns ier."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    fn = _lib.fmm3d_l3dtaevalhess_device if kind == "local" else _lib.fmm3d_l3dmpevalhess_device
    ctr = np.ascontiguousarray(center, np.float64)
    return fn(float(rscale), _ptr(ctr), ptr(coef), nterms, targ.shape[0], ptr(targ), ptr(pot), int(fld is not None),
              ptr(fld), int(hess is not None), ptr(hess), _P(stream))


def lfmm3dparttarg_hess_device(iprec, source, charge, dipstr, dipvec, pot, fld, hess, target=None, pottarg=None,
                               fldtarg=None, hesstarg=None, stream=0):
    """lfmm3dparttarg_device with Hessians: ``hess`` / ``hesstarg`` (N,12) float64 tensors or None."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    n = source.shape[0]
    m = 0 if target is None else target.shape[0]
    return _lib.fmm3d_lfmm3dparttarg_hess_device(
        iprec, n, ptr(source), int(charge is not None), ptr(charge), int(dipstr is not None), ptr(dipstr),
        ptr(dipvec), int(pot is not None), ptr(pot), int(fld is not None), ptr(fld), int(hess is not None),
        ptr(hess), m, ptr(target), int(pottarg is not None), ptr(pottarg), int(fldtarg is not None), ptr(fldtarg),
        int(hesstarg is not None), ptr(hesstarg), _P(stream))


def _tri_args(triaflat, trianorm, source, charge, dipstr, target):
    tri = np.ascontiguousarray(triaflat, dtype=np.float64).reshape(-1, 3, 3)
    n = tri.shape[0]
    nrm = np.ascontiguousarray(trianorm, dtype=np.float64).reshape(-1, 3) if trianorm is not None else None
    if nrm is None:
        e = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
        nrm = np.ascontiguousarray(e / np.linalg.norm(e, axis=1)[:, None])
    src = _pts(source) if source is not None else np.ascontiguousarray(tri.mean(axis=1))
    trg = _pts(target) if target is not None else np.zeros((0, 3))
    return tri, n, nrm, src, trg, _cplx(charge, n), _cplx(dipstr, n)


def lfmm3dtriatarg(iprec, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, ifpot, iffld,
                   target=None, ifpottarg=0, iffldtarg=0):
    """Laplace layer potentials of flat triangles (lfmm3dtriatarg, src/lfmm3dtria.f:121);
    returns (ier, pot, fld, pottarg, fldtarg).  triaflat (N,3,3) vertices, trianorm (N,3) unit
    normals (None: from the vertex order), source (N,3) centroids (None: computed)."""
    tri, n, nrm, src, trg, q, ds = _tri_args(triaflat, trianorm, source, charge, dipstr, target)
    m = trg.shape[0]
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = ctypes.c_int(0)
    dv = np.zeros((max(n, 1), 3))
    _lib.lfmm3dtriatarg_(ctypes.byref(ier), _iref(iprec), _iref(n), _ptr(tri), _ptr(nrm), _ptr(src), _iref(ifcharge),
                         _ptr(q), _iref(ifdipole), _ptr(ds), _ptr(dv), _iref(ifpot), _ptr(pot), _iref(iffld),
                         _ptr(fld), _iref(m), _ptr(trg if m else src), _iref(ifpottarg), _ptr(pt), _iref(iffldtarg),
                         _ptr(ft))
    return ier.value, pot[:n], fld[:n], pt[:m], ft[:m]


def hfmm3dtriatarg(iprec, zk, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, ifpot, iffld,
                   target=None, ifpottarg=0, iffldtarg=0):
    """Helmholtz layer potentials of flat triangles (hfmm3dtriatarg, src/hfmm3dtria.f:133);
    returns (ier, pot, fld, pottarg, fldtarg); arguments as lfmm3dtriatarg plus zk."""
    tri, n, nrm, src, trg, q, ds = _tri_args(triaflat, trianorm, source, charge, dipstr, target)
    m = trg.shape[0]
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = ctypes.c_int(0)
    dv = np.zeros((max(n, 1), 3))
    z = np.array([complex(zk).real, complex(zk).imag])
    _lib.hfmm3dtriatarg_(ctypes.byref(ier), _iref(iprec), _ptr(z), _iref(n), _ptr(tri), _ptr(nrm), _ptr(src),
                         _iref(ifcharge), _ptr(q), _iref(ifdipole), _ptr(ds), _ptr(dv), _iref(ifpot), _ptr(pot),
                         _iref(iffld), _ptr(fld), _iref(m), _ptr(trg if m else src), _iref(ifpottarg), _ptr(pt),
                         _iref(iffldtarg), _ptr(ft))
    return ier.value, pot[:n], fld[:n], pt[:m], ft[:m]


def hfmm3dtriaself(iprec, zk, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, ifpot, iffld):
    ier, pot, fld, _, _ = hfmm3dtriatarg(iprec, zk, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr,
                                         ifpot, iffld)
    return ier, pot, fld


def h3dtriadirect(nqtri, zk, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, ifpot, iffld,
                  target=None, ifpottarg=0, iffldtarg=0):
    """O(N^2) Helmholtz layer potentials (h3dtriadirect) with near-field quadrature degree nqtri."""
    tri, n, nrm, src, trg, q, ds = _tri_args(triaflat, trianorm, source, charge, dipstr, target)
    m = trg.shape[0]
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    dv = np.zeros((max(n, 1), 3))
    z = np.array([complex(zk).real, complex(zk).imag])
    _lib.h3dtriadirect_(_iref(nqtri), _ptr(z), _iref(n), _ptr(tri), _ptr(nrm), _ptr(src), _iref(ifcharge), _ptr(q),
                        _iref(ifdipole), _ptr(ds), _ptr(dv), _iref(ifpot), _ptr(pot), _iref(iffld), _ptr(fld),
                        _iref(m), _ptr(trg if m else src), _iref(ifpottarg), _ptr(pt), _iref(iffldtarg), _ptr(ft))
    return pot[:n], fld[:n], pt[:m], ft[:m]


def htri_direct_points_device(nqtri, zk, triaflat, charge, dipstr, pts, self_idx, pot, fld, stream=0):
    """Helmholtz triangle direct sum at device points; layouts as tri_direct_points_device."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    z = np.array([complex(zk).real, complex(zk).imag])
    return _lib.fmm3d_h3dtriadirect_points_device(nqtri, _ptr(z), triaflat.shape[0], ptr(triaflat),
                                                  int(charge is not None), ptr(charge), int(dipstr is not None),
                                                  ptr(dipstr), pts.shape[0], ptr(pts), ptr(self_idx), 0, ptr(pot),
                                                  ptr(fld), _P(stream))


def hfmm3dtriatarg_device(iprec, zk, triaflat, trianorm, source, charge, dipstr, pot, fld, target=None, pottarg=None,
                          fldtarg=None, stream=0):
    """hfmm3dtriatarg on device tensors (layouts as lfmm3dtriatarg_device).  Returns ier."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    n = source.shape[0]
    m = 0 if target is None else target.shape[0]
    z = np.array([complex(zk).real, complex(zk).imag])
    return _lib.fmm3d_hfmm3dtriatarg_device(
        iprec, _ptr(z), n, ptr(triaflat), ptr(trianorm), ptr(source), int(charge is not None), ptr(charge),
        int(dipstr is not None), ptr(dipstr), None, int(pot is not None), ptr(pot), int(fld is not None), ptr(fld), m,
        ptr(target), int(pottarg is not None), ptr(pottarg), int(fldtarg is not None), ptr(fldtarg), _P(stream))


def lfmm3dtriaself(iprec, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, ifpot, iffld):
    """lfmm3dtriaself: (ier, pot, fld) at the centroids."""
    ier, pot, fld, _, _ = lfmm3dtriatarg(iprec, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr,
                                         ifpot, iffld)
    return ier, pot, fld


def l3dtriadirect(triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, ifpot, iffld,
                  target=None, ifpottarg=0, iffldtarg=0):
    """O(N^2) layer potentials by exact integrals (l3dtriadirect); returns (pot, fld, pottarg, fldtarg)."""
    tri, n, nrm, src, trg, q, ds = _tri_args(triaflat, trianorm, source, charge, dipstr, target)
    m = trg.shape[0]
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    dv = np.zeros((max(n, 1), 3))
    _lib.l3dtriadirect_(_iref(n), _ptr(tri), _ptr(nrm), _ptr(src), _iref(ifcharge), _ptr(q), _iref(ifdipole),
                        _ptr(ds), _ptr(dv), _iref(ifpot), _ptr(pot), _iref(iffld), _ptr(fld), _iref(m),
                        _ptr(trg if m else src), _iref(ifpottarg), _ptr(pt), _iref(iffldtarg), _ptr(ft))
    return pot[:n], fld[:n], pt[:m], ft[:m]


def lfmm3dtriatarg_device(iprec, triaflat, trianorm, source, charge, dipstr, pot, fld, target=None, pottarg=None,
                          fldtarg=None, stream=0):
    """lfmm3dtriatarg on device tensors: triaflat (N,9), trianorm / source / target (N,3) float64;
    charge / dipstr (N,2); outputs pot (N,2), fld (N,6) or None.  Returns ier."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    n = source.shape[0]
    m = 0 if target is None else target.shape[0]
    return _lib.fmm3d_lfmm3dtriatarg_device(
        iprec, n, ptr(triaflat), ptr(trianorm), ptr(source), int(charge is not None), ptr(charge),
        int(dipstr is not None), ptr(dipstr), None, int(pot is not None), ptr(pot), int(fld is not None), ptr(fld), m,
        ptr(target), int(pottarg is not None), ptr(pottarg), int(fldtarg is not None), ptr(fldtarg), _P(stream))


def tri_direct_points_device(triaflat, charge, dipstr, pts, self_idx, pot, fld, stream=0):
    """Triangle direct sum at device points ``pts`` (M,3); ``self_idx`` int32 (M,) (the triangle whose
    centroid the point is, or -1) or None; ``pot`` (M,2), ``fld`` (M,6) float64.  Returns ier."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    n = triaflat.shape[0]
    return _lib.fmm3d_l3dtriadirect_points_device(n, ptr(triaflat), int(charge is not None), ptr(charge),
                                                  int(dipstr is not None), ptr(dipstr), pts.shape[0], ptr(pts),
                                                  ptr(self_idx), ptr(pot), ptr(fld), _P(stream))


def lfmm3dpartself(iprec, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, iffld):
    """Laplace FMM among sources; returns (ier, pot, fld) as lfmm3dpartself."""
    ier, pot, fld, _, _ = lfmm3dparttarg(iprec, source, ifcharge, charge, ifdipole, dipstr, dipvec,
                                         ifpot, iffld)
    return ier, pot, fld


lfmm3dpart = lfmm3dpartself


def l3dpartdirect(source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, iffld,
                  target=None, ifpottarg=0, iffldtarg=0):
    """O(N^2) Laplace sum on the GPU; returns (pot, fld, pottarg, fldtarg) as l3dpartdirect."""
    src = _pts(source)
    n = src.shape[0]
    trg = _pts(target) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _cplx(charge, n)
    ds = _cplx(dipstr, n)
    dv = _pts(dipvec) if (ifdipole == 1 and dipvec is not None) else np.zeros((max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    _lib.l3dpartdirect_(_iref(n), _ptr(src), _iref(ifcharge), _ptr(q), _iref(ifdipole), _ptr(ds), _ptr(dv),
                        _iref(ifpot), _ptr(pot), _iref(iffld), _ptr(fld), _iref(m), _ptr(trg if m else src),
                        _iref(ifpottarg), _ptr(pt), _iref(iffldtarg), _ptr(ft))
    return pot[:n], fld[:n], pt[:m], ft[:m]


def lfmm3dparttarg_device(iprec, source, charge, dipstr, dipvec, pot, fld, target=None, pottarg=None,
                          fldtarg=None, stream=0):
    """FMM on device-resident torch tensors (float64 views of the Fortran layouts).

    ``source``/``target``/``dipvec``: (N,3) float64 CUDA tensors; ``charge``/
    ``dipstr``: (N,2) float64 (re, im); outputs ``pot`` (N,2) and ``fld``
    (N,6) float64, or None when not requested.  Returns ier.
    """
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    n = source.shape[0]
    m = 0 if target is None else target.shape[0]
    return _lib.fmm3d_lfmm3dparttarg_device(
        iprec, n, ptr(source), int(charge is not None), ptr(charge), int(dipstr is not None), ptr(dipstr),
        ptr(dipvec), int(pot is not None), ptr(pot), int(fld is not None), ptr(fld), m, ptr(target),
        int(pottarg is not None), ptr(pottarg), int(fldtarg is not None), ptr(fldtarg), _P(stream))


def direct_points_device(source, charge, dipstr, dipvec, pts, skip, pot, fld, stream=0):
    """Direct sum at device points ``pts`` (M,3) with per-point excluded source ``skip``
    (int32 (M,) or None); ``pot`` (M,2), ``fld`` (M,6) float64 outputs.  Returns ier."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    return _lib.fmm3d_l3ddirect_points_device(
        source.shape[0], ptr(source), int(charge is not None), ptr(charge), int(dipstr is not None), ptr(dipstr),
        ptr(dipvec), pts.shape[0], ptr(pts), ptr(skip), ptr(pot), ptr(fld), _P(stream))


def lfmm3dparttarg_batched_device(iprec, src_offsets, source, charge, dipstr, dipvec, pot, fld, trg_offsets=None,
                                  target=None, pottarg=None, fldtarg=None, stream=0):
    """Many independent Laplace FMMs in one call on device-resident torch tensors.

    ``src_offsets`` (ninst+1 ints, from 0): instance i owns rows
    src_offsets[i]:src_offsets[i+1] of the concatenated ``source``/``charge``/...
    arrays (layouts as lfmm3dparttarg_device); ``trg_offsets`` likewise for
    ``target``.  Outputs are written in the concatenated order.  Returns ier.
    """
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    so = np.ascontiguousarray(src_offsets, dtype=np.int32)
    to = None if trg_offsets is None else np.ascontiguousarray(trg_offsets, dtype=np.int32)
    return _lib.fmm3d_lfmm3dparttarg_batched_device(
        iprec, len(so) - 1, _ptr(so), ptr(source), int(charge is not None), ptr(charge), int(dipstr is not None),
        ptr(dipstr), ptr(dipvec), int(pot is not None), ptr(pot), int(fld is not None), ptr(fld),
        None if to is None else _ptr(to), ptr(target), int(pottarg is not None), ptr(pottarg),
        int(fldtarg is not None), ptr(fldtarg), _P(stream))


TUNING_KNOBS = ("m2l_kt", "trans_kt", "tc_variant", "overlap", "p2p_ept")
TUNING_FORMS = ("fp64-rotation", "fp64-dense", "mixed-cuda", "mixed-tc")


def _knob_array(knobs):
    if isinstance(knobs, dict):
        unknown = set(knobs) - set(TUNING_KNOBS)
        if unknown:
            raise ValueError("unknown tuning knobs: %s" % sorted(unknown))
        return [int(knobs.get(k, 0)) for k in TUNING_KNOBS]
    a = [int(v) for v in knobs]
    if len(a) != len(TUNING_KNOBS):
        raise ValueError("expected %d knobs" % len(TUNING_KNOBS))
    return a


def _tuning_dict(out):
    d = {k: int(out[i]) for i, k in enumerate(TUNING_KNOBS)}
    d["form"] = TUNING_FORMS[int(out[len(TUNING_KNOBS)])]
    d["from_cache"] = bool(out[len(TUNING_KNOBS) + 1])
    return d


def set_tuning_cache(path):
    """Tuning cache file for later calls: a path, None (the default: $FMM3D_TUNING_CACHE,
    else tuning_cache.json beside the library) or "" (no cache)."""
    _lib.fmm3d_set_tuning_cache(None if path is None else str(path).encode())


def tuning_reload():
    """Re-read the tuning cache; returns the number of entries."""
    return _lib.fmm3d_tuning_reload()


def tuning_cache_path():
    n = _lib.fmm3d_tuning_cache_path(None, 0)
    buf = ctypes.create_string_buffer(max(n, 1))
    _lib.fmm3d_tuning_cache_path(buf, len(buf))
    return buf.value.decode()


def last_tuning():
    """(knobs dict, signature) of this thread's last single Laplace call."""
    out = np.zeros(len(TUNING_KNOBS) + 2, np.int32)
    buf = ctypes.create_string_buffer(1024)
    _lib.fmm3d_last_tuning(_ptr(out), len(out), buf, len(buf))
    return _tuning_dict(out), buf.value.decode()


class LaplacePlan:
    """A Laplace FMM geometry kept on the device: build once for fixed sources and
    targets (device tensors, layouts as lfmm3dparttarg_device), then ``execute`` for
    new charges / dipoles.  ``use_graph`` replays a CUDA graph of the passes.
    ``getb`` / ``getl`` answer d3tgetb / d3tgetl queries (1-based boxes)."""

    def __init__(self, iprec, source, ifcharge=1, ifdipole=0, ifpot=1, iffld=1, target=None, ifpottarg=0,
                 iffldtarg=0, stream=0, src_offsets=None, trg_offsets=None):
        """``src_offsets`` / ``trg_offsets`` (ninst+1 ints): a batch of independent instances."""
        h = _P()
        m = 0 if target is None else target.shape[0]
        tp = None if target is None else _P(target.data_ptr())
        if src_offsets is None:
            ier = _lib.fmm3d_lfmm3d_plan_create(
                iprec, source.shape[0], _P(source.data_ptr()), ifcharge, ifdipole, ifpot, iffld, m, tp, ifpottarg,
                iffldtarg, _P(stream), ctypes.byref(h))
        else:
            so = np.ascontiguousarray(src_offsets, dtype=np.int32)
            to = None if trg_offsets is None else np.ascontiguousarray(trg_offsets, dtype=np.int32)
            ier = _lib.fmm3d_lfmm3d_plan_create_batched(
                iprec, len(so) - 1, _ptr(so), _P(source.data_ptr()), ifcharge, ifdipole, ifpot, iffld,
                None if to is None else _ptr(to), tp, ifpottarg, iffldtarg, _P(stream), ctypes.byref(h))
        if ier != 0:
            raise RuntimeError("plan creation failed, ier=%d: %s" % (ier, last_error()))
        self._h = h

    def execute(self, charge=None, dipstr=None, dipvec=None, pot=None, fld=None, pottarg=None, fldtarg=None,
                use_graph=True, stream=0):
        def ptr(t):
            return None if t is None else _P(t.data_ptr())
        return _lib.fmm3d_lfmm3d_plan_execute(self._h, ptr(charge), ptr(dipstr), ptr(dipvec), ptr(pot), ptr(fld),
                                              ptr(pottarg), ptr(fldtarg), int(bool(use_graph)), _P(stream))

    def info(self):
        out = np.zeros(10)
        _lib.fmm3d_lfmm3d_plan_info(self._h, _ptr(out), 10)
        keys = ["nboxes", "nlev", "nleaves", "nterms", "nsource", "ntarget"]
        d = {k: int(out[i]) for i, k in enumerate(keys)}
        d["center"], d["size"] = out[6:9].copy(), float(out[9])
        return d

    def getb(self, ibox):
        box = np.zeros(20, np.int32)
        c = np.zeros(3)
        corners = np.zeros((8, 3))
        ier = _lib.fmm3d_lfmm3d_plan_getb(self._h, int(ibox), _ptr(box), _ptr(c), _ptr(corners))
        return ier, box, c, corners

    def getl(self, ibox, itype):
        n = _I(0)
        _lib.fmm3d_lfmm3d_plan_getl(self._h, int(ibox), int(itype), None, ctypes.byref(n))
        lst = np.zeros(max(n.value, 1), np.int32)
        ier = _lib.fmm3d_lfmm3d_plan_getl(self._h, int(ibox), int(itype), _ptr(lst), ctypes.byref(n))
        return ier, lst[:n.value]

    def set_tuning(self, knobs):
        """Launch-shape knobs (dict with keys of ``TUNING_KNOBS`` or a sequence of five;
        0 = automatic).  Returns 0, or 2 if this problem cannot take a value (the
        plan keeps its previous knobs)."""
        a = np.asarray(_knob_array(knobs), np.int32)
        return _lib.fmm3d_lfmm3d_plan_set_tuning(self._h, _ptr(a), len(a))

    def get_tuning(self):
        """The knobs in use (0 where the form has none), the form and whether they came
        from the tuning cache."""
        out = np.zeros(len(TUNING_KNOBS) + 2, np.int32)
        _lib.fmm3d_lfmm3d_plan_get_tuning(self._h, _ptr(out), len(out))
        return _tuning_dict(out)

    def signature(self):
        """The plan's problem signature (the tuning cache key)."""
        n = _lib.fmm3d_lfmm3d_plan_signature(self._h, None, 0)
        buf = ctypes.create_string_buffer(max(n, 1))
        _lib.fmm3d_lfmm3d_plan_signature(self._h, buf, len(buf))
        return buf.value.decode()

    def close(self):
        if getattr(self, "_h", None):
            _lib.fmm3d_lfmm3d_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass


class OctTree(LaplacePlan):
    """d3tstrcrem (src/d3tstrcr.f:264-460): the adaptive octree of device tensors
    ``source`` (N, 3) and ``target`` (M, 3) alone, with the reference's options
    (``ifempty`` = 1 keeps empty boxes; every box above ``minlevel`` is split;
    none at ``maxlevel`` or deeper, capped at 21 levels).  Answers ``info``,
    ``getb`` and ``getl`` like a plan; it has no charges to execute."""

    def __init__(self, source, nbox, target=None, ifempty=0, minlevel=0, maxlevel=100, stream=0):
        h = _P()
        m = 0 if target is None else target.shape[0]
        tp = None if target is None else _P(target.data_ptr())
        ier = _lib.fmm3d_d3tstrcrem(source.shape[0], _P(source.data_ptr()), int(nbox), m, tp, int(ifempty),
                                    int(minlevel), int(maxlevel), _P(stream), ctypes.byref(h))
        if ier != 0:
            raise RuntimeError("d3tstrcrem failed, ier=%d: %s" % (ier, last_error()))
        self._h = h


def _zk(zk):
    z = complex(zk)
    return np.array([z.real, z.imag], np.float64)


def hfmm3dparttarg(iprec, zk, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, iffld,
                   target=None, ifpottarg=0, iffldtarg=0):
    """Helmholtz FMM over sources and targets; returns (ier, pot, fld, pottarg, fldtarg).

    Same arguments and outputs as hfmm3dparttarg (src/hfmm3dpart.f:141-539):
    the kernel is e^{i zk r}/r; unrequested outputs are returned as zeros.
    """
    src = _pts(source)
    n = src.shape[0]
    trg = _pts(target) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _cplx(charge, n)
    ds = _cplx(dipstr, n)
    dv = _pts(dipvec) if (ifdipole == 1 and dipvec is not None) else np.zeros((max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = ctypes.c_int(0)
    k = _zk(zk)
    _lib.hfmm3dparttarg_(ctypes.byref(ier), _iref(iprec), _ptr(k), _iref(n), _ptr(src), _iref(ifcharge), _ptr(q),
                         _iref(ifdipole), _ptr(ds), _ptr(dv), _iref(ifpot), _ptr(pot), _iref(iffld), _ptr(fld),
                         _iref(m), _ptr(trg if m else src), _iref(ifpottarg), _ptr(pt), _iref(iffldtarg),
                         _ptr(ft))
    return ier.value, pot[:n], fld[:n], pt[:m], ft[:m]


def hfmm3dpartself(iprec, zk, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, iffld):
    """Helmholtz FMM among sources; returns (ier, pot, fld) as hfmm3dpartself."""
    ier, pot, fld, _, _ = hfmm3dparttarg(iprec, zk, source, ifcharge, charge, ifdipole, dipstr, dipvec,
                                         ifpot, iffld)
    return ier, pot, fld


hfmm3dpart = hfmm3dpartself


def h3dpartdirect(zk, source, ifcharge, charge, ifdipole, dipstr, dipvec, ifpot, iffld,
                  target=None, ifpottarg=0, iffldtarg=0):
    """O(N^2) Helmholtz sum on the GPU; returns (pot, fld, pottarg, fldtarg) as h3dpartdirect."""
    src = _pts(source)
    n = src.shape[0]
    trg = _pts(target) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _cplx(charge, n)
    ds = _cplx(dipstr, n)
    dv = _pts(dipvec) if (ifdipole == 1 and dipvec is not None) else np.zeros((max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    k = _zk(zk)
    _lib.h3dpartdirect_(_ptr(k), _iref(n), _ptr(src), _iref(ifcharge), _ptr(q), _iref(ifdipole), _ptr(ds), _ptr(dv),
                        _iref(ifpot), _ptr(pot), _iref(iffld), _ptr(fld), _iref(m), _ptr(trg if m else src),
                        _iref(ifpottarg), _ptr(pt), _iref(iffldtarg), _ptr(ft))
    return pot[:n], fld[:n], pt[:m], ft[:m]


def hfmm3dparttarg_device(iprec, zk, source, charge, dipstr, dipvec, pot, fld, target=None, pottarg=None,
                          fldtarg=None, stream=0):
    """Helmholtz FMM on device-resident torch tensors (layouts as lfmm3dparttarg_device)."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    n = source.shape[0]
    m = 0 if target is None else target.shape[0]
    k = _zk(zk)
    return _lib.fmm3d_hfmm3dparttarg_device(
        iprec, _ptr(k), n, ptr(source), int(charge is not None), ptr(charge), int(dipstr is not None), ptr(dipstr),
        ptr(dipvec), int(pot is not None), ptr(pot), int(fld is not None), ptr(fld), m, ptr(target),
        int(pottarg is not None), ptr(pottarg), int(fldtarg is not None), ptr(fldtarg), _P(stream))


def hdirect_points_device(zk, source, charge, dipstr, dipvec, pts, skip, pot, fld, stream=0):
    """Helmholtz direct sum at device points (as direct_points_device).  Returns ier."""
    def ptr(t):
        return None if t is None else _P(t.data_ptr())
    k = _zk(zk)
    return _lib.fmm3d_h3ddirect_points_device(
        _ptr(k), source.shape[0], ptr(source), int(charge is not None), ptr(charge), int(dipstr is not None),
        ptr(dipstr), ptr(dipvec), pts.shape[0], ptr(pts), ptr(skip), ptr(pot), ptr(fld), _P(stream))


def last_launches():
    """Kernel launches issued by the last library call on this thread."""
    return _lib.fmm3d_last_launches()


def set_timing(on=True):
    _lib.fmm3d_set_timing(1 if on else 0)


def set_stats(on=True):
    """Gather tree and interaction statistics on the following calls (last_stats())."""
    _lib.fmm3d_set_stats(1 if on else 0)


def set_m2l_mode(mode):
    """0 automatic, 1 rotate-shift-rotate, 2 dense per-offset operators (nterms <= 16)."""
    _lib.fmm3d_set_m2l_mode(int(mode))


def set_precision(mode):
    """0 FP64 throughout (default), 1 mixed FP32 P2P/M2L for iprec <= 1."""
    _lib.fmm3d_set_precision(int(mode))


def set_precision_thread(mode):
    """Arithmetic form for later calls on this host thread only: 0 FP64, 1 mixed (iprec <= 1),
    -1 follow the process-wide ``set_precision``."""
    if _lib.fmm3d_set_precision_thread(int(mode)) != 0:
        raise ValueError("unknown precision mode %r" % (mode,))


def set_tensor_m2l(mode):
    """Mixed-form M2L: 0 FP32 CUDA cores, 1 (default) / 2 tensor cores (tcgen05, split TF32; staging variants)."""
    if _lib.fmm3d_set_tensor_m2l(int(mode)) != 0:
        raise ValueError("unknown tensor M2L mode %r" % (mode,))


def set_overlap(on=True):
    """Laplace: near field concurrent with the far field (default) or all passes serial (same results)."""
    _lib.fmm3d_set_overlap(1 if on else 0)


def set_tensor_m2l_group(slots):
    """Tensor-core M2L: list-2 slots per TMEM sum before it is added into FP32 registers (0: one per tile)."""
    if _lib.fmm3d_set_tensor_m2l_group(int(slots)) != 0:
        raise ValueError("bad group %r" % (slots,))


def tc_selftest(A, B, nprod=3):
    """D = A @ B.T on the tensor cores (A: 128 x K, B: N x K float32).  Returns (status, D)."""
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    D = np.zeros((128, B.shape[0]), np.float32)
    st = _lib.fmm3d_tc_selftest(B.shape[0], A.shape[1], _ptr(A), _ptr(B), _ptr(D), int(nprod))
    return st, D


def last_timing():
    """Per-pass device milliseconds of the last call on this thread."""
    out = np.zeros(len(PASSES))
    k = _lib.fmm3d_last_timing(_ptr(out), len(PASSES))
    return dict(zip(PASSES[:k], out[:k]))


def last_stats():
    out = np.zeros(9 + 128 + 22, np.int64)
    k = _lib.fmm3d_last_stats(_ptr(out), out.size)
    if k == 0:
        return {}
    names = ["nboxes", "nlev", "nleaves", "nterms", "_l1", "_l3", "_l4", "p2p_pairs", "m2l_pairs"]
    d = {nm: int(out[i]) for i, nm in enumerate(names) if not nm.startswith("_")}
    d["m2l_pt_hist"] = {i: int(out[9 + i]) for i in range(128) if out[9 + i]}
    if k > 9 + 128:  # Helmholtz: expansion order per level
        d["nterms_level"] = [int(v) for v in out[9 + 128:k]]
    return d


def last_depth_capped():
    """Boxes of level 21 in this thread's last tree that the reference (100 levels) would split further."""
    return _lib.fmm3d_last_depth_capped()


def last_error():
    return _lib.fmm3d_last_error().decode()
