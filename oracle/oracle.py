"""ctypes binding of oracle/fmm3d_oracle.c (test infrastructure only).

The C file restates FMMLIB3D's Laplace particle FMM (lfmm3dparttarg and its
tree, lists, expansion orders and operators) and the O(N^2) direct sum
l3dpartdirect.  See the header of fmm3d_oracle.c for the parity status.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle_fmm3d.so")
_lib = None

c_int = ctypes.c_int
c_dbl = ctypes.c_double
P = ctypes.c_void_p


def build():
    """Compile the oracle with the committed Makefile (gcc, OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        _lib.oracle_hkrand.restype = c_dbl
        _lib.oracle_hkrand.argtypes = [c_int]
        _lib.oracle_l3dterms.restype = c_int
        _lib.oracle_l3dterms.argtypes = [c_dbl]
        _lib.oracle_lap_eps.restype = c_dbl
        _lib.oracle_lap_eps.argtypes = [c_int]
        _lib.oracle_lap_nbox.restype = c_int
        _lib.oracle_lap_nbox.argtypes = [c_int, c_int, c_int]
        _lib.oracle_tree_build.restype = P
        _lib.oracle_tree_build.argtypes = [c_int, P, c_int, P, c_int]
        _lib.oracle_tree_build_em.restype = P
        _lib.oracle_tree_build_em.argtypes = [c_int, P, c_int, P, c_int, c_int, c_int, c_int]
        for f in ("oracle_tree_nboxes", "oracle_tree_nlev"):
            getattr(_lib, f).restype = c_int
            getattr(_lib, f).argtypes = [P]
        _lib.oracle_tree_list_len.restype = c_int
        _lib.oracle_tree_list_len.argtypes = [P, c_int]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(P)


def _c128(a, n):
    if a is None:
        return np.zeros(max(n, 1), np.complex128)
    return np.ascontiguousarray(a, dtype=np.complex128)


def _f64(a, shape):
    if a is None:
        return np.zeros(shape, np.float64)
    return np.ascontiguousarray(a, dtype=np.float64)


def hkrand_stream(count, reset=True):
    """`count` successive values of the examples/hkrand.f generator."""
    L = lib()
    if reset:
        L.oracle_hkrand_reset()
    return np.array([L.oracle_hkrand(0) for _ in range(count)])


def l3dterms(eps):
    return lib().oracle_l3dterms(eps)


def l3dterms_list2(eps):
    t = np.zeros(343, np.int32)
    lib().oracle_l3dterms_list2(c_dbl(eps), _p(t))
    return t.reshape(7, 7, 7)


def lap_eps(iprec):
    return lib().oracle_lap_eps(iprec)


def lap_nbox(iprec, ns, nt):
    return lib().oracle_lap_nbox(iprec, ns, nt)


def l3dpartdirect(source, charge=None, dipstr=None, dipvec=None, target=None,
                  ifpot=1, iffld=1, ifpottarg=1, iffldtarg=1):
    """Full O(N^2) direct sum.  Arrays are (N,3) / (N,) numpy arrays."""
    src = _f64(source, (0, 3))
    n = src.shape[0]
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _c128(charge, n)
    ds = _c128(dipstr, n)
    dv = _f64(dipvec, (max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    lib().oracle_l3dpartdirect(
        c_int(n), _p(src), c_int(int(charge is not None)), _p(q), c_int(int(dipstr is not None)),
        _p(ds), _p(dv), c_int(ifpot), _p(pot), c_int(iffld), _p(fld), c_int(m), _p(trg),
        c_int(ifpottarg if m else 0), _p(pt), c_int(iffldtarg if m else 0), _p(ft))
    return pot[:n], fld[:n], pt[:m], ft[:m]


def direct_at(source, pts, skip=None, charge=None, dipstr=None, dipvec=None):
    """Direct pot/fld at arbitrary points; skip[k] = source index excluded."""
    src = _f64(source, (0, 3))
    n = src.shape[0]
    pts = _f64(pts, (0, 3))
    k = pts.shape[0]
    q = _c128(charge, n)
    ds = _c128(dipstr, n)
    dv = _f64(dipvec, (max(n, 1), 3))
    sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.int64)
    pot = np.zeros(max(k, 1), np.complex128)
    fld = np.zeros((max(k, 1), 3), np.complex128)
    lib().oracle_l3ddirect_points(
        c_int(n), _p(src), c_int(int(charge is not None)), _p(q), c_int(int(dipstr is not None)),
        _p(ds), _p(dv), c_int(k), _p(pts), _p(sk), _p(pot), _p(fld))
    return pot[:k], fld[:k]


def lfmm3dparttarg(iprec, source, charge=None, dipstr=None, dipvec=None, target=None,
                   ifpot=1, iffld=1, ifpottarg=1, iffldtarg=1, timing=False):
    src = _f64(source, (0, 3))
    n = src.shape[0]
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _c128(charge, n)
    ds = _c128(dipstr, n)
    dv = _f64(dipvec, (max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = c_int(0)
    tinfo = np.zeros(8)
    lib().oracle_lfmm3dparttarg(
        ctypes.byref(ier), c_int(iprec), c_int(n), _p(src), c_int(int(charge is not None)), _p(q),
        c_int(int(dipstr is not None)), _p(ds), _p(dv), c_int(ifpot), _p(pot), c_int(iffld), _p(fld),
        c_int(m), _p(trg if m else np.zeros((1, 3))), c_int(ifpottarg if m else 0), _p(pt),
        c_int(iffldtarg if m else 0), _p(ft), _p(tinfo))
    out = (ier.value, pot[:n], fld[:n], pt[:m], ft[:m])
    return out + (tinfo,) if timing else out


def lfmm3dparttarg_hess(iprec, source, charge=None, dipstr=None, dipvec=None, target=None,
                        ifpot=1, iffld=1, ifhess=1, ifpottarg=1, iffldtarg=1, ifhesstarg=1):
    """lfmm3dparttarg with Hessians (dxx,dyy,dzz,dxy,dxz,dyz per point):
    returns (ier, pot, fld, hess, pottarg, fldtarg, hesstarg)."""
    src = _f64(source, (0, 3))
    n = src.shape[0]
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    q = _c128(charge, n)
    ds = _c128(dipstr, n)
    dv = _f64(dipvec, (max(n, 1), 3))
    pot = np.zeros(max(n, 1), np.complex128)
    fld = np.zeros((max(n, 1), 3), np.complex128)
    hs = np.zeros((max(n, 1), 6), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128)
    ft = np.zeros((max(m, 1), 3), np.complex128)
    ht = np.zeros((max(m, 1), 6), np.complex128)
    ier = c_int(0)
    lib().oracle_lfmm3dparttarg_hess(
        ctypes.byref(ier), c_int(iprec), c_int(n), _p(src), c_int(int(charge is not None)), _p(q),
        c_int(int(dipstr is not None)), _p(ds), _p(dv), c_int(ifpot), _p(pot), c_int(iffld), _p(fld),
        c_int(ifhess), _p(hs), c_int(m), _p(trg if m else np.zeros((1, 3))), c_int(ifpottarg if m else 0), _p(pt),
        c_int(iffldtarg if m else 0), _p(ft), c_int(ifhesstarg if m else 0), _p(ht))
    return ier.value, pot[:n], fld[:n], hs[:n], pt[:m], ft[:m], ht[:m]


# ---------------------------------------------------------------- triangles

def tri_near(tri, pts, self=False):
    """Exact single / double layer integrals of one flat triangle (3,3) at pts:
    (S, grad S, D, grad D); self: pts are the triangle's own centroid (in-plane values)."""
    v = _f64(tri, (3, 3))
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    S, D = np.zeros(k), np.zeros(k)
    gS, gD = np.zeros((k, 3)), np.zeros((k, 3))
    lib().oracle_tri_near(_p(v), c_int(k), _p(pts), c_int(int(self)), _p(S), _p(gS), _p(D), _p(gD))
    return S, gS, D, gD


def tri_rule(norder):
    xi, eta, w = np.zeros(64), np.zeros(64), np.zeros(64)
    nq = c_int(0)
    lib().oracle_tri_rule(c_int(norder), _p(xi), _p(eta), _p(w), ctypes.byref(nq))
    return xi[:nq.value], eta[:nq.value], w[:nq.value]


def tri_nbox(iprec, ns, nt=0):
    lib().oracle_tri_nbox.restype = c_int
    return lib().oracle_tri_nbox(c_int(iprec), c_int(ns), c_int(nt))


def l3dtriadirect(triaflat, source, charge=None, dipstr=None, target=None, ifpot=1, iffld=1, ifpottarg=1,
                  iffldtarg=1):
    """O(N^2) layer potentials (l3dtriadirect): (pot, fld, pottarg, fldtarg)."""
    tri = _f64(triaflat, (0, 3, 3)); n = tri.shape[0]
    src = _f64(source, (0, 3))
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3)); m = trg.shape[0]
    pot = np.zeros(max(n, 1), np.complex128); fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128); ft = np.zeros((max(m, 1), 3), np.complex128)
    lib().oracle_l3dtriadirect(c_int(n), _p(tri), _p(src), c_int(int(charge is not None)), _p(_c128(charge, n)),
                               c_int(int(dipstr is not None)), _p(_c128(dipstr, n)), c_int(ifpot), _p(pot),
                               c_int(iffld), _p(fld), c_int(m), _p(trg if m else np.zeros((1, 3))),
                               c_int(ifpottarg if m else 0), _p(pt), c_int(iffldtarg if m else 0), _p(ft))
    return pot[:n], fld[:n], pt[:m], ft[:m]


def tri_direct_at(triaflat, pts, self_idx=None, charge=None, dipstr=None):
    """Triangle direct sum at pts; self_idx[k]: the triangle whose centroid point k is (or -1)."""
    tri = _f64(triaflat, (0, 3, 3)); n = tri.shape[0]
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    sk = None if self_idx is None else np.ascontiguousarray(self_idx, np.int64)
    pot = np.zeros(max(k, 1), np.complex128); fld = np.zeros((max(k, 1), 3), np.complex128)
    lib().oracle_tri_direct_points(c_int(n), _p(tri), c_int(int(charge is not None)), _p(_c128(charge, n)),
                                   c_int(int(dipstr is not None)), _p(_c128(dipstr, n)), c_int(k), _p(pts),
                                   None if sk is None else _p(sk), _p(pot), _p(fld))
    return pot[:k], fld[:k]


def htri_near(zk, tri, pts, self=False, nqtri=6):
    """Helmholtz single / double layer integrals of one flat triangle (3,3) at pts (the near-field
    formulas of the triangle FMM): (S, grad S, D, grad D), complex."""
    v = _f64(tri, (3, 3))
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    S, D = np.zeros(k, np.complex128), np.zeros(k, np.complex128)
    gS, gD = np.zeros((k, 3), np.complex128), np.zeros((k, 3), np.complex128)
    zk = complex(zk)
    lib().oracle_htri_near(c_dbl(zk.real), c_dbl(zk.imag), _p(v), c_int(k), _p(pts), c_int(int(self)),
                           c_int(nqtri), _p(S), _p(gS), _p(D), _p(gD))
    return S, gS, D, gD


def htri_nqtri(iprec):
    lib().oracle_htri_nqtri.restype = c_int
    return lib().oracle_htri_nqtri(c_int(iprec))


def htri_direct_at(zk, triaflat, pts, self_idx=None, charge=None, dipstr=None, nqtri=6):
    """Helmholtz triangle direct sum at pts (self_idx[k]: the triangle whose centroid point k is, or -1)."""
    tri = _f64(triaflat, (0, 3, 3)); n = tri.shape[0]
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    sk = None if self_idx is None else np.ascontiguousarray(self_idx, np.int64)
    pot = np.zeros(max(k, 1), np.complex128); fld = np.zeros((max(k, 1), 3), np.complex128)
    zk = complex(zk)
    lib().oracle_htri_direct_points(c_dbl(zk.real), c_dbl(zk.imag), c_int(n), _p(tri), c_int(int(charge is not None)),
                                    _p(_c128(charge, n)), c_int(int(dipstr is not None)), _p(_c128(dipstr, n)),
                                    c_int(k), _p(pts), None if sk is None else _p(sk), c_int(nqtri), _p(pot), _p(fld))
    return pot[:k], fld[:k]


def hfmm3dtriatarg(iprec, zk, triaflat, trianorm, source, charge=None, dipstr=None, target=None, ifpot=1, iffld=1,
                   ifpottarg=1, iffldtarg=1):
    """hfmm3dtriatarg: (ier, pot, fld, pottarg, fldtarg)."""
    tri = _f64(triaflat, (0, 3, 3)); n = tri.shape[0]
    nrm = _f64(trianorm, (0, 3))
    src = _f64(source, (0, 3))
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3)); m = trg.shape[0]
    pot = np.zeros(max(n, 1), np.complex128); fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128); ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = c_int(0)
    zk = complex(zk)
    lib().oracle_hfmm3dtriatarg(ctypes.byref(ier), c_int(iprec), c_dbl(zk.real), c_dbl(zk.imag), c_int(n), _p(tri),
                                _p(nrm), _p(src), c_int(int(charge is not None)), _p(_c128(charge, n)),
                                c_int(int(dipstr is not None)), _p(_c128(dipstr, n)), c_int(ifpot), _p(pot),
                                c_int(iffld), _p(fld), c_int(m), _p(trg if m else np.zeros((1, 3))),
                                c_int(ifpottarg if m else 0), _p(pt), c_int(iffldtarg if m else 0), _p(ft))
    return ier.value, pot[:n], fld[:n], pt[:m], ft[:m]


def lfmm3dtriatarg(iprec, triaflat, trianorm, source, charge=None, dipstr=None, target=None, ifpot=1, iffld=1,
                   ifpottarg=1, iffldtarg=1):
    """lfmm3dtriatarg: (ier, pot, fld, pottarg, fldtarg)."""
    tri = _f64(triaflat, (0, 3, 3)); n = tri.shape[0]
    nrm = _f64(trianorm, (0, 3))
    src = _f64(source, (0, 3))
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3)); m = trg.shape[0]
    pot = np.zeros(max(n, 1), np.complex128); fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128); ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = c_int(0)
    lib().oracle_lfmm3dtriatarg(ctypes.byref(ier), c_int(iprec), c_int(n), _p(tri), _p(nrm), _p(src),
                                c_int(int(charge is not None)), _p(_c128(charge, n)), c_int(int(dipstr is not None)),
                                _p(_c128(dipstr, n)), c_int(ifpot), _p(pot), c_int(iffld), _p(fld), c_int(m),
                                _p(trg if m else np.zeros((1, 3))), c_int(ifpottarg if m else 0), _p(pt),
                                c_int(iffldtarg if m else 0), _p(ft))
    return ier.value, pot[:n], fld[:n], pt[:m], ft[:m]


class Tree:
    """The oracle's octree (d3tstrcr semantics) exported as numpy arrays."""

    def __init__(self, source, target, nbox, ifempty=0, minlevel=0, maxlevel=100):
        """ifempty / minlevel / maxlevel: the options of d3tstrcrem (the defaults are d3tstrcr's)."""
        L = lib()
        src = _f64(source, (0, 3))
        trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3))
        n, m = src.shape[0], trg.shape[0]
        h = L.oracle_tree_build_em(c_int(n), _p(src), c_int(m), _p(trg if m else np.zeros((1, 3))), c_int(nbox),
                                   c_int(ifempty), c_int(minlevel), c_int(maxlevel))
        try:
            nb = L.oracle_tree_nboxes(h)
            self.nboxes = nb
            self.nlev = L.oracle_tree_nlev(h)
            g = np.zeros(4)
            L.oracle_tree_geometry(P(h), _p(g))
            self.center0, self.size = g[:3].copy(), g[3]
            self.box = np.zeros((nb, 20), np.int32)
            self.centers = np.zeros((nb, 3))
            self.iz = np.zeros(max(n, 1), np.int32)
            self.iztarg = np.zeros(max(m, 1), np.int32)
            L.oracle_tree_boxes(P(h), _p(self.box), _p(self.centers), _p(self.iz), _p(self.iztarg),
                                c_int(n), c_int(m))
            self.iz = self.iz[:n]
            self.iztarg = self.iztarg[:m]
            self.lists = {}
            for ty in range(1, 6):
                ln = L.oracle_tree_list_len(P(h), c_int(ty))
                st = np.zeros(nb + 1, np.int32)
                ix = np.zeros(max(ln, 1), np.int32)
                L.oracle_tree_list(P(h), c_int(ty), _p(st), _p(ix))
                self.lists[ty] = (st, ix[:ln])
        finally:
            L.oracle_tree_free(P(h))

    def list_of(self, ty, b):
        st, ix = self.lists[ty]
        return ix[st[b]:st[b + 1]]


def _cdouble_arr(n):
    return np.zeros(n, np.complex128)


def formmp(src, c, p, charge=None, dipstr=None, dipvec=None):
    src = _f64(src, (0, 3)); n = src.shape[0]
    mp = _cdouble_arr((p + 1) ** 2)
    lib().oracle_formmp(c_int(n), _p(src), c_int(int(charge is not None)), _p(_c128(charge, n)),
                        c_int(int(dipstr is not None)), _p(_c128(dipstr, n)), _p(_f64(dipvec, (max(n, 1), 3))),
                        _p(_f64(c, (3,))), c_int(p), _p(mp))
    return mp


def formta(src, c, p, charge=None, dipstr=None, dipvec=None):
    src = _f64(src, (0, 3)); n = src.shape[0]
    lo = _cdouble_arr((p + 1) ** 2)
    lib().oracle_formta(c_int(n), _p(src), c_int(int(charge is not None)), _p(_c128(charge, n)),
                        c_int(int(dipstr is not None)), _p(_c128(dipstr, n)), _p(_f64(dipvec, (max(n, 1), 3))),
                        _p(_f64(c, (3,))), c_int(p), _p(lo))
    return lo


def mpeval(c, mp, p, pts):
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    pot = _cdouble_arr(k); fld = np.zeros((k, 3), np.complex128)
    lib().oracle_mpeval(_p(_f64(c, (3,))), _p(np.ascontiguousarray(mp, np.complex128)), c_int(p), c_int(k),
                        _p(pts), _p(pot), _p(fld))
    return pot, fld


def taeval(c, lo, p, pts):
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    pot = _cdouble_arr(k); fld = np.zeros((k, 3), np.complex128)
    lib().oracle_taeval(_p(_f64(c, (3,))), _p(np.ascontiguousarray(lo, np.complex128)), c_int(p), c_int(k),
                        _p(pts), _p(pot), _p(fld))
    return pot, fld


def taevalhess(c, lo, p, pts, rscale=1.0):
    """l3dtaevalhessd_trunc at each point: (pot, fld, hess[dxx,dyy,dzz,dxy,dxz,dyz])."""
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    pot = _cdouble_arr(k); fld = np.zeros((k, 3), np.complex128); hess = np.zeros((k, 6), np.complex128)
    lib().oracle_taevalhess(c_dbl(rscale), _p(_f64(c, (3,))), _p(np.ascontiguousarray(lo, np.complex128)),
                            c_int(p), c_int(k), _p(pts), _p(pot), _p(fld), _p(hess))
    return pot, fld, hess


def mpevalhess(c, mp, p, pts, rscale=1.0):
    """l3dmpevalhessd_trunc at each point: (pot, fld, hess)."""
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    pot = _cdouble_arr(k); fld = np.zeros((k, 3), np.complex128); hess = np.zeros((k, 6), np.complex128)
    lib().oracle_mpevalhess(c_dbl(rscale), _p(_f64(c, (3,))), _p(np.ascontiguousarray(mp, np.complex128)),
                            c_int(p), c_int(k), _p(pts), _p(pot), _p(fld), _p(hess))
    return pot, fld, hess


def direct_hess_at(source, pts, skip=None, charge=None, dipstr=None, dipvec=None):
    """Direct-sum Hessians (lpotfld3dhess, lpotfld3dhess_dp) at pts; skip[k] is excluded at point k."""
    source = _f64(source, (0, 3)); n = source.shape[0]
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    hess = np.zeros((k, 6), np.complex128)
    sk = None if skip is None else np.ascontiguousarray(skip, np.int64)
    lib().oracle_l3ddirect_points_hess(c_int(n), _p(source), c_int(int(charge is not None)), _p(_c128(charge, n)),
                                       c_int(int(dipstr is not None)), _p(_c128(dipstr, n)),
                                       _p(_f64(dipvec, (max(n, 1), 3))), c_int(k), _p(pts),
                                       None if sk is None else _p(sk), _p(hess))
    return hess


def translate(kind, c_from, c_to, coef, p, nt=None):
    """kind 0 = M2M, 1 = M2L (truncated to nt), 2 = L2L; returns the new expansion."""
    out = _cdouble_arr((p + 1) ** 2)
    lib().oracle_translate(c_int(kind), _p(_f64(c_from, (3,))), _p(_f64(c_to, (3,))),
                           _p(np.ascontiguousarray(coef, np.complex128)), c_int(p),
                           c_int(p if nt is None else nt), _p(out))
    return out


# ---------------------------------------------------------------- Helmholtz
def h3dall(nterms, z, scale):
    """Scaled spherical Hankel functions h_n(z) * scale^n and derivatives."""
    h = _cdouble_arr(nterms + 2); hd = _cdouble_arr(nterms + 2)
    lib().oracle_h3dall(c_int(nterms), c_dbl(z.real), c_dbl(complex(z).imag), c_dbl(scale), _p(h), _p(hd))
    return h[:nterms + 1], hd[:nterms + 1]


def jfuns3d(nterms, z, scale):
    """Scaled spherical Bessel functions j_n(z) / scale^n and derivatives."""
    f = _cdouble_arr(nterms + 2); fd = _cdouble_arr(nterms + 2)
    L = lib()
    L.oracle_jfuns3d.restype = c_int
    ier = L.oracle_jfuns3d(c_int(nterms), c_dbl(z.real), c_dbl(complex(z).imag), c_dbl(scale), _p(f), _p(fd))
    return ier, f[:nterms + 1], fd[:nterms + 1]


def h3dterms(size, zk, eps):
    L = lib()
    L.oracle_h3dterms.restype = c_int
    ier = c_int(0)
    n = L.oracle_h3dterms(c_dbl(size), c_dbl(complex(zk).real), c_dbl(complex(zk).imag), c_dbl(eps),
                          ctypes.byref(ier))
    return n, ier.value


def h3dterms_list2(size, zk, eps):
    t = np.zeros(343, np.int32)
    ier = c_int(0)
    lib().oracle_h3dterms_list2(c_dbl(size), c_dbl(complex(zk).real), c_dbl(complex(zk).imag), c_dbl(eps), _p(t),
                                ctypes.byref(ier))
    return t.reshape(7, 7, 7)


def rotviaproj(beta, nterms, coef):
    """Rotation about the y axis by projection (rotviaprojf90); coef: (nterms+1)^2 complex."""
    a = np.ascontiguousarray(coef, dtype=np.complex128)
    out = np.zeros((nterms + 1) ** 2, np.complex128)
    lib().oracle_rotviaproj(c_dbl(beta), c_int(nterms), _p(a), _p(out))
    return out


def rotviarecur(beta, nterms, coef):
    """The same rotation by the three-term recursion (rotviarecur3p_init / _apply)."""
    a = np.ascontiguousarray(coef, dtype=np.complex128)
    out = np.zeros((nterms + 1) ** 2, np.complex128)
    lib().oracle_rotviarecur(c_dbl(beta), c_int(nterms), _p(a), _p(out))
    return out


def legewhts(n):
    x = np.zeros(n); w = np.zeros(n)
    lib().oracle_legewhts(c_int(n), _p(x), _p(w))
    return x, w


def h3dpartdirect(zk, source, charge=None, dipstr=None, dipvec=None, target=None,
                  ifpot=1, iffld=1, ifpottarg=1, iffldtarg=1):
    src = _f64(source, (0, 3)); n = src.shape[0]
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    zk = complex(zk)
    pot = np.zeros(max(n, 1), np.complex128); fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128); ft = np.zeros((max(m, 1), 3), np.complex128)
    lib().oracle_h3dpartdirect(
        c_dbl(zk.real), c_dbl(zk.imag), c_int(n), _p(src), c_int(int(charge is not None)), _p(_c128(charge, n)),
        c_int(int(dipstr is not None)), _p(_c128(dipstr, n)), _p(_f64(dipvec, (max(n, 1), 3))), c_int(ifpot),
        _p(pot), c_int(iffld), _p(fld), c_int(m), _p(trg), c_int(ifpottarg if m else 0), _p(pt),
        c_int(iffldtarg if m else 0), _p(ft))
    return pot[:n], fld[:n], pt[:m], ft[:m]


def hdirect_at(zk, source, pts, skip=None, charge=None, dipstr=None, dipvec=None):
    """Helmholtz direct pot/fld at arbitrary points; skip[k] = excluded source."""
    src = _f64(source, (0, 3)); n = src.shape[0]
    pts = _f64(pts, (0, 3)); k = pts.shape[0]
    zk = complex(zk)
    sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.int64)
    pot = np.zeros(max(k, 1), np.complex128); fld = np.zeros((max(k, 1), 3), np.complex128)
    lib().oracle_h3ddirect_points(
        c_dbl(zk.real), c_dbl(zk.imag), c_int(n), _p(src), c_int(int(charge is not None)), _p(_c128(charge, n)),
        c_int(int(dipstr is not None)), _p(_c128(dipstr, n)), _p(_f64(dipvec, (max(n, 1), 3))), c_int(k), _p(pts),
        _p(sk), _p(pot), _p(fld))
    return pot[:k], fld[:k]


def hfmm3dparttarg(iprec, zk, source, charge=None, dipstr=None, dipvec=None, target=None,
                   ifpot=1, iffld=1, ifpottarg=1, iffldtarg=1, timing=False, nterms=False):
    src = _f64(source, (0, 3)); n = src.shape[0]
    trg = _f64(target, (0, 3)) if target is not None else np.zeros((0, 3))
    m = trg.shape[0]
    zk = complex(zk)
    pot = np.zeros(max(n, 1), np.complex128); fld = np.zeros((max(n, 1), 3), np.complex128)
    pt = np.zeros(max(m, 1), np.complex128); ft = np.zeros((max(m, 1), 3), np.complex128)
    ier = c_int(0)
    tinfo = np.zeros(8)
    nt = np.zeros(202, np.int32)
    lib().oracle_hfmm3dparttarg(
        ctypes.byref(ier), c_int(iprec), c_dbl(zk.real), c_dbl(zk.imag), c_int(n), _p(src),
        c_int(int(charge is not None)), _p(_c128(charge, n)), c_int(int(dipstr is not None)), _p(_c128(dipstr, n)),
        _p(_f64(dipvec, (max(n, 1), 3))), c_int(ifpot), _p(pot), c_int(iffld), _p(fld), c_int(m),
        _p(trg if m else np.zeros((1, 3))), c_int(ifpottarg if m else 0), _p(pt), c_int(iffldtarg if m else 0),
        _p(ft), _p(tinfo), _p(nt))
    out = (ier.value, pot[:n], fld[:n], pt[:m], ft[:m])
    if timing:
        out = out + (tinfo,)
    if nterms:
        out = out + (nt,)
    return out


def hformmp(zk, rscale, src, c, p, charge=None, dipstr=None, dipvec=None):
    src = _f64(src, (0, 3)); n = src.shape[0]; zk = complex(zk)
    mp = _cdouble_arr((p + 1) ** 2)
    lib().oracle_hformmp(c_dbl(zk.real), c_dbl(zk.imag), c_dbl(rscale), c_int(n), _p(src),
                         c_int(int(charge is not None)), _p(_c128(charge, n)), c_int(int(dipstr is not None)),
                         _p(_c128(dipstr, n)), _p(_f64(dipvec, (max(n, 1), 3))), _p(_f64(c, (3,))), c_int(p), _p(mp))
    return mp


def hformta(zk, rscale, src, c, p, charge=None, dipstr=None, dipvec=None):
    src = _f64(src, (0, 3)); n = src.shape[0]; zk = complex(zk)
    lo = _cdouble_arr((p + 1) ** 2)
    lib().oracle_hformta(c_dbl(zk.real), c_dbl(zk.imag), c_dbl(rscale), c_int(n), _p(src),
                         c_int(int(charge is not None)), _p(_c128(charge, n)), c_int(int(dipstr is not None)),
                         _p(_c128(dipstr, n)), _p(_f64(dipvec, (max(n, 1), 3))), _p(_f64(c, (3,))), c_int(p), _p(lo))
    return lo


def hmpeval(zk, rscale, c, mp, p, pts):
    pts = _f64(pts, (0, 3)); k = pts.shape[0]; zk = complex(zk)
    pot = _cdouble_arr(k); fld = np.zeros((k, 3), np.complex128)
    lib().oracle_hmpeval(c_dbl(zk.real), c_dbl(zk.imag), c_dbl(rscale), _p(_f64(c, (3,))),
                         _p(np.ascontiguousarray(mp, np.complex128)), c_int(p), c_int(k), _p(pts), _p(pot), _p(fld))
    return pot, fld


def htaeval(zk, rscale, c, lo, p, pts):
    pts = _f64(pts, (0, 3)); k = pts.shape[0]; zk = complex(zk)
    pot = _cdouble_arr(k); fld = np.zeros((k, 3), np.complex128)
    lib().oracle_htaeval(c_dbl(zk.real), c_dbl(zk.imag), c_dbl(rscale), _p(_f64(c, (3,))),
                         _p(np.ascontiguousarray(lo, np.complex128)), c_int(p), c_int(k), _p(pts), _p(pot), _p(fld))
    return pot, fld


def htranslate(kind, zk, c_from, c_to, coef, nin, sc1, nout, sc2, radius, nq):
    """kind 0 = M2M, 1 = M2L, 2 = L2L by the reference's sphere projection."""
    zk = complex(zk)
    out = _cdouble_arr((max(nin, nout) + 1) ** 2)
    lib().oracle_htranslate(c_int(kind), c_dbl(zk.real), c_dbl(zk.imag), _p(_f64(c_from, (3,))),
                            _p(_f64(c_to, (3,))), _p(np.ascontiguousarray(coef, np.complex128)), c_int(nin),
                            c_dbl(sc1), c_int(nout), c_dbl(sc2), c_dbl(radius), c_int(nq), _p(out))
    return out[:(nout + 1) ** 2]
