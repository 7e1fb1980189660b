"""Inputs of the reference's sample driver, regenerated from its own RNG.

examples/lfmm3dpart_driver.f:49-102 draws, from hkrand (examples/hkrand.f,
LAPACK dlaran with seed (0,0,0,1)): one discarded value; per source theta
(x pi) and phi (x 2 pi) on a sphere of radius 0.5; per target the same on a
sphere shifted by +2 in x; per source a complex charge; per source a complex
dipole strength and a dipole vector (three values).  The Helmholtz driver
(examples/hfmm3dpart_driver.f:46-50) uses the same geometry with the target
sphere shifted by +1.
"""
import numpy as np


def driver_inputs(n, shift=2.0):
    import oracle
    vals = oracle.hkrand_stream(1 + 4 * n + 2 * n + 5 * n)
    it = iter(vals[1:])
    src = np.zeros((n, 3))
    trg = np.zeros((n, 3))
    for i in range(n):
        th = next(it) * np.pi
        ph = next(it) * 2 * np.pi
        src[i] = (.5 * np.cos(ph) * np.sin(th), .5 * np.sin(ph) * np.sin(th), .5 * np.cos(th))
    for i in range(n):
        th = next(it) * np.pi
        ph = next(it) * 2 * np.pi
        trg[i] = (.5 * np.cos(ph) * np.sin(th) + shift, .5 * np.sin(ph) * np.sin(th), .5 * np.cos(th))
    q = np.array([next(it) + 1j * next(it) for _ in range(n)])
    ds = np.zeros(n, complex)
    dv = np.zeros((n, 3))
    for i in range(n):
        ds[i] = next(it) + 1j * next(it)
        dv[i] = (next(it), next(it), next(it))
    return src, trg, q, ds, dv
