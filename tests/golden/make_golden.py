"""Regenerates tests/golden/driver_{lap,helm}_n2000.npz (run from the repository root).

The reference ships no golden output files and cannot be compiled here (no
Fortran compiler), so the fixture records, for the reference driver's own
inputs at N = 2000 (examples/lfmm3dpart_driver.f geometry, charges and
dipoles, iprec = 1): the first 20 hkrand values, the FP64 direct sum and the
oracle FMM at the first 100 sources and targets (the points the driver's
accuracy check uses, examples/lfmm3dpart_driver.f:130-264).  The Helmholtz
fixture does the same for examples/hfmm3dpart_driver.f (targets shifted by
+1, zk = 1 + 0.1i, iprec = 1).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)


def main():
    import oracle
    from driver_inputs import driver_inputs
    n = 2000
    src, trg, q, ds, dv = driver_inputs(n)
    ier, pot, fld, pt, ft = oracle.lfmm3dparttarg(1, src, q, ds, dv, trg)
    assert ier == 0
    k = 100
    dp, df = oracle.direct_at(src, src[:k], np.arange(k), q, ds, dv)
    dpt, dft = oracle.direct_at(src, trg[:k], None, q, ds, dv)
    np.savez_compressed(os.path.join(HERE, "driver_lap_n2000.npz"), hkrand20=oracle.hkrand_stream(20),
                        pot=pot[:k], fld=fld[:k], pottarg=pt[:k], fldtarg=ft[:k], dpot=dp, dfld=df,
                        dpottarg=dpt, dfldtarg=dft)
    src, trg, q, ds, dv = driver_inputs(n, shift=1.0)
    zk = 1 + 0.1j
    ier, pot, fld, pt, ft = oracle.hfmm3dparttarg(1, zk, src, q, ds, dv, trg)
    assert ier == 0
    dp, df = oracle.hdirect_at(zk, src, src[:k], np.arange(k), q, ds, dv)
    dpt, dft = oracle.hdirect_at(zk, src, trg[:k], None, q, ds, dv)
    np.savez_compressed(os.path.join(HERE, "driver_helm_n2000.npz"), zk=zk, pot=pot[:k], fld=fld[:k],
                        pottarg=pt[:k], fldtarg=ft[:k], dpot=dp, dfld=df, dpottarg=dpt, dfldtarg=dft)


if __name__ == "__main__":
    main()
