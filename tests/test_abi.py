"""The C ABI library loads and exports every symbol declared in include/*.h (no GPU call)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\s*\*?\s*(\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_reference_entry_points():
    names = declared_symbols()
    for s in ("lfmm3dpart_", "lfmm3dpartself_", "lfmm3dparttarg_", "l3dpartdirect_"):
        assert s in names


def test_library_exports_all_declared_symbols():
    import fmmlib3d_b200 as F
    lib = ctypes.CDLL(F.LIBPATH)
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing, missing


def test_package_has_no_cpu_fallback():
    src = open(os.path.join(ROOT, "fmmlib3d_b200", "__init__.py")).read()
    assert "import oracle" not in src and "from oracle" not in src


def test_fortran_module_binds_exported_symbols():
    """include/fmm3d_b200.f90 (iso_c_binding interfaces) names only symbols the library exports,
    and covers every reference entry point (no Fortran compiler here to build the module)."""
    import fmmlib3d_b200 as F
    src = open(os.path.join(ROOT, "include", "fmm3d_b200.f90")).read()
    bound = set(re.findall(r'bind\(C,\s*name="(\w+)"\)', src))
    lib = ctypes.CDLL(F.LIBPATH)
    assert bound and not [s for s in bound if not hasattr(lib, s)]
    for s in ("lfmm3dpart_", "lfmm3dpartself_", "lfmm3dparttarg_", "l3dpartdirect_",
              "hfmm3dpart_", "hfmm3dpartself_", "hfmm3dparttarg_", "h3dpartdirect_"):
        assert s in bound
