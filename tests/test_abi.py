"""The C ABI library loads and exports every function include/dynlattice.h declares."""
import ctypes as C
import re
from pathlib import Path

import pytest

from dynlattice_b200.engine import LIB_PATH, load_library

HEADER = Path(__file__).resolve().parent.parent / "include" / "dynlattice.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"DL_API[^;(]*?\b(dl_\w+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "dl_create" in names and "dl_run" in names and len(names) > 15


def test_library_exports_all_declared_symbols():
    lib = load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"symbols declared but not exported: {missing}"


def test_version_and_device_query():
    lib = load_library()
    lib.dl_version.restype = C.c_char_p
    assert b"sm_100a" in lib.dl_version()
    n = C.c_int(-1)
    assert lib.dl_device_count(C.byref(n)) == 0
    assert n.value >= 0


def test_create_without_device_fails_loudly():
    """The engine has no CPU path: without a CUDA device dl_create must fail."""
    from dynlattice_b200 import lattices
    from dynlattice_b200.engine import DLError, Lattice, device_count
    if device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(DLError) as ei:
        Lattice(lattices.straight_rod(n_elems=4))
    assert ei.value.code == 11  # DL_ERR_NO_DEVICE


def test_build_targets_sm100a():
    """The engine's build compiles every CUDA source for sm_100a only."""
    mk = (Path(__file__).resolve().parent.parent / "dynlattice_b200" / "csrc" / "Makefile").read_text()
    assert "ARCH := -gencode arch=compute_100a,code=sm_100a" in mk
    assert LIB_PATH.exists()


@pytest.mark.gpu
def test_kernels_report_sm100_binary(gpu):
    """The runtime sees sm_100 device code in the loaded library."""
    lib = load_library()
    v = C.c_int32(0)
    assert lib.dl_device_binary_version(C.byref(v)) == 0, lib.dl_last_error()
    assert v.value == 100


@pytest.mark.parametrize("precision", [0, 1])
def test_runtime_compiled_kernels_build_for_sm100a(precision):
    """The step and adjoint kernels that NVRTC specialises per yield function
    compile for sm_100a from the embedded device sources (no device needed)."""
    from dynlattice_b200 import lattices
    lib = load_library()
    spec = lattices.lattice_impact(n=1)
    d = spec.desc()
    n = C.c_size_t()
    log = C.create_string_buffer(1 << 16)
    rc = lib.dl_jit_check(C.byref(d), precision, C.byref(n), log, C.c_size_t(1 << 16))
    assert rc == 0, log.value.decode(errors="replace")
    assert n.value > 0
