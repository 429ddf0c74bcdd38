"""The .pro entry point on the GPU: dl_create_from_pro on the reference's
swinging-rod input, against the oracle reading the same file."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from dynlattice_b200.abi import DL_PLAIN_FP64
from dynlattice_b200.engine import Lattice, load_library
from dynlattice_b200.pro import ProModel
from helpers import rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu

PRO = Path(__file__).resolve().parent / "golden" / "pro" / "transient"


def test_create_from_pro_matches_oracle(gpu):
    """dl_create_from_pro applies the file's MilneDevice module; the oracle
    reads the same file and runs the same integrator."""
    lib = load_library()
    lib.dl_create_from_pro.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
    h = C.c_void_p()
    assert lib.dl_create_from_pro(str(PRO / "test2.pro").encode(), DL_PLAIN_FP64, C.byref(h)) == 0
    lib.dl_run(h, 100000)
    assert lib.dl_synchronize(h) == 0
    p = ProModel(PRO / "test2.pro")
    u = np.zeros((p.n_nodes, 3)); th = np.zeros((p.n_nodes, 3)); v = np.zeros((p.n_nodes, 6))
    dp = C.POINTER(C.c_double)
    lib.dl_get_state(h, u.ctypes.data_as(dp), th.ctypes.data_as(dp), v.ctypes.data_as(dp))
    t = C.c_double()
    lib.dl_get_time(h, C.byref(t), None, None, None)
    lib.dl_destroy(h)
    o = Oracle(p)
    o.set_integrator(p.integrator)
    o.run(100000)
    uo, _, vo = o.state()
    assert t.value == pytest.approx(o.time()[0], rel=1e-10)
    assert rel_err(u, uo) < 1e-8 and rel_err(v, vo) < 1e-7
    # the same model through the Python ProModel object, LeapFrog at fixed dt
    g = Lattice(p, DL_PLAIN_FP64)
    g.run(1000)
    o2 = Oracle(p)
    o2.run(1000)
    assert rel_err(g.state()[0], o2.state()[0]) < 1e-9
