"""GPU element tables (dl_element_table) against the oracle: the strain,
stress and plastic-strain tables of an elastoplastic lattice after an
impact, in both frames.  Plain FP64 to 1e-9 of each table's largest entry;
the mixed path forms strains and stresses in FP32, to 1e-5."""
import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import DLError, Lattice
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu

NAMES = ("strain", "stress", "mat_strain", "mat_stress", "plast_strain")


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, 1e-9), (DL_MIXED, 1e-5)])
def test_tables_match_oracle(gpu, precision, tol):
    spec = lattices.lattice_impact(n=2)
    o = Oracle(spec, threads=4)
    g = Lattice(spec, precision)
    o.run(1500)
    g.run(1500)
    g.synchronize()
    for name in NAMES:
        to, tg = o.element_table(name), g.element_table(name)
        scale = np.abs(to).max()
        assert scale > 0.0, name
        err = np.abs(tg - to).max() / scale
        assert err < tol, f"{name}: {err:.3e}"


def test_unknown_table(gpu):
    g = Lattice(lattices.lattice_impact(n=2), DL_PLAIN_FP64)
    with pytest.raises(DLError, match="element table"):
        g.element_table("hard_params")
