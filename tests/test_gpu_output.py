"""Output modules of a .pro run on the GPU (dl_pro_run): GroupOutput
variables, Sample rows, CSVOutput state vectors and ParaView VTU/PVD files
for the reference's swinging-rod input (tests/golden/pro/transient/test2.pro)
with an extra Sample module, under MilneDevice (step-by-step loop) and
LeapFrog (runs chunked up to the next output step)."""
import gzip
import shutil
import xml.etree.ElementTree as ET
from pathlib import Path

import numpy as np
import pytest

from dynlattice_b200.abi import DL_INTEG_LEAPFROG, DL_PLAIN_FP64
from dynlattice_b200.engine import VTU_FEXT, VTU_FINT, VTU_FRES, Lattice
from dynlattice_b200.pro import ProModel

pytestmark = pytest.mark.gpu

SRC = Path(__file__).resolve().parent / "golden" / "pro" / "transient"


def _case(tmp_path, integrator="MilneDevice", sample_when=None):
    for f in ("test2.pro", "input.pro", "model.pro", "output.pro"):
        shutil.copy(SRC / f, tmp_path / f)
    shutil.copy(SRC / "test2.geo", tmp_path / "case.geo")  # the input module reads $(CASE_NAME).geo
    lines = ['include "test2.pro";',
             f'Solver.integrator.type = "{integrator}";',
             'Output.modules += "energy";',
             'Output.energy.type = "Sample";',
             'Output.energy.file = "$(CASE_NAME)/energy.txt";',
             'Output.energy.dataSets = [ "i", "t", "free.disp.dx", "free.disp.dz", "fixed.resp.dz", '
             '"fixed.load.dz", "free.velo.dz", "kineticEnergy" ];',
             'Output.energy.separator = ",";',
             'Output.modules += "pv2";',
             'Output.pv2.type = "ParaView";',
             'Output.pv2.output_format = "$(CASE_NAME)/pv2/frame%i";',
             'Output.pv2.groups = [ "beams" ];',
             'Output.pv2.beams.node_data = [ "fint", "fext", "fres" ];',
             'Output.pv2.beams.el_data = [ "strain", "stress", "mat_stress", "mat_strain", "plast_strain" ];',
             'Output.pv2.sampleWhen = "i % 100 == 0";']
    if sample_when:
        lines.append(f'Output.energy.sampleWhen = "{sample_when}";')
    (tmp_path / "case.pro").write_text("\n".join(lines) + "\n")
    p = ProModel(tmp_path / "case.pro")
    g = Lattice(p, DL_PLAIN_FP64)
    if p.integrator.kind != DL_INTEG_LEAPFROG:
        g.set_integrator(p.integrator)
    return p, g


def _vtu_arrays(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    out = {}
    for da in piece.iter("DataArray"):
        name = da.get("Name") or "Points"
        vals = np.array(da.text.split(), dtype=float)
        k = int(da.get("NumberOfComponents") or 1)
        out[name] = vals.reshape(-1, k) if k > 1 else vals
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), out


def test_milne_run_with_outputs(gpu, tmp_path):
    p, g = _case(tmp_path)
    n = p.run(g, tmp_path, max_steps=300)
    assert n == 300
    t, _, step, _ = g.time()
    assert step == 300
    free, fixed = int(p.group("free")[0]), int(p.group("fixed")[0])
    u, th, v = g.state()
    # Sample: one row per step, GroupOutput variables of the final state
    rows = np.loadtxt(tmp_path / "case" / "energy.txt", delimiter=",")
    assert rows.shape == (300, 8)
    assert np.array_equal(rows[:, 0], np.arange(1, 301)) and (np.diff(rows[:, 1]) > 0).all()
    assert rows[-1, 1] == pytest.approx(t, rel=1e-15)
    assert rows[-1, 2] == pytest.approx(u[free, 0], rel=1e-12, abs=1e-300)
    assert rows[-1, 3] == pytest.approx(u[free, 2], rel=1e-12)
    assert rows[-1, 6] == pytest.approx(v[free, 2], rel=1e-12)
    f = g.internal_force(u, th)
    assert rows[-1, 4] == pytest.approx(f[fixed, 2], rel=1e-10, abs=1e-12 * np.abs(f).max())
    w = np.pi * (5e-3) ** 2 * 0.1 * 1.1e3 * 9.81
    assert rows[-1, 5] == pytest.approx(-0.5 * w, rel=1e-12)   # -w (all) + w/2 (fixed)
    assert rows[-1, 7] == pytest.approx(g.energies()["kinetic"], rel=1e-12)
    # CSVOutput: header, then "t,disp,<6N values>" rows where saveWhen held
    with gzip.open(tmp_path / "case" / "disp.gz", "rt") as fh:
        lines = fh.read().splitlines()
    head = lines[0].split(",")
    assert head[:2] == ["time", "label"] and len(head) == 2 + 6 * p.n_nodes
    assert head[2:8] == ["dx[0]", "dy[0]", "dz[0]", "rx[0]", "ry[0]", "rz[0]"]
    body = [ln.split(",") for ln in lines[1:]]
    assert len(body) >= 1 and all(r[1] == "disp" for r in body)
    # ParaView: the files of steps 100, 200, 300 and their collection
    pv = tmp_path / "case" / "pv2"
    assert sorted(x.name for x in pv.glob("*.vtu")) == ["frame0.vtu", "frame1.vtu", "frame2.vtu"]
    coll = ET.parse(pv / "frame.pvd").getroot().findall("Collection/DataSet")
    assert [d.get("file") for d in coll] == ["frame0.vtu", "frame1.vtu", "frame2.vtu"]
    assert float(coll[-1].get("timestep")) == pytest.approx(t, rel=1e-15)
    npts, ncells, arr = _vtu_arrays(pv / "frame2.vtu")
    assert (npts, ncells) == (p.n_nodes, p.n_elems)
    assert np.allclose(arr["Points"], p.coords, rtol=1e-7, atol=1e-9)
    assert np.allclose(arr["Displacement"], u, rtol=1e-6, atol=1e-7 * np.abs(u).max())
    assert np.allclose(arr["otherDofsVelo"], v[:, 3:], rtol=1e-6, atol=1e-7 * np.abs(v[:, 3:]).max())
    fx = np.zeros((p.n_nodes, 3))
    fx[:, 2] = -w
    fx[free, 2] += 0.5 * w
    fx[fixed, 2] += 0.5 * w
    assert np.allclose(arr["External Forces"], fx, rtol=1e-6, atol=1e-9)
    assert np.allclose(arr["Resulting Forces"], fx - f[:, :3], rtol=1e-5, atol=1e-6 * np.abs(f).max())
    conn = arr["connectivity"].reshape(-1, 2)
    assert np.array_equal(conn, p.conn) and (arr["types"] == 3).all()
    # cell data: the element tables of the final state in single precision
    for name in ("strain", "stress", "mat_stress", "mat_strain", "plast_strain"):
        tab = g.element_table(name)
        assert arr[name].shape == (p.n_elems, 6)
        assert np.allclose(arr[name], tab, rtol=1e-6, atol=1e-7 * max(np.abs(tab).max(), 1e-30))
    assert not arr["plast_strain"].any()


def test_leapfrog_chunked_outputs(gpu, tmp_path):
    """With time-only conditions a LeapFrog run advances to the next output
    step in one launch; the rows equal a separately sampled run."""
    p, g = _case(tmp_path, integrator="LeapFrog", sample_when="i % 50 == 0")
    n = p.run(g, tmp_path, max_steps=300)
    assert n == 300
    rows = np.loadtxt(tmp_path / "case" / "energy.txt", delimiter=",")
    assert np.array_equal(rows[:, 0], np.arange(50, 301, 50))
    free = int(p.group("free")[0])
    ref = Lattice(p, DL_PLAIN_FP64)
    ref.set_sampling(50, [free], capacity=10)
    ref.run(300)
    steps, srows, en = ref.samples()
    assert np.array_equal(steps, rows[:, 0])
    assert np.allclose(rows[:, 2], srows[:, 0, 0], rtol=1e-12, atol=0)
    assert np.allclose(rows[:, 3], srows[:, 0, 2], rtol=1e-12, atol=0)
    assert np.allclose(rows[:, 1], steps * p.dt, rtol=1e-12)
