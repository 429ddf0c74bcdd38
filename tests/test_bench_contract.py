"""bench.py's output contract, checked on the host.

The reference arm (the CPU restatement of the reference's explicit step, timed
on the host cores) prints one JSON line with the keys a harness reads.  Under a
multi-rank launch, every rank but 0 exits 0 without output.  The GPU arm fails
loudly without a device instead of falling back to the CPU.
"""
import json
import os
import subprocess
import sys
import types
from pathlib import Path

import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]


def _run(args, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=timeout)


def test_reference_arm_line():
    r = _run(["--impl", "reference", "--steps", "1", "--warmup", "3"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config"):
        assert k in d, k
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 1, 3)
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e2e = d["e2e"]
    assert (e2e["value"], e2e["unit"]) == (d["value"], d["unit"])
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"],
             env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


@pytest.mark.skipif(torch.cuda.is_available(), reason="the behaviour without a GPU")
def test_gpu_arm_fails_without_device():
    r = _run(["--steps", "3", "--warmup", "3"])
    assert r.returncode != 0
    assert r.stdout.strip() == ""  # no number from a fallback path


def test_workload_sizes():
    """The bench's workloads at the sizes its lines state: the 20^3 BCC impact,
    the 8^3 BCC adjoint case, the 32-element rod and the 20 000-rod network."""
    sys.path.insert(0, str(ROOT))
    import bench
    from dynlattice_b200 import lattices
    s = bench.workload(20)
    assert (s.n_elems, s.n_nodes, s.dt, s.n_gauss) == (128000, 81261, 5e-8, 2)
    a = bench.adjoint_case()
    assert (a.n_elems, len(a.strut_radius), a.dt) == (8192, 4096, 5e-8)
    r = lattices.straight_rod()
    assert (r.n_elems, r.n_nodes, r.dt) == (32, 33, 2e-6)
    f = bench.fibre_spec(types.SimpleNamespace(rods=20000))
    assert (f.n_elems, f.n_nodes, f.dt) == (80000, 100000, 1e-8)
