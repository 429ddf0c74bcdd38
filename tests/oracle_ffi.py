"""ctypes loader of the CPU oracle (test infrastructure; see oracle/oracle.h).

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
use this module.  It builds ``oracle/_build/liboracle.so`` on first use if the
library is missing (``make -C oracle``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from dynlattice_b200.abi import Integrator, ModelSpec, dl_energies, dl_integrator_desc, dl_model_desc

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "oracle" / "_build" / "liboracle.so"
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True,
                       stdout=subprocess.DEVNULL)
    lib = C.CDLL(str(LIB))
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    lib.orc_last_error.restype = C.c_char_p
    lib.orc_create.argtypes = [C.POINTER(dl_model_desc), C.POINTER(P)]
    lib.orc_destroy.argtypes = [P]
    lib.orc_run.argtypes = [P, C.c_int64]
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_set_sampling.argtypes = [P, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]
    lib.orc_get_samples.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), dp,
                                    C.POINTER(dl_energies), C.c_int64]
    lib.orc_get_state.argtypes = [P, dp, dp, dp]
    lib.orc_set_state.argtypes = [P, dp, dp, dp]
    lib.orc_get_energies.argtypes = [P, C.POINTER(dl_energies)]
    lib.orc_static_force.argtypes = [P, dp, dp, dp]
    lib.orc_static_commit.argtypes = [P, dp, dp]
    lib.orc_internal_force.argtypes = [P, dp, dp, dp]
    lib.orc_elastic_energy.argtypes = [P, dp, dp, dp]
    lib.orc_get_history.argtypes = [P, dp, dp, dp]
    lib.orc_get_frames.argtypes = [P, dp, dp]
    lib.orc_mass.argtypes = [P, dp, dp, dp]
    lib.orc_error_word.argtypes = [P, C.POINTER(C.c_uint32)]
    lib.orc_group_sums.argtypes = [P, C.c_int32, C.POINTER(C.c_int32), dp, dp]
    lib.orc_contact_pairs.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int32), dp, C.c_int64]
    lib.orc_blacklist_size.argtypes = [P, C.POINTER(C.c_int64)]
    lib.orc_element_table.argtypes = [P, C.c_char_p, dp]
    lib.orc_joint_contact_pairs.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int32), dp, C.c_int64]
    lib.orc_plate_reaction.argtypes = [P, dp]
    lib.orc_set_integrator.argtypes = [P, C.POINTER(dl_integrator_desc)]
    lib.orc_get_time.argtypes = [P, dp, dp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.orc_get_sample_times.argtypes = [P, dp, C.c_int64]
    _lib = lib
    return lib


def _dp(a):
    if a is None:
        return C.POINTER(C.c_double)()
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """FP64 CPU restatement of the reference explicit path for one model."""

    def __init__(self, spec: ModelSpec, threads: int = 1):
        self.lib = load()
        self.spec = spec
        self.lib.orc_set_threads(threads)
        self._desc = spec.desc()
        h = C.c_void_p()
        rc = self.lib.orc_create(C.byref(self._desc), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"orc_create failed ({rc}): {self.lib.orc_last_error().decode()}")
        self.h = h
        self.N = spec.n_nodes
        self.E = spec.n_elems
        self.G = spec.n_gauss
        self.watch = np.zeros(0, np.int32)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle error {rc}: {self.lib.orc_last_error().decode()}")

    def run(self, nsteps: int):
        self._check(self.lib.orc_run(self.h, int(nsteps)))

    def set_sampling(self, every: int, watch):
        self.watch = np.ascontiguousarray(watch, dtype=np.int32)
        self._check(self.lib.orc_set_sampling(self.h, every, self.watch.size,
                                              self.watch.ctypes.data_as(C.POINTER(C.c_int32))))

    def samples(self):
        n = C.c_int64()
        self._check(self.lib.orc_get_samples(self.h, C.byref(n), None, None, None, 0))
        m = n.value
        steps = np.zeros(m, np.int64)
        rows = np.zeros((m, self.watch.size, 12))
        en = (dl_energies * max(1, m))()
        self._check(self.lib.orc_get_samples(self.h, C.byref(n),
                                             steps.ctypes.data_as(C.POINTER(C.c_int64)),
                                             _dp(rows), en, m))
        energies = np.array([[e.kinetic, e.potential, e.dissipated, e.external_work, e.contact]
                             for e in en[:m]]).reshape(m, 5)
        return steps, rows, energies

    def set_integrator(self, integ: Integrator):
        d = integ.desc()
        self._check(self.lib.orc_set_integrator(self.h, C.byref(d)))

    def time(self):
        """(t, dt, accepted steps, rejected attempts)"""
        t, dt = C.c_double(), C.c_double()
        st, rj = C.c_int64(), C.c_int64()
        self._check(self.lib.orc_get_time(self.h, C.byref(t), C.byref(dt), C.byref(st), C.byref(rj)))
        return t.value, dt.value, st.value, rj.value

    def sample_times(self, n: int):
        out = np.zeros(max(n, 1))
        self._check(self.lib.orc_get_sample_times(self.h, _dp(out), n))
        return out[:n]

    def state(self):
        u = np.zeros((self.N, 3)); th = np.zeros((self.N, 3)); v = np.zeros((self.N, 6))
        self._check(self.lib.orc_get_state(self.h, _dp(u), _dp(th), _dp(v)))
        return u, th, v

    def set_state(self, u=None, theta=None, v=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        u, theta, v = c(u), c(theta), c(v)
        self._check(self.lib.orc_set_state(self.h, _dp(u), _dp(theta), _dp(v)))

    def energies(self):
        e = dl_energies()
        self._check(self.lib.orc_get_energies(self.h, C.byref(e)))
        return e.as_dict()

    def internal_force(self, u, theta):
        u = np.ascontiguousarray(u, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        f = np.zeros((self.N, 6))
        self._check(self.lib.orc_internal_force(self.h, _dp(u), _dp(theta), _dp(f)))
        return f

    def static_force(self, u, theta):
        """Internal force [N, 6] of a static Newton iteration at (u, theta):
        return map from the committed history, contact forces included,
        history untouched (orc_static_force)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        f = np.zeros((self.N, 6))
        self._check(self.lib.orc_static_force(self.h, _dp(u), _dp(theta), _dp(f)))
        return f

    def static_commit(self, u, theta):
        """Commit a converged static load step at (u, theta) (orc_static_commit)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        self._check(self.lib.orc_static_commit(self.h, _dp(u), _dp(theta)))

    def elastic_energy(self, u, theta):
        u = np.ascontiguousarray(u, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        e = C.c_double()
        self._check(self.lib.orc_elastic_energy(self.h, _dp(u), _dp(theta), C.byref(e)))
        return e.value

    def history(self):
        NG = self.E * self.G
        ep = np.zeros((NG, 6)); hp = np.zeros((NG, 7)); ed = np.zeros(NG)
        self._check(self.lib.orc_get_history(self.h, _dp(ep), _dp(hp), _dp(ed)))
        return ep.reshape(self.E, self.G, 6), hp.reshape(self.E, self.G, 7), ed.reshape(self.E, self.G)

    def frames(self):
        nen = self.spec.conn.shape[1]
        L = np.zeros((self.E * nen, 3, 3)); s0 = np.zeros((self.E, self.G, 6))
        self._check(self.lib.orc_get_frames(self.h, _dp(L), _dp(s0)))
        return L.reshape(self.E, nen, 3, 3), s0

    def mass(self, theta=None):
        th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
        mt = np.zeros(self.N); mr = np.zeros((self.N, 3, 3))
        self._check(self.lib.orc_mass(self.h, _dp(th), _dp(mt), _dp(mr)))
        return mt, mr

    def error_word(self):
        w = C.c_uint32()
        self._check(self.lib.orc_error_word(self.h, C.byref(w)))
        return w.value

    def group_sums(self, nodes):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        r = np.zeros(6); l = np.zeros(6)
        self._check(self.lib.orc_group_sums(self.h, nodes.size,
                                            nodes.ctypes.data_as(C.POINTER(C.c_int32)), _dp(r), _dp(l)))
        return r, l

    def contact_pairs(self):
        """Closed element pairs of the last step, sorted: ([K, 2], gaps [K])."""
        n = C.c_int64()
        self._check(self.lib.orc_contact_pairs(self.h, C.byref(n), None, None, 0))
        k = n.value
        pairs = np.zeros((max(k, 1), 2), dtype=np.int32)
        gaps = np.zeros(max(k, 1))
        self._check(self.lib.orc_contact_pairs(self.h, C.byref(n), pairs.ctypes.data_as(C.POINTER(C.c_int32)),
                                               _dp(gaps), k))
        pairs, gaps = pairs[:k], gaps[:k]
        order = np.lexsort((pairs[:, 1], pairs[:, 0]))
        return pairs[order], gaps[order]

    def joint_contact_pairs(self):
        """Joint pairs in contact in the last step, sorted: ([K, 2] nodes, gaps [K])."""
        n = C.c_int64()
        self._check(self.lib.orc_joint_contact_pairs(self.h, C.byref(n), None, None, 0))
        k = n.value
        pairs = np.zeros((max(k, 1), 2), dtype=np.int32)
        gaps = np.zeros(max(k, 1))
        self._check(self.lib.orc_joint_contact_pairs(self.h, C.byref(n),
                                                     pairs.ctypes.data_as(C.POINTER(C.c_int32)), _dp(gaps), k))
        return pairs[:k], gaps[:k]

    def element_table(self, name):
        """[E, 6] element table at the current state (see dl_element_table)."""
        out = np.zeros((self.E, 6))
        self._check(self.lib.orc_element_table(self.h, name.encode(), _dp(out)))
        return out

    def blacklist_size(self):
        n = C.c_int64()
        self._check(self.lib.orc_blacklist_size(self.h, C.byref(n)))
        return n.value

    def plate_reaction(self):
        out = np.zeros(6)
        self._check(self.lib.orc_plate_reaction(self.h, _dp(out)))
        return out.reshape(2, 3)
