"""ctypes binding of ``libdynlattice_b200.so`` (the C ABI of ``include/dynlattice.h``).

The Python class :class:`Lattice` mirrors the life cycle of the reference's
explicit path: INIT (``dl_create``), repeated explicit steps (``dl_run``, the
LeapFrog module), output sampling (``dl_set_sampling``/``dl_get_samples``, the
Sample/GroupOutput modules) and state/energy queries.  There is no CPU path:
creating a lattice without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from .abi import (DL_MIXED, DL_PLAIN_FP64, Integrator, ModelSpec, dl_energies, dl_integrator_desc,
                  dl_model_desc)

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libdynlattice_b200.so"
_lib = None

DL_ERR_NAMES = {
    1: "DL_ERR_INVALID", 2: "DL_ERR_CUDA", 3: "DL_ERR_PARSE", 4: "DL_ERR_RETURN_MAP",
    5: "DL_ERR_NONFINITE", 6: "DL_ERR_MASS", 7: "DL_ERR_TIMEOUT", 8: "DL_ERR_UNSUPPORTED",
    9: "DL_ERR_IO", 10: "DL_ERR_NOMEM", 11: "DL_ERR_NO_DEVICE", 12: "DL_ERR_CONTACT",
}


class DLError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{DL_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def load_library():
    """Load the engine library (built in-tree by ``python -m dynlattice_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `python -m dynlattice_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    i32p = C.POINTER(C.c_int32)
    lib.dl_last_error.restype = C.c_char_p
    lib.dl_version.restype = C.c_char_p
    lib.dl_device_count.argtypes = [C.POINTER(C.c_int)]
    lib.dl_create.argtypes = [C.POINTER(dl_model_desc), C.c_int, C.POINTER(P)]
    lib.dl_destroy.argtypes = [P]
    lib.dl_set_stream.argtypes = [P, P]
    lib.dl_set_exec_mode.argtypes = [P, C.c_int]
    lib.dl_run.argtypes = [P, C.c_int64]
    lib.dl_get_info.argtypes = [P, i32p, i32p, C.POINTER(C.c_char_p)]
    lib.dl_set_sampling.argtypes = [P, C.c_int32, C.c_int32, i32p, C.c_int64]
    lib.dl_get_samples.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), dp,
                                   C.POINTER(dl_energies), C.c_int64]
    lib.dl_get_error_word.argtypes = [P, C.POINTER(C.c_uint32)]
    lib.dl_synchronize.argtypes = [P]
    lib.dl_get_sizes.argtypes = [P, i32p, i32p, i32p, C.POINTER(C.c_int64)]
    lib.dl_get_state.argtypes = [P, dp, dp, dp]
    lib.dl_set_state.argtypes = [P, dp, dp, dp]
    lib.dl_get_energies.argtypes = [P, C.POINTER(dl_energies)]
    lib.dl_internal_force.argtypes = [P, dp, dp, dp]
    lib.dl_get_history.argtypes = [P, dp, dp, dp]
    lib.dl_group_sums.argtypes = [P, C.c_int32, i32p, dp, dp]
    lib.dl_eval_expression.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_char_p), dp, dp]
    lib.dl_contact_pairs.argtypes = [P, C.POINTER(C.c_int64), i32p, dp, C.c_int64]
    lib.dl_joint_contact_pairs.argtypes = [P, C.POINTER(C.c_int64), i32p, dp, C.c_int64]
    lib.dl_element_table.argtypes = [P, C.c_char_p, dp]
    lib.dl_plate_reaction.argtypes = [P, dp]
    lib.dl_contact_stats.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.dl_launch_count.argtypes = [P, C.POINTER(C.c_int64)]
    lib.dl_set_tape_budget.argtypes = [P, C.c_int64]
    lib.dl_autotune.argtypes = [P, C.c_int64, i32p, i32p, dp]
    lib.dl_set_threads.argtypes = [P, C.c_int32]
    lib.dl_set_group_output.argtypes = [P, C.c_int32]
    lib.dl_set_integrator.argtypes = [P, C.POINTER(dl_integrator_desc)]
    lib.dl_get_time.argtypes = [P, dp, dp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.dl_get_sample_times.argtypes = [P, dp, C.c_int64]
    lib.dl_write_vtu.argtypes = [P, C.c_char_p, C.c_int32]
    lib.dl_write_pvd.argtypes = [C.c_char_p, C.c_int32, dp, C.POINTER(C.c_char_p)]
    lib.dl_trim_retained_memory.argtypes = []
    lib.dl_adjoint_radius.argtypes = [P, C.c_int64, C.c_int32, C.c_int32, i32p, C.c_int32, i32p, C.c_int32,
                                      C.c_double, dp, dp]
    lib.dl_adjoint_branch_mode.argtypes = [P, C.c_int32]
    lib.dl_adjoint_branch_tape.argtypes = [P, C.c_int32, C.POINTER(C.c_uint8), C.c_int64, C.POINTER(C.c_int64),
                                           dp]
    lib.dl_adjoint_branch_bytes.argtypes = [P, C.POINTER(C.c_int64)]
    lib.dl_device_binary_version.argtypes = [C.POINTER(C.c_int32)]
    lib.dl_clear_error.argtypes = [P]
    lib.dl_set_barrier_test.argtypes = [P, C.c_uint32, C.c_uint32]
    _lib = lib
    return lib


def _dp(a):
    if a is None:
        return C.POINTER(C.c_double)()
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(lib, rc):
    if rc != 0:
        raise DLError(rc, lib.dl_last_error().decode())


def trim_retained_memory():
    """Return the unused part of the adjoint's retained tape pool (current
    device) to the driver."""
    lib = load_library()
    _check(lib, lib.dl_trim_retained_memory())


VTU_FINT, VTU_FEXT, VTU_FRES = 1, 2, 4


def write_pvd(path, times, files):
    """ParaView collection of VTU files with their times."""
    lib = load_library()
    t = np.ascontiguousarray(times, dtype=np.float64)
    arr = (C.c_char_p * max(1, len(files)))(*[str(f).encode() for f in files])
    _check(lib, lib.dl_write_pvd(str(path).encode(), len(files), _dp(t), arr))


def device_count() -> int:
    lib = load_library()
    n = C.c_int()
    lib.dl_device_count(C.byref(n))
    return n.value


def eval_expression(expr: str, **variables) -> float:
    """Evaluate a .pro expression with the engine's parser."""
    lib = load_library()
    names = list(variables)
    arr = (C.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
    vals = np.array([float(variables[n]) for n in names] or [0.0])
    out = C.c_double()
    _check(lib, lib.dl_eval_expression(expr.encode(), len(names), arr, _dp(vals), C.byref(out)))
    return out.value


class Lattice:
    """One rod lattice resident on the GPU."""

    def __init__(self, spec: ModelSpec, precision: int = DL_PLAIN_FP64, stream: Optional[int] = None):
        self.lib = load_library()
        self.spec = spec
        self._desc = spec.desc()
        h = C.c_void_p()
        _check(self.lib, self.lib.dl_create(C.byref(self._desc), int(precision), C.byref(h)))
        self.h = h
        self.precision = precision
        self.N = spec.n_nodes
        self.E = spec.n_elems
        self.G = spec.n_gauss
        self.watch = np.zeros(0, np.int32)
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if getattr(self, "h", None):
            self.lib.dl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        _check(self.lib, rc)

    def set_stream(self, stream: int):
        self._c(self.lib.dl_set_stream(self.h, C.c_void_p(int(stream))))

    def set_exec_mode(self, mode: int):
        self._c(self.lib.dl_set_exec_mode(self.h, int(mode)))

    def info(self) -> dict:
        """Kernel variant: {"jit": bool, "persistent_blocks": int, "jit_log": str}."""
        j = C.c_int32(); b = C.c_int32(); l = C.c_char_p()
        self._c(self.lib.dl_get_info(self.h, C.byref(j), C.byref(b), C.byref(l)))
        return {"jit": bool(j.value), "persistent_blocks": b.value,
                "jit_log": (l.value or b"").decode(errors="replace")}

    def run(self, nsteps: int):
        self._c(self.lib.dl_run(self.h, int(nsteps)))

    def synchronize(self):
        self._c(self.lib.dl_synchronize(self.h))

    def clear_error(self):
        """Clear the device error word and reset the grid barrier (dl_clear_error)."""
        self._c(self.lib.dl_clear_error(self.h))

    def set_barrier_test(self, limit_us: int, phantom_blocks: int):
        """Failure-path hook (dl_set_barrier_test): bound one grid-barrier
        wait and let the barrier expect blocks that never arrive."""
        self._c(self.lib.dl_set_barrier_test(self.h, int(limit_us), int(phantom_blocks)))

    @property
    def step(self) -> int:
        s = C.c_int64()
        self._c(self.lib.dl_get_sizes(self.h, None, None, None, C.byref(s)))
        return s.value

    def set_sampling(self, every: int, watch: Sequence[int] = (), capacity: int = 0):
        self.watch = np.ascontiguousarray(watch, dtype=np.int32)
        self._c(self.lib.dl_set_sampling(self.h, int(every), int(self.watch.size),
                                         self.watch.ctypes.data_as(C.POINTER(C.c_int32)),
                                         int(capacity)))

    def write_vtu(self, path, node_data: int = 0):
        """ParaView file of the current state; node_data: VTU_FINT | VTU_FEXT | VTU_FRES."""
        self._c(self.lib.dl_write_vtu(self.h, str(path).encode(), int(node_data)))

    def set_integrator(self, integ: Integrator):
        """LeapFrog (fixed dt) or MilneDevice (error-controlled dt); with
        MilneDevice, run(n) advances n accepted steps."""
        d = integ.desc()
        self._c(self.lib.dl_set_integrator(self.h, C.byref(d)))

    def time(self):
        """(t, dt of the next step, accepted steps, rejected attempts)"""
        t, dt = C.c_double(), C.c_double()
        st, rj = C.c_int64(), C.c_int64()
        self._c(self.lib.dl_get_time(self.h, C.byref(t), C.byref(dt), C.byref(st), C.byref(rj)))
        return t.value, dt.value, st.value, rj.value

    def sample_times(self):
        n = C.c_int64()
        self._c(self.lib.dl_get_samples(self.h, C.byref(n), None, None, None, 0))
        out = np.zeros(max(n.value, 1))
        self._c(self.lib.dl_get_sample_times(self.h, _dp(out), n.value))
        return out[:n.value]

    def samples(self):
        n = C.c_int64()
        self._c(self.lib.dl_get_samples(self.h, C.byref(n), None, None, None, 0))
        m = n.value
        steps = np.zeros(m, np.int64)
        rows = np.zeros((m, max(1, self.watch.size), 12))
        en = (dl_energies * max(1, m))()
        self._c(self.lib.dl_get_samples(self.h, C.byref(n), steps.ctypes.data_as(C.POINTER(C.c_int64)),
                                        _dp(rows), en, m))
        energies = np.array([[e.kinetic, e.potential, e.dissipated, e.external_work, e.contact]
                             for e in en[:m]]).reshape(m, 5)
        return steps, rows[:, :self.watch.size], energies

    def state(self):
        u = np.zeros((self.N, 3)); th = np.zeros((self.N, 3)); v = np.zeros((self.N, 6))
        self._c(self.lib.dl_get_state(self.h, _dp(u), _dp(th), _dp(v)))
        return u, th, v

    def set_state(self, u=None, theta=None, v=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        u, theta, v = c(u), c(theta), c(v)
        self._c(self.lib.dl_set_state(self.h, _dp(u), _dp(theta), _dp(v)))

    def set_state_ptrs(self, u_ptr: int, theta_ptr: int, v_ptr: int):
        """dl_set_state from raw host pointers (e.g. pinned torch tensors)."""
        dp = C.POINTER(C.c_double)
        cast = lambda p: C.cast(C.c_void_p(p), dp) if p else dp()
        self._c(self.lib.dl_set_state(self.h, cast(u_ptr), cast(theta_ptr), cast(v_ptr)))

    def get_state_ptrs(self, u_ptr: int, theta_ptr: int, v_ptr: int):
        dp = C.POINTER(C.c_double)
        cast = lambda p: C.cast(C.c_void_p(p), dp) if p else dp()
        self._c(self.lib.dl_get_state(self.h, cast(u_ptr), cast(theta_ptr), cast(v_ptr)))

    def energies(self):
        e = dl_energies()
        self._c(self.lib.dl_get_energies(self.h, C.byref(e)))
        return e.as_dict()

    def error_word(self) -> int:
        w = C.c_uint32()
        self._c(self.lib.dl_get_error_word(self.h, C.byref(w)))
        return w.value

    def internal_force(self, u, theta):
        u = np.ascontiguousarray(u, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        f = np.zeros((self.N, 6))
        self._c(self.lib.dl_internal_force(self.h, _dp(u), _dp(theta), _dp(f)))
        return f

    def history(self):
        NG = self.E * self.G
        ep = np.zeros((NG, 6)); hp = np.zeros((NG, 7)); ed = np.zeros(NG)
        self._c(self.lib.dl_get_history(self.h, _dp(ep), _dp(hp), _dp(ed)))
        return ep.reshape(self.E, self.G, 6), hp.reshape(self.E, self.G, 7), ed.reshape(self.E, self.G)

    def set_group_output(self, on: bool = True):
        """Record the internal force of the last step of every run (needed by
        group_sums' first result; off by default)."""
        self._c(self.lib.dl_set_group_output(self.h, int(bool(on))))

    def group_sums(self, nodes):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        r = np.zeros(6); l = np.zeros(6)
        self._c(self.lib.dl_group_sums(self.h, int(nodes.size),
                                       nodes.ctypes.data_as(C.POINTER(C.c_int32)), _dp(r), _dp(l)))
        return r, l

    def contact_pairs(self):
        """Closed element pairs of the last step: ([K, 2] int32 sorted, gaps [K])."""
        n = C.c_int64()
        self._c(self.lib.dl_contact_pairs(self.h, C.byref(n), None, None, 0))
        k = n.value
        pairs = np.zeros((max(k, 1), 2), dtype=np.int32)
        gaps = np.zeros(max(k, 1))
        self._c(self.lib.dl_contact_pairs(self.h, C.byref(n), pairs.ctypes.data_as(C.POINTER(C.c_int32)),
                                          _dp(gaps), k))
        return pairs[:k], gaps[:k]

    def element_table(self, name: str) -> np.ndarray:
        """[E, 6] element table at the current state (dl_element_table):
        "strain", "stress", "mat_strain", "mat_stress" or "plast_strain"."""
        out = np.zeros((self.E, 6))
        self._c(self.lib.dl_element_table(self.h, name.encode(), _dp(out)))
        return out

    def joint_contact_pairs(self):
        """Joint pairs in contact in the last step: ([K, 2] node indices, sorted; gaps [K])."""
        n = C.c_int64()
        self._c(self.lib.dl_joint_contact_pairs(self.h, C.byref(n), None, None, 0))
        k = n.value
        pairs = np.zeros((max(k, 1), 2), dtype=np.int32)
        gaps = np.zeros(max(k, 1))
        self._c(self.lib.dl_joint_contact_pairs(self.h, C.byref(n), pairs.ctypes.data_as(C.POINTER(C.c_int32)),
                                                _dp(gaps), k))
        return pairs[:k], gaps[:k]

    def adjoint_radius(self, nsteps: int, checkpoint_every: int = 100, elem_param=None, n_params=None,
                       react_nodes=None, react_dof: int = 2, react_weight: float = 0.0):
        """Run nsteps forward and back (dl_adjoint_radius): returns (J, dJ/dp) for
        J = E_diss(T) + react_weight * max_k |sum_{react_nodes} fint[react_dof](k)|,
        p = element radii, or per-parameter sums through elem_param."""
        if elem_param is not None:
            elem_param = np.ascontiguousarray(elem_param, dtype=np.int32)
            n_params = int(elem_param.max()) + 1 if n_params is None else int(n_params)
            ep_ptr = elem_param.ctypes.data_as(C.POINTER(C.c_int32))
        else:
            n_params = self.E
            ep_ptr = C.POINTER(C.c_int32)()
        if react_nodes is not None and len(react_nodes) > 0:
            react_nodes = np.ascontiguousarray(react_nodes, dtype=np.int32)
            rn_ptr, n_react = react_nodes.ctypes.data_as(C.POINTER(C.c_int32)), int(react_nodes.size)
        else:
            rn_ptr, n_react = C.POINTER(C.c_int32)(), 0
        J = C.c_double()
        grad = np.zeros(n_params)
        self._c(self.lib.dl_adjoint_radius(self.h, int(nsteps), int(checkpoint_every), n_params, ep_ptr, n_react,
                                           rn_ptr, int(react_dof), float(react_weight), C.byref(J), _dp(grad)))
        return J.value, grad

    def set_branch_mode(self, mode: int):
        """Branch tape of the next adjoint_radius run (dl_adjoint_branch_mode):
        0 off, 1 record the return map's iteration counts and the peak step,
        2 impose a tape set with set_branch_tape (objective-only runs)."""
        self._c(self.lib.dl_adjoint_branch_mode(self.h, int(mode)))

    def branch_tape(self):
        """The recorded tape ([nsteps][n_gauss][n_elems] uint8, engine element
        order), the peak step (1-based within the run) and the peak's sign."""
        n = C.c_int64()
        self._c(self.lib.dl_adjoint_branch_bytes(self.h, C.byref(n)))
        tape = np.zeros(n.value, dtype=np.uint8)
        ps, sg = C.c_int64(), C.c_double()
        self._c(self.lib.dl_adjoint_branch_tape(self.h, 1, tape.ctypes.data_as(C.POINTER(C.c_uint8)),
                                                int(n.value), C.byref(ps), C.byref(sg)))
        return tape, ps.value, sg.value

    def set_branch_tape(self, tape, peak_step: int, peak_sign: float):
        tape = np.ascontiguousarray(tape, dtype=np.uint8)
        ps, sg = C.c_int64(int(peak_step)), C.c_double(float(peak_sign))
        self._c(self.lib.dl_adjoint_branch_tape(self.h, 0, tape.ctypes.data_as(C.POINTER(C.c_uint8)),
                                                int(tape.size), C.byref(ps), C.byref(sg)))

    def autotune(self, steps: int = 200):
        """Pick the fastest launch shape for this lattice (dl_autotune):
        returns (exec mode, threads per block, ms for `steps` steps)."""
        mode, tpb, ms = C.c_int32(), C.c_int32(), C.c_double()
        self._c(self.lib.dl_autotune(self.h, int(steps), C.byref(mode), C.byref(tpb), C.byref(ms)))
        return mode.value, tpb.value, ms.value

    def set_launch_shape(self, mode: int, threads: int):
        """Exec mode and threads per block (e.g. an autotune result)."""
        self.set_exec_mode(mode)
        self._c(self.lib.dl_set_threads(self.h, int(threads)))

    def set_tape_budget(self, nbytes: int):
        """Device memory for the adjoint's state tape (-1: half the free memory;
        0: checkpoints only, every segment recomputed)."""
        self._c(self.lib.dl_set_tape_budget(self.h, int(nbytes)))

    def launch_count(self) -> int:
        """Kernels this handle has launched in run() so far."""
        n = C.c_int64()
        self._c(self.lib.dl_launch_count(self.h, C.byref(n)))
        return n.value

    def contact_stats(self):
        """(candidate pairs in the current list, list builds so far)."""
        a, b = C.c_int64(), C.c_int64()
        self._c(self.lib.dl_contact_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def plate_reaction(self):
        """Force of each rigid plate on the nodes in the last step, [2, 3]."""
        out = np.zeros(6)
        self._c(self.lib.dl_plate_reaction(self.h, _dp(out)))
        return out.reshape(2, 3)


class Batch(Lattice):
    """Many independent lattices stepped together in one launch (dl_create_batch)."""

    def __init__(self, specs, precision: int = DL_PLAIN_FP64, stream: Optional[int] = None):
        self.lib = load_library()
        lib = self.lib
        lib.dl_create_batch.argtypes = [C.POINTER(dl_model_desc), C.c_int32, C.c_int, C.POINTER(C.c_void_p)]
        lib.dl_batch_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32)]
        lib.dl_batch_get_state.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.dl_batch_get_energies.argtypes = [C.c_void_p, C.c_int32, C.POINTER(dl_energies)]
        self.specs = list(specs)
        self._descs = (dl_model_desc * len(self.specs))(*[s.desc() for s in self.specs])
        h = C.c_void_p()
        _check(lib, lib.dl_create_batch(self._descs, len(self.specs), int(precision), C.byref(h)))
        self.h = h
        self.precision = precision
        self.spec = self.specs[0]
        self.N = sum(s.n_nodes for s in self.specs)
        self.E = sum(s.n_elems for s in self.specs)
        self.G = self.specs[0].n_gauss
        self.watch = np.zeros(0, np.int32)
        n = len(self.specs)
        self.node_off = np.zeros(n + 1, np.int32)
        self.elem_off = np.zeros(n + 1, np.int32)
        cnt = C.c_int32()
        self._c(lib.dl_batch_sizes(self.h, C.byref(cnt), self.node_off.ctypes.data_as(C.POINTER(C.c_int32)),
                                   self.elem_off.ctypes.data_as(C.POINTER(C.c_int32))))
        if stream is not None:
            self.set_stream(stream)

    def lattice_state(self, k: int):
        n = self.specs[k].n_nodes
        u = np.zeros((n, 3)); th = np.zeros((n, 3)); v = np.zeros((n, 6))
        self._c(self.lib.dl_batch_get_state(self.h, int(k), _dp(u), _dp(th), _dp(v)))
        return u, th, v

    def lattice_energies(self, k: int) -> dict:
        e = dl_energies()
        self._c(self.lib.dl_batch_get_energies(self.h, int(k), C.byref(e)))
        return e.as_dict()
