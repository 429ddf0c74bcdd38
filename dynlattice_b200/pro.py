"""A dynLattice .pro input file as an engine model (dl_pro_open)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import Integrator, dl_integrator_desc, dl_model_desc
from .engine import DLError, load_library


class ProModel:
    """Parsed .pro file: ``desc()`` (for :class:`~dynlattice_b200.engine.Lattice`),
    the run length ``steps`` and ``t_end`` (control.runWhile), the explicit
    module ``integrator`` (apply with ``Lattice.set_integrator``) and node
    ``groups``."""

    def __init__(self, path: str):
        lib = load_library()
        lib.dl_pro_open.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
        lib.dl_pro_desc.argtypes = [C.c_void_p, C.POINTER(C.POINTER(dl_model_desc))]
        lib.dl_pro_steps.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        lib.dl_pro_group.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32),
                                     C.POINTER(C.POINTER(C.c_int32))]
        lib.dl_pro_close.argtypes = [C.c_void_p]
        lib.dl_pro_integrator.argtypes = [C.c_void_p, C.POINTER(dl_integrator_desc)]
        lib.dl_pro_end_time.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.dl_pro_run.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)]
        lib.dl_pro_note.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_char_p)]
        self.lib = lib
        h = C.c_void_p()
        rc = lib.dl_pro_open(str(path).encode(), C.byref(h))
        if rc != 0:
            raise DLError(rc, lib.dl_last_error().decode())
        self.h = h
        p = C.POINTER(dl_model_desc)()
        lib.dl_pro_desc(h, C.byref(p))
        self._desc = p.contents
        n = C.c_int64()
        lib.dl_pro_steps(h, C.byref(n))
        self.steps = n.value
        te = C.c_double()
        lib.dl_pro_end_time(h, C.byref(te))
        self.t_end = te.value
        ig = dl_integrator_desc()
        lib.dl_pro_integrator(h, C.byref(ig))
        self.integrator = Integrator(ig.kind, ig.precision, ig.min_dt, ig.max_dt, ig.safety, ig.increase,
                                     ig.decrease, ig.length_scale)
        d = self._desc
        self.n_nodes, self.n_elems, self.n_gauss = d.n_nodes, d.n_elems, d.n_gauss
        self.nodes_per_elem = d.nodes_per_elem
        self.dt = d.dt
        self.coords = np.ctypeslib.as_array(d.coords, shape=(d.n_nodes, 3)).copy()
        self.conn = np.ctypeslib.as_array(d.conn, shape=(d.n_elems, d.nodes_per_elem)).copy()

    def desc(self):
        return self._desc

    @property
    def notes(self):
        """Properties the file sets that the engine reads but does not apply."""
        n = C.c_int32()
        self.lib.dl_pro_note(self.h, 0, C.byref(n), None)
        out = []
        for i in range(n.value):
            t = C.c_char_p()
            self.lib.dl_pro_note(self.h, i, None, C.byref(t))
            out.append(t.value.decode())
        return out

    def group(self, name: str) -> np.ndarray:
        n = C.c_int32()
        ptr = C.POINTER(C.c_int32)()
        rc = self.lib.dl_pro_group(self.h, name.encode(), C.byref(n), C.byref(ptr))
        if rc != 0:
            raise DLError(rc, self.lib.dl_last_error().decode())
        return np.ctypeslib.as_array(ptr, shape=(n.value,)).copy() if n.value else np.zeros(0, np.int32)

    def run(self, lattice, out_dir: str = ".", max_steps: int = -1) -> int:
        """Run the file's control loop on ``lattice`` (built from this file,
        with ``integrator`` applied) with its output modules writing under
        ``out_dir``; returns the steps run."""
        n = C.c_int64()
        rc = self.lib.dl_pro_run(self.h, lattice.h, str(out_dir).encode(), int(max_steps), C.byref(n))
        if rc != 0:
            raise DLError(rc, self.lib.dl_last_error().decode())
        return n.value

    def close(self):
        if self.h:
            self.lib.dl_pro_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
