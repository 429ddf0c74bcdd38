"""ctypes mirror of ``include/dynlattice.h`` and a Python builder for model descriptions.

The structures here are byte-for-byte the C structs of the engine's C ABI.  A
:class:`ModelSpec` owns the numpy arrays of one model and produces a
``dl_model_desc`` whose pointers stay valid while the spec lives.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

DL_OK = 0
DL_PLAIN_FP64 = 0
DL_MIXED = 1

DL_MAT_ELASTIC_ROD = 0
DL_MAT_ELASTOPLASTIC_ROD = 1

DL_BC_DIRICHLET = 0
DL_BC_NEUMANN = 1
DL_BC_INIT_VELO = 2
DL_BC_INIT_DISP = 3
DL_BC_MASS = 4

DL_MASS_CONSISTENT = 0
DL_MASS_LUMPED = 1

DL_EW_RETURN_MAP = 0x1
DL_EW_NONFINITE = 0x2
DL_EW_TIMEOUT = 0x4
DL_EW_MASS = 0x8
DL_EW_CONTACT_OVERFLOW = 0x10

DOF_NAMES = ("dx", "dy", "dz", "rx", "ry", "rz")


class dl_material_desc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("young", C.c_double),
        ("shear_modulus", C.c_double),
        ("shear_correction", C.c_double),
        ("area", C.c_double),
        ("area_moment", C.c_double * 2),
        ("polar_moment", C.c_double),
        ("density", C.c_double),
        ("inertia_correct", C.c_double),
        ("circle", C.c_int32),
        ("radius", C.c_double),
        ("yield_cond", C.c_char_p),
        ("yield_deriv", C.POINTER(C.c_char_p)),
        ("n_yield_deriv", C.c_int32),
        ("has_isotropic", C.c_int32),
        ("isotropic_coefficient", C.c_double),
        ("kinematic_tensor", C.POINTER(C.c_double)),
        ("max_iter", C.c_int32),
        ("precision", C.c_double),
    ]


class dl_bc_desc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("dof", C.c_int32),
        ("n_nodes", C.c_int32),
        ("nodes", C.POINTER(C.c_int32)),
        ("factor", C.c_double),
        ("scale", C.c_char_p),
    ]


class dl_plate_desc(C.Structure):
    _fields_ = [
        ("normal", C.c_double * 3),
        ("point0", C.c_double * 3),
        ("velocity", C.c_double * 3),
        ("penalty", C.c_double),
    ]


class dl_contact_desc(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("radius", C.c_double),
        ("penalty_sts", C.c_double),
        ("penalty_nts", C.c_double),
        ("margin", C.c_double),
        ("max_pairs", C.c_int32),
        ("n_plates", C.c_int32),
        ("plates", dl_plate_desc * 2),
    ]


class dl_joint_contact_desc(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("radius", C.c_double),
        ("penalty", C.c_double),
        ("n_joints", C.c_int32),
        ("joints", C.POINTER(C.c_int32)),
        ("margin", C.c_double),
    ]


class dl_model_desc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int32),
        ("coords", C.POINTER(C.c_double)),
        ("n_elems", C.c_int32),
        ("nodes_per_elem", C.c_int32),
        ("conn", C.POINTER(C.c_int32)),
        ("elem_rod", C.POINTER(C.c_int32)),
        ("n_rods", C.c_int32),
        ("elem_mat", C.POINTER(C.c_int32)),
        ("elem_radius", C.POINTER(C.c_double)),
        ("n_materials", C.c_int32),
        ("materials", C.POINTER(dl_material_desc)),
        ("dof_names", C.POINTER(C.c_char_p)),
        ("n_gauss", C.c_int32),
        ("has_material_ey", C.c_int32),
        ("material_ey", C.c_double * 3),
        ("n_given_dirs", C.c_int32),
        ("given_dir_nodes", C.POINTER(C.c_int32)),
        ("given_dirs", C.POINTER(C.c_double)),
        ("n_bcs", C.c_int32),
        ("bcs", C.POINTER(dl_bc_desc)),
        ("dt", C.c_double),
        ("so3_update", C.c_int32),
        ("gyroscopic", C.c_int32),
        ("contact", dl_contact_desc),
        ("joint_contact", dl_joint_contact_desc),
        ("mass_mode", C.c_int32),
        ("n_ties", C.c_int32),
        ("ties", C.POINTER(C.c_int32)),
    ]


class dl_energies(C.Structure):
    _fields_ = [
        ("kinetic", C.c_double),
        ("potential", C.c_double),
        ("dissipated", C.c_double),
        ("external_work", C.c_double),
        ("contact", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


DL_INTEG_LEAPFROG = 0
DL_INTEG_MILNE = 1


class dl_integrator_desc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("precision", C.c_double),
        ("min_dt", C.c_double),
        ("max_dt", C.c_double),
        ("safety", C.c_double),
        ("increase", C.c_double),
        ("decrease", C.c_double),
        ("length_scale", C.c_double),
    ]


@dataclass
class Integrator:
    """Explicit module settings (dl_integrator_desc): LeapFrog with fixed dt, or
    MilneDevice with error-controlled dt.  Zero means the reference default."""
    kind: int = DL_INTEG_LEAPFROG
    precision: float = 0.0
    min_dt: float = 0.0
    max_dt: float = 0.0
    safety: float = 0.0
    increase: float = 0.0
    decrease: float = 0.0
    length_scale: float = 0.0

    @classmethod
    def milne(cls, precision: float, **kw) -> "Integrator":
        return cls(kind=DL_INTEG_MILNE, precision=precision, **kw)

    def desc(self) -> dl_integrator_desc:
        return dl_integrator_desc(self.kind, self.precision, self.min_dt, self.max_dt, self.safety,
                                  self.increase, self.decrease, self.length_scale)


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.POINTER(ctype)()
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class Material:
    """Keys of ElasticRodMaterial / ElastoPlasticRodMaterial (.pro names in comments)."""

    young: float                      # young
    shear_modulus: float              # shear_modulus (or from poisson_ratio)
    area: float
    area_moment: Sequence[float]
    polar_moment: float
    density: float = 0.0              # density
    shear_correction: float = 5.0 / 6.0
    inertia_correct: float = 1.0      # inertia_correct
    circle: bool = False
    radius: float = 0.0
    yield_cond: Optional[str] = None  # yieldCond
    yield_deriv: Optional[List[str]] = None  # yieldDeriv
    isotropic_coefficient: Optional[float] = None  # isotropicCoefficient
    kinematic_tensor: Optional[Sequence[float]] = None  # kinematicTensor
    max_iter: int = 20
    precision: float = 1e-5

    @staticmethod
    def circle_section(radius: float, young: float, poisson_ratio: float = None,
                       shear_modulus: float = None, density: float = 0.0, **kw) -> "Material":
        """cross_section = "circle" (ElasticRodMaterial.cpp:159-165): A = pi r^2,
        I = pi r^4 / 4, J = I1 + I2, shear correction 9/10."""
        if shear_modulus is None:
            shear_modulus = young / 2.0 / (poisson_ratio + 1.0)
        A = np.pi * radius ** 2
        I = np.pi * radius ** 4 / 4.0
        kw.setdefault("shear_correction", 9.0 / 10.0)
        return Material(young=young, shear_modulus=shear_modulus, area=A, area_moment=(I, I),
                        polar_moment=2 * I, density=density, circle=True, radius=radius, **kw)

    @property
    def plastic(self) -> bool:
        return self.yield_cond is not None


@dataclass
class BC:
    kind: int
    dof: int
    nodes: np.ndarray
    factor: float = 0.0
    scale: Optional[str] = None


@dataclass
class Contact:
    """RodContact keys (RodContactModel.cpp:24-97) plus the engine's rigid plates."""

    radius: float = 0.0
    penalty: float = 0.0              # penalty (both STS and NTS)
    penalty_nts: Optional[float] = None
    enabled: bool = True
    margin: float = 0.0
    max_pairs: int = 0
    plates: List[dict] = field(default_factory=list)  # {"normal", "point0", "velocity", "penalty"}


@dataclass
class JointContact:
    """JointContact keys (JointContactModel.cpp:24-60): joints are the nodes
    of the element group "points", in that group's order."""

    joints: Sequence[int]
    radius: float
    penalty: float
    margin: float = 0.0


@dataclass
class ModelSpec:
    """Plain-array description of one rod lattice (see ``dl_model_desc``)."""

    coords: np.ndarray                      # [N, 3]
    conn: np.ndarray                        # [E, nen]
    elem_rod: np.ndarray                    # [E]
    materials: List[Material]
    elem_mat: Optional[np.ndarray] = None
    elem_radius: Optional[np.ndarray] = None
    n_gauss: int = 2
    dt: float = 1e-6
    so3_update: bool = True
    gyroscopic: bool = True
    lumped_mass: bool = False               # explicit module's mass: diagonal, no gyroscopic term
    ties: Optional[np.ndarray] = None       # [K, 2] (master, slave) rigid hinge ties
    bcs: List[BC] = field(default_factory=list)
    material_ey: Optional[Sequence[float]] = None
    contact: Optional[Contact] = None
    joint_contact: Optional[JointContact] = None
    groups: dict = field(default_factory=dict)   # named node sets (not passed to C)
    name: str = "model"

    def __post_init__(self):
        self.coords = np.ascontiguousarray(self.coords, dtype=np.float64)
        self.conn = np.ascontiguousarray(self.conn, dtype=np.int32)
        self.elem_rod = np.ascontiguousarray(self.elem_rod, dtype=np.int32)
        if self.elem_mat is not None:
            self.elem_mat = np.ascontiguousarray(self.elem_mat, dtype=np.int32)
        if self.elem_radius is not None:
            self.elem_radius = np.ascontiguousarray(self.elem_radius, dtype=np.float64)
        self._keep = []

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])

    def desc(self) -> dl_model_desc:
        """Build the C description; pointers borrow this object's arrays."""
        keep = []
        d = dl_model_desc()
        d.n_nodes = self.n_nodes
        d.coords = _ptr(self.coords, C.c_double)
        d.n_elems = self.n_elems
        d.nodes_per_elem = int(self.conn.shape[1])
        d.conn = _ptr(self.conn, C.c_int32)
        d.elem_rod = _ptr(self.elem_rod, C.c_int32)
        d.n_rods = int(self.elem_rod.max()) + 1 if self.n_elems else 0
        d.elem_mat = _ptr(self.elem_mat, C.c_int32)
        d.elem_radius = _ptr(self.elem_radius, C.c_double)
        mats = (dl_material_desc * len(self.materials))()
        for i, m in enumerate(self.materials):
            md = mats[i]
            md.type = DL_MAT_ELASTOPLASTIC_ROD if m.plastic else DL_MAT_ELASTIC_ROD
            md.young = m.young
            md.shear_modulus = m.shear_modulus
            md.shear_correction = m.shear_correction
            md.area = m.area
            md.area_moment[0] = m.area_moment[0]
            md.area_moment[1] = m.area_moment[1] if len(m.area_moment) > 1 else m.area_moment[0]
            md.polar_moment = m.polar_moment
            md.density = m.density
            md.inertia_correct = m.inertia_correct
            md.circle = 1 if m.circle else 0
            md.radius = m.radius
            if m.plastic:
                yc = m.yield_cond.encode()
                keep.append(yc)
                md.yield_cond = yc
                if m.yield_deriv:
                    arr = (C.c_char_p * len(m.yield_deriv))(*[s.encode() for s in m.yield_deriv])
                    keep.append(arr)
                    md.yield_deriv = arr
                    md.n_yield_deriv = len(m.yield_deriv)
                if m.isotropic_coefficient is not None:
                    md.has_isotropic = 1
                    md.isotropic_coefficient = m.isotropic_coefficient
                if m.kinematic_tensor is not None:
                    kt = np.ascontiguousarray(m.kinematic_tensor, dtype=np.float64)
                    keep.append(kt)
                    md.kinematic_tensor = _ptr(kt, C.c_double)
                md.max_iter = m.max_iter
                md.precision = m.precision
        keep.append(mats)
        d.n_materials = len(self.materials)
        d.materials = mats
        d.dof_names = C.POINTER(C.c_char_p)()
        d.n_gauss = self.n_gauss
        if self.material_ey is not None:
            d.has_material_ey = 1
            for k in range(3):
                d.material_ey[k] = self.material_ey[k]
        bcs = (dl_bc_desc * max(1, len(self.bcs)))()
        for i, b in enumerate(self.bcs):
            nodes = np.ascontiguousarray(b.nodes, dtype=np.int32)
            keep.append(nodes)
            bcs[i].kind = b.kind
            bcs[i].dof = b.dof
            bcs[i].n_nodes = int(nodes.size)
            bcs[i].nodes = _ptr(nodes, C.c_int32)
            bcs[i].factor = b.factor
            if b.scale:
                s = b.scale.encode()
                keep.append(s)
                bcs[i].scale = s
        keep.append(bcs)
        d.n_bcs = len(self.bcs)
        d.bcs = bcs
        d.dt = self.dt
        d.so3_update = 1 if self.so3_update else 0
        d.gyroscopic = 1 if self.gyroscopic else 0
        d.mass_mode = DL_MASS_LUMPED if self.lumped_mass else DL_MASS_CONSISTENT
        if self.ties is not None and len(self.ties) > 0:
            ties = np.ascontiguousarray(self.ties, dtype=np.int32).reshape(-1, 2)
            keep.append(ties)
            d.n_ties = int(ties.shape[0])
            d.ties = _ptr(ties, C.c_int32)
        if self.contact is not None:
            c = self.contact
            d.contact.enabled = 1 if (c.enabled and c.penalty > 0) else 0
            d.contact.radius = c.radius
            d.contact.penalty_sts = c.penalty
            d.contact.penalty_nts = c.penalty if c.penalty_nts is None else c.penalty_nts
            d.contact.margin = c.margin
            d.contact.max_pairs = c.max_pairs
            d.contact.n_plates = len(c.plates)
            for i, pl in enumerate(c.plates[:2]):
                for k in range(3):
                    d.contact.plates[i].normal[k] = pl["normal"][k]
                    d.contact.plates[i].point0[k] = pl["point0"][k]
                    d.contact.plates[i].velocity[k] = pl["velocity"][k]
                d.contact.plates[i].penalty = pl["penalty"]
        if self.joint_contact is not None:
            jc = self.joint_contact
            joints = np.ascontiguousarray(jc.joints, dtype=np.int32)
            keep.append(joints)
            d.joint_contact.enabled = 1
            d.joint_contact.radius = jc.radius
            d.joint_contact.penalty = jc.penalty
            d.joint_contact.n_joints = int(joints.size)
            d.joint_contact.joints = _ptr(joints, C.c_int32)
            d.joint_contact.margin = jc.margin
        self._keep = keep
        return d
