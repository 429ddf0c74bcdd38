"""torch.autograd wrapper of the engine's adjoint (dl_adjoint_radius).

``impact_objective(radii, spec, ...)`` returns the scalar
J = E_diss(T) + react_weight * max_k |R(k)| of an explicit run (R(k): the summed
internal force component ``react_dof`` of the ``react`` node group in step k)
as a differentiable function of the strut radii: the forward runs the engine
(checkpointed forward plus reverse sweep on the GPU, one call), the backward
returns the engine's gradient.  The radii may live on any device; the result
is a 0-d tensor on the same device and dtype.
"""
from __future__ import annotations

import copy
from typing import Optional

import numpy as np
import torch

from .abi import DL_MIXED, DL_PLAIN_FP64, ModelSpec
from .engine import Lattice


class _ImpactObjective(torch.autograd.Function):

    @staticmethod
    def forward(ctx, radii, spec, elem_param, nsteps, checkpoint_every, react_nodes, react_dof, react_weight,
                precision):
        r = radii.detach().to("cpu", torch.float64).numpy()
        s2 = copy.copy(spec)
        s2.elem_radius = r[elem_param]
        eng = Lattice(s2, precision)
        J, grad = eng.adjoint_radius(nsteps, checkpoint_every, elem_param=elem_param, n_params=r.size,
                                     react_nodes=react_nodes, react_dof=react_dof, react_weight=react_weight)
        eng.synchronize()
        ctx.save_for_backward(torch.as_tensor(grad, dtype=radii.dtype, device=radii.device))
        return torch.as_tensor(J, dtype=radii.dtype, device=radii.device)

    @staticmethod
    def backward(ctx, gJ):
        (g,) = ctx.saved_tensors
        return gJ * g, None, None, None, None, None, None, None, None


def impact_objective(radii: torch.Tensor, spec: ModelSpec, nsteps: int, elem_param: Optional[np.ndarray] = None,
                     checkpoint_every: int = 100, react_nodes: Optional[np.ndarray] = None, react_dof: int = 2,
                     react_weight: float = -0.1, precision: int = DL_MIXED) -> torch.Tensor:
    """J(radii) for the lattice ``spec`` (circular sections).  ``elem_param``
    maps elements to entries of ``radii`` (default: ``spec.elem_rod``, one
    radius per strut); ``react_nodes`` defaults to ``spec.groups["top"]``."""
    if elem_param is None:
        elem_param = np.asarray(spec.elem_rod, dtype=np.int32)
    if react_nodes is None:
        react_nodes = spec.groups.get("top", np.zeros(0, np.int32))
    return _ImpactObjective.apply(radii, spec, np.asarray(elem_param, dtype=np.int32), int(nsteps),
                                  int(checkpoint_every), np.asarray(react_nodes, dtype=np.int32), int(react_dof),
                                  float(react_weight), int(precision))


__all__ = ["impact_objective", "DL_MIXED", "DL_PLAIN_FP64"]
