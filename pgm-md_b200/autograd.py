"""Parameter gradients of the pGM energy as a ``torch.autograd.Function``.

``PGMEnergy.apply(q_type, strength_type, alpha_type, radius_type, engine, system)`` maps per-type parameters
(charges, covalent-dipole strengths, polarizabilities, Gaussian radii; float64 tensors) to per-atom and
per-dipole values through ``system.types`` / ``system.cov_types``, evaluates the total energy on the GPU and,
in backward, returns dE/d(parameter) per type.  The energy is stationary in the induced dipoles, so the
gradient is the partial derivative at the solved dipoles (the engine's analytic adjoint, no unrolled
iterations): run the engine with peek = 0 (the peek step breaks stationarity).  Torch carries the tensors;
the arithmetic is the engine's CUDA kernels.
"""

from __future__ import annotations

import numpy as np
import torch


def _per_type(values, index, ntypes):
    out = np.zeros(ntypes)
    np.add.at(out, index, values)
    return out


class PGMEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q_type, strength_type, alpha_type, radius_type, engine, system):
        types = np.asarray(system.types)
        ctypes_ = np.asarray(system.cov_types)
        q = q_type.detach().cpu().numpy()[types]
        al = alpha_type.detach().cpu().numpy()[types]
        R = radius_type.detach().cpu().numpy()[types]
        c = strength_type.detach().cpu().numpy()[ctypes_] if len(ctypes_) else np.zeros(0)
        engine.set_atoms(q, R, al)
        engine.set_covalent(system.cov_atom, system.cov_partner, c)
        res = engine.compute(system.pos, system.box, new_step=True)
        g = engine.param_grad()
        ctx.grads = (
            torch.from_numpy(_per_type(g["q"], types, len(q_type))),
            torch.from_numpy(_per_type(g["cov_strength"], ctypes_, len(strength_type))) if len(ctypes_) else
            torch.zeros(len(strength_type), dtype=torch.float64),
            torch.from_numpy(_per_type(g["alpha"], types, len(alpha_type))),
            torch.from_numpy(_per_type(g["radius"], types, len(radius_type))),
        )
        ctx.result = res
        return torch.tensor(res.energy, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        gq, gc, ga, gR = ctx.grads
        return grad_out * gq, grad_out * gc, grad_out * ga, grad_out * gR, None, None


def energy(engine, system, q_type, strength_type, alpha_type, radius_type):
    """Total electrostatic energy [kJ/mol] as a differentiable function of the per-type parameters."""
    return PGMEnergy.apply(q_type, strength_type, alpha_type, radius_type, engine, system)


def type_parameters(system):
    """Per-type parameter tensors (float64) of a system whose atoms share their type's parameters."""
    types = np.asarray(system.types)
    nt = int(types.max()) + 1
    q = np.zeros(nt)
    al = np.zeros(nt)
    R = np.zeros(nt)
    q[types] = system.q
    al[types] = system.alpha
    R[types] = system.radius
    ct = np.asarray(system.cov_types)
    c = np.zeros(int(ct.max()) + 1 if len(ct) else 0)
    if len(ct):
        c[ct] = system.cov_strength
    t = lambda a: torch.tensor(a, dtype=torch.float64, requires_grad=True)
    return t(q), t(c), t(al), t(R)
