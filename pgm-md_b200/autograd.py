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


def force_matching_atom_grads(engine, system, F_target, tol=1e-10):
    """dL/d(per-atom q, radius, alpha; per-dipole strength) of L = sum |F - F_target|^2 by one adjoint solve.

    With w = 2 (F - F_target), g_theta = dE/dtheta at fixed induced dipoles mu and E_tot the total field at fixed
    mu:  dL/dtheta = -D_w g_theta + D_u g_theta,  (alpha^-1 - T) u = -D_w E_tot,  D_w the derivative along the
    displacement w of the positions (mu fixed), D_u along u of the dipoles.  The engine forms every derivative
    analytically on the GPU (tangent pair and PME passes, the radial kernels recomputed per pair) and solves for
    u with its own CG kernels (pgm_engine_force_matching_grad); no iterations are unrolled.  Run the engine with
    peek = 0 (the energy is then stationary in mu).  Works for batched engines (system = a list of systems, the
    target forces concatenated).  Returns (L, grads, F)."""
    if isinstance(system, (list, tuple)):
        pos = np.concatenate([s.pos for s in system])
        boxes = np.stack([s.box for s in system])
        F = engine.compute_batch(pos, boxes)["forces"]
    else:
        F = engine.compute(system.pos, system.box, new_step=True).forces
    L, grads, _ = engine.force_matching_grad(np.asarray(F_target, np.float64), tol=tol)
    return L, grads, F


class PGMForceMatching(torch.autograd.Function):
    """L = sum |F - F_target|^2 as a differentiable function of per-type parameters (adjoint gradient)."""

    @staticmethod
    def forward(ctx, q_type, strength_type, alpha_type, radius_type, engine, system, F_target):
        types = np.asarray(system.types)
        ctypes_ = np.asarray(system.cov_types)
        q = q_type.detach().cpu().numpy()[types]
        al = alpha_type.detach().cpu().numpy()[types]
        R = radius_type.detach().cpu().numpy()[types]
        c = strength_type.detach().cpu().numpy()[ctypes_] if len(ctypes_) else np.zeros(0)
        engine.set_atoms(q, R, al)
        engine.set_covalent(system.cov_atom, system.cov_partner, c)
        L, g, _ = force_matching_atom_grads(engine, system, np.asarray(F_target))
        ctx.grads = (
            torch.from_numpy(_per_type(g["q"], types, len(q_type))),
            torch.from_numpy(_per_type(g["cov_strength"], ctypes_, len(strength_type))) if len(ctypes_) else
            torch.zeros(len(strength_type), dtype=torch.float64),
            torch.from_numpy(_per_type(g["alpha"], types, len(alpha_type))),
            torch.from_numpy(_per_type(g["radius"], types, len(radius_type))),
        )
        return torch.tensor(L, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        gq, gc, ga, gR = ctx.grads
        return grad_out * gq, grad_out * gc, grad_out * ga, grad_out * gR, None, None, None


def force_matching_loss(engine, system, F_target, q_type, strength_type, alpha_type, radius_type):
    """L = sum |F - F_target|^2 [(kJ/mol/nm)^2] as a differentiable function of the per-type parameters."""
    return PGMForceMatching.apply(q_type, strength_type, alpha_type, radius_type, engine, system, F_target)


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
