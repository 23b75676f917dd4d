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


def force_matching_atom_grads(engine, system, F_target, tol=1e-10, probe=1e-5):
    """dL/d(per-atom q, radius, alpha; per-dipole strength) of L = sum |F - F_target|^2 by one adjoint solve.

    With w = 2 (F - F_target), E the energy at fixed induced dipoles mu, g_theta = dE/dtheta at fixed mu and
    E_tot the total field at fixed mu:
        dL/dtheta = -D_w g_theta + D_u g_theta,   u = -(alpha^-1 - T)^-1 D_w E_tot,
    where D_w is the derivative along the displacement w of the positions (mu fixed) and D_u the derivative
    along u of the dipoles (positions fixed).  D_w comes from central differences of the analytic g_theta and
    E_tot (step `probe` nm for the largest displacement, the pair list of the solution kept, so the function
    is smooth); D_u from central differences in mu, exact here because g_theta is at most quadratic in mu.
    The engine must run with peek = 0 (the energy is then stationary in mu).  Returns (L, grads, F)."""
    res = engine.compute(system.pos, system.box, new_step=True)
    F = res.forces
    mu = engine.induced_dipoles()
    w = 2.0 * (F - F_target)
    L = float(np.sum((F - F_target) ** 2))
    h = probe / max(np.abs(w).max(), 1e-300)

    def probe_at(pos, m):
        r = engine.evaluate_fixed(pos, system.box, m, keep_list=True)
        return engine.param_grad(), r.extra["field"]

    gp, Ep = probe_at(system.pos + h * w, mu)
    gm, Em = probe_at(system.pos - h * w, mu)
    Dw_g = {k: (gp[k] - gm[k]) / (2 * h) for k in gp}
    Dw_E = (Ep - Em) / (2 * h)
    engine.evaluate_fixed(system.pos, system.box, mu, keep_list=True)   # the solution's geometry again
    u, _ = engine.solve(-Dw_E, tol=tol)
    hu = 1e-3 * max(np.abs(mu).max(), 1e-30) / max(np.abs(u).max(), 1e-300)
    gup, _ = probe_at(system.pos, mu + hu * u)
    gum, _ = probe_at(system.pos, mu - hu * u)
    grads = {k: -Dw_g[k] + (gup[k] - gum[k]) / (2 * hu) for k in Dw_g}
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
