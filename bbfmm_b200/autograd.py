"""Differentiable FMM: phi_i = q_i * sum_{j != i} q_j / |x_i - x_j| with a hand-written
backward.

The FMM-approximated interaction matrix K is symmetric (the compressed operators satisfy
E_{-v} = E_v^T and the same Chebyshev interpolation is used on the source and the target
side), so for a loss with g = dL/dphi:

    dL/dq_k = g_k pot_k(q) + pot_k(g o q)                       (the transposed FMM)
    dL/dx_k = q_k (g_k field_k(q) + field_k(g o q))             (field = grad pot)

Two ways to get pot(q) and field(q) to the backward (``save``):

  "fields"     checkpoint: the forward runs bbfmm_b200_solve_fields and keeps pot and
               field (4 values per particle); the backward is ONE more solve, with charges
               g o q.
  "recompute"  the forward runs the plain solve and keeps nothing but q; the backward
               solves for both charge vectors q and g o q in one call (solve_fields2:
               two far fields, one near-field pass over the pairs for both).

Neither keeps per-level expansions between the passes (each solve rebuilds them on the
device in its own work buffers), so the saved state is O(N) either way.
The reference has no derivative code; the interpolant derivative (Clenshaw recurrence
differentiated) and the P2P gradient kernel are new.
"""
from __future__ import annotations

import torch


class _FMMPhi(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, x, solver, need_field, recompute):
        ctx.solver = solver
        ctx.need_field = need_field
        ctx.recompute = recompute
        empty = torch.empty(0, device=q.device)
        if recompute:
            ctx.save_for_backward(q, empty, empty)
            return solver.solve(q)
        pot, fld = solver.solve_fields(q, want_field=need_field)
        ctx.save_for_backward(q, pot, fld if fld is not None else empty)
        return q.to(pot.dtype) * pot

    @staticmethod
    def backward(ctx, g):
        q, pot, fld = ctx.saved_tensors
        solver = ctx.solver
        if ctx.recompute:
            qs = q.to(solver.dtype)
            g = g.to(solver.dtype).contiguous()
            pot, fld, pot2, fld2 = solver.solve_fields2(qs, g * qs, want_field=ctx.need_field)
            q = qs
        else:
            g = g.to(pot.dtype).contiguous()
            q = q.to(pot.dtype)
            pot2, fld2 = solver.solve_fields(g * q, want_field=ctx.need_field)
        dq = torch.addcmul(pot2, g, pot) if ctx.needs_input_grad[0] else None
        dx = None
        if ctx.needs_input_grad[1] and ctx.need_field:
            dx = torch.addcmul(fld2, fld, g[:, None]).mul_(q[:, None])
        return dq, dx, None, None, None


def fmm_phi(solver, q: torch.Tensor, x: torch.Tensor | None = None, save: str = "fields") -> torch.Tensor:
    """q_i * phi_i on the solver's particles, differentiable in q and (if given and
    requiring grad) in the positions x, an (N, 3) tensor equal to the solver's particles.
    Positions define the tree: pass the same x that was given to solver.set_particles.
    save: "fields" (keep pot and field from the forward) or "recompute" (keep only q)."""
    if save not in ("fields", "recompute"):
        raise ValueError(f"save must be 'fields' or 'recompute', not {save!r}")
    need_field = x is not None and x.requires_grad
    if x is None:
        x = torch.empty(0, device=q.device)
    return _FMMPhi.apply(q, x, solver, need_field, save == "recompute")
