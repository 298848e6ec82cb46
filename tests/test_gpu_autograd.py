"""Differentiation through the FMM (-m gpu): fmm_phi's hand-written backward against
central finite differences in FP64 (h = 1e-5) and against the FP64 direct-sum analytic
gradient, for L = sum_i w_i phi_i, phi_i = q_i sum_{j != i} q_j / r_ij.

Tolerances: finite differences vs autograd, relative 1e-6 (charges; L is quadratic in q)
and 1e-5 (positions, Richardson-extrapolated from h and h/2), plus the rounding of L
divided by h; FMM gradient vs the direct-sum gradient, relative L2 2e-5 (n = 8, the
truncation error of the FMM field).
"""
import numpy as np
import pytest

from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu


def _clustered(N, seed):
    """Positions from 8 isotropic Gaussian clusters (sigma 0.05, centres U[0.15, 0.85]^3)
    shifted onto the origin-centred root cell; charges U[-1, 1]; weights N(0, 1)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.15, 0.85, (8, 3))
    x = c[rng.integers(0, 8, N)] + 0.05 * rng.standard_normal((N, 3))
    x = np.clip(x, 0.0, np.nextafter(1.0, 0.0)) - 0.5
    return x, rng.uniform(-1, 1, N), rng.standard_normal(N)


def _loss(solver, x, q, w, save="fields"):
    import torch
    from bbfmm_b200.autograd import fmm_phi
    solver.set_particles(x)
    xt = torch.as_tensor(x, device="cuda").requires_grad_(True)
    qt = torch.as_tensor(q, device="cuda").requires_grad_(True)
    L = (torch.as_tensor(w, device="cuda") * fmm_phi(solver, qt, xt, save=save)).sum()
    return L, qt, xt


def test_gradients_match_finite_differences():
    from bbfmm_b200 import Solver
    N = 8192
    x, q, w = _clustered(N, 1)
    s = Solver(8, 3, 1.0, mode="d")
    L, qt, xt = _loss(s, x, q, w)
    L.backward()
    gq, gx = qt.grad.cpu().numpy(), xt.grad.cpu().numpy()
    rng = np.random.default_rng(2)
    h = 1e-5
    # rounding of L itself (~1e-13 relative in FP64) divided by the step
    atol = 1e-11 * abs(L.item()) / h
    for k in rng.choice(N, 64, replace=False):
        qp, qm = q.copy(), q.copy()
        qp[k] += h
        qm[k] -= h
        fd = (_loss(s, x, qp, w)[0].item() - _loss(s, x, qm, w)[0].item()) / (2 * h)
        assert abs(fd - gq[k]) <= 1e-6 * abs(gq[k]) + atol, (k, fd, gq[k])
    leaf = 1.0 / 8
    picked = 0
    for k in rng.permutation(N):
        a = int(rng.integers(0, 3))
        frac = ((x[k, a] + 0.5) / leaf) % 1.0
        if min(frac, 1 - frac) * leaf < 1e-4:
            continue  # stay inside the leaf: the tree is piecewise constant in x
        def central(step):
            xp, xm = x.copy(), x.copy()
            xp[k, a] += step
            xm[k, a] -= step
            return (_loss(s, xp, q, w)[0].item() - _loss(s, xm, q, w)[0].item()) / (2 * step)
        # Richardson extrapolation of h and h/2 removes the h^2 term, which close pairs of
        # the clustered input make visible
        fd = (4 * central(h / 2) - central(h)) / 3
        assert abs(fd - gx[k, a]) <= 1e-5 * abs(gx[k, a]) + 2 * atol, (k, a, fd, gx[k, a])
        picked += 1
        if picked == 64:
            break
    s.close()


@pytest.mark.parametrize("mode,save", [("d", "fields"), ("mixed", "fields"), ("mixed", "recompute")])
def test_gradients_match_direct_sum(oracle_d, mode, save):
    from bbfmm_b200 import Solver
    N = 16384
    x, q, w = _clustered(N, 3)
    s = Solver(8, 3 if mode == "d" else 4, 1.0, mode=mode)
    L, qt, xt = _loss(s, x, q, w, save)
    L.backward()
    gq, gx = qt.grad.cpu().numpy(), xt.grad.cpu().numpy()
    t = np.arange(N)
    p1, f1 = oracle_d.direct_field_fp64(x, q, t)
    p2, f2 = oracle_d.direct_field_fp64(x, w * q, t)
    dq = w * p1 + p2
    dx = q[:, None] * (w[:, None] * f1 + f2)
    assert rel_l2(gq, dq) < 2e-5
    assert rel_l2(gx.reshape(-1), dx.reshape(-1)) < 2e-5
    s.close()


@pytest.mark.parametrize("save,n_fields,n_plain,n_pair", [("fields", 2, 0, 0), ("recompute", 0, 1, 1)])
def test_solves_per_forward_backward(save, n_fields, n_plain, n_pair):
    """fields: forward + backward = two solves of fields (the backward is one solve);
    recompute: one plain solve forward, one solve of fields for both charge vectors backward."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200.autograd import fmm_phi
    N = 100000
    x, q, w = _clustered(N, 4)
    s = Solver(8, 4, 1.0, mode="mixed")
    s.set_particles(x)
    qt = torch.as_tensor(q, device="cuda").requires_grad_(True)
    xt = torch.as_tensor(x, device="cuda").requires_grad_(True)
    wt = torch.as_tensor(w, device="cuda")
    calls = {"fields": 0, "plain": 0, "pair": 0}
    of, op, o2 = s.solve_fields, s.solve, s.solve_fields2

    def count(kind, f):
        def g(*a, **k):
            calls[kind] += 1
            return f(*a, **k)
        return g
    s.solve_fields, s.solve, s.solve_fields2 = count("fields", of), count("plain", op), count("pair", o2)
    (wt * fmm_phi(s, qt, xt, save=save)).sum().backward()
    assert calls == {"fields": n_fields, "plain": n_plain, "pair": n_pair}
    assert qt.grad is not None and xt.grad is not None
    s.close()


@pytest.mark.parametrize("mode", ["d", "s", "mixed"])
def test_fields_for_two_charge_vectors_equal_two_solves(mode):
    """bbfmm_b200_solve_fields2 gives, bitwise, what two bbfmm_b200_solve_fields calls give: the
    same far-field passes per charge vector and, in its single near-field pass, each pair's
    terms for both vectors with the arithmetic and summation order of one vector's pass
    (clustered input: sparse and dense near-field items)."""
    import torch
    from bbfmm_b200 import Solver
    x, q, w = _clustered(150000, 6)
    s = Solver(8, 4, 1.0, mode=mode)
    s.set_particles(x)
    q1 = torch.as_tensor(q, device="cuda")
    q2 = torch.as_tensor(w * q, device="cuda")
    a = s.solve_fields(q1) + s.solve_fields(q2)
    b = s.solve_fields2(q1, q2)
    for u, v in zip(a, b):
        assert torch.equal(u, v)
    p1, _, p2, _ = s.solve_fields2(q1, q2, want_field=False)
    assert torch.equal(p1, a[0]) and torch.equal(p2, a[2])
    s.close()


def test_save_modes_agree():
    import torch
    from bbfmm_b200 import Solver
    x, q, w = _clustered(20000, 5)
    s = Solver(8, 4, 1.0, mode="s")
    grads = []
    for save in ("fields", "recompute"):
        L, qt, xt = _loss(s, x, q, w, save)
        L.backward()
        grads.append((qt.grad.cpu().numpy(), xt.grad.cpu().numpy()))
    assert np.array_equal(grads[0][0], grads[1][0]) and np.array_equal(grads[0][1], grads[1][1])
    s.close()


def test_direct_field_matches_oracle(oracle_d):
    """The GPU FP64 direct potential/gradient used for the gradient error of the N = 1M
    benchmark agrees with the oracle's (relative L2 1e-14: summation order only)."""
    import torch
    from bbfmm_b200.fmm import direct_field
    x, q, _ = _clustered(6000, 6)
    t = np.random.default_rng(7).choice(6000, 500, replace=False).astype(np.int32)
    pot, fld = direct_field(torch.as_tensor(x, device="cuda"), torch.as_tensor(q, device="cuda"),
                            torch.as_tensor(t, device="cuda"))
    p0, f0 = oracle_d.direct_field_fp64(x, q, t)
    assert rel_l2(pot.cpu().numpy(), p0) < 1e-14
    assert rel_l2(fld.cpu().numpy().reshape(-1), f0.reshape(-1)) < 1e-14


def test_fields_after_growing_particle_set():
    """solve_fields after set_particles with more particles (the field scratch is resized)."""
    import torch
    from bbfmm_b200 import Solver
    x1, q1, _ = _clustered(5000, 8)
    x2, q2, _ = _clustered(40000, 9)
    s = Solver(4, 3, 1.0, mode="d")
    s.set_particles(x1)
    s.solve_fields(torch.as_tensor(q1, device="cuda"))
    s.set_particles(x2)
    p, f = s.solve_fields(torch.as_tensor(q2, device="cuda"))
    t = Solver(4, 3, 1.0, mode="d")
    t.set_particles(x2)
    p0, f0 = t.solve_fields(torch.as_tensor(q2, device="cuda"))
    assert torch.equal(p, p0) and torch.equal(f, f0)
    s.close()
    t.close()
