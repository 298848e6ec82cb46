"""Host-side Python interface of the B200 bbFMM solver.

Mirrors the reference's user-facing call ``bbfmm(field, source, q, Nf, Ns, L, n, phi, l)``
(bbfmm.h:97, bbfmm.c:15-87) with field = source, and exposes a handle (``Solver``) that
keeps the tree, the operators and every expansion on the GPU between solves.

Conventions follow the reference: the root cell is [-L/2, L/2]^3, the output is
q_i * phi_i (bbfmm.c:501), the rank is r = n^3/2 and the depth formula of FMMSetup
(bbfmm.c:151-160) is available as ``reference_depth``.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from . import operators as ops


def reference_depth(N: int, level_modifier: int = 0) -> int:
    """maxlev as the reference's FMMSetup computes it: the integer cast binds to log(N)
    only, then one level is subtracted, with a floor of MINLEV = 2 (bbfmm.c:151-160)."""
    l = level_modifier + int(math.log(N)) / math.log(8.0) if N > 0 else float(level_modifier)
    l = int(l)
    if l > 0:
        l -= 1
    return max(l, 2)


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if isinstance(a, np.ndarray) else C.c_void_p(a.data_ptr())


def _check_count(what: str, got: int, want: int):
    """The C-ABI takes bare pointers sized by the particle count it holds: a shorter buffer
    would be read or written past its end, so sizes are checked here, before any copy."""
    if got != want:
        raise ValueError(f"{what} has {got} entries; {want} expected")


def _check_out(out, like):
    if out.dtype != like.dtype or out.device != like.device or out.numel() != like.numel() or not out.is_contiguous():
        raise ValueError("out must be a contiguous tensor of q's dtype, device and size")


class Solver:
    """Device-resident FMM for one particle set.

    mode: "d" (FP64 everywhere), "s" (FP32 everywhere), "mixed" (FP64 passes,
    split-precision tensor-core M2L whose leading operator block -- outputs i < ``lead_rows``,
    components j < ``lead`` -- runs in FP64, split-precision tensor-core projections with 16
    FP64 components, P2P with FP64 separations and compensated FP32 sums).
    kernel: "laplacian" (1/r), "laplacianforce" (x/r^3, x the first component of source -
    target; modes "d" and "s") or "oneoverr4" (1/r^4, modes "d" and "s"), the reference's
    LAPLACIAN, LAPLACIANFORCE and ONEOVERR4 builds."""

    def __init__(self, n: int, maxlev: int, L: float = 1.0, mode: str = "d", lead: int = 16,
                 lead_rows: int = 32, device: int = 0, operators=None, stream=None, rank: int | None = None,
                 tol: float | None = None, kernel: str = "laplacian"):
        import torch
        self.torch = torch
        self.n, self.maxlev, self.L, self.mode = n, maxlev, float(L), mode
        self.r = n ** 3 // 2
        self.lead = lead if mode == "mixed" else 0
        self.lead_rows = lead_rows if mode == "mixed" else 0
        self.device = device
        self.dtype = torch.float32 if mode == "s" else torch.float64
        self.np_dtype = np.float32 if mode == "s" else np.float64
        if kernel not in ops.KERNELS:
            raise ValueError(f"unknown kernel {kernel!r} ({', '.join(ops.KERNELS)})")
        self.kernel = kernel
        if operators is None:
            _, U, E = ops.load_operators(n, single=(mode == "s"), kernel=kernel)
        else:
            U, E = operators
        # tolerance-rank mode: an SVD cut at relative singular value `tol` (or an explicit rank),
        # the truncated operators zero-padded to r and the zero blocks skipped by the kernels
        if tol is not None and rank is None:
            rank = ops.tolerance_rank(n, tol, kernel=kernel)
        self.rank = self.r if rank is None else int(rank)
        if self.rank != self.r:
            U, E = ops.truncate_operators(n, U, E, self.rank)
        U = np.ascontiguousarray(U)
        E = np.ascontiguousarray(E)
        fp32 = int(U.dtype == np.float32)
        assert E.dtype == U.dtype
        cfg = _lib.Config(n=n, maxlev=maxlev, L=self.L, mode=_lib.MODES[mode], lead=self.lead, lead_rows=self.lead_rows,
                          device=device, stream=C.c_void_p(stream) if stream else None)
        h = C.c_void_p()
        _lib.check(_lib.lib().bbfmm_b200_create(C.byref(cfg), _ptr(U), _ptr(E), fp32, C.byref(h)))
        self.h = h
        self.N = 0
        if self.rank != self.r:
            _lib.check(_lib.lib().bbfmm_b200_set_rank(h, self.rank))
        if kernel != "laplacian":
            _lib.check(_lib.lib().bbfmm_b200_set_kernel(h, ops.KERNELS[kernel][1]))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            try:
                _lib.lib().bbfmm_b200_destroy(h)
            except (TypeError, AttributeError):  # interpreter shutdown: the module is gone
                pass

    def close(self):
        self.__del__()

    @property
    def stream(self):
        return _lib.lib().bbfmm_b200_stream(self.h)

    def set_particles(self, xyz):
        """Particle positions, N x 3 inside [-L/2, L/2]^3: a host array (the tree is built on
        the host), or a CUDA tensor (the tree is built on the GPU; same particle order)."""
        torch = self.torch
        if isinstance(xyz, torch.Tensor) and xyz.is_cuda:
            x = xyz.to(device=f"cuda:{self.device}", dtype=self.dtype).reshape(-1, 3).contiguous()
            self.N = x.shape[0]
            torch.cuda.synchronize(x.device)  # the solver's stream reads x
            _lib.check(_lib.lib().bbfmm_b200_set_particles_device(self.h, self.N, C.c_void_p(x.data_ptr())))
            return
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=self.np_dtype).reshape(-1, 3))
        self.N = xyz.shape[0]
        _lib.check(_lib.lib().bbfmm_b200_set_particles(self.h, self.N, _ptr(xyz)))

    def solve(self, q, out=None):
        """q: CUDA tensor (N,) -> q_i * phi_i as a CUDA tensor, on the solver's stream."""
        torch = self.torch
        _check_count("q", q.numel(), self.N)
        q = q.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        if out is None:
            out = torch.empty_like(q)
        _check_out(out, q)
        # order the solver's stream after the caller's work on q, and the caller's stream
        # after the solve: both buffers belong to the caller's stream, which cannot reuse
        # them before the solve has finished with them
        caller = torch.cuda.current_stream(q.device)
        mine = torch.cuda.ExternalStream(self.stream, device=q.device)
        ready = torch.cuda.Event()
        ready.record(caller)
        mine.wait_event(ready)
        _lib.check(_lib.lib().bbfmm_b200_solve(self.h, C.c_void_p(q.data_ptr()), C.c_void_p(out.data_ptr())))
        done = torch.cuda.Event()
        done.record(mine)
        caller.wait_event(done)
        return out

    def solve_fields(self, q, want_field=True):
        """q: CUDA tensor (N,) -> (pot, field): pot_i = sum_j q_j / r_ij and field = grad pot
        at every particle, (N,) and (N, 3) CUDA tensors (field None unless want_field)."""
        torch = self.torch
        _check_count("q", q.numel(), self.N)
        q = q.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        pot = torch.empty_like(q)
        fld = torch.empty((q.numel(), 3), dtype=self.dtype, device=q.device) if want_field else None
        caller = torch.cuda.current_stream(q.device)
        mine = torch.cuda.ExternalStream(self.stream, device=q.device)
        ready = torch.cuda.Event()
        ready.record(caller)
        mine.wait_event(ready)
        _lib.check(_lib.lib().bbfmm_b200_solve_fields(self.h, C.c_void_p(q.data_ptr()), C.c_void_p(pot.data_ptr()),
                                                       C.c_void_p(fld.data_ptr()) if fld is not None else None))
        done = torch.cuda.Event()
        done.record(mine)
        caller.wait_event(done)
        return pot, fld

    def solve_fields2(self, q1, q2, want_field=True):
        """solve_fields for two charge vectors in one call (bbfmm_b200_solve_fields2: the
        near-field pairs evaluated once for both) -> (pot1, field1, pot2, field2)."""
        torch = self.torch
        _check_count("q1", q1.numel(), self.N)
        _check_count("q2", q2.numel(), self.N)
        q1 = q1.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        q2 = q2.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        pot1, pot2 = torch.empty_like(q1), torch.empty_like(q2)
        mk = lambda: torch.empty((q1.numel(), 3), dtype=self.dtype, device=q1.device) if want_field else None
        fld1, fld2 = mk(), mk()
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        caller = torch.cuda.current_stream(q1.device)
        mine = torch.cuda.ExternalStream(self.stream, device=q1.device)
        ready = torch.cuda.Event()
        ready.record(caller)
        mine.wait_event(ready)
        _lib.check(_lib.lib().bbfmm_b200_solve_fields2(self.h, ptr(q1), ptr(q2), ptr(pot1), ptr(fld1), ptr(pot2),
                                                        ptr(fld2)))
        done = torch.cuda.Event()
        done.record(mine)
        caller.wait_event(done)
        return pot1, fld1, pot2, fld2

    def solve_host(self, q, out=None):
        """Host charges -> host q_i * phi_i (copies in, solves, copies out, synchronises).
        out: an optional host array of the same size (pinned memory makes the copy direct)."""
        q = np.ascontiguousarray(np.asarray(q, dtype=self.np_dtype))
        _check_count("q", q.size, self.N)
        phi = np.empty_like(q) if out is None else out
        if phi.dtype != self.np_dtype or phi.size != q.size or not phi.flags.c_contiguous:
            raise ValueError("out must be a contiguous array of the solver's dtype and q's size")
        _lib.check(_lib.lib().bbfmm_b200_solve_host(self.h, _ptr(q), _ptr(phi)))
        return phi

    def set_tc_products(self, nprod: int):
        """Mixed mode: 0 (adaptive, default: split BF16 where one product would not do),
        3 (split BF16 for every term) or 1 (plain BF16) products per M2L term."""
        _lib.check(_lib.lib().bbfmm_b200_set_tc_products(self.h, int(nprod)))

    def set_target_region(self, level: int, active=None):
        """Results wanted only at the particles inside the active cells of `level` (a bool or
        uint8 array of 8^level cells in Morton order; level < 0 clears): the near field skips
        the other targets and the tensor-core M2L above `level` runs only above active cells."""
        if level < 0:
            _lib.check(_lib.lib().bbfmm_b200_set_target_region(self.h, -1, None))
            return
        a = np.ascontiguousarray(np.asarray(active).astype(np.uint8).reshape(-1))
        _check_count("active", a.size, 8 ** level)
        _lib.check(_lib.lib().bbfmm_b200_set_target_region(self.h, int(level), _ptr(a)))

    def set_first_m2l_level(self, level: int):
        """The local expansions start at `level`: the solve gathers, for every target, only the
        sources in the 3 x 3 x 3 neighbourhood of its ancestor at level - 1."""
        _lib.check(_lib.lib().bbfmm_b200_set_first_m2l_level(self.h, int(level)))

    def set_leaf_slab(self, cells: int):
        """Leaf cells per slab of the leaf level (multiple of 64; 0 = automatic)."""
        _lib.check(_lib.lib().bbfmm_b200_set_leaf_slab(self.h, int(cells)))

    def autotune(self, q):
        """Time the per-level M2L and near-field launch choices on this tree (an upward pass
        with charges q, a CUDA tensor) and keep the fastest; returns the choices."""
        _check_count("q", q.numel(), self.N)
        q = q.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        self.torch.cuda.synchronize(q.device)
        _lib.check(_lib.lib().bbfmm_b200_autotune(self.h, C.c_void_p(q.data_ptr())))
        return self.tuning()

    def set_tuning(self, choices):
        """Set launch choices (the dict of tuning(): P2P threads, per-level M2L kind and groups)."""
        v = [int(choices["p2p_threads"])] + [int(k) for k in choices["m2l_kind"]] + [int(g) for g in choices["m2l_groups"]]
        info = (C.c_int * 23)(*v)
        _lib.check(_lib.lib().bbfmm_b200_set_tuning(self.h, info))

    def tuning(self):
        info = (C.c_int * 23)()
        _lib.check(_lib.lib().bbfmm_b200_tuning(self.h, info))
        v = list(info)
        return {"p2p_threads": v[0], "m2l_kind": v[1:12], "m2l_groups": v[12:23]}

    def set_timing(self, on: bool):
        _lib.check(_lib.lib().bbfmm_b200_set_timing(self.h, int(on)))

    def stage_times(self):
        ms = (C.c_float * len(_lib.STAGES))()
        nl = _lib.lib().bbfmm_b200_stage_times(self.h, ms, len(_lib.STAGES))
        return dict(zip(_lib.STAGES, list(ms))), nl

    def time_m2l(self, level: int, reps: int = 3):
        ms = (C.c_float * 2)()
        _lib.check(_lib.lib().bbfmm_b200_time_m2l(self.h, level, reps, ms))
        return float(ms[0]), float(ms[1])

    def multipoles(self, level: int):
        out = np.empty(8 ** level * self.r, dtype=self.np_dtype)
        _lib.check(_lib.lib().bbfmm_b200_copy_multipoles(self.h, level, _ptr(out)))
        return out

    def m2l_output(self, level: int):
        """The level's M2L output L = sum E_k M (before the post-M2L projection), recomputed
        from the multipoles of the last solve; shape (8^level, r), Morton cell order."""
        out = np.empty(8 ** level * self.r, dtype=self.np_dtype)
        _lib.check(_lib.lib().bbfmm_b200_copy_m2l(self.h, level, _ptr(out)))
        return out.reshape(8 ** level, self.r)


def morton_to_grid(m, level: int):
    """Grid coordinates of Morton cell indices (the reference's bit order,
    anotherFMMDistribute.c:239-253)."""
    m = np.asarray(m, np.int64)
    ix, iy, iz = (np.zeros_like(m) for _ in range(3))
    for b in range(level):
        t = (m >> (3 * b)) & 7
        ix |= ((t >> 2) & 1) << b
        iy |= ((t >> 1) & 1) << b
        iz |= (t & 1) << b
    return ix, iy, iz


def leaf_of_particles(xyz, L: float, level: int, fp32: bool = False):
    """Morton leaf of every particle at `level` (the library's own leaf assignment, from FP32
    positions as an FP32 solver has them when fp32), and the particle count of every leaf."""
    x = np.ascontiguousarray(np.asarray(xyz, np.float32 if fp32 else np.float64).reshape(-1, 3))
    N = x.shape[0]
    perm = np.zeros(N, np.int32)
    ls = np.zeros(8 ** level + 1, np.int32)
    _lib.check(_lib.lib().bbfmm_b200_sort_particles(N, int(fp32), _ptr(x), float(L), level,
                                                    perm.ctypes.data_as(C.POINTER(C.c_int)),
                                                    ls.ctypes.data_as(C.POINTER(C.c_int))))
    counts = np.diff(ls)
    leaf = np.empty(N, np.int64)
    leaf[perm] = np.repeat(np.arange(8 ** level, dtype=np.int64), counts)
    return leaf, counts


def refinement_plan(xyz, L: float, depth: int, cap: int, fp32: bool = False):
    """Heavy leaves of a set at `depth` (more than cap particles; a Morton-order mask of 8^depth
    cells), the particles inside their 3 x 3 x 3 neighbourhoods (`sel`, indices into xyz) and,
    among those, the ones in heavy leaves (`keep`, a mask over sel). Leaves are assigned as the
    solvers assign them: from FP32 positions when fp32 (an FP32 solver's own view; a particle
    within FP32 rounding of a leaf face can sit in another leaf than its FP64 position says).
    xyz a torch tensor: the same plan computed on its device, returned as tensors there."""
    if type(xyz).__module__.startswith("torch"):
        return _refinement_plan_tensor(xyz, L, depth, cap, fp32)
    leaf, counts = leaf_of_particles(xyz, L, depth, fp32=fp32)
    heavy = counts > cap
    if not heavy.any():
        return heavy, np.zeros(0, np.int64), np.zeros(0, bool)
    m = 2 ** depth
    gx, gy, gz = morton_to_grid(np.arange(8 ** depth), depth)
    g = np.zeros((m + 2, m + 2, m + 2), bool)
    g[gx + 1, gy + 1, gz + 1] = heavy
    d = np.zeros_like(g)
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            for c in (-1, 0, 1):
                d |= np.roll(np.roll(np.roll(g, a, 0), b, 1), c, 2)
    near_region = d[gx + 1, gy + 1, gz + 1]  # Morton order
    sel = np.nonzero(near_region[leaf])[0]
    return heavy, sel, heavy[leaf[sel]]


def _refinement_plan_tensor(xyz, L: float, depth: int, cap: int, fp32: bool):
    """refinement_plan on the tensor's device: the leaf sort's arithmetic ((x + L/2) times the
    reciprocal leaf length, each operation rounded in the solver's precision, truncated and
    clamped to the last leaf; anotherFMMDistribute.c:258-298), counts by bincount and the
    3 x 3 x 3 neighbourhoods of the heavy leaves by a max filter."""
    import torch
    npdt, dt = (np.float32, torch.float32) if fp32 else (np.float64, torch.float64)
    x = xyz.to(dt).reshape(-1, 3)
    cel = npdt(L)
    for _ in range(depth):
        cel = npdt(cel * npdt(0.5))
    half, inv = float(npdt(npdt(L) / npdt(2))), float(npdt(npdt(1) / cel))  # exact in dt
    m = 2 ** depth
    g = ((x + half) * inv).to(torch.int64).clamp_(max=m - 1)
    key = (g[:, 0] * m + g[:, 1]) * m + g[:, 2]
    heavy_g = torch.bincount(key, minlength=m ** 3) > cap
    gx, gy, gz = morton_to_grid(np.arange(8 ** depth), depth)
    heavy = heavy_g[torch.as_tensor((gx * m + gy) * m + gz, device=x.device)]  # Morton order
    if not bool(heavy_g.any()):
        return heavy, torch.zeros(0, dtype=torch.int64, device=x.device), torch.zeros(0, dtype=torch.bool,
                                                                                      device=x.device)
    near_g = torch.nn.functional.max_pool3d(heavy_g.view(1, 1, m, m, m).float(), 3, stride=1, padding=1).view(-1) > 0
    sel = torch.nonzero(near_g[key]).squeeze(1)
    return heavy, sel, heavy_g[key[sel]]


class AdaptiveSolver:
    """Two-level adaptive refinement over uniform solvers (no counterpart in the reference,
    whose octrees are uniform, anotherBuildFMMHierachy.c:44-55).

    A coarse solver of depth `coarse_depth` takes every particle; its leaves holding more than
    `cap` particles are heavy. For a target in a heavy leaf A, the near field -- the direct sum
    over A's 3 x 3 x 3 neighbourhood N(A) -- is computed instead by a refined solver of depth
    `fine_depth` over the particles of the heavy leaves' neighbourhoods, whose local expansions
    start at level coarse_depth + 1: its interaction lists at the levels below and its leaf-level
    near field together cover exactly N(A), so it returns that near field, FMM-approximated at
    the finer depth. So

        phi = coarse (far field of everyone, near field of the light leaves)
            + refined (near field of the heavy leaves' particles)

    The coarse solver's near field skips the heavy leaves and the refined solver's skips the
    rest (target regions), and the refined tensor-core M2L runs only on the tiles above heavy
    leaves, so its cost follows the heavy volume rather than the whole grid. Positions and
    charges are in the caller's order throughout."""

    def __init__(self, n: int, coarse_depth: int, fine_depth: int, L: float = 1.0, mode: str = "mixed",
                 cap: int = 256, device: int = 0, **kw):
        if fine_depth <= coarse_depth:
            raise ValueError("fine_depth must exceed coarse_depth")
        self.n, self.Dc, self.Df, self.L, self.mode, self.cap, self.device = (
            n, coarse_depth, fine_depth, float(L), mode, int(cap), device)
        self.kw = kw
        self.coarse = Solver(n, coarse_depth, L, mode=mode, device=device, **kw)
        self.fine = None

    def close(self):
        for s in (self.coarse, self.fine):
            if s is not None:
                s.close()

    def set_particles(self, xyz):
        """Positions as for Solver.set_particles: a host array, or a CUDA tensor (the trees and
        the refinement plan are then built on the GPU)."""
        torch = self.coarse.torch
        on_device = isinstance(xyz, torch.Tensor) and xyz.is_cuda
        if on_device:
            x = xyz.to(f"cuda:{self.device}").reshape(-1, 3)
        else:
            x = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
        self.N = x.shape[0]
        self.coarse.set_particles(x)
        heavy, sel, keep = refinement_plan(x, self.L, self.Dc, self.cap, fp32=self.mode == "s")
        if on_device:
            heavy = heavy.cpu().numpy()
        self.heavy_leaves = int(heavy.sum())
        if self.fine is not None:
            self.fine.close()
            self.fine = None
        if not heavy.any():
            self.coarse.set_target_region(-1)
            return
        self.coarse.set_target_region(self.Dc, ~heavy)
        self.fine = Solver(self.n, self.Df, self.L, mode=self.mode, device=self.device, **self.kw)
        self.fine.set_particles(x[sel])
        self.fine.set_first_m2l_level(self.Dc + 1)
        self.fine.set_target_region(self.Dc, heavy)
        dev = f"cuda:{self.device}"
        self.sel = torch.as_tensor(sel, device=dev)
        self.keep_local = torch.nonzero(keep).squeeze(1) if on_device else torch.as_tensor(np.nonzero(keep)[0], device=dev)
        self.keep_global = torch.as_tensor(sel[keep], device=dev)
        self.fine_particles = int(sel.shape[0])

    def solve(self, q, out=None):
        """q: CUDA tensor (N,) -> q_i * phi_i (CUDA tensor) on the caller's stream."""
        phi = self.coarse.solve(q, out=out)
        if self.fine is not None:
            pf = self.fine.solve(q.index_select(0, self.sel))
            phi.index_add_(0, self.keep_global, pf.index_select(0, self.keep_local))
        return phi


def batch_depth(N: int, per_leaf: float = 32.0) -> int:
    """Leaf depth for about `per_leaf` particles per leaf: round(log8(N / per_leaf)), >= 2."""
    return max(2, int(round(math.log(max(N, 1) / per_leaf, 8)))) if N > 0 else 2



class AdaptiveBatch:
    """Two-level adaptive refinement of a batch (AdaptiveSolver for many sets): a coarse Batch of
    the sets as given, whose near field skips the heavy leaves (more than `cap` particles), and a
    refined Batch of each set with heavy leaves -- the particles of their neighbourhoods, at the
    set's depth + `refine`, local expansions starting one level below the coarse leaves -- whose
    results are added at the heavy leaves' particles. Charges and results as for Batch; positions
    host arrays, or all CUDA tensors (the trees and the refinement plans built on the GPU)."""

    def __init__(self, sets, mode: str = "mixed", cap: int = 256, refine: int = 2, L: float = 1.0, **kw):
        import torch
        self.torch = torch
        self.coarse = Batch(sets, mode=mode, L=L, **kw)
        self.offsets = self.coarse.offsets
        self.N = self.coarse.N
        on_device = len(sets) > 0 and all(isinstance(x, torch.Tensor) and x.is_cuda for x, _, _ in sets)
        nonzero = (lambda k: torch.nonzero(k).squeeze(1)) if on_device else (lambda k: np.nonzero(k)[0])
        cat = torch.cat if on_device else np.concatenate
        light, refined, heavy_masks, sel_all, keep_local, keep_global = [], [], [], [], [], []
        rbase = 0
        self.heavy_leaves = 0
        for s, (x, n, lev) in enumerate(sets):
            x = x.reshape(-1, 3) if on_device else np.asarray(x, np.float64).reshape(-1, 3)
            heavy, sel, keep = refinement_plan(x, L, lev, cap, fp32=mode == "s")
            if on_device:
                heavy = heavy.cpu().numpy()
            light.append(~heavy)
            off = int(self.offsets[s])
            if heavy.any() and lev + refine <= 10:
                self.heavy_leaves += int(heavy.sum())
                refined.append((x[sel], n, lev + refine))
                heavy_masks.append(heavy)
                sel_all.append(off + sel)
                keep_global.append(off + sel[keep])
                keep_local.append(rbase + nonzero(keep))
                rbase += int(sel.shape[0])
            else:
                light[-1] = np.ones_like(heavy)
        self.coarse.set_target_regions(0, np.concatenate(light))
        self.refined = None
        self.refined_particles = rbase
        if refined:
            self.refined = Batch(refined, mode=mode, L=L, **kw)
            self.refined.set_target_regions(refine, np.concatenate(heavy_masks), first_m2l=True)
            dev = f"cuda:{self.coarse.device}"
            self.sel = torch.as_tensor(cat(sel_all), device=dev)
            self.keep_local = torch.as_tensor(cat(keep_local), device=dev)
            self.keep_global = torch.as_tensor(cat(keep_global), device=dev)
            # fixed buffers for the refined batch, whose captured graph is tied to its pointers
            self.q_ref = torch.empty(rbase, dtype=self.coarse.dtype, device=dev)
            self.phi_ref = torch.empty_like(self.q_ref)

    def close(self):
        for b in (self.coarse, self.refined):
            if b is not None:
                b.close()

    def autotune(self, q):
        """Both batches' launch choices, then the submission (replayed graphs or launches) that
        runs the two batches faster side by side: their graphs each run every group as a
        parallel branch, which can crowd the two batches' kernels onto the SMs together."""
        self.coarse.autotune(q)
        torch = self.torch
        if self.refined is not None:
            torch.index_select(q.to(self.q_ref.dtype), 0, self.sel, out=self.q_ref)
            self.refined.autotune(self.q_ref)
        out = torch.empty_like(q.to(self.coarse.dtype))
        ms = {}
        for graph in (True, False):
            for _ in range(2):
                self.solve(q, out=out, graph=graph)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(3):
                self.solve(q, out=out, graph=graph)
            b.record()
            b.synchronize()
            ms[graph] = a.elapsed_time(b)
        self.graph = ms[True] <= ms[False]

    graph = True  # submission of solve(graph=None): replayed graphs (set by autotune)

    def solve(self, q, out=None, graph: bool | None = None):
        """As Batch.solve (graph None: the submission autotune chose). The coarse and the
        refined batch run at the same time on their own streams (both read charges gathered
        before either starts); the refined results are added on the caller's stream once both
        are done."""
        torch = self.torch
        if graph is None:
            graph = self.graph
        if self.refined is None:
            return self.coarse.solve(q, out=out, graph=graph)
        _check_count("q", q.numel(), self.N)
        q = q.to(device=f"cuda:{self.coarse.device}", dtype=self.coarse.dtype).contiguous()
        if out is None:
            out = torch.empty_like(q)
        torch.index_select(q, 0, self.sel, out=self.q_ref)
        done = [self.coarse._submit(q, out, graph), self.refined._submit(self.q_ref, self.phi_ref, graph)]
        caller = torch.cuda.current_stream(q.device)
        for d in done:
            caller.wait_event(d)
        out.index_add_(0, self.keep_global, self.phi_ref.index_select(0, self.keep_local))
        return out

def set_cost(N: int, n: int, maxlev: int) -> float:
    """Model of one set's device work: M2L flops 2 r^2 x (about 189 8^l pairs per level) plus
    near-field pairs (27 neighbour leaves of N / 8^maxlev particles each, uniform estimate)."""
    r = n ** 3 // 2
    m2l = 2.0 * r * r * sum(189.0 * 8 ** l for l in range(2, maxlev + 1))
    p2p = 27.0 * N * N / 8 ** maxlev
    return m2l + 20.0 * p2p  # a pair costs about 20 flops


def shard_sets(costs, world: int):
    """Split set indices over `world` ranks, longest job first onto the least loaded rank
    (greedy LPT: the largest load is within 4/3 of the optimum). Deterministic; returns one
    sorted index list per rank."""
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


class Batch:
    """Many independent particle sets solved together (bbfmm_b200_batch_*).

    sets: a list of (xyz, n, maxlev) with xyz an (N_s, 3) array inside [-L/2, L/2]^3: host
    arrays (the trees are sorted on the host) or, all of them, CUDA tensors (the trees are built
    on the GPU, bbfmm_b200_batch_create_device; the same particle order and leaf ranges).
    Charges and results are CUDA tensors holding the sets back to back in list order
    (``offsets[s]:offsets[s + 1]``). kernel: as for Solver, one for every set."""

    def __init__(self, sets, mode: str = "mixed", L: float = 1.0, lead: int = 16, lead_rows: int = 32,
                 device: int = 0, kernel: str = "laplacian"):
        import torch
        self.torch = torch
        self.mode, self.L, self.device = mode, float(L), device
        self.dtype = torch.float32 if mode == "s" else torch.float64
        np_dtype = np.float32 if mode == "s" else np.float64
        on_device = len(sets) > 0 and all(isinstance(x, torch.Tensor) and x.is_cuda for x, _, _ in sets)
        counts = np.array([(x.numel() if on_device else np.asarray(x).size) // 3 for x, _, _ in sets], dtype=np.int32)
        ns = np.array([n for _, n, _ in sets], dtype=np.int32)
        levs = np.array([lv for _, _, lv in sets], dtype=np.int32)
        self.depths = levs.tolist()
        self.offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.N = int(self.offsets[-1])
        if on_device:
            xyz = torch.cat([x.to(device=f"cuda:{device}", dtype=self.dtype).reshape(-1, 3) for x, _, _ in sets])
            xyz = xyz.contiguous()
            torch.cuda.synchronize(xyz.device)  # the batch's streams read xyz
        else:
            xyz = np.ascontiguousarray(np.concatenate([np.asarray(x, np_dtype).reshape(-1, 3) for x, _, _ in sets])
                                       if len(sets) else np.zeros((0, 3), np_dtype))
        if kernel not in ops.KERNELS:
            raise ValueError(f"unknown kernel {kernel!r} ({', '.join(ops.KERNELS)})")
        self.kernel = kernel
        ops_ = {}
        for n in sorted(set(ns.tolist())):
            _, U, E = ops.load_operators(n, single=(mode == "s"), kernel=kernel)
            ops_[n] = (np.ascontiguousarray(U), np.ascontiguousarray(E))
        fp32 = int(mode == "s")
        p = lambda n, k: _ptr(ops_[n][k]) if n in ops_ else None
        cfg = _lib.Config(n=0, maxlev=0, L=self.L, mode=_lib.MODES[mode], lead=lead if mode == "mixed" else 0,
                          lead_rows=lead_rows if mode == "mixed" else 0, device=device, stream=None)
        h = C.c_void_p()
        ip = C.POINTER(C.c_int)
        create = _lib.lib().bbfmm_b200_batch_create_device if on_device else _lib.lib().bbfmm_b200_batch_create
        _lib.check(create(C.byref(cfg), len(sets), ns.ctypes.data_as(ip), levs.ctypes.data_as(ip),
                          counts.ctypes.data_as(ip), _ptr(xyz),
                          p(4, 0), p(4, 1), p(8, 0), p(8, 1), fp32, C.byref(h)))
        self.h = h
        if kernel != "laplacian":
            _lib.check(_lib.lib().bbfmm_b200_batch_set_kernel(h, ops.KERNELS[kernel][1]))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            try:
                _lib.lib().bbfmm_b200_batch_destroy(h)
            except (TypeError, AttributeError):  # interpreter shutdown: the module is gone
                pass

    def close(self):
        self.__del__()

    @property
    def stream(self):
        return _lib.lib().bbfmm_b200_batch_stream(self.h)

    def set_target_regions(self, levels_up: int, active=None, first_m2l: bool = False):
        """Target regions of every set at level depth_s - levels_up: `active` concatenates, in
        set order, each set's mask over the 8^(depth_s - levels_up) cells of that level (None
        clears); first_m2l also starts each set's local expansions one level below it."""
        if active is None:
            _lib.check(_lib.lib().bbfmm_b200_batch_set_target_regions(self.h, 0, None, 0))
            return
        a = np.ascontiguousarray(np.asarray(active).astype(np.uint8).reshape(-1))
        _check_count("active", a.size, int(sum(8 ** (lv - levels_up) for lv in self.depths)))
        _lib.check(_lib.lib().bbfmm_b200_batch_set_target_regions(self.h, int(levels_up), _ptr(a), int(first_m2l)))

    def _order(self, q):
        torch = self.torch
        caller = torch.cuda.current_stream(q.device)
        mine = torch.cuda.ExternalStream(self.stream, device=q.device)
        ev = torch.cuda.Event()
        ev.record(caller)
        mine.wait_event(ev)
        return caller, mine

    def _submit(self, q, out, graph: bool):
        """Launches the solve of q (on this device, this dtype, contiguous) into out on the
        batch's stream after the work already queued on the caller's stream; returns the event
        that marks its end, which the caller's stream does not wait for."""
        _check_out(out, q)
        _, mine = self._order(q)
        _lib.check(_lib.lib().bbfmm_b200_batch_solve(self.h, C.c_void_p(q.data_ptr()), C.c_void_p(out.data_ptr()),
                                                      int(graph)))
        done = self.torch.cuda.Event()
        done.record(mine)
        return done

    def solve(self, q, out=None, graph: bool = True):
        """q: CUDA tensor (N_total,) -> q_i * phi_i of every set (same layout)."""
        torch = self.torch
        _check_count("q", q.numel(), self.N)
        q = q.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        if out is None:
            out = torch.empty_like(q)
        done = self._submit(q, out, graph)
        torch.cuda.current_stream(q.device).wait_event(done)
        return out

    def set_tc_products(self, nprod: int):
        """Mixed mode: 0 (adaptive, default: split BF16 where one product would not do),
        3 (split BF16 for every term) or 1 (plain BF16) products per M2L term."""
        _lib.check(_lib.lib().bbfmm_b200_set_tc_products(self.h, int(nprod)))

    def set_leaf_slab(self, cells: int):
        """Leaf cells per slab of the leaf level (multiple of 64; 0 = automatic)."""
        _lib.check(_lib.lib().bbfmm_b200_set_leaf_slab(self.h, int(cells)))

    def autotune(self, q):
        _check_count("q", q.numel(), self.N)
        q = q.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        self.torch.cuda.synchronize(q.device)
        _lib.check(_lib.lib().bbfmm_b200_batch_autotune(self.h, C.c_void_p(q.data_ptr())))
        return self.groups()

    def groups(self):
        out = []
        for g in range(_lib.lib().bbfmm_b200_batch_groups(self.h)):
            info = (C.c_int * 27)()
            _lib.check(_lib.lib().bbfmm_b200_batch_group_info(self.h, g, info))
            v = list(info)
            out.append({"n": v[0], "maxlev": v[1], "sets": v[2], "particles": v[3], "p2p_threads": v[4],
                        "m2l_kind": v[5:5 + v[1] + 1], "m2l_groups": v[16:16 + v[1] + 1]})
        return out

    def group_stage_times(self, q, g: int):
        """Stage times (ms) of group g solved alone (q: CUDA tensor of all sets)."""
        _check_count("q", q.numel(), self.N)
        q = q.to(device=f"cuda:{self.device}", dtype=self.dtype).contiguous()
        out = self.torch.empty_like(q)
        ms = (C.c_float * len(_lib.STAGES))()
        _lib.check(_lib.lib().bbfmm_b200_batch_group_stage_times(self.h, g, C.c_void_p(q.data_ptr()),
                                                                  C.c_void_p(out.data_ptr()), ms, len(_lib.STAGES)))
        return dict(zip(_lib.STAGES, [round(v, 3) for v in ms]))

    @property
    def graph_nodes(self) -> int:
        return int(_lib.lib().bbfmm_b200_batch_graph_nodes(self.h))


def _check_direct(xyz, q, targets):
    """Sizes, devices and target indices of a direct sum: the kernel reads xyz[3 t + k] and
    q[t] for every target t, so each must lie in [0, N)."""
    _check_count("xyz", xyz.numel(), 3 * q.numel())
    if not (xyz.device == q.device == targets.device) or q.device.type != "cuda":
        raise ValueError("xyz, q and targets must be CUDA tensors on one device")
    if targets.numel() and (int(targets.min()) < 0 or int(targets.max()) >= q.numel()):
        raise ValueError("targets must be particle indices in [0, N)")


def direct(xyz, q, targets, stream=None):
    """FP64 direct sum q_i sum_{j != i} q_j / r_ij on the GPU for the given targets
    (torch CUDA tensors: xyz (N,3) float64, q (N,) float64, targets (T,) int32)."""
    import torch
    xyz = xyz.to(torch.float64).contiguous()
    q = q.to(torch.float64).contiguous()
    targets = targets.to(torch.int32).contiguous()
    _check_direct(xyz, q, targets)
    out = torch.empty(targets.numel(), dtype=torch.float64, device=q.device)
    st = torch.cuda.current_stream(q.device).cuda_stream if stream is None else stream
    _lib.check(_lib.lib().bbfmm_b200_direct(q.numel(), C.c_void_p(xyz.data_ptr()), C.c_void_p(q.data_ptr()),
                                             targets.numel(), C.c_void_p(targets.data_ptr()),
                                             C.c_void_p(out.data_ptr()), C.c_void_p(st)))
    return out


def direct_field(xyz, q, targets, stream=None):
    """FP64 direct potential sum_{j != i} q_j / r_ij and its gradient at the given targets
    (torch CUDA tensors as in ``direct``) -> (pot (T,), field (T, 3))."""
    import torch
    xyz = xyz.to(torch.float64).contiguous()
    q = q.to(torch.float64).contiguous()
    targets = targets.to(torch.int32).contiguous()
    _check_direct(xyz, q, targets)
    pot = torch.empty(targets.numel(), dtype=torch.float64, device=q.device)
    fld = torch.empty((targets.numel(), 3), dtype=torch.float64, device=q.device)
    st = torch.cuda.current_stream(q.device).cuda_stream if stream is None else stream
    _lib.check(_lib.lib().bbfmm_b200_direct_field(q.numel(), C.c_void_p(xyz.data_ptr()), C.c_void_p(q.data_ptr()),
                                                   targets.numel(), C.c_void_p(targets.data_ptr()),
                                                   C.c_void_p(pot.data_ptr()), C.c_void_p(fld.data_ptr()),
                                                   C.c_void_p(st)))
    return pot, fld


def bbfmm(xyz, q, L: float = 1.0, n: int = 4, level_modifier: int = 0, mode: str = "d", maxlev=None,
          operators=None, kernel: str = "laplacian"):
    """One solve from host arrays, like the reference's ``bbfmm()`` with field = source; the
    kernel, a compile-time choice there (bbfmm.c:109-144), is an argument here.

    Returns q_i * phi_i in the input order."""
    xyz = np.asarray(xyz)
    N = xyz.shape[0]
    lev = maxlev if maxlev is not None else reference_depth(N, level_modifier)
    s = Solver(n, lev, L, mode=mode, operators=operators, kernel=kernel)
    try:
        s.set_particles(xyz)
        return s.solve_host(q)
    finally:
        s.close()
