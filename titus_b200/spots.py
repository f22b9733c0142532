"""Pencil-beam plans sharded across GPUs by spot (one process per GPU).

A plan is a set of independent pencil beams (energy, entry y0) with weights on
one phantom. Spots do not interact, so rank k of W takes spots k, k+W, ...
(round robin: spot counts differ by at most one), solves them in one batched
launch (``titus_solve_batched``). The exchanges are SUM all-reduces over the
process group (NCCL between GPUs, gloo on CPU): the weighted total dose (n
words) and, for the objective below, the spot-weight gradient (one word per
spot). Per-spot doses never leave their rank.

For the plan objective J(w) = sum_c mask_c (sum_s w_s D_s[c] - P[c])^2 the
spot-weight gradient dJ/dw_s = 2 sum_c mask_c (D[c] - P[c]) D_s[c] needs only
the reduced total dose and the rank's own spot doses, so it is computed where
the spots were solved. ``plan_adjoint`` adds the gradient with respect to the
voxel densities through the discrete adjoint of the full-rank sweep
(``DoseAdjoint``): spots of one energy share one solve whose inflow profile is
their weighted sum (the sweep is linear in the inflow), the energy groups are
sharded over the ranks, and dJ/drho and dJ/dw are summed by all-reduce.
"""
from __future__ import annotations

import numpy as np


def partition(nspots: int, world: int, rank: int) -> np.ndarray:
    """Indices of the spots rank `rank` of `world` solves (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if nspots < 0:
        raise ValueError("negative spot count")
    return np.arange(rank, nspots, world, dtype=np.int64)


def _world():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def _allreduce_sum(a: np.ndarray, device=None) -> np.ndarray:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return a
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def plan_dose(solver, spots, weights=None, method: str = "bug", team_ctas: int = 1, max_steps: int = 0,
              device=None, solve=None):
    """Weighted total dose of a plan, sharded by spot over the default process
    group (a single process solves everything when none is initialised).

    ``solve(solver, local_spots, method, team_ctas, max_steps)`` returns the
    per-spot doses (len(local_spots) x n); the default is the batched CUDA path
    (``SolveBatchedPencilBeams``). Every rank must call this with the same
    spots and weights. Returns (total dose (n), local spot indices, local
    per-spot doses).
    """
    spots = list(spots)
    ns = len(spots)
    w = np.ones(ns) if weights is None else np.asarray(weights, dtype=np.float64)
    if w.shape != (ns,):
        raise ValueError(f"{w.shape[0] if w.ndim else 0} weights for {ns} spots")
    world, rank = _world()
    idx = partition(ns, world, rank)
    if solve is None:
        from .solver import SolveBatchedPencilBeams

        def solve(sv, sp, m, t, k):
            return SolveBatchedPencilBeams(sv, sp, m, t, k)[0]
    n = solver.n
    if idx.size:
        local = np.asarray(solve(solver, [spots[i] for i in idx], method, team_ctas, max_steps), dtype=np.float64)
        if local.shape != (idx.size, n):
            raise ValueError(f"solve returned {local.shape}, expected {(idx.size, n)}")
    else:
        local = np.zeros((0, n))
    part = w[idx] @ local if idx.size else np.zeros(n)
    return _allreduce_sum(part, device), idx, local


def plan_objective(solver, spots, weights, prescription, mask=None, method: str = "bug", team_ctas: int = 1,
                   max_steps: int = 0, device=None, solve=None):
    """J(w) = sum_c mask_c (D[c] - P[c])^2 with D = sum_s w_s D_s, and dJ/dw.

    Returns (J, gradient over all spots, total dose). The gradient entries of
    other ranks' spots are filled by one more SUM all-reduce of an nspots
    vector (zeros outside each rank's spots), so every rank returns the whole
    gradient.
    """
    spots = list(spots)
    D, idx, local = plan_dose(solver, spots, weights, method, team_ctas, max_steps, device, solve)
    P = np.asarray(prescription, dtype=np.float64)
    m = np.ones_like(D) if mask is None else np.asarray(mask, dtype=np.float64)
    if P.shape != D.shape or m.shape != D.shape:
        raise ValueError("prescription and mask must have one entry per cell")
    res = m * (D - P)
    J = float(res @ (D - P))
    g = np.zeros(len(spots))
    if idx.size:
        g[idx] = 2.0 * (local @ res)
    return J, _allreduce_sum(g, device), D


def _full_rank_forward(solver, profile):
    from .solver import SolveFirstCollisionSource

    solver.set_beam_profile(profile)
    return SolveFirstCollisionSource(solver)[1]


def _full_rank_adjoint(solver, profile, dj_ddose, checkpoint_every):
    from .solver import DoseAdjoint

    solver.set_beam_profile(profile)
    _, dose, grho, gprof = DoseAdjoint(solver, dj_ddose=dj_ddose, checkpoint_every=checkpoint_every)
    return dose, grho, gprof


def plan_adjoint(make_solver, spots, weights, prescription, mask=None, checkpoint_every: int = 0, device=None,
                 forward=None, adjoint=None):
    """J(w, rho) = sum_c mask_c (D[c] - P[c])^2 of a plan solved with the
    full-rank sweep, and its gradients with respect to the spot weights and the
    voxel densities (the adjoint-optimisation objective of a treatment plan).

    ``spots`` = [(energy, y0), ...]; ``make_solver(energy)`` returns a solver
    (``SolverCSD``) of the phantom for beams of that energy; ``beam_profile(y0=...)``
    of that solver gives a spot's inflow profile. Spots of equal energy share
    one solve with inflow sum_s w_s p_s. Groups are sharded round robin over
    the default process group: each rank solves its groups forward, the total
    dose D is summed by all-reduce, each rank then runs the adjoint of its groups
    with dJ/dD = 2 mask (D - P) (``titus_dose_adjoint`` checkpointing every
    ``checkpoint_every`` steps), and dJ/drho and dJ/dw = p_s . dJ/dprofile are
    summed by all-reduce. ``forward(solver, profile) -> dose`` and
    ``adjoint(solver, profile, dj_ddose, checkpoint_every) -> (dose, dJ/drho,
    dJ/dprofile)`` replace the GPU calls (tests). Returns (J, dJ/dw (nspots),
    dJ/drho (n), D).
    """
    forward = forward or _full_rank_forward
    adjoint = adjoint or _full_rank_adjoint
    spots = list(spots)
    ns = len(spots)
    w = np.asarray(weights, dtype=np.float64)
    if w.shape != (ns,):
        raise ValueError(f"{w.shape[0] if w.ndim else 0} weights for {ns} spots")
    energies = sorted({float(e) for e, _ in spots})
    world, rank = _world()
    mine = partition(len(energies), world, rank)
    groups = []
    for gi in mine:
        e = energies[gi]
        members = [i for i, (ei, _) in enumerate(spots) if float(ei) == e]
        sv = make_solver(e)
        profs = [np.asarray(sv.beam_profile(y0=spots[i][1]), dtype=np.float64) for i in members]
        profile = sum(w[i] * p for i, p in zip(members, profs))
        groups.append((sv, members, profs, profile))
    n = None
    part = None
    for sv, _, _, profile in groups:
        d = np.asarray(forward(sv, profile), dtype=np.float64)
        part = d if part is None else part + d
        n = d.size
    P = np.asarray(prescription, dtype=np.float64)
    if n is None:
        n = P.size
        part = np.zeros(n)
    D = _allreduce_sum(part, device)
    m = np.ones_like(D) if mask is None else np.asarray(mask, dtype=np.float64)
    if P.shape != D.shape or m.shape != D.shape:
        raise ValueError("prescription and mask must have one entry per cell")
    res = m * (D - P)
    J = float(res @ (D - P))
    djdd = 2.0 * res
    grho = np.zeros(n)
    gw = np.zeros(ns)
    for sv, members, profs, profile in groups:
        _, gr, gp = adjoint(sv, profile, djdd, checkpoint_every)
        grho += np.asarray(gr, dtype=np.float64)
        for i, p in zip(members, profs):
            gw[i] = float(p @ np.asarray(gp, dtype=np.float64))
    return J, _allreduce_sum(gw, device), _allreduce_sum(grho, device), D
