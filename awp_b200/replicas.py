"""Independent simulations dealt across GPUs (one process per GPU).

The single-rank time step does not shard: its domain decomposition (halo
exchange of velocity, stress, yield-factor and swap-zone planes between
ranks) is outside this library.  Several GPUs therefore take independent
work -- the instances of a source ensemble, or the shots of a multi-shot
misfit gradient on one shared model -- and the only collective is the one
that combines results: a sum of the per-shot misfits and gradients.

``deal`` assigns items to ranks largest first, round-robin, so the ranks'
loads stay within one item of each other.  ``misfit_gradient_shots`` runs a
rank's shots on its own GPU (``awp_b200.adjoint.misfit_gradient``, each shot
from a zero wavefield on the same workspace), sums them in float64, and one
all-reduce over the process group gives every rank the sum over all shots.
"""
from __future__ import annotations

import numpy as np


def deal(n_items: int, rank: int, world: int, sizes=None) -> list[int]:
    """Indices of the items rank `rank` of `world` takes: sorted by `sizes`
    (largest first; item order when None), then dealt round-robin."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    order = list(range(n_items))
    if sizes is not None:
        if len(sizes) != n_items:
            raise ValueError("one size per item")
        order = sorted(order, key=lambda i: (-sizes[i], i))
    return order[rank::world]


def _default_shot(solver, nsteps, shot, nsnap, want_q):
    from . import adjoint
    src_pos, src_data, rec_xyz, rec_comp, d_obs = shot
    solver.upload_sources(src_pos, src_data)
    solver.reset()
    out = adjoint.misfit_gradient(solver, nsteps, rec_xyz, rec_comp, d_obs, nsnap,
                                  want_q=want_q)
    return out[0], out[2:]


def misfit_gradient_shots(solver, nsteps: int, shots, dist=None, nsnap: int = 0,
                          want_q: bool = False, run_shot=None):
    """Multi-shot misfit and gradient on one model over every rank of the
    default process group of `dist` (torch.distributed; None = this process
    alone).  `shots` is the full list on every rank, each (src_pos, src_data,
    rec_xyz, rec_comp, d_obs); a rank runs the shots ``deal`` gives it.
    Returns (J, [g_lambda, g_mu, g_rho (, g_qpinv, g_qsinv)]) as float64 sums
    over all shots, identical on every rank.  `run_shot(solver, nsteps, shot,
    nsnap, want_q) -> (J, gradients)` replaces the per-shot call (tests)."""
    import torch
    shots = list(shots)
    if not shots:
        raise ValueError("shots is empty")
    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    run = run_shot or _default_shot
    J = 0.0
    acc = None
    for i in deal(len(shots), rank, world):
        Js, g = run(solver, nsteps, shots[i], nsnap, want_q)
        J += Js
        if acc is None:
            acc = [np.asarray(x, np.float64).copy() for x in g]
        else:
            for a, x in zip(acc, g):
                a += x
    if acc is None:  # more ranks than shots: this rank contributes zeros
        p = solver.params
        acc = [np.zeros((p.nz, p.ny, p.nx)) for _ in range(5 if want_q else 3)]
    if dist is None or world == 1:
        return J, acc
    # one flat buffer: the misfit and every gradient, summed in one collective
    backend = dist.get_backend()
    device = (torch.device("cuda", torch.cuda.current_device()) if backend == "nccl"
              else torch.device("cpu"))
    flat = torch.from_numpy(np.concatenate([np.array([J])] + [a.ravel() for a in acc]))
    flat = flat.to(device)
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    flat = flat.cpu().numpy()
    J = float(flat[0])
    out, off = [], 1
    for a in acc:
        out.append(flat[off:off + a.size].reshape(a.shape))
        off += a.size
    return J, out
