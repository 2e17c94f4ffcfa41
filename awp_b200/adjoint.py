"""Seismogram misfit and its material gradient through the C ABI.

``misfit_gradient`` runs the checkpointed forward / discrete-adjoint pair of
``awp_misfit_gradient`` (include/awp_b200.h); ``Misfit`` wraps it as a
``torch.autograd.Function`` of the Lame moduli and the density, so a model
held as torch tensors can be optimised with torch's optimisers.  Receivers
are velocity samples at interior cells: ``rec_xyz`` [nrec][3] = (x, y, z) with
z counted from the surface, ``rec_comp`` [nrec] = 0 (vx), 1 (vy), 2 (vz).
Model arrays are [nz][ny][nx], surface first (the mesh-file order).
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_double

import numpy as np

from ._lib import check

_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def seismograms(solver, nsteps: int, rec_xyz, rec_comp) -> np.ndarray:
    """nsteps forward steps from the solver's current state; samples
    [nsteps][nrec] taken after each step."""
    xyz, comp = _i32(rec_xyz).reshape(-1, 3), _i32(rec_comp).reshape(-1)
    out = np.zeros((nsteps, comp.size), np.float32)
    check(solver.lib.awp_seismograms(solver.ctx, int(nsteps), comp.size, xyz.ctypes.data_as(_I),
                                     comp.ctypes.data_as(_I), out.ctypes.data_as(_F)),
          "awp_seismograms")
    return out


def _ptr(x):
    """ctypes float pointer of a numpy array or of a CUDA tensor's storage."""
    if isinstance(x, np.ndarray):
        return x.ctypes.data_as(_F)
    return ctypes.cast(ctypes.c_void_p(x.data_ptr()), _F)


def misfit_gradient(solver, nsteps: int, rec_xyz, rec_comp, d_obs, nsnap: int = 0,
                    want_q: bool = False, out=None):
    """J = 1/2 sum (seis - d_obs)^2 over nsteps steps from the solver's current
    state, and dJ/dlambda, dJ/dmu, dJ/drho ([nz][ny][nx]); with want_q also
    dJ/dQp^-1 and dJ/dQs^-1.  Returns (J, seis, g_lambda, g_mu, g_rho[, g_qpinv,
    g_qsinv]).  `out` (optional): the gradient arrays to fill -- numpy arrays
    or contiguous float32 CUDA tensors, written in place by the library."""
    xyz, comp = _i32(rec_xyz).reshape(-1, 3), _i32(rec_comp).reshape(-1)
    d = _f32(d_obs).reshape(nsteps, comp.size)
    p = solver.params
    shape = (p.nz, p.ny, p.nx)
    seis = np.zeros((nsteps, comp.size), np.float32)
    ng = 5 if want_q else 3
    g = list(out) if out is not None else [np.zeros(shape, np.float32) for _ in range(ng)]
    if len(g) != ng:
        raise ValueError(f"out must hold {ng} arrays")
    J = c_double()
    ptrs = [_ptr(x) for x in g] + [None] * (5 - ng)
    check(solver.lib.awp_misfit_gradient_q(solver.ctx, int(nsteps), comp.size,
                                           xyz.ctypes.data_as(_I), comp.ctypes.data_as(_I),
                                           d.ctypes.data_as(_F), int(nsnap), byref(J),
                                           seis.ctypes.data_as(_F), *ptrs),
          "awp_misfit_gradient_q")
    return (J.value, seis, *g)


def misfit_gradient_shots(solver, nsteps: int, shots, nsnap: int = 0):
    """Multi-shot misfit on one model: J = sum over shots of each shot's
    1/2 sum (seis - d_obs)^2 and its gradient (the sum of the shots'
    gradients).  `shots` is a sequence of (src_pos, src_data, rec_xyz,
    rec_comp, d_obs), each run from a zero wavefield with its own sources;
    the solver keeps one workspace for all of them.  Returns (J, g_lambda,
    g_mu, g_rho) with float64 sums of the float32 per-shot gradients."""
    shots = list(shots)
    if not shots:
        raise ValueError("shots is empty")
    J = 0.0
    g = None
    for src_pos, src_data, rec_xyz, rec_comp, d_obs in shots:
        solver.upload_sources(src_pos, src_data)
        solver.reset()
        Js, _, gl, gm, gr = misfit_gradient(solver, nsteps, rec_xyz, rec_comp, d_obs, nsnap)
        J += Js
        if g is None:
            g = [x.astype(np.float64) for x in (gl, gm, gr)]
        else:
            for acc, x in zip(g, (gl, gm, gr)):
                acc += x
    return J, g[0], g[1], g[2]


def adjoint_plan(solver, nsteps: int, nsnap: int = 0) -> dict:
    """The forward-state storage ``misfit_gradient`` would use now: steps whose
    velocities are kept, the recomputed segment length, the snapshot count and
    the workspace in GB."""
    m, l, n, gb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), c_double()
    check(solver.lib.awp_adjoint_plan(solver.ctx, int(nsteps), int(nsnap), byref(m), byref(l),
                                      byref(n), byref(gb)), "awp_adjoint_plan")
    return {"tail_steps": m.value, "segment_steps": l.value, "snapshots": n.value,
            "workspace_gb": gb.value}


def adjoint_reserve(solver, nsteps: int, nsnap: int = 0) -> None:
    """Allocate the workspace ``misfit_gradient`` needs for nsteps steps now
    (it stays with the solver for later calls)."""
    check(solver.lib.awp_adjoint_reserve(solver.ctx, int(nsteps), int(nsnap)),
          "awp_adjoint_reserve")


def _autograd_function():
    import torch

    class Misfit(torch.autograd.Function):
        """J(lambda, mu, rho) of one shot: set the model, reset the wavefield,
        run forward and adjoint; backward returns the stored gradients."""

        @staticmethod
        def forward(ctx, lam, mu, rho, solver, nsteps, rec_xyz, rec_comp, d_obs, nsnap=0):
            # the library reads the model and writes the gradients through
            # device pointers when the tensors live on the GPU (no host copy);
            # host tensors go through their host memory the same way
            m = [t.detach().to(torch.float32).contiguous() for t in (lam, mu, rho)]
            if m[0].is_cuda:
                torch.cuda.current_stream(m[0].device).synchronize()
            solver.set_moduli(*m)
            solver.reset()
            g = [torch.empty_like(x) for x in m]
            J, _, gl, gm, gr = misfit_gradient(solver, nsteps, rec_xyz, rec_comp, d_obs, nsnap,
                                               out=g)
            ctx.save_for_backward(gl, gm, gr)
            return torch.tensor(J, dtype=torch.float64, device=lam.device)

        @staticmethod
        def backward(ctx, gJ):
            gl, gm, gr = ctx.saved_tensors
            s = gJ.to(gl.dtype)
            return s * gl, s * gm, s * gr, None, None, None, None, None, None

    return Misfit


_MISFIT = None


def misfit(lam, mu, rho, solver, nsteps, rec_xyz, rec_comp, d_obs, nsnap: int = 0):
    """Differentiable misfit of torch tensors lam, mu, rho ([nz][ny][nx])."""
    global _MISFIT
    if _MISFIT is None:
        _MISFIT = _autograd_function()
    return _MISFIT.apply(lam, mu, rho, solver, nsteps, rec_xyz, rec_comp, d_obs, nsnap)
