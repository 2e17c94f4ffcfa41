"""x-slab domain decomposition of a single-grid run.

The reference decomposes pmcl3d over MPI ranks in x and y and exchanges
velocity and stress halos between the kernels of every step
(pmcl3d.c:1657-1721, 1838-1924; swap.c).  Here a grid is cut along x, the
slowest axis of the padded layout, so each halo is a run of whole x planes:
one contiguous copy per field and side.  A part is a context made with
:meth:`Solver.set_subdomain`; the halos of a step are the stresses and
velocities at its start, the velocities after the velocity update and, with
plasticity, the yield factors between the two plasticity kernels, plus the
media once (include/awp_b200.h).

* :func:`split_x` -- widths and even offsets of the parts.
* :class:`LocalDecomposition` -- several parts on one device stepped in
  lockstep by the library (awp_decomp_*), halos copied in device memory.
* :class:`SlabRank` -- one part per process; the exchange hook moves the
  halos through torch.distributed (NCCL between GPUs, gloo on host buffers).
"""
from __future__ import annotations

from ctypes import byref, c_void_p

import numpy as np

from . import _lib
from ._lib import HALO_MEDIA, HALO_PLANES, HALO_STRESS, HALO_VELOCITY, HALO_YLDFAC, check

NGSL = 8

__all__ = ["split_x", "part_media", "part_sources", "halo_fields", "LocalDecomposition",
           "SlabRank"]


def split_x(nx: int, nparts: int) -> list[tuple[int, int]]:
    """(x0, width) of each part: near-equal widths, every offset even (the
    attenuation parity pattern of a part is then the grid's), every width at
    least the halo."""
    if nparts < 1:
        raise ValueError("nparts >= 1")
    w = max(2, 2 * round(nx / (2 * nparts)))
    out, x0 = [], 0
    for p in range(nparts):
        width = nx - x0 if p == nparts - 1 else w
        if width < HALO_PLANES:
            raise ValueError(f"{nparts} parts of a grid {nx} wide leave a part of {width}")
        out.append((x0, width))
        x0 += width
    return out


def part_media(media: np.ndarray, x0: int, nx: int) -> np.ndarray:
    """The part's columns of a media volume [nz][ny][nx][nvar]."""
    return np.ascontiguousarray(np.asarray(media)[:, :, x0:x0 + nx])


def part_sources(pos, data, x0: int, nx: int, first: bool, last: bool):
    """The point sources of one part in its own coordinates: x (1-based, as
    INSRC) in (x0, x0 + nx], the ghost columns beyond the grid's edges going
    to the outer parts."""
    pos = np.asarray(pos, np.int32).reshape(-1, 3)
    data = np.asarray(data, np.float32)
    x = pos[:, 0]
    sel = np.ones(len(pos), bool)
    if not first:
        sel &= x > x0
    if not last:
        sel &= x <= x0 + nx
    p = pos[sel].copy()
    p[:, 0] -= x0
    return p, data[sel]


def halo_fields(hset: int) -> int:
    """Fields in a halo set."""
    return 3 * bool(hset & HALO_VELOCITY) + 6 * bool(hset & HALO_STRESS) + \
        5 * bool(hset & HALO_MEDIA) + bool(hset & HALO_YLDFAC)


class LocalDecomposition:
    """A grid cut into x slabs on the current device, stepped in lockstep."""

    def __init__(self, params, nparts: int | None = None, parts=None):
        from .solver import Solver, default_params
        self.lib = _lib.load()
        nxg = params.nx
        self.layout = parts if parts is not None else split_x(nxg, nparts or 2)
        self.nx_global = nxg
        fields = {f: getattr(params, f) for f, _ in params._fields_}
        self.parts = []
        for x0, w in self.layout:
            s = Solver(default_params(**dict(fields, nx=w)))
            s.set_subdomain(nxg, x0)
            self.parts.append(s)
        arr = (c_void_p * len(self.parts))(*[s.ctx for s in self.parts])
        d = c_void_p()
        check(self.lib.awp_decomp_create(arr, len(self.parts), byref(d)), "awp_decomp_create")
        self.d = d
        s0 = self.parts[0]
        self.shape = (nxg + 4 + 2 * NGSL, s0.shape[1], s0.shape[2])

    def upload_media(self, media) -> None:
        for s, (x0, w) in zip(self.parts, self.layout):
            s.upload_media(part_media(media, x0, w))

    def upload_sources(self, pos, data) -> None:
        n = len(self.parts)
        for q, (s, (x0, w)) in enumerate(zip(self.parts, self.layout)):
            p, d = part_sources(pos, data, x0, w, q == 0, q == n - 1)
            if len(p):
                s.upload_sources(p, d)

    def topography(self, intopo: str) -> None:
        """The whole grid's topography file; each part keeps its planes of the
        metrics."""
        for s in self.parts:
            s.topography(intopo)

    def upload_plasticity(self, sigma2, cohes, phi, fmajor, fminor, strike, dip) -> None:
        """NVE 3 inputs of the whole padded grid; each part takes its planes."""
        for s, (x0, w) in zip(self.parts, self.layout):
            sl = slice(x0, x0 + w + 4 + 2 * NGSL)
            s.upload_plasticity(*(np.ascontiguousarray(np.asarray(a)[sl])
                                  for a in (sigma2, cohes, phi)), fmajor, fminor, strike, dip)

    def set_stream(self, stream: int | None) -> None:
        """Run the parts and the halo copies on this cudaStream_t handle."""
        check(self.lib.awp_decomp_set_stream(self.d, c_void_p(stream or None)),
              "awp_decomp_set_stream")

    def step(self, n: int = 1) -> None:
        check(self.lib.awp_decomp_step(self.d, int(n)), "awp_decomp_step")

    def synchronize(self) -> None:
        check(self.lib.awp_decomp_synchronize(self.d), "awp_decomp_synchronize")

    def field(self, name: str) -> np.ndarray:
        """The whole padded field: each part's interior planes, the outer
        ghost planes from the outer parts."""
        out = np.zeros(self.shape, np.float32)
        lo = 2 + NGSL
        for q, (s, (x0, w)) in enumerate(zip(self.parts, self.layout)):
            f = s.field(name)
            out[x0 + lo:x0 + lo + w] = f[lo:lo + w]
            if q == 0:
                out[:lo] = f[:lo]
            if q == len(self.parts) - 1:
                out[x0 + lo + w:] = f[lo + w:]
        return out

    def close(self) -> None:
        if getattr(self, "d", None):
            self.lib.awp_decomp_destroy(self.d)
            self.d = None
        for s in getattr(self, "parts", []):
            s.close()
        self.parts = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class SlabRank:
    """One x slab per process.  The solver's exchange hook packs the planes
    next to each neighbour into a send buffer, trades them with
    torch.distributed point-to-point operations and unpacks the received
    planes into the ghost planes.  On a GPU the solver runs on torch's
    current stream, so the packing, the NCCL transfers and the unpacking keep
    stream order; `device="cpu"` stages through host buffers (gloo)."""

    def __init__(self, solver, rank: int, world: int, device="cuda",
                 planes: int = HALO_PLANES, group=None, comm=None):
        """`comm`: an object with torch.distributed's isend / irecv (the
        module itself by default)."""
        import torch
        if comm is None:
            import torch.distributed as comm
        self.dist = comm
        self.group = group
        self.s = solver
        self.rank, self.world = rank, world
        self.left = rank - 1 if rank > 0 else None
        self.right = rank + 1 if rank < world - 1 else None
        self.planes = planes
        self.per_field = planes * solver.shape[1] * solver.shape[2]
        n = 9 * self.per_field  # the largest set: velocities and stresses
        kw = {"dtype": torch.float32, "device": device}
        if str(device) == "cpu":
            kw["pin_memory"] = torch.cuda.is_available()
        self.send = [torch.empty(n, **kw), torch.empty(n, **kw)]
        self.recv = [torch.empty(n, **kw), torch.empty(n, **kw)]
        self.exchanges = 0
        if str(device) != "cpu" and hasattr(solver, "set_stream"):
            solver.set_stream(torch.cuda.current_stream().cuda_stream)
        solver.set_exchange(self.exchange)

    def _sides(self):
        return [(side, nbr) for side, nbr in ((0, self.left), (1, self.right)) if nbr is not None]

    def exchange(self, hset: int) -> None:
        """Trade the halo of `hset` with both neighbours (every rank calls
        this at the same points of the step)."""
        n = halo_fields(hset) * self.per_field
        if n > self.send[0].numel():
            raise ValueError(f"halo set {hset} exceeds the exchange buffers")
        sides = self._sides()
        for side, _ in sides:
            self.s.halo_copy(False, side, hset, self.planes, self.send[side].data_ptr())
        if self.send[0].device.type == "cpu":
            self.s.synchronize()  # host staging: the packed planes must have landed
        reqs = []
        for side, nbr in sides:
            reqs.append(self.dist.isend(self.send[side][:n], nbr, group=self.group, tag=side))
            reqs.append(self.dist.irecv(self.recv[side][:n], nbr, group=self.group,
                                        tag=1 - side))
        for r in reqs:
            r.wait()
        for side, _ in sides:
            self.s.halo_copy(True, side, hset, self.planes, self.recv[side].data_ptr())
        self.exchanges += 1

    def exchange_media(self) -> None:
        """The media halos, once after the media upload."""
        self.exchange(HALO_MEDIA)
