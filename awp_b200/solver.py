"""Python mirror of the pmcl3d time-step interface over the C ABI.

``Solver`` owns one ``awp_ctx`` (include/awp_b200.h).  Its methods map one to
one onto the context entry points, which in turn replace the set-up and time
loop of pmcl3d (src/awp/pmcl3d.c:370-2490) for a single rank.  Errors are
raised as :class:`awp_b200._lib.AwpError` carrying the library's status code.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_float, c_int, c_longlong, c_void_p

import numpy as np

from . import _lib
from ._lib import FIELD_ID, awp_params, check

NGSL = 8
ALIGN = 32


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(c_float))


def default_params(**kw) -> awp_params:
    """pmcl3d's defaults (command.c:71-136) overridden by keyword arguments."""
    lib = _lib.load()
    p = awp_params()
    lib.awp_params_default(byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


def padded_shape(nx: int, ny: int, nz: int) -> tuple[int, int, int]:
    return (nx + 4 + 2 * NGSL, ny + 4 + 2 * NGSL, nz + 2 * ALIGN)


class Solver:
    """One single-rank, single-grid simulation on the current CUDA device
    (or one block of a :class:`Mesh`, which owns it)."""

    def __init__(self, params: awp_params | None = None, stream: int | None = None, **kw):
        self.lib = _lib.load()
        self.params = params if params is not None else default_params(**kw)
        ctx = c_void_p()
        check(self.lib.awp_ctx_create(byref(self.params), byref(ctx)), "awp_ctx_create")
        self.ctx = ctx
        if stream is not None:
            check(self.lib.awp_set_stream(self.ctx, c_void_p(stream)), "awp_set_stream")
        dims = (c_longlong * 3)()
        check(self.lib.awp_padded_dims(self.ctx, dims), "awp_padded_dims")
        self.shape = tuple(int(d) for d in dims)

    @classmethod
    def _borrow(cls, lib, ctx, params, owner):
        s = cls.__new__(cls)
        s.lib = lib
        s.params = params
        s.ctx = ctx
        s._owner = owner  # the Mesh destroys the context
        dims = (c_longlong * 3)()
        check(lib.awp_padded_dims(ctx, dims), "awp_padded_dims")
        s.shape = tuple(int(d) for d in dims)
        return s

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_owner", None) is not None:
            self.ctx = None
            return
        if getattr(self, "ctx", None):
            self.lib.awp_ctx_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- inputs ------------------------------------------------------------
    def upload_media(self, media: np.ndarray) -> None:
        """media: float32 [nz][ny][nx][nvar] in the mesh-file order (surface first)."""
        media = np.ascontiguousarray(media, dtype=np.float32)
        if media.ndim != 4:
            raise ValueError("media must be [nz][ny][nx][nvar]")
        p = self.params
        if media.shape[:3] != (p.nz, p.ny, p.nx):
            raise ValueError(f"media shape {media.shape} does not match {p.nz, p.ny, p.nx}")
        check(self.lib.awp_upload_media(self.ctx, int(media.shape[3]), _fptr(media)),
              "awp_upload_media")

    def upload_media_device(self, ptr: int, nvar: int) -> None:
        check(self.lib.awp_upload_media_device(self.ctx, nvar, c_void_p(ptr)),
              "awp_upload_media_device")

    def upload_sources(self, pos: np.ndarray, data: np.ndarray) -> None:
        """pos: int32 [nsrc][3] INSRC coordinates; data: float32 [nsrc][read_step][6]."""
        pos = np.ascontiguousarray(pos, dtype=np.int32)
        data = np.ascontiguousarray(data, dtype=np.float32)
        n = int(pos.shape[0])
        check(self.lib.awp_upload_sources(self.ctx, n,
                                          pos.ctypes.data_as(ctypes.POINTER(c_int)),
                                          _fptr(data)), "awp_upload_sources")

    def upload_plane_wave(self, vx, vy, vz) -> None:
        """IFAULT=6 plane-wave input: three float series of NST samples (the
        columns of the INSRC text file, ini_plane_wave)."""
        xs = [np.ascontiguousarray(v, dtype=np.float32) for v in (vx, vy, vz)]
        n = int(xs[0].size)
        if any(x.size != n for x in xs):
            raise ValueError("the three plane-wave series differ in length")
        check(self.lib.awp_upload_plane_wave(self.ctx, n, *[c_void_p(x.ctypes.data) for x in xs]),
              "awp_upload_plane_wave")

    def set_source_filter(self, b, a) -> None:
        b = np.ascontiguousarray(b, dtype=np.float64)
        a = np.ascontiguousarray(a, dtype=np.float64)
        check(self.lib.awp_set_source_filter(
            self.ctx, len(b) - 1, b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "awp_set_source_filter")

    def download_moment(self, nsrc: int) -> np.ndarray:
        out = np.zeros(nsrc, np.float32)
        check(self.lib.awp_download_moment(self.ctx, _fptr(out)), "awp_download_moment")
        return out

    def upload_plasticity(self, sigma2, cohes, phi, fmajor, fminor, strike, dip) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (sigma2, cohes, phi)]
        st = np.ascontiguousarray(strike, dtype=np.float32)
        dp = np.ascontiguousarray(dip, dtype=np.float32)
        check(self.lib.awp_upload_plasticity(self.ctx, *[_fptr(a) for a in arrs],
                                             c_float(fmajor), c_float(fminor),
                                             _fptr(st), _fptr(dp)), "awp_upload_plasticity")

    def _model_ptrs(self, arrays):
        """float pointers of [nz][ny][nx] model arrays: numpy arrays (host) or
        contiguous float32 torch tensors (host or CUDA, passed in place)."""
        n = self.params.nx * self.params.ny * self.params.nz
        keep, ptrs = [], []
        for x in arrays:
            if isinstance(x, np.ndarray) or not hasattr(x, "data_ptr"):
                x = np.ascontiguousarray(x, np.float32)
                size = x.size
                ptrs.append(_fptr(x))
            else:
                import torch
                if x.dtype != torch.float32 or not x.is_contiguous():
                    raise ValueError("model tensors must be contiguous float32")
                size = x.numel()
                ptrs.append(ctypes.cast(ctypes.c_void_p(x.data_ptr()), ctypes.POINTER(c_float)))
            if size != n:
                raise ValueError("model arrays must have nz*ny*nx elements")
            keep.append(x)
        return keep, ptrs

    def set_moduli(self, lam, mu, rho) -> None:
        """Lame moduli and density of the interior, arrays [nz][ny][nx] (surface
        first; numpy arrays or float32 tensors, CUDA tensors by device
        pointer), into the kernel arrays; Q stays from the media upload."""
        keep, ptrs = self._model_ptrs((lam, mu, rho))
        check(self.lib.awp_set_moduli(self.ctx, *ptrs), "awp_set_moduli")
        del keep

    def set_qinv(self, qpinv, qsinv) -> None:
        """Inverse quality factors Qp^-1, Qs^-1 of the interior ([nz][ny][nx],
        surface first) into the kernel arrays; moduli and density stay."""
        keep, ptrs = self._model_ptrs((qpinv, qsinv))
        check(self.lib.awp_set_qinv(self.ctx, *ptrs), "awp_set_qinv")
        del keep

    def reset(self) -> None:
        """Wavefield and memory variables to zero, back to step 0."""
        check(self.lib.awp_reset(self.ctx), "awp_reset")

    def topography(self, intopo: str) -> None:
        """Curvilinear topography of this (top) grid from an INTOPO elevation
        file; call before receivers() and sourcefile()."""
        check(self.lib.awp_topography_init(self.ctx, intopo.encode()), "awp_topography_init")

    def set_topo_plasticity(self, consistent: bool) -> None:
        """NVE 3 on a curvilinear top grid: False (default) keeps the
        reference's single-rank behaviour (Cartesian stress on the middle band
        only), True runs the curvilinear stress everywhere before the return."""
        check(self.lib.awp_set_topo_plasticity(self.ctx, 1 if consistent else 0),
              "awp_set_topo_plasticity")

    def receivers(self, recvfile: str, nt: int) -> None:
        """RECVFILE receivers (ASCII v2); records the current step at once."""
        check(self.lib.awp_receivers_init(self.ctx, recvfile.encode(), int(nt)),
              "awp_receivers_init")

    def sgt(self, sgtfile: str, nt: int) -> None:
        """SGTFILE stress receivers and material output (ASCII v2); writes the
        material files and records the current stresses at once (with the
        step-1 source sample of IFAULT < 4 added first, as the reference has
        it before its loop: upload the sources before this call)."""
        check(self.lib.awp_sgt_init(self.ctx, sgtfile.encode(), int(nt)), "awp_sgt_init")

    def receiver_counts(self) -> tuple[int, int, int]:
        c = (c_int * 3)()
        check(self.lib.awp_receivers_count(self.ctx, c), "awp_receivers_count")
        return tuple(int(v) for v in c)

    def sourcefile(self, sourcefile: str) -> None:
        """SOURCEFILE moment-tensor sources (ASCII v2 + <file>_<xx..yz> rates)."""
        check(self.lib.awp_sourcefile_init(self.ctx, sourcefile.encode()), "awp_sourcefile_init")

    def forcefile(self, forcefile: str) -> None:
        """FORCEFILE boundary forces on the curvilinear top block (ASCII v2
        + <file>_<fx|fy|fz> rates); after topography()."""
        check(self.lib.awp_forcefile_init(self.ctx, forcefile.encode()), "awp_forcefile_init")

    def velocity_forcing(self, pos, vx, vy, vz, tskp: int, window: int) -> None:
        """IFAULT=4 prescribed velocities: pos int32 [npsrc][3] (read_src_ifault_4
        positions), frames vx, vy, vz float32 [nframes][npsrc] handed to the
        library window by window, tskp steps per frame."""
        pos = np.ascontiguousarray(pos, np.int32).reshape(-1, 3)
        frames = [np.ascontiguousarray(a, np.float32) for a in (vx, vy, vz)]
        npsrc = pos.shape[0]
        nframes = frames[0].shape[0]
        for a in frames:
            assert a.shape == (nframes, npsrc), (a.shape, nframes, npsrc)

        def read(_user, first, n, px, py, pz):
            try:
                for a, ptr in zip(frames, (px, py, pz)):
                    dst = np.ctypeslib.as_array(ptr, shape=(n * npsrc,))
                    dst[:] = a[first:first + n].reshape(-1)
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a status
                return 1

        self._frame_reader = _lib.FRAME_READER(read)  # kept alive with the context
        self._frames = (pos, frames)
        check(self.lib.awp_velocity_forcing_init(self.ctx, npsrc,
                                                 pos.ctypes.data_as(POINTER(c_int)), nframes,
                                                 int(tskp), int(window), self._frame_reader,
                                                 None), "awp_velocity_forcing_init")

    # -- time stepping -----------------------------------------------------
    def step(self, n: int = 1) -> None:
        check(self.lib.awp_step(self.ctx, int(n)), "awp_step")

    def synchronize(self) -> None:
        check(self.lib.awp_synchronize(self.ctx), "awp_synchronize")

    @property
    def current_step(self) -> int:
        s = c_longlong()
        check(self.lib.awp_current_step(self.ctx, byref(s)), "awp_current_step")
        return s.value

    # -- fields --------------------------------------------------------------
    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, np.float32)
        check(self.lib.awp_field_download(self.ctx, FIELD_ID[name], _fptr(out)),
              f"awp_field_download({name})")
        return out

    def set_field(self, name: str, arr: np.ndarray) -> None:
        arr = np.ascontiguousarray(arr, dtype=np.float32).reshape(self.shape)
        check(self.lib.awp_field_upload(self.ctx, FIELD_ID[name], _fptr(arr)),
              f"awp_field_upload({name})")

    def device_ptr(self, name: str) -> int:
        p = c_void_p()
        check(self.lib.awp_field_device_ptr(self.ctx, FIELD_ID[name], byref(p)),
              f"awp_field_device_ptr({name})")
        return int(p.value)

    def gather(self, nbgx, nedx, nskpx, nbgy, nedy, nskpy, nbgz, nedz, nskpz,
               bufx: int, bufy: int, bufz: int, bufeta: int = 0) -> None:
        """velbuffer gather into device (or pinned) buffers given as addresses."""
        check(self.lib.awp_gather_output(self.ctx, nbgx, nedx, nskpx, nbgy, nedy, nskpy,
                                         nbgz, nedz, nskpz, c_void_p(bufx), c_void_p(bufy),
                                         c_void_p(bufz), c_void_p(bufeta or None)),
              "awp_gather_output")

    def bathymetry(self) -> np.ndarray:
        """FOLLOWBATHY surface level per padded column of this grid's media,
        int32 [ny_pad][nx_pad], as pmcl3d derives it (0 where no level has
        vs > 0.001)."""
        nxp, nyp = self.shape[0], self.shape[1]
        out = np.zeros((nyp, nxp), np.int32)
        check(self.lib.awp_compute_bathymetry(self.ctx, out.ctypes.data_as(POINTER(c_int))),
              "awp_compute_bathymetry")
        return out

    def set_bathymetry(self, bathy: np.ndarray | None) -> None:
        """Make gather() follow the given surface levels ([ny_pad][nx_pad]
        int32), or plain levels again with None."""
        if bathy is None:
            check(self.lib.awp_set_bathymetry(self.ctx, None), "awp_set_bathymetry")
            return
        b = np.ascontiguousarray(bathy, np.int32).reshape(self.shape[1], self.shape[0])
        check(self.lib.awp_set_bathymetry(self.ctx, b.ctypes.data_as(POINTER(c_int))),
              "awp_set_bathymetry")

    def set_stream(self, stream: int | None) -> None:
        """Run on this cudaStream_t handle from now on (None or 0: the legacy
        default stream)."""
        check(self.lib.awp_set_stream(self.ctx, c_void_p(stream or None)), "awp_set_stream")

    # -- x-slab sub-domains -------------------------------------------------
    def set_subdomain(self, nx_global: int, x0: int) -> None:
        """This context is the part [x0, x0 + nx) of a grid nx_global wide
        (before the media)."""
        check(self.lib.awp_set_subdomain(self.ctx, int(nx_global), int(x0)), "awp_set_subdomain")

    def halo_copy(self, unpack: bool, side: int, hset: int, planes: int, buf: int) -> None:
        """awp_halo_copy on the context's stream; buf is a device or pinned
        address of nfields * planes * ny_pad * nz_pad floats."""
        check(self.lib.awp_halo_copy(self.ctx, int(bool(unpack)), int(side), int(hset),
                                     int(planes), c_void_p(buf)), "awp_halo_copy")

    def set_exchange(self, fn) -> None:
        """fn(hset) -> None runs at the two exchange points of every step
        (None removes it); an exception is reported as a failed step."""
        if fn is None:
            self._exchange = None
            check(self.lib.awp_set_exchange(self.ctx, _lib.EXCHANGE_FN(), None),
                  "awp_set_exchange")
            return

        def hook(_user, hset):
            try:
                fn(int(hset))
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a status
                import traceback
                traceback.print_exc()
                return 1

        self._exchange = _lib.EXCHANGE_FN(hook)  # kept alive with the context
        check(self.lib.awp_set_exchange(self.ctx, self._exchange, None), "awp_set_exchange")

    def check_finite(self) -> bool:
        ok = c_int()
        check(self.lib.awp_check_finite(self.ctx, byref(ok)), "awp_check_finite")
        return bool(ok.value)

    PHASES = ("velocity", "stress", "sources", "plasticity", "fstr")

    def profile_phases(self, enable: bool = True) -> None:
        check(self.lib.awp_profile_phases(self.ctx, int(enable)), "awp_profile_phases")

    def phase_times(self) -> dict:
        ms = (ctypes.c_double * 5)()
        n = (c_longlong * 5)()
        check(self.lib.awp_phase_times(self.ctx, ms, n), "awp_phase_times")
        return {p: (ms[i], n[i]) for i, p in enumerate(self.PHASES)}

    @property
    def kernel_launches(self) -> int:
        n = c_longlong()
        check(self.lib.awp_kernel_launches(self.ctx, byref(n)), "awp_kernel_launches")
        return n.value

    @property
    def device_bytes(self) -> int:
        b = c_longlong()
        check(self.lib.awp_device_bytes(self.ctx, byref(b)), "awp_device_bytes")
        return b.value


class Mesh:
    """A discontinuous mesh: blocks 0 (top, finest) .. n-1, each 3x coarser in
    x and y than the one above.  ``grid(p)`` gives block p's Solver for
    uploads and field access; ``step`` advances the whole mesh."""

    def __init__(self, params_list, stream: int | None = None):
        self.lib = _lib.load()
        n = len(params_list)
        arr = (awp_params * n)(*params_list)
        m = c_void_p()
        check(self.lib.awp_mesh_create(arr, n, byref(m)), "awp_mesh_create")
        self.mesh = m
        if stream is not None:
            check(self.lib.awp_mesh_set_stream(self.mesh, c_void_p(stream)),
                  "awp_mesh_set_stream")
        self.grids = []
        for p in range(n):
            ctx = c_void_p()
            check(self.lib.awp_mesh_grid(self.mesh, p, byref(ctx)), "awp_mesh_grid")
            self.grids.append(Solver._borrow(self.lib, ctx, params_list[p], self))

    def grid(self, p: int) -> Solver:
        return self.grids[p]

    def step(self, n: int = 1) -> None:
        check(self.lib.awp_mesh_step(self.mesh, int(n)), "awp_mesh_step")

    def synchronize(self) -> None:
        check(self.lib.awp_mesh_synchronize(self.mesh), "awp_mesh_synchronize")

    def close(self) -> None:
        if getattr(self, "mesh", None):
            for g in self.grids:
                g.ctx = None
            self.lib.awp_mesh_destroy(self.mesh)
            self.mesh = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent single-grid simulations advanced together
    (awp_batch_*): one persistent launch per half-step over the tiles of every
    instance, the step replayed as a CUDA graph.  ``solvers`` are ordinary
    Solvers set up as for ``step``; keep them alive while the batch lives."""

    def __init__(self, solvers):
        self.lib = _lib.load()
        self.solvers = list(solvers)
        n = len(self.solvers)
        arr = (c_void_p * n)(*[s.ctx for s in self.solvers])
        b = c_void_p()
        check(self.lib.awp_batch_create(arr, n, byref(b)), "awp_batch_create")
        self.batch = b

    def step(self, n: int = 1) -> None:
        check(self.lib.awp_batch_step(self.batch, int(n)), "awp_batch_step")

    def synchronize(self) -> None:
        check(self.lib.awp_batch_synchronize(self.batch), "awp_batch_synchronize")

    def set_shape(self, ty: int, ichunk: int) -> None:
        check(self.lib.awp_batch_set_shape(self.batch, int(ty), int(ichunk)),
              "awp_batch_set_shape")

    @property
    def shape(self) -> tuple[int, int]:
        ty, ich = c_int(), c_int()
        check(self.lib.awp_batch_get_shape(self.batch, byref(ty), byref(ich)),
              "awp_batch_get_shape")
        return ty.value, ich.value

    def set_graph(self, use_graph: bool) -> None:
        check(self.lib.awp_batch_set_graph(self.batch, int(bool(use_graph))),
              "awp_batch_set_graph")

    def set_mode(self, mode: int) -> None:
        """0: persistent tile-queue launches; 1: graph of each instance's own
        launches as parallel branches."""
        check(self.lib.awp_batch_set_mode(self.batch, int(mode)), "awp_batch_set_mode")

    @property
    def mode(self) -> int:
        return self.lib.awp_batch_get_mode(self.batch)

    def set_branches(self, branches: int) -> None:
        """Mode 1: parallel graph branches the instances are dealt onto
        (0: one per instance)."""
        check(self.lib.awp_batch_set_branches(self.batch, int(branches)),
              "awp_batch_set_branches")

    def info(self) -> dict:
        v = (c_longlong * 6)()
        check(self.lib.awp_batch_info(self.batch, v), "awp_batch_info")
        keys = ("instances", "cells", "velocity_tiles", "stress_tiles", "grid_velocity",
                "grid_stress")
        return dict(zip(keys, (int(x) for x in v)))

    def close(self) -> None:
        if getattr(self, "batch", None):
            self.lib.awp_batch_destroy(self.batch)
            self.batch = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
