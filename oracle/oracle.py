"""Python wrapper of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

``OracleSim`` runs the CPU restatement of the reference time step
(oracle/awp_oracle.cpp) on inputs assembled by ``refbind.model_setup``, i.e. by
the reference's own host set-up code.  precision=64 is the FP64 oracle;
precision=32 with OpenMP threads is the CPU baseline bench.py times.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_longlong, c_void_p

import numpy as np

from . import refbind

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_F = POINTER(c_float)
_I = POINTER(c_int)

FIELD = {n: i for i, n in enumerate(
    ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5", "r6",
     "d1", "mu", "lam", "qp", "qs", "sigma2", "cohes", "phi", "yldfac", "neta", "vx1", "vx2",
     "wwo"])}

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        lib = ctypes.CDLL(LIB, mode=ctypes.RTLD_LOCAL)
        lib.oracle_create.restype = c_void_p
        lib.oracle_create.argtypes = [c_int, c_int, c_int, c_int, c_float, c_float, c_int, c_int]
        lib.oracle_destroy.argtypes = [c_void_p]
        lib.oracle_set_field.argtypes = [c_void_p, c_int, _F]
        lib.oracle_get_field.argtypes = [c_void_p, c_int, _F]
        lib.oracle_get_field_f64.argtypes = [c_void_p, c_int, POINTER(c_double)]
        lib.oracle_set_ww.argtypes = [c_void_p, _I]
        lib.oracle_set_sponge.argtypes = [c_void_p, _F, _F, _F]
        lib.oracle_set_coeff.argtypes = [c_void_p, _F]
        lib.oracle_compute_lam_mu.argtypes = [c_void_p]
        lib.oracle_set_sources.argtypes = [c_void_p, c_int, c_int, _I, c_int, c_int] + [_F] * 6
        lib.oracle_set_filter.argtypes = [c_void_p, c_int, POINTER(c_double), POINTER(c_double)]
        lib.oracle_get_moment.argtypes = [c_void_p, _F]
        lib.oracle_set_plasticity.argtypes = [c_void_p, c_float, c_float, _F, _F]
        lib.oracle_set_plane_wave.argtypes = [c_void_p, c_int, c_int, _F, _F, _F]
        lib.oracle_step.argtypes = [c_void_p, c_int, c_int]
        lib.oracle_set_flush_denormals.argtypes = [c_void_p, c_int]
        lib.oracle_add_point_sources.argtypes = ([c_void_p, c_int, c_int, c_int] + [_I] * 3 +
                                                 [_F] * 3 + [c_int, _F, c_int])
        lib.oracle_current_step.restype = c_longlong
        lib.oracle_current_step.argtypes = [c_void_p]
        lib.oracle_gather.argtypes = [c_void_p] + [c_int] * 9 + [_F] * 3
        lib.oracle_set_tangent.argtypes = [c_void_p, c_int, POINTER(c_double)]
        lib.oracle_get_tangent.argtypes = [c_void_p, c_int, POINTER(c_double)]
        _lib = lib
    return _lib


def fp(a):
    return a.ctypes.data_as(_F)


class OracleSim:
    def __init__(self, scn, setup=None, precision=64, nthreads=0, flush_denormals=False):
        lib = load()
        self.lib = lib
        self.scn = scn
        p = scn.params
        self.p = p
        self.shape = refbind.padded_shape(p["nx"], p["ny"], p["nz"])
        setup = setup if setup is not None else refbind.model_setup(scn)
        self.setup = setup
        self.o = lib.oracle_create(precision, p["nx"], p["ny"], p["nz"], p["dh"], p["dt"],
                                   p.get("npc", 0), nthreads)
        # the CPU baseline flushes FP32 subnormals like the reference's
        # -use_fast_math CUDA build
        lib.oracle_set_flush_denormals(self.o, 1 if flush_denormals else 0)
        m = setup["media"]
        for k in ("d1", "mu", "lam", "qp", "qs"):
            lib.oracle_set_field(self.o, FIELD[k], fp(np.ascontiguousarray(m[k], np.float32)))
        for k in ("vx1", "vx2", "wwo"):
            lib.oracle_set_field(self.o, FIELD[k], fp(np.ascontiguousarray(setup[k], np.float32)))
        lib.oracle_set_ww(self.o, np.ascontiguousarray(setup["ww"], np.int32).ctypes.data_as(_I))
        lib.oracle_set_sponge(self.o, fp(setup["dcrjx"]), fp(setup["dcrjy"]), fp(setup["dcrjz"]))
        lib.oracle_set_coeff(self.o, fp(np.ascontiguousarray(setup["coeff"], np.float32)))
        lib.oracle_compute_lam_mu(self.o)
        psrc = np.ascontiguousarray(setup["psrc"], np.int32)
        comps = [np.ascontiguousarray(c, np.float32) for c in setup["src"]]
        lib.oracle_set_sources(self.o, p["ifault"], int(psrc.shape[0]), psrc.ctypes.data_as(_I),
                               setup["src_stride"], p["nst"], *[fp(c) for c in comps])
        self._keep = (psrc, comps)

    def set_field(self, name, arr):
        self.lib.oracle_set_field(self.o, FIELD[name],
                                  fp(np.ascontiguousarray(arr, np.float32).reshape(self.shape)))

    def set_tangent(self, name, arr):
        """Tangent part of a field (precision 65, dual numbers)."""
        a = np.ascontiguousarray(arr, np.float64).reshape(self.shape)
        self.lib.oracle_set_tangent(self.o, FIELD[name], a.ctypes.data_as(POINTER(c_double)))

    def tangent(self, name):
        out = np.empty(self.shape, np.float64)
        self.lib.oracle_get_tangent(self.o, FIELD[name], out.ctypes.data_as(POINTER(c_double)))
        return out

    def compute_lam_mu(self):
        self.lib.oracle_compute_lam_mu(self.o)

    def set_plane_wave(self, vx, vy, vz):
        """IFAULT 6 plane-wave series (ini_plane_wave), entering on level
        align + ND + 1 of this grid."""
        xs = [np.ascontiguousarray(v, np.float32) for v in (vx, vy, vz)]
        self._plane = xs
        self.lib.oracle_set_plane_wave(self.o, int(xs[0].size), int(self.p["nd"]),
                                       *[x.ctypes.data_as(_F) for x in xs])

    def set_plasticity(self, fmajor, fminor, Rz, RzT):
        self.lib.oracle_set_plasticity(self.o, fmajor, fminor,
                                       fp(np.ascontiguousarray(Rz, np.float32)),
                                       fp(np.ascontiguousarray(RzT, np.float32)))

    def set_filter(self, b, a):
        b = np.ascontiguousarray(b, np.float64)
        a = np.ascontiguousarray(a, np.float64)
        self.lib.oracle_set_filter(self.o, len(b) - 1, b.ctypes.data_as(POINTER(c_double)),
                                   a.ctypes.data_as(POINTER(c_double)))

    def add_point_sources(self, field, coefs, values, stride):
        """coefs: ix/iy/iz [nq], lx/ly/lz [nq][nb]; values [nsamples][nq]."""
        I = lambda a: np.ascontiguousarray(a, np.int32).ctypes.data_as(_I)  # noqa: E731
        keep = [np.ascontiguousarray(coefs[k], np.int32) for k in ("ix", "iy", "iz")]
        keepf = [np.ascontiguousarray(coefs[k], np.float32) for k in ("lx", "ly", "lz")]
        vals = np.ascontiguousarray(values, np.float32)
        nq, nb = keepf[0].shape
        self.lib.oracle_add_point_sources(self.o, FIELD[field], nq, nb,
                                          *[a.ctypes.data_as(_I) for a in keep],
                                          *[fp(a) for a in keepf], vals.shape[0], fp(vals),
                                          stride)
        del I

    def step(self, n=1):
        self.lib.oracle_step(self.o, self.p.get("nve", 1), n)

    @property
    def current_step(self):
        return self.lib.oracle_current_step(self.o)

    def field(self, name, f64=False):
        if f64:
            out = np.empty(self.shape, np.float64)
            self.lib.oracle_get_field_f64(self.o, FIELD[name], out.ctypes.data_as(POINTER(c_double)))
            return out
        out = np.empty(self.shape, np.float32)
        self.lib.oracle_get_field(self.o, FIELD[name], fp(out))
        return out

    def moment(self, nsrc):
        out = np.zeros(nsrc, np.float32)
        self.lib.oracle_get_moment(self.o, fp(out))
        return out

    def gather(self, nbgx, nedx, nskpx, nbgy, nedy, nskpy, nbgz, nedz, nskpz):
        n = (((nedx - nbgx) // nskpx + 1) * ((nedy - nbgy) // nskpy + 1) *
             ((nedz - nbgz) // nskpz + 1))
        bx, by, bz = (np.zeros(n, np.float32) for _ in range(3))
        self.lib.oracle_gather(self.o, nbgx, nedx, nskpx, nbgy, nedy, nskpy, nbgz, nedz, nskpz,
                               fp(bx), fp(by), fp(bz))
        return bx, by, bz

    def close(self):
        if self.o:
            self.lib.oracle_destroy(self.o)
            self.o = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
