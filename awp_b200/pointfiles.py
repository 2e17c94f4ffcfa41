"""Writers for the ASCII v2 point-set files (RECVFILE / SOURCEFILE) and their
binary side files, plus a reader of the receiver output files.

Formats (reference: readers/input.h:15-50, readers/input.c:48-78,
topography/sources/source.c:434-447, topography/receivers/receiver.c:47-113):

* input file: a version line ("2.0.0"), ``key=value`` header lines, the word
  ``coordinates``, then one ``type x y z`` line per point (type 0: volume
  coordinates, z <= 0 below the surface; type 1: surface coordinates);
* SOURCEFILE rates: ``<file>_<xx|yy|zz|xy|xz|yz>``, float32, source-major,
  ``steps`` samples per source;
* receiver output: ``<file>_<x|y|z>_<step>``, float32, receiver-major,
  ``num_writes`` rings of ``gpu_buffer_size*cpu_buffer_size`` samples each;
  SGT output the same as ``<file>_<Gxx..Gyz>_<step>`` (topography/receivers/sgt.c)
  plus one sample per point in ``<file>_d1``, ``<file>_lami``, ``<file>_mui``.
"""
from __future__ import annotations

import math
import os

import numpy as np

COMPONENTS_SRC = ("xx", "yy", "zz", "xy", "xz", "yz")
COMPONENTS_RECV = ("x", "y", "z")
COMPONENTS_SGT = ("Gxx", "Gyy", "Gzz", "Gxy", "Gxz", "Gyz")


def write_input(path, file, coords, types=None, *, steps=1, stride=1, degree=3,
                gpu_buffer_size=1, cpu_buffer_size=1, num_writes=1, version="2.0.0"):
    coords = np.asarray(coords, np.float64).reshape(-1, 3)
    types = np.zeros(len(coords), np.int32) if types is None else np.asarray(types, np.int32)
    with open(path, "w") as fh:
        fh.write(f"{version}\n")
        fh.write(f"file={file}\n")
        fh.write(f"length={len(coords)}\n")
        fh.write(f"gpu_buffer_size={gpu_buffer_size}\n")
        fh.write(f"cpu_buffer_size={cpu_buffer_size}\n")
        fh.write(f"steps={steps}\n")
        fh.write(f"num_writes={num_writes}\n")
        fh.write(f"stride={stride}\n")
        fh.write(f"degree={degree}\n")
        fh.write("coordinates\n")
        for t, (x, y, z) in zip(types, coords):
            fh.write(f"{int(t)} {x:.9g} {y:.9g} {z:.9g}\n")


def write_source_rates(file, rates):
    """rates: float32 [nsrc][steps][6] in (xx, yy, zz, xy, xz, yz) order."""
    rates = np.asarray(rates, np.float32)
    for c, name in enumerate(COMPONENTS_SRC):
        np.ascontiguousarray(rates[:, :, c]).tofile(f"{file}_{name}")


def receiver_file_step(step, gpu, cpu, num_writes, stride):
    unit = gpu * cpu * num_writes * stride
    return (1 + step // unit) * unit


def receiver_file_name(base, comp, step, nt, gpu, cpu, num_writes, stride):
    zeros = int(math.ceil(math.log10(nt))) + 1
    return f"{base}_{comp}_{receiver_file_step(step, gpu, cpu, num_writes, stride):0{zeros}d}"


def read_receiver_series(base, nrecv, nt, gpu, cpu, num_writes, stride,
                         components=COMPONENTS_RECV):
    """Reassemble the recorded samples of every complete file of a run:
    returns {comp: float32 [nrecv][nsamples]} with sample s taken at step
    s*stride, s from 0 (components: COMPONENTS_RECV for a RECVFILE,
    COMPONENTS_SGT for an SGTFILE)."""
    ne = gpu * cpu
    unit = ne * num_writes * stride
    out = {}
    for comp in components:
        series = []
        fstep = unit
        while True:
            name = receiver_file_name(base, comp, fstep - 1, nt, gpu, cpu, num_writes, stride)
            if not os.path.exists(name):
                break
            a = np.fromfile(name, np.float32).reshape(nrecv, num_writes * ne)
            series.append(a)
            fstep += unit
        out[comp] = np.concatenate(series, axis=1) if series else np.zeros((nrecv, 0), np.float32)
    return out
