"""The link-time drop-in: the reference's own pmcl3d host code links against
libawpb200 in place of the `awp` kernel library.

src/awp/CMakeLists.txt builds kernel.cu into the `awp` library and links it
with the host files of `lpmcl3d` (calc.c, cerjan.c, command.c, dump.c,
grid.c, init.c, io.c, mesh.c, source.c, swap.c, utils.c) and pmcl3d.c.  Here
those host files are compiled as they are (against the single-rank MPI
stand-in of oracle/mpi_stub, which only needs to make them compile), every
launcher of include/awp/kernel_launch.h they call is listed, and the objects
are linked against libawpb200.so: every such launcher must resolve there.
What stays unresolved belongs to the other libraries pmcl3d links (MPI, the
topography, receiver and buffer libraries), none of which kernel.cu
provides.  Needs the reference source tree (AWP_REFERENCE); CPU only."""
import os
import re
import shutil
import subprocess

import pytest

from awp_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("AWP_REFERENCE", "/root/reference")
HOST = ["pmcl3d", "calc", "cerjan", "command", "dump", "grid", "init", "io", "mesh", "source",
        "swap", "utils"]

pytestmark = pytest.mark.skipif(not os.path.isfile(os.path.join(REF, "src", "awp", "pmcl3d.c"))
                                or shutil.which("gcc") is None,
                                reason="reference source tree or gcc missing")


def launcher_names():
    """Function names declared in the reference's include/awp/kernel_launch.h."""
    text = open(os.path.join(REF, "include", "awp", "kernel_launch.h")).read()
    return set(re.findall(r"^void\s+(\w+)\s*\(", text, flags=re.M))


def symbols(objs, flag):
    out = subprocess.run(["nm", flag] + objs, check=True, capture_output=True, text=True).stdout
    names = set()
    for ln in out.splitlines():
        parts = ln.split()
        if flag == "-u" and len(parts) == 2 and parts[0] == "U":
            names.add(parts[1])
        elif flag == "--defined-only" and len(parts) == 3 and parts[1] in "TDBRC":
            names.add(parts[2])
    return names


@pytest.fixture(scope="module")
def objects(tmp_path_factory):
    d = tmp_path_factory.mktemp("pmcl3d_host")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    objs = []
    for f in HOST:
        o = str(d / f"{f}.o")
        subprocess.run(["gcc", "-c", "-w", "-std=gnu99", "-fcommon", "-D_GNU_SOURCE",
                        "-I" + os.path.join(ROOT, "oracle", "mpi_stub"),
                        "-I" + os.path.join(REF, "include"), "-I" + os.path.join(cuda, "include"),
                        "-I" + os.path.join(cuda, "include", "nvtx3"),
                        os.path.join(REF, "src", "awp", f + ".c"), "-o", o],
                       check=True, capture_output=True)
        objs.append(o)
    return d, objs


def test_every_called_launcher_is_exported(objects):
    _, objs = objects
    called = (symbols(objs, "-u") - symbols(objs, "--defined-only")) & launcher_names()
    # the launchers pmcl3d's time loop and swap.c call at least
    for name in ("SetDeviceConstValue", "dvelcx_H_opt", "dstrqc_H", "dvelc2_H", "dstrqc2_H",
                 "intp3d_H", "swap_H", "drprecpc_calc_H_opt", "velbuffer_H",
                 "update_swapzone_buffer_x_H", "update_bound_y_H"):
        assert name in called, name
    have = set(_lib.declared_symbols())
    missing = sorted(called - have)
    assert not missing, missing


def test_pmcl3d_links_against_libawpb200(objects):
    d, objs = objects
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = str(d / "pmcl3d_linked")
    r = subprocess.run(["gcc", "-o", exe] + objs +
                       ["-L" + libdir, "-lawpb200", "-lm",
                        "-Wl,--warn-unresolved-symbols", "-Wl,-rpath," + libdir],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    unresolved = set(re.findall(r"undefined reference to `(\w+)'", r.stderr))
    launchers = launcher_names()
    assert not (unresolved & launchers), sorted(unresolved & launchers)
    # what is left comes from the other libraries pmcl3d links, never kernel.cu
    assert unresolved, "expected MPI / topography symbols to stay unresolved"
