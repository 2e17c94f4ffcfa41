"""The C-ABI library loads and exports every entry point include/awp_b200.h declares."""
import ctypes
import os
import subprocess

from awp_b200 import _lib


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], check=True,
                         capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_loads():
    lib = _lib.load()
    assert isinstance(lib, ctypes.CDLL)


def test_every_declared_symbol_is_exported():
    declared = _lib.declared_symbols()
    assert "awp_ctx_create" in declared and "dstrqc_H" in declared
    have = exported(_lib.LIB_PATH)
    missing = [s for s in declared if s not in have]
    assert not missing, missing


def test_no_stray_exports():
    # only the declared ABI leaves the library (exports.map)
    declared = set(_lib.declared_symbols())
    extra = {s for s in exported(_lib.LIB_PATH) if not s.startswith("_")} - declared
    assert not extra, sorted(extra)


def test_status_strings_and_defaults():
    lib = _lib.load()
    assert lib.awp_status_string(0) == b"ok"
    assert lib.awp_status_string(6) == b"non-finite wavefield"
    p = _lib.awp_params()
    lib.awp_params_default(ctypes.byref(p))
    # pmcl3d defaults (command.c:71-136)
    assert (p.nx, p.ny, p.nz) == (256, 256, 1024)
    assert abs(p.dh - 200.0) < 1e-6 and abs(p.dt - 0.01) < 1e-9
    assert p.nd == 20 and abs(p.arbc - 0.92) < 1e-7 and p.nve == 1 and p.socalq == 1
    assert p.nst == 91 and p.read_step == 91


def test_tuning_keys_and_ranges():
    # host-side settings only: no GPU work is queued
    lib = _lib.load()
    assert lib.awp_get_tuning(b"spin_limit") == 1 << 26
    assert lib.awp_set_tuning(b"spin_limit", -1) != 0
    assert lib.awp_set_tuning(b"spin_limit", (1 << 30) + 1) != 0
    assert lib.awp_set_tuning(b"spin_limit", 1 << 20) == 0
    assert lib.awp_get_tuning(b"spin_limit") == 1 << 20
    assert lib.awp_set_tuning(b"spin_limit", 1 << 26) == 0
    assert lib.awp_set_tuning(b"ichunk", 3) != 0
    assert lib.awp_get_tuning(b"nonsense") == -1
