#!/usr/bin/env python3
"""Benchmark of the B200 AWP-ODC time step (Gcell-updates/s and % of HBM roofline).

Workload (default): the anelastic heterogeneous forward run -- 512 x 512 x 256
cells, h = 50 m, dt = 3.5 ms, 1-D vs gradient 1000..3500 m/s with a seeded
von Karman perturbation (5 %, 500 m, Hurst 0.1), Qs = 50 vs[km/s], Qp = 2 Qs,
200 seeded kinematic subfaults (IFAULT=5, Brune).  A "step" is one full time
step of that grid (velocity, stress + memory variables, sources, free-surface
images).  The 15 state fields plus 5 media fields (about 7 GB) are far larger
than the 126 MB L2, so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs an independent replica (the single-rank
path does not shard; "replicas only"), timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG = {"anelastic": 140, "elastic": 84}          # bytes per cell-update, whole step
B_STRESS = {"anelastic": 124, "elastic": 68}       # stress kernel: 19 (11) reads + 12 (6) writes
B_VEL = 52                                         # velocity kernel: 10 reads + 3 writes
L2_BYTES = 126 << 20                               # B200 L2


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def reduce_max(value: float, dist, device: str = "cuda") -> float:
    """Max over ranks of a per-rank timing (every rank takes part)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def build_workload(name: str, grid=None):
    from awp_b200 import scenarios
    kw = {}
    if grid:
        kw = dict(nx=grid[0], ny=grid[1], nz=grid[2])
    if name == "layered_vk":
        return scenarios.layered_vk(**kw), "anelastic"
    if name == "halfspace":
        return scenarios.halfspace(**kw), "elastic"
    raise SystemExit(f"unknown workload {name}")


def host_cpu() -> dict:
    """The host's processor as lscpu reports it (model, sockets, cores, threads)."""
    info = {"nproc": os.cpu_count()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for ln in out.splitlines():
            k, _, v = ln.partition(":")
            k = k.strip()
            if k in ("Model name", "Socket(s)", "Core(s) per socket", "Thread(s) per core",
                     "CPU max MHz"):
                info[k] = v.strip()
    except Exception:
        pass
    return info


def cpu_baseline(workload: str, steps: int = 10, warmup: int = 3, grid=None) -> dict:
    """FP32 OpenMP restatement of the reference kernels (oracle/) on every host
    core, on the workload's full grid: `warmup` untimed steps, then `steps`
    timed ones.  FP32 subnormals are flushed to zero on the stepping threads,
    as the reference's -use_fast_math CUDA build flushes them, so the timing
    does not depend on how far the wavefield has spread."""
    from oracle import oracle as orc
    from oracle import refbind
    scn, _ = build_workload(workload, grid)
    p = scn.params
    setup = refbind.model_setup(scn)
    ncores = os.cpu_count() or 1
    sim = orc.OracleSim(scn, setup, precision=32, nthreads=ncores, flush_denormals=True)
    del setup
    sim.step(max(1, warmup))
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    cells = p["nx"] * p["ny"] * p["nz"]
    val = cells * steps / dt / 1e9
    sim.close()
    return {"value": val, "unit": "Gcell-updates/s", "cores": ncores, "kind": "port",
            "sample": (f"the full {p['nx']}x{p['ny']}x{p['nz']} grid of the {workload} "
                       f"workload, FP32 with subnormals flushed, {steps} timed steps after "
                       f"{max(1, warmup)} warm-up, {dt:.1f} s"),
            "host": host_cpu()}


def texture_arrays(nx, ny, nz, tau1, tau2, w8):
    """init_texture (mesh.c:1103-1137) arrays from its visit-parity pattern."""
    shp = (nx + 20, ny + 20, nz + 64)
    vx1 = np.zeros(shp, np.float32)
    vx2 = np.zeros(shp, np.float32)
    wwo = np.zeros(shp, np.float32)
    ww = np.zeros(shp, np.int32)
    i = np.arange(nx)[:, None, None]
    j = np.arange(ny)[None, :, None]
    k = np.arange(nz)[None, None, :]
    ij = i * ny + j
    itx = (i + 1) & 1
    ity = (ij + 1) & 1
    itz = (nz * (ij + 1) + k) & 1
    t = (4 * itx + 2 * ity + itz).astype(np.int64)
    sl = (slice(10, nx + 10), slice(10, ny + 10), slice(32, nz + 32))
    vx1[sl] = np.asarray(tau1, np.float32)[t]
    vx2[sl] = np.asarray(tau2, np.float32)[t]
    wwo[sl] = (8.0 * np.asarray(w8, np.float64)).astype(np.float32)[t]
    ww[sl] = (t + 1).astype(np.int32)
    return vx1, vx2, ww, wwo


def reference_gpu(scn, solver, steps=20, warmup=3, topo_path=None, variant="as_shipped") -> dict:
    """The reference's own CUDA build on the same workload, inputs taken from
    the product's set-up: `variant` "as_shipped" (oracle/_ref/libawpref.so,
    2 x 2 x 4-thread blocks of include/awp/pmcl3d_cons.h) or "block_64x8"
    (oracle/_ref/libawpref_b64x8.so: the same source with only the launch block
    raised to 64 z x 8 y threads, as dstrqc_H_new picks it); with a topography
    file, its curvilinear kernels (oracle/_ref/libawpref_topo.so) in place of
    dvelcx / dstrqc."""
    import torch
    from oracle import refbind
    p = scn.params
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    host = refbind.RefHost()
    import ctypes
    from ctypes import byref, c_float
    taumax, taumin = c_float(), c_float()
    tau8 = np.zeros(8, np.float32)
    w8 = np.zeros(8, np.float32)
    coeff = np.zeros(16, np.float32)
    F = ctypes.POINTER(c_float)
    solver.lib.awp_q_tau(0.0, 0.005, byref(taumax), byref(taumin), tau8.ctypes.data_as(F))
    solver.lib.awp_q_weights(0.0, 0.005, w8.ctypes.data_as(F), coeff.ctypes.data_as(F))
    tau1, tau2 = refbind.tau12(tau8, p["dt"])
    vx1, vx2, ww, wwo = texture_arrays(nx, ny, nz, tau1, tau2, w8)
    dx, dy, dz = host.inicrj(p["arbc"], nx, ny, nz, p["nd"], 1, p["npc"])
    media = {k: solver.field(k) for k in ("d1", "mu", "lam", "qp", "qs")}
    psrc, comps, rs = refbind.map_sources(scn)
    setup = dict(media=media, vx1=vx1, vx2=vx2, ww=ww, wwo=wwo, dcrjx=dx, dcrjy=dy, dcrjz=dz,
                 lam_mu=refbind.lam_mu_ref(media["lam"], media["mu"], nx, ny, nz),
                 coeff=coeff, psrc=psrc, src=comps, src_stride=rs)
    del media
    with torch.cuda.stream(torch.cuda.default_stream()):
        # the reference launchers run on the legacy default stream
        lib = None
        if variant == "block_64x8":
            if nz % 64 or ny % 8:
                raise ValueError("the 64x8-block build needs nzt % 64 == 0 and nyt % 8 == 0")
            lib = os.path.join(refbind.REF_DIR, "libawpref_b64x8.so")
        if topo_path:
            sim = refbind.RefTopoSim(scn, setup, topo_path, path=lib)
        else:
            sim = refbind.RefGpuSim(scn, setup, path=lib)
        del setup, vx1, vx2, ww, wwo
        sim.step(warmup)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s0.record()
        sim.step(steps)
        s1.record()
        torch.cuda.synchronize()
        ms = s0.elapsed_time(s1) / steps
    out = {"value": nx * ny * nz / (ms * 1e-3) / 1e9, "unit": "Gcell-updates/s",
           "ms_per_step": ms, "steps": steps,
           "build": "reference src/awp/kernel.cu, nvcc sm_100a -O3 -use_fast_math, " +
                    ("BLOCK_SIZE 2x2x4 as shipped" if variant == "as_shipped" else
                     "BLOCK_SIZE_Z/Y raised to 64/8 (DEFINITIONS_H), nothing else changed") +
                    f"; launched in the pmcl3d single-rank order; {steps} steps timed after "
                    f"{warmup} warm-up"}
    if topo_path:
        out["build"] += ("; curvilinear top grid: the reference's topo_velocity_interior_H "
                         "and topo_stress_{interior,left,right}_H (opt_topography kernels)")
    if hasattr(sim, "close"):
        sim.close()
    del sim
    torch.cuda.empty_cache()
    return out


def _lib_handle():
    from awp_b200 import _lib
    return _lib.load()


def load_traffic(kernel: str, workload: str):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return d.get(workload, {}).get(kernel)
    except Exception:
        return None


def run_ours(args, rank, world, dist) -> dict | None:
    import torch
    from awp_b200 import Solver, default_params

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    scn, kind = build_workload(args.workload, args.grid)
    p = scn.params
    cells = p["nx"] * p["ny"] * p["nz"]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    hbm, peak_kind = peaks()

    # ---- device-resident timing -------------------------------------------------
    topo_path = None
    if args.topography:
        # a Gaussian hill with rough relief over the workload's surface (the
        # curvilinear top-grid operators replace the Cartesian ones)
        import tempfile
        from awp_b200 import scenarios as _sc
        topo_path = os.path.join(tempfile.mkdtemp(prefix="awp_topo_"), "topography.bin")
        depth = p["dh"] * (p["nz"] - 2)
        _sc.write_topography(topo_path, p["nx"], p["ny"], p["dh"], amplitude=0.1 * depth,
                             width=0.2 * p["nx"] * p["dh"], rough_rms=0.005 * depth, seed=3)
    if args.l2_promotion is not None:
        from awp_b200 import tune as _t
        _t.set_tuning(_lib_handle(), "l2_promotion", args.l2_promotion)
    s = Solver(default_params(**p), stream=stream.cuda_stream)
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    if topo_path:
        s.topography(topo_path)
    tuning = None
    if topo_path:
        pass  # the tuning keys select Cartesian kernel families only
    elif args.tma is not None:
        from awp_b200 import tune
        tune.set_tuning(s.lib, "tma", args.tma)
    elif not args.no_tune:
        from awp_b200 import tune
        tuning = tune.autotune(s)
    s.step(args.warmup)
    s.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    s.profile_phases(True)
    launches0 = s.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dev_bytes = s.device_bytes
    if dev_bytes < 8 * L2_BYTES:
        # a working set within a few L2 sizes (the 128^3 half-space): write a
        # buffer twice the L2 before each step and time the steps one by one
        flush_buf = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda")
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        for k, (ea, eb) in enumerate(ev):
            flush_buf.fill_(k & 0xFF)
            ea.record(stream)
            s.step(1)
            eb.record(stream)
        torch.cuda.synchronize()
        ms_flushed = sum(ea.elapsed_time(eb) for ea, eb in ev)
        l2_note = (f"working set {dev_bytes / 1e9:.2f} GB: L2 flushed (a {2 * L2_BYTES >> 20} MB "
                   "write) before each timed step, steps timed one by one")
        del flush_buf
    else:
        e0.record(stream)
        s.step(args.steps)
        e1.record(stream)
        ms_flushed = None
        l2_note = f"working set {dev_bytes / 1e9:.1f} GB >> 126 MB L2, no flush needed"
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    launches = s.kernel_launches - launches0
    ms = ms_flushed if ms_flushed is not None else e0.elapsed_time(e1)
    phases = s.phase_times()
    s.profile_phases(False)
    ok = s.check_finite()
    t_max = reduce_max(ms, dist)
    ms_step = t_max / args.steps
    value = world * cells * args.steps / (t_max * 1e-3) / 1e9

    st_ms, st_n = phases["stress"]
    ve_ms, ve_n = phases["velocity"]
    stress_ms = st_ms / max(st_n, 1)
    vel_ms = ve_ms / max(ve_n, 1)
    b_st = B_STRESS[kind] * cells
    achieved = b_st / (stress_ms * 1e-3) / 1e9
    if topo_path:
        tkey = "topo_stress"
    else:
        # the stress kernel family the run used (autotuned, forced or default)
        from awp_b200 import tune as _tune
        tkey = "stress_tma" if _tune.get_tuning(s.lib)["tma_str"] == 1 else "stress"
    traffic = load_traffic(tkey, args.workload)
    kname = {"topo_stress": "k_topo_stress (curvilinear stress + memory variables)",
             "stress_tma": "k_stress_tma (TMA-pipelined stress + memory variables)",
             "stress": "k_stress (stress + memory variables)"}[tkey]
    roofline = {"bound": "hbm", "kernel": kname,
                "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_kind": f"{peak_kind} hbm_gbs", "traffic": traffic,
                "alg_bytes_per_launch": b_st, "alg_bytes_per_cell": B_STRESS[kind],
                "avg_launch_ms": stress_ms}
    step_bw = B_ALG[kind] * cells / (ms_step * 1e-3) / 1e9
    kernels = {name: {"ms_per_launch": v[0] / max(v[1], 1), "launches": v[1]}
               for name, v in phases.items()}
    kernels["velocity"]["achieved_GBs"] = B_VEL * cells / (vel_ms * 1e-3) / 1e9
    kernels["stress"]["achieved_GBs"] = achieved
    s.close()
    del s
    torch.cuda.empty_cache()

    # ---- end to end through the C ABI with host buffers ----------------------------
    e2e = None
    e2e_steps = args.e2e_steps or (scn.steps if args.grid is None else args.steps)
    if not args.no_e2e:
        media = torch.from_numpy(scn.media).pin_memory()
        nvar = scn.media.shape[3]
        h2d = media.numel() * 4 + scn.src_pos.nbytes + scn.src_data.nbytes
        rec = (p["nx"] * p["ny"])
        out = [torch.empty(rec, dtype=torch.float32).pin_memory() for _ in range(3)]
        dev = [torch.empty(rec, dtype=torch.float32, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        # host clock of each set-up call (the device is idle meanwhile, so the
        # events see their sum)
        h0 = time.perf_counter()
        se = Solver(default_params(**p), stream=stream.cuda_stream)
        h1 = time.perf_counter()
        se.lib.awp_upload_media(se.ctx, nvar, media.numpy().ctypes.data_as(
            __import__("ctypes").POINTER(__import__("ctypes").c_float)))
        h2 = time.perf_counter()
        se.upload_sources(scn.src_pos, scn.src_data)
        if topo_path:
            se.topography(topo_path)
        h3 = time.perf_counter()
        setup_host = {"context_create_ms": (h1 - h0) * 1e3, "media_upload_ms": (h2 - h1) * 1e3,
                      "sources_ms": (h3 - h2) * 1e3}
        t_setup = torch.cuda.Event(enable_timing=True)
        t_setup.record(stream)
        se.step(e2e_steps)
        t_steps = torch.cuda.Event(enable_timing=True)
        t_steps.record(stream)
        # free-surface snapshot (velbuffer, NBGZ=NEDZ=1) back to the host
        se.gather(0, p["nx"] - 1, 1, 0, p["ny"] - 1, 1, 0, 0, 1,
                  dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr())
        for o, d in zip(out, dev):
            o.copy_(d, non_blocking=True)
        t1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = reduce_max(t0.elapsed_time(t1), dist)
        setup_ms = t0.elapsed_time(t_setup)
        steps_ms = t_setup.elapsed_time(t_steps)
        d2h = 3 * rec * 4
        e2e = {"value": world * cells * e2e_steps / (e2e_ms * 1e-3) / 1e9,
               "unit": "Gcell-updates/s", "h2d_bytes_per_step": h2d / e2e_steps,
               "d2h_bytes_per_step": d2h / e2e_steps, "ms_total": e2e_ms,
               "steps": e2e_steps,
               # where the time goes (rank 0's events): set-up (context, media H2D
               # and mapping, sources) and the steps, against the timed region's
               # step time (a long run may sit under the power cap)
               "setup_ms": setup_ms, "setup_host_ms": setup_host,
               "ms_per_step": steps_ms / max(e2e_steps, 1),
               "includes": "the whole run through the C ABI: context create, media H2D + "
                           "on-device inimesh mapping, sources, every time step of the run, "
                           "surface snapshot D2H"}
        se.close()
        del se, media

    if rank != 0:
        return None
    line = {
        "metric": "Gcell-updates/s (whole time step) & %HBM roofline on 1 B200",
        "value": value, "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": scn.name, "description": scn.description,
                   "grid": [p["nx"], p["ny"], p["nz"]], "cells": cells,
                   "dh": p["dh"], "dt": p["dt"], "ifault": p["ifault"], "nve": p["nve"],
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": l2_note,
                   "topography": ("Gaussian hill + rough relief (curvilinear top grid)"
                                  if topo_path else None),
                   "finite_after_run": ok},
        "roofline": roofline,
        "step_roofline": {"bytes_per_cell_alg": B_ALG[kind], "achieved": step_bw,
                          "peak": hbm, "unit": "GB/s", "frac": step_bw / hbm},
        "kernels": kernels,
        "clocks": clocks,
        "gpu_launches": launches,
        "tuning": tuning["chosen"] if tuning else None,
        "tuning_table": tuning["table"] if tuning else None,
    }
    if e2e:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload, steps=10, warmup=3, grid=args.grid)
    if world == 1 and not args.no_ref_gpu:
        rg = {}
        for variant in ("as_shipped", "block_64x8"):
            try:
                s2 = Solver(default_params(**p))
                s2.upload_media(scn.media)
                rg[variant] = reference_gpu(scn, s2, topo_path=topo_path, variant=variant)
                s2.close()
            except Exception as exc:  # reported, never substituted
                rg[variant] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        line["reference_gpu_build"] = rg
    return line


def reference_config(args) -> dict:
    """The workload keys of the GPU arm's `config` (the same model and size),
    from the scenario's parameters without generating its medium."""
    from awp_b200 import scenarios
    g = args.grid or (None, None, None)
    p, desc = scenarios.workload_meta(args.workload, *g)
    return {"workload": args.workload, "description": desc,
            "grid": [p["nx"], p["ny"], p["nz"]], "cells": p["nx"] * p["ny"] * p["nz"],
            "dh": p["dh"], "dt": p["dt"], "ifault": p["ifault"], "nve": p["nve"],
            "parallelism": "the single-GPU workload's full grid, timed on the host cores",
            "l2": "working set ~7 GB >> 126 MB L2, no flush needed", "topography": None}


def run_reference(args, rank) -> dict | None:
    """Reference arm: the reference path's CPU restatement on the host cores,
    W warm-up and K timed steps on the workload's full grid."""
    if rank != 0:
        return None
    cb = cpu_baseline(args.workload, steps=args.steps, warmup=args.warmup, grid=args.grid)
    return {"metric": "Gcell-updates/s (whole time step) & %HBM roofline on 1 B200",
            "value": cb["value"], "unit": "Gcell-updates/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "impl": "reference", "dtype": "f32", "data": "synthetic (seeded)",
            "config": reference_config(args),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference ships only CUDA for this path; its arm is the OpenMP "
                    "restatement of the same kernels (oracle/awp_oracle.cpp) on the host cores"}


def run_batched(args) -> dict:
    """Batched ensemble: the same instances advanced (a) by the plain path,
    one context per simulation, each on its own stream (so independent
    simulations may overlap on the GPU), and (b) by awp_batch_step (persistent
    tile-queue launches, one CUDA graph per step).  Both timed on the device
    with CUDA events; value = batched Gcell-updates/s."""
    import torch
    from awp_b200 import Batch, Solver, default_params, scenarios, tune

    ens = scenarios.batch_ensemble(n=args.batch_n, seed=6, steps=args.steps + args.warmup + 64)
    cells = sum(sc.params["nx"] * sc.params["ny"] * sc.params["nz"] for sc in ens)
    root = torch.cuda.Stream()
    streams = [torch.cuda.Stream() for _ in ens]
    solvers = []
    for sc, st in zip(ens, streams):
        s = Solver(default_params(**sc.params), stream=st.cuda_stream)
        s.upload_media(sc.media)
        s.upload_sources(sc.src_pos, sc.src_data)
        solvers.append(s)
    torch.cuda.synchronize()

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(root)
        for st in streams:
            st.wait_event(e0)
        fn()
        for st in streams:
            root.wait_stream(st)
        e1.record(root)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def plain(k):
        for s in solvers:
            s.step(k)

    def plain_seq(k):  # one simulation after another
        for q, s in enumerate(solvers):
            if q:
                streams[q].wait_stream(streams[q - 1])
            s.step(k)

    timed(lambda: plain(args.warmup))
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    ms_plain = timed(lambda: plain(args.steps))
    ms_seq = timed(lambda: plain_seq(args.steps))
    launches_plain = sum(s.kernel_launches for s in solvers)

    b = Batch(solvers)
    tuning = tune.autotune_batch(b, steps=3, timer=timed)
    b.step(args.warmup)
    b.synchronize()
    l0 = sum(s.kernel_launches for s in solvers)
    ms_batch = timed(lambda: b.step(args.steps))
    launches_batch = sum(s.kernel_launches for s in solvers) - l0
    clocks = sampler.stop()
    info = b.info()
    ok = all(s.check_finite() for s in solvers)
    b.close()
    for s in solvers:
        s.close()
    hbm, peak_kind = peaks()
    v_b = cells * args.steps / (ms_batch * 1e-3) / 1e9
    v_p = cells * args.steps / (ms_plain * 1e-3) / 1e9
    v_s = cells * args.steps / (ms_seq * 1e-3) / 1e9
    step_bw = 140 * cells / (ms_batch / args.steps * 1e-3) / 1e9
    sizes = [[sc.params["nx"], sc.params["ny"], sc.params["nz"]] for sc in ens]
    return {
        "metric": "batched vs plain Gcell-updates/s (ensemble of uneven grids) on 1 B200",
        "value": v_b, "unit": "Gcell-updates/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_batch / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"batched ensemble of {len(ens)} anelastic grids",
                   "sizes_drawn": "nx, ny in [64, 256], nz in [64, 128] (seed 6)",
                   "cells": cells, "instances": len(ens), "first_sizes": sizes[:8],
                   "l2": "working set of tens of GB >> 126 MB L2, no flush needed",
                   "finite_after_run": ok},
        "plain": {"value": v_s, "ms_per_step": ms_seq / args.steps,
                  "kernel_launches_per_step": launches_plain / max(2 * args.steps + args.warmup, 1),
                  "mode": "one context per simulation, the simulations one after another"},
        "plain_concurrent": {"value": v_p, "ms_per_step": ms_plain / args.steps,
                             "mode": "one context per simulation, each on its own stream, "
                                     "all enqueued together (the GPU overlaps them)"},
        "batched_over_plain": v_b / v_s,
        "batched_over_plain_concurrent": v_b / v_p,
        "batch": {"tuning": tuning["chosen"], "tuning_table": tuning["table"], **info,
                  "graph": True},
        "step_roofline": {"bytes_per_cell_alg": 140, "achieved": step_bw, "peak": hbm,
                          "unit": "GB/s", "frac": step_bw / hbm,
                          "peak_kind": f"{peak_kind} hbm_gbs"},
        "clocks": clocks,
        "gpu_launches": launches_batch,
    }


def run_adjoint(args) -> dict:
    """Misfit gradient (discrete adjoint; stored velocities for the last steps,
    sqrt snapshots and recomputation for the rest): its cost against the
    forward run of the same steps, and central finite differences of the
    misfit along seeded directions (eps = 1e-3 relative)."""
    import torch
    from awp_b200 import Solver, adjoint, default_params, scenarios

    nx, ny, nz = args.grid if args.grid else (256, 256, 128)
    steps = args.adj_steps or 1500
    scn, m_true, m0, xyz, comp = scenarios.adjoint_case(nx=nx, ny=ny, nz=nz, steps=steps)
    stream = torch.cuda.Stream()
    s = Solver(default_params(**scn.params), stream=stream.cuda_stream)
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.set_moduli(*m_true)
    s.reset()
    d_obs = adjoint.seismograms(s, steps, xyz, comp)

    def timed(fn):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    s.set_moduli(*m0)
    s.reset()
    adjoint.seismograms(s, min(steps, 20), xyz, comp)  # warm-up
    # the workspace (snapshots, velocity store) is allocated once per solver
    # and kept for later gradients; its allocation is timed on its own
    ms_alloc, _ = timed(lambda: adjoint.adjoint_reserve(s, steps))
    # one untimed gradient: the first pass over a freshly allocated workspace
    # of ~170 GB runs up to ~50 % slower than the following ones
    s.reset()
    adjoint.misfit_gradient(s, steps, xyz, comp, d_obs)
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    # --adj-reps (default five) forward runs and gradients, alternating; the
    # medians are reported with every run listed (single runs vary with the
    # power-capped clocks, a gradient by up to ~20 % on some boxes)
    fwd_runs, adj_runs = [], []
    for _ in range(args.adj_reps):
        s.reset()
        fwd_runs.append(timed(lambda: adjoint.seismograms(s, steps, xyz, comp))[0])
        s.reset()
        ms, (J, seis, gl, gm, gr) = timed(
            lambda: adjoint.misfit_gradient(s, steps, xyz, comp, d_obs))
        adj_runs.append(ms)
    ms_fwd = float(np.median(fwd_runs))
    ms_adj = float(np.median(adj_runs))
    clocks = sampler.stop()
    plan = adjoint.adjoint_plan(s, steps)  # the storage the timed call used
    # the plain sqrt(N) plan (nsnap = ~sqrt(steps) snapshots, every segment run
    # forward again): the configuration's "~39 checkpoints in HBM"
    nsnap_sqrt = int(round(np.sqrt(steps)))
    plan_sqrt = adjoint.adjoint_plan(s, steps, nsnap_sqrt)
    adjoint.adjoint_reserve(s, steps, nsnap_sqrt)
    s.reset()
    ms_sqrt, _ = timed(lambda: adjoint.misfit_gradient(s, steps, xyz, comp, d_obs, nsnap_sqrt))
    # finite differences along seeded relative directions
    rng = np.random.default_rng(8)
    eps = 1e-3
    fd_rows = []

    def J_of(mp):
        s.set_moduli(*mp)
        s.reset()
        sp = adjoint.seismograms(s, steps, xyz, comp).astype(np.float64)
        return 0.5 * float(np.sum((sp - d_obs) ** 2))
    for d in range(args.fd_dirs):
        dm = [(x * rng.standard_normal(x.shape)).astype(np.float64) for x in m0]
        adj_dir = float(sum(np.sum(g.astype(np.float64) * x) for g, x in zip((gl, gm, gr), dm)))
        row = {"adjoint": adj_dir}
        # eps = 1e-3 as the configuration states; 1e-2 beside it, where the
        # FP32 rounding of the two forward runs weighs ten times less against
        # the difference of the misfits
        for e_, key in ((eps, ""), (10 * eps, "_eps1e-2")):
            fd = (J_of([(x + e_ * y).astype(np.float32) for x, y in zip(m0, dm)]) -
                  J_of([(x - e_ * y).astype(np.float32) for x, y in zip(m0, dm)])) / (2 * e_)
            row["fd" + key] = fd
            row["rel_err" + key] = abs(adj_dir - fd) / max(abs(fd), 1e-300)
        fd_rows.append(row)
    cells = nx * ny * nz
    s.close()
    return {
        "metric": "adjoint gradient cost / forward cost on 1 B200",
        "value": ms_adj / ms_fwd, "unit": "x forward", "n_gpus": 1, "steps": steps,
        "warmup": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": scn.description, "grid": [nx, ny, nz], "cells": cells,
                   "receivers": int(len(comp)), "storage": plan,
                   "l2": "state of GBs >> 126 MB L2, no flush needed"},
        "forward_ms": ms_fwd, "adjoint_ms": ms_adj, "workspace_alloc_ms": ms_alloc,
        "forward_runs_ms": fwd_runs, "adjoint_runs_ms": adj_runs,
        "sqrt_plan": {"nsnap": nsnap_sqrt, "storage": plan_sqrt, "adjoint_ms": ms_sqrt,
                      "x_forward": ms_sqrt / ms_fwd},
        "forward_gcell_updates_s": cells * steps / (ms_fwd * 1e-3) / 1e9,
        "misfit": J,
        "fd_check": {"eps_rel": eps, "directions": fd_rows,
                     "max_rel_err": max(r["rel_err"] for r in fd_rows) if fd_rows else None,
                     "max_rel_err_eps1e-2": (max(r["rel_err_eps1e-2"] for r in fd_rows)
                                             if fd_rows else None),
                     # errors against the typical size of a directional derivative
                     # (one seeded direction can be nearly orthogonal to the gradient)
                     "max_err_over_rms_fd": (max(abs(r["adjoint"] - r["fd"]) for r in fd_rows) /
                                             max(float(np.sqrt(np.mean([r["fd"] ** 2 for r in fd_rows]))),
                                                 1e-300)) if fd_rows else None},
        "clocks": clocks,
    }


def run_shots(args, rank, world, dist) -> dict | None:
    """Multi-shot misfit gradient on one shared model: `--shots` shots (default
    32) on the 384 x 384 x 192 anelastic layered + von Karman model (h = 100 m),
    `--adj-steps` steps each (the configuration's 1000), 64 shared surface
    receivers, each shot a moment-tensor point source (Mxy Ricker') at a seeded
    position; gradients summed over the shots (float64).  Under torchrun the
    shots are dealt across the ranks and one all-reduce sums the misfit and
    the lambda / mu / rho gradients (awp_b200.replicas).  The observed traces
    are zero (the cost does not depend on their values).  Timed with CUDA
    events from the first shot to the summed gradient, max over ranks; value =
    shots x steps x cells / time, beside the same shots' forward runs."""
    import torch
    from awp_b200 import Solver, adjoint, default_params, replicas, scenarios

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    nx, ny, nz = args.grid if args.grid else (384, 384, 192)
    steps = args.adj_steps or 1000
    scn = scenarios.layered_vk(nx=nx, ny=ny, nz=nz, h=100.0, dt=0.005, steps=steps, nsub=1,
                               seed_medium=7, seed_src=8)
    rng = np.random.default_rng(9)
    nst = steps + 1
    stf = scenarios.ricker_derivative(nst, 0.005, 2.0) * 1e15
    shots = []
    rec = np.stack([rng.integers(nx // 8, nx - nx // 8, 64), rng.integers(ny // 8, ny - ny // 8, 64),
                    np.zeros(64, np.int64)], 1).astype(np.int32)
    comp = rng.integers(0, 3, 64).astype(np.int32)
    d_obs = np.zeros((steps, 64), np.float32)
    for k in range(args.shots):
        pos = np.array([[rng.integers(nx // 4, 3 * nx // 4), rng.integers(ny // 4, 3 * ny // 4),
                         rng.integers(nz // 8, nz // 2)]], np.int32)
        data = np.zeros((1, nst, 6), np.float32)
        data[0, :, 5] = stf
        shots.append((pos, data, rec, comp, d_obs))
    stream = torch.cuda.Stream()
    s = Solver(default_params(**dict(scn.params, ifault=1, nst=nst, read_step=nst)),
               stream=stream.cuda_stream)
    s.upload_media(scn.media)
    mine = replicas.deal(len(shots), rank, world)
    adjoint.adjoint_reserve(s, steps)
    # one untimed shot: the first pass over a fresh workspace runs slower
    s.upload_sources(*shots[mine[0]][:2] if mine else shots[0][:2])
    s.reset()
    adjoint.misfit_gradient(s, steps, rec, comp, d_obs)

    def timed(fn):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return reduce_max(e0.elapsed_time(e1), dist), out

    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    ms, (J, g) = timed(lambda: replicas.misfit_gradient_shots(s, steps, shots, dist=dist))

    def forwards():
        for i in mine:
            s.upload_sources(*shots[i][:2])
            s.reset()
            s.step(steps)
        s.synchronize()
    ms_fwd, _ = timed(forwards)
    clocks = sampler.stop()
    plan = adjoint.adjoint_plan(s, steps)
    s.close()
    if rank != 0:
        return None
    cells = nx * ny * nz
    return {
        "metric": "multi-shot misfit gradient (shared model, summed) on B200",
        "value": len(shots) * steps * cells / (ms * 1e-3) / 1e9, "unit": "Gcell-updates/s",
        "n_gpus": world, "steps": steps, "warmup": 1, "ms_total": ms,
        "ms_per_shot": ms * world / len(shots), "higher_is_better": True,
        "scaling": "weak" if world == 1 else "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded); observed traces zero",
        "config": {"workload": "shots", "grid": [nx, ny, nz], "shots": len(shots),
                   "steps_per_shot": steps, "receivers": 64,
                   "parallelism": f"shots dealt over {world} rank(s), one all-reduce",
                   "storage": plan},
        "x_forward": ms / ms_fwd, "forward_ms_total": ms_fwd, "misfit": J,
        "gradient_rms": [float(np.sqrt(np.mean(x * x))) for x in g],
        "clocks": clocks,
    }


def run_decomp(args, rank, world, dist) -> dict | None:
    """x-slab domain decomposition of the 512 x 512 x 256 anelastic layered +
    von Karman run (strong scaling: the grid is fixed).  One process: `--parts`
    parts on the GPU in lockstep (awp_decomp_*), beside the whole grid on the
    same GPU, so the line gives the cost of the halo copies.  Under torchrun:
    one part per rank, halos over NCCL (awp_b200.decomp.SlabRank); the time is
    the max over ranks."""
    import torch
    from awp_b200 import Solver, default_params, scenarios
    from awp_b200.decomp import (LocalDecomposition, SlabRank, part_media, part_sources,
                                 split_x)

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    nx, ny, nz = args.grid if args.grid else (512, 512, 256)
    scn = scenarios.layered_vk(nx=nx, ny=ny, nz=nz, steps=args.warmup + args.steps + 2)
    p = scn.params
    cells = nx * ny * nz
    stream = torch.cuda.current_stream()

    def timed(step, count):
        """(max over ranks of the device time of the timed steps, kernels
        this rank launched in them)."""
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        n0 = count()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        return reduce_max(t0.elapsed_time(t1), dist), count() - n0

    nparts = world if world > 1 else args.parts
    layout = split_x(nx, nparts)
    line = {"metric": "Gcell-updates/s (strong scaling of an x-slab decomposition)",
            "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "layered_vk_decomp", "grid": [nx, ny, nz], "parts": layout,
                       "halo_planes": 4,
                       "l2": "working set ~7 GB >> 126 MB L2, no flush needed"}}
    if world == 1:
        whole = Solver(default_params(**p), stream=stream.cuda_stream)
        whole.upload_media(scn.media)
        whole.upload_sources(scn.src_pos, scn.src_data)
        ms_whole, _ = timed(lambda: whole.step(1), lambda: whole.kernel_launches)
        whole.close()
        del whole
        torch.cuda.empty_cache()
        d = LocalDecomposition(default_params(**p), parts=layout)
        d.set_stream(stream.cuda_stream)
        d.upload_media(scn.media)
        d.upload_sources(scn.src_pos, scn.src_data)
        ms, launches = timed(lambda: d.step(1),
                             lambda: sum(s.kernel_launches for s in d.parts))
        d.close()
        line["whole_grid_ms_per_step"] = ms_whole / args.steps
        line["halo_cost_frac"] = ms / ms_whole - 1.0
    else:
        x0, w = layout[rank]
        s = Solver(default_params(**dict(p, nx=w)))
        s.set_subdomain(nx, x0)
        s.upload_media(part_media(scn.media, x0, w))
        ps, ds = part_sources(scn.src_pos, scn.src_data, x0, w, rank == 0, rank == world - 1)
        if len(ps):
            s.upload_sources(ps, ds)
        slab = SlabRank(s, rank, world, group=None)
        slab.exchange_media()
        ms, launches = timed(lambda: s.step(1), lambda: s.kernel_launches)
        s.close()
    line["value"] = cells * args.steps / (ms * 1e-3) / 1e9
    line["ms_per_step"] = ms / args.steps
    line["gpu_launches"] = launches
    return line if rank == 0 else None


def run_config3(args) -> dict:
    """Topography + discontinuous mesh + plasticity + attenuation: a 639 x 639
    x 320 block at h = 40 m (640 is not a multiple of 3) over a 213 x 213 x 96
    block at h = 120 m, a Gaussian hill of 1 km (5 km width) with 100 m rms
    seeded roughness on the fine block, Drucker-Prager plasticity with 1 MPa
    cohesion, 30 degree friction and lithostatic initial stress on both blocks,
    attenuation on, a moment-tensor point source at 8 km depth.  W warm-up and
    K timed steps (the configuration's run is 3000) with CUDA events on the
    mesh's stream; value = cells of both blocks x steps / time.  Timed with the
    consistent topography + plasticity path (curvilinear stress everywhere,
    then the return); the reference's single-rank behaviour (only the middle
    band of the fine block's stress updated) is timed after it for context."""
    import tempfile

    import torch
    from awp_b200 import Mesh, default_params, scenarios

    torch.cuda.set_device(0)
    hbm, peak_kind = peaks()
    kw = {}
    if args.grid:  # profiling cases: coarse nx, ny and the fine block's nz
        kw = dict(nxc=args.grid[0], nyc=args.grid[1], nz_fine=args.grid[2],
                  nz_coarse=max(12, args.grid[2] // 3 // 4 * 4),
                  src_depth_m=40.0 * args.grid[2] * 0.6)
    blocks = scenarios.config3_blocks(steps=args.steps + args.warmup + 4, **kw)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    m = Mesh([default_params(**b.params) for b in blocks], stream=stream.cuda_stream)
    for p, b in enumerate(blocks):
        g = m.grid(p)
        g.upload_media(b.media)
        if b.src_pos.shape[0]:
            g.upload_sources(b.src_pos, b.src_data)
        q = b.params
        s2 = scenarios.lithostatic_sigma2(g.field("d1"), q["nx"], q["ny"], q["nz"], q["dh"])
        g.upload_plasticity(s2, np.full_like(s2, 1e6), np.full_like(s2, 30.0), 1.0, 1.0,
                            (0.0, 0.0, 0.0), (0.0, 90.0, 0.0))
        del s2
    p0 = blocks[0].params
    topo = os.path.join(tempfile.mkdtemp(prefix="awp_cfg3_"), "topography.bin")
    scenarios.write_topography(topo, p0["nx"], p0["ny"], p0["dh"], amplitude=1000.0,
                               width=5000.0, rough_rms=100.0, seed=4)
    m.grid(0).topography(topo)
    cells = sum(b.params["nx"] * b.params["ny"] * b.params["nz"] for b in blocks)
    block_params = [b.params for b in blocks]
    del blocks

    def timed(nsteps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.step(nsteps)
        e1.record(stream)
        torch.cuda.synchronize()
        m.synchronize()
        return e0.elapsed_time(e1)

    m.grid(0).set_topo_plasticity(True)
    m.step(args.warmup)
    m.synchronize()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    for g in m.grids:
        g.profile_phases(True)
    launches0 = sum(g.kernel_launches for g in m.grids)
    ms = timed(args.steps)
    clocks = sampler.stop()
    launches = sum(g.kernel_launches for g in m.grids) - launches0
    phases = [g.phase_times() for g in m.grids]
    for g in m.grids:
        g.profile_phases(False)
    ok = all(g.check_finite() for g in m.grids)
    m.grid(0).set_topo_plasticity(False)
    ms_ref_mode = timed(args.steps)
    m.close()
    ms_step = ms / args.steps
    value = cells * args.steps / (ms * 1e-3) / 1e9
    step_bw = 160 * cells / (ms_step * 1e-3) / 1e9
    return {
        "metric": "Gcell-updates/s (topography + DM + plasticity + attenuation step) on 1 B200",
        "value": value, "unit": "Gcell-updates/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": "config3",
                   "blocks": [f"{q['nx']}x{q['ny']}x{q['nz']} h={q['dh']:g}" +
                              (" (curvilinear)" if n == 0 else "")
                              for n, q in enumerate(block_params)],
                   "cells": cells, "dt": p0["dt"], "nve": 3,
                   "topography": "Gaussian hill 1 km / 5 km width + 100 m rms roughness (seed 4)",
                   "plasticity": "cohesion 1 MPa, friction 30 deg, lithostatic sigma2",
                   "topo_plasticity": "consistent (curvilinear stress everywhere, then return)",
                   "steps_note": f"{args.steps} timed steps of the configuration's 3000",
                   "finite_after_run": ok},
        "step_roofline": {"bytes_per_cell_alg": 160, "achieved": step_bw, "peak": hbm,
                          "unit": "GB/s", "frac": step_bw / hbm,
                          "peak_kind": f"{peak_kind} hbm_gbs"},
        "kernels": [{name: {"ms_per_launch": v[0] / max(v[1], 1), "launches": v[1]}
                     for name, v in ph.items()} for ph in phases],
        "reference_behaviour_ms_per_step": ms_ref_mode / args.steps,
        "clocks": clocks, "gpu_launches": launches,
    }


def run_extras(args) -> dict:
    """The other two parts of the metric, as sub-objects of the headline line:
    batched vs plain on the 96-instance ensemble, and the adjoint gradient's
    cost against the forward run (with its finite-difference check)."""
    out = {}
    sub = argparse.Namespace(**{**vars(args), "steps": 20, "warmup": 3, "batch_n": 96,
                                "adj_steps": 1500, "fd_dirs": 8, "grid": None})
    try:
        b = run_batched(sub)
        out["batched"] = {k: b[k] for k in ("metric", "value", "unit", "ms_per_step", "plain",
                                             "plain_concurrent", "batched_over_plain",
                                             "batched_over_plain_concurrent", "gpu_launches")}
        out["batched"]["config"] = {k: b["config"][k] for k in ("workload", "cells", "instances",
                                                              "sizes_drawn")}
        out["batched"]["tuning"] = b["batch"]["tuning"]
    except Exception as exc:  # reported, never substituted
        out["batched"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    try:
        a = run_adjoint(sub)
        out["adjoint"] = {k: a[k] for k in ("metric", "value", "unit", "forward_ms",
                                             "adjoint_ms", "workspace_alloc_ms",
                                             "forward_runs_ms", "adjoint_runs_ms", "misfit",
                                             "sqrt_plan")}
        out["adjoint"]["config"] = a["config"]
        out["adjoint"]["fd_check"] = a["fd_check"]
    except Exception as exc:
        out["adjoint"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="layered_vk",
                    choices=["layered_vk", "halfspace", "batched", "adjoint", "config3",
                             "shots", "decomp"])
    ap.add_argument("--parts", type=int, default=2,
                    help="x slabs of --workload decomp on one GPU")
    ap.add_argument("--shots", type=int, default=32,
                    help="shots of the multi-shot gradient (--workload shots)")
    ap.add_argument("--adj-steps", type=int, default=None,
                    help="time steps of a misfit-gradient run: config 4's 1500 for "
                         "--workload adjoint, config 5b's 1000 per shot for --workload shots")
    ap.add_argument("--adj-reps", type=int, default=5,
                    help="timed forward runs and gradients, alternating (--workload adjoint)")
    ap.add_argument("--fd-dirs", type=int, default=8,
                    help="finite-difference directions (--workload adjoint)")
    ap.add_argument("--batch-n", type=int, default=96,
                    help="instances of the batched ensemble (--workload batched)")
    ap.add_argument("--topography", action="store_true",
                    help="curvilinear top grid (INTOPO) on the same workload")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and adjoint sub-measurements of the default line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--l2-promotion", type=int, choices=[0, 1, 2, 3], default=None,
                    help="L2 fetch granule of the TMA tiles (profiling cases)")
    ap.add_argument("--tma", type=int, choices=[0, 1], default=None,
                    help="force the kernel family (profiling cases; implies --no-tune)")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="steps of the end-to-end run (default: the workload's full run)")
    ap.add_argument("--grid", type=lambda v: tuple(int(x) for x in v.split(",")), default=None,
                    help="nx,ny,nz override of the workload grid (profiling cases)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        line = run_reference(args, rank)
    elif args.workload == "batched":
        line = run_batched(args) if rank == 0 else None
    elif args.workload == "adjoint":
        line = run_adjoint(args) if rank == 0 else None
    elif args.workload == "config3":
        line = run_config3(args) if rank == 0 else None
    elif args.workload == "decomp":
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist_mod
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
            dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
            dist = dist_mod
        line = run_decomp(args, rank, world, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    elif args.workload == "shots":
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist_mod
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
            dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
            dist = dist_mod
        line = run_shots(args, rank, world, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    else:
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist_mod
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
            dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
            dist = dist_mod
        line = run_ours(args, rank, world, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    if (line is not None and args.impl == "ours" and world == 1 and
            args.workload == "layered_vk" and not args.no_extras and args.grid is None and
            not args.topography):
        line.update(run_extras(args))
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
