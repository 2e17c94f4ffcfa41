"""Launch-shape autotuner for the stencil kernels.

Times every candidate (kernel family: TMA-pipelined or read-only path; x
planes marched per CTA; then, for the TMA kernels, the L2 fetch granule of
their tiles) with the library's own per-phase CUDA events on a live context,
keeps the fastest per kernel and installs it process-wide through
awp_set_tuning.  The arithmetic does not depend on the launch shape or on the
caching (every cell is computed by exactly one thread with the same
expression), so tuning never changes results -- tests/test_tuning_gpu.py
checks that bit for bit.
"""
from __future__ import annotations

import itertools

CANDIDATES = {
    "tma": (1, 0),
    # longer marches re-read fewer x-halo planes per chunk and keep the CTAs
    # that share j/k halos closer in time; 512 covers a whole 512-plane grid
    "ichunk": (16, 32, 64, 128, 256, 512),
}
# L2 promotion of the TMA tiles: 3 = 256 B (the library default), 2 = 128 B,
# 1 = 64 B, 0 = none
PROMOTIONS = (3, 2, 1, 0)
KEYS = ("tma_vel", "tma_str", "ichunk", "l2_promotion")


def set_tuning(lib, key: str, value: int) -> None:
    if lib.awp_set_tuning(key.encode(), int(value)) != 0:
        raise ValueError(f"tuning {key}={value} rejected")


def get_tuning(lib) -> dict:
    return {k: lib.awp_get_tuning(k.encode()) for k in KEYS}


def autotune(solver, steps: int = 3) -> dict:
    """Time every (kernel family, ichunk) on `solver` (advancing it), then
    install the fastest family per half-step and the ichunk that minimises
    their sum; when a TMA family won a half-step, time the L2 promotion
    granules with that choice and install the fastest.  Returns the choice and
    the timing table."""
    lib = solver.lib
    table = []
    solver.profile_phases(True)
    solver.phase_times()  # drop earlier events
    for tma, ich in itertools.product(*CANDIDATES.values()):
        set_tuning(lib, "tma", tma)
        set_tuning(lib, "ichunk", ich)
        solver.step(1)  # settle
        solver.phase_times()
        solver.step(steps)
        t = solver.phase_times()
        table.append({"tma": tma, "ichunk": ich,
                      "velocity_ms": t["velocity"][0] / max(t["velocity"][1], 1),
                      "stress_ms": t["stress"][0] / max(t["stress"][1], 1)})
    solver.profile_phases(False)
    best = None
    for ich in CANDIDATES["ichunk"]:
        rows = [r for r in table if r["ichunk"] == ich]
        v = min(rows, key=lambda r: r["velocity_ms"])
        s = min(rows, key=lambda r: r["stress_ms"])
        cand = (v["velocity_ms"] + s["stress_ms"], ich, v["tma"], s["tma"])
        if best is None or cand < best:
            best = cand
    _, ich, tv, ts = best
    chosen = {"tma_vel": tv, "tma_str": ts, "ichunk": ich}
    for k, v in chosen.items():
        set_tuning(lib, k, v)
    promo = lib.awp_get_tuning(b"l2_promotion")
    if tv == 1 or ts == 1:
        # the context re-encodes its tensor maps before the next TMA launch
        solver.profile_phases(True)
        solver.phase_times()
        rows = []
        for pr in PROMOTIONS:
            set_tuning(lib, "l2_promotion", pr)
            solver.step(1)  # settle
            solver.phase_times()
            solver.step(steps)
            t = solver.phase_times()
            rows.append({"l2_promotion": pr, "tma": 1, "ichunk": ich,
                         "velocity_ms": t["velocity"][0] / max(t["velocity"][1], 1),
                         "stress_ms": t["stress"][0] / max(t["stress"][1], 1)})
        solver.profile_phases(False)
        # only the TMA half-steps depend on it
        cost = lambda r: (r["velocity_ms"] if tv == 1 else 0.0) + \
            (r["stress_ms"] if ts == 1 else 0.0)
        promo = min(rows, key=cost)["l2_promotion"]
        table.extend(rows)
    set_tuning(lib, "l2_promotion", promo)
    chosen["l2_promotion"] = promo
    return {"chosen": chosen, "table": table}


BATCH_CANDIDATES = {"ty": (8, 4), "ichunk": (8, 16, 32)}


def autotune_batch(batch, steps: int = 3, timer=None) -> dict:
    """Pick the batched execution: the persistent tile-queue mode with its
    tile shape (ty j rows x ichunk x planes, threads per CTA = 32 ty), or the
    graph of the instances' own launches, by timing `steps` batched steps per
    candidate (advancing the instances); `timer(fn)` returns the milliseconds
    fn takes.  No choice changes results (each cell is computed by the same
    expression)."""
    table = []
    batch.set_mode(0)
    for ty, ich in itertools.product(*BATCH_CANDIDATES.values()):
        batch.set_shape(ty, ich)
        batch.step(1)  # build the tile lists and the graph
        batch.synchronize()
        ms = timer(lambda: batch.step(steps))
        table.append({"mode": 0, "ty": ty, "ichunk": ich, "ms_per_step": ms / steps})
    # mode 1 captures each instance's launches with the process-wide kernel
    # families and x chunk in force at capture time: try those too, then put
    # the process-wide values back (the captured graph keeps its own)
    lib = batch.lib
    saved = get_tuning(lib)
    # the mode-1 rows below are one branch per instance (branches = 0)
    batch.set_branches(0)
    for tv, ich in itertools.product((1, 0), (16, 32, 64)):
        set_tuning(lib, "tma_vel", tv)
        set_tuning(lib, "ichunk", ich)
        batch.set_mode(0)
        batch.set_mode(1)  # recapture
        batch.step(1)
        batch.synchronize()
        ms = timer(lambda: batch.step(steps))
        table.append({"mode": 1, "ty": None, "ichunk": ich, "tma_vel": tv,
                      "ms_per_step": ms / steps})
    best = min(table, key=lambda r: r["ms_per_step"])
    if best["mode"] == 1:
        set_tuning(lib, "tma_vel", best["tma_vel"])
        set_tuning(lib, "ichunk", best["ichunk"])
        best["branches"] = 0
        for nb in (32, 16, 8):  # fewer, longer branches
            batch.set_branches(nb)
            batch.step(1)
            batch.synchronize()
            ms = timer(lambda: batch.step(steps))
            row = {"mode": 1, "ty": None, "ichunk": best["ichunk"], "tma_vel": best["tma_vel"],
                   "branches": nb, "ms_per_step": ms / steps}
            table.append(row)
            if row["ms_per_step"] < best["ms_per_step"]:
                best = row
        batch.set_branches(best["branches"])
        batch.set_mode(0)
        batch.set_mode(1)
        batch.step(1)  # capture with the chosen values
        batch.synchronize()
    else:
        batch.set_mode(0)
        batch.set_shape(best["ty"], best["ichunk"])
    for k, v in saved.items():
        set_tuning(lib, k, v)
    return {"chosen": {k: best.get(k) for k in ("mode", "ty", "ichunk", "tma_vel", "branches")},
            "table": table}
