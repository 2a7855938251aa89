"""Canonicalisation helpers for comparing the GPU sort/grid with the oracle.

The reference assigns block header ids and orders particles inside a sort
bucket with atomics, so only these are deterministic: the set of active
blocks (by virtual id), each block's per-bucket particle sets, and the
neighbour relation expressed in virtual ids.  Deterministic mode also fixes
the order inside every bucket (ascending id).
"""
from __future__ import annotations

import numpy as np

NONE = 0xFFFFFFFF


def vid_index(headers: np.ndarray) -> dict:
    return {tuple(int(v) for v in h[:3]): i for i, h in enumerate(headers)}


def buckets(header_row: np.ndarray, sorted_ids: np.ndarray) -> list:
    """Particle ids of each of the 10 buckets of one block (cursors are
    bucket ends after the sort's finalize pass)."""
    out = []
    start = int(header_row[3])
    for k in range(10):
        end = int(header_row[6 + k])
        out.append(sorted_ids[start:end])
        start = end
    return out


def compare_sort(gpu_h, gpu_sorted, orc_h, orc_sorted, exact_order: bool) -> list:
    """Returns a list of mismatch descriptions (empty = identical)."""
    errs = []
    gi, oi = vid_index(gpu_h), vid_index(orc_h)
    if set(gi) != set(oi):
        errs.append(f"active block sets differ: gpu-only {sorted(set(gi) - set(oi))[:5]}, "
                    f"oracle-only {sorted(set(oi) - set(gi))[:5]}")
        return errs
    for vid, o in oi.items():
        g = gi[vid]
        gr, orow = gpu_h[g], orc_h[o]
        if gr[4] != orow[4] or gr[5] != orow[5]:
            errs.append(f"block {vid}: counts gpu ({gr[4]},{gr[5]}) oracle ({orow[4]},{orow[5]})")
            continue
        gb, ob = buckets(gr, gpu_sorted), buckets(orow, orc_sorted)
        for k in range(10):
            a, b = gb[k], ob[k]
            if not exact_order:
                a, b = np.sort(a), np.sort(b)
            if a.shape != b.shape or not np.array_equal(a, b):
                errs.append(f"block {vid} bucket {k}: ids differ")
        for i in range(7):
            gn, on = int(gr[16 + i]) & 0xFFFFFFFF, int(orow[16 + i]) & 0xFFFFFFFF
            gv = None if gn == NONE else tuple(int(v) for v in gpu_h[gn][:3])
            ov = None if on == NONE else tuple(int(v) for v in orc_h[on][:3])
            if gv != ov:
                errs.append(f"block {vid} neighbour {i}: gpu {gv} oracle {ov}")
        if len(errs) > 20:
            break
    return errs


def nodes_in_oracle_order(gpu_h, gpu_nodes, orc_h) -> np.ndarray:
    """GPU node array (nb, 64, 4) permuted into the oracle's block order."""
    gi = vid_index(gpu_h)
    order = [gi[tuple(int(v) for v in h[:3])] for h in orc_h]
    return gpu_nodes[np.asarray(order, dtype=np.int64)]


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


# ---------------------------------------------------------------------------
# Accuracy of a run against the oracle, measured on what the run changed.
#
# A relative L2 of positions divides by |x|, which is of order 1 in a unit
# domain, while 100 steps move the particles by 1e-4 to 1e-3 of that: a step
# that returned its inputs unchanged would score below a 1e-3 bound.  The
# errors below divide by the oracle's own change from the starting state
# instead, so an unmoved result scores exactly 1 in every field that moved.
# A field that only moves by rounding (F and C of a body in free fall) is
# measured against a noise floor instead of its change: 100 float32 ulps
# (1.2e-5) of the field's scale (the largest |x| for positions, the CFL speed
# dx/dt for v, m/dt for C = m grad v - stress term, 1 for F), so that rounding
# noise is not scored as error.

STATE_KEYS = ("pos", "vel", "aff", "def_grad")

# Fast mode (atomic scatter P2G, fused multiply-adds, fast model forms) after a
# full run: bounds on change_rel_l2 per field.  The position bound is the
# accuracy target of the path (1e-3); v, C and F get looser bounds because
# Drucker-Prager sand amplifies rounding differences through its return map.
FAST_BOUNDS = {"pos": 1e-3, "vel": 1e-2, "aff": 5e-2, "def_grad": 1e-2}
# Deterministic mode (gather P2G in the reference's order, --fmad=false).
DET_BOUNDS = {"pos": 1e-5, "vel": 1e-4, "aff": 1e-3, "def_grad": 1e-4}
# Where a run moves the particles by only a few hundred float32 ulps of their
# positions (the mixed-materials scene moves 2e-4 in 50 steps at |x| ~ 0.5),
# single precision alone limits these errors: the FP32 oracle itself is
# 4.6e-4 from the FP64 oracle there.  A field's bound is therefore the larger
# of its fixed bound and NOISE_FACTOR times the FP32 oracle's own error
# against the FP64 oracle in that field.
NOISE_FACTOR = 4.0


def change_rel_l2(got, want, start, floor: float = 0.0) -> float:
    """||got - want|| / max(||want - start||, floor * sqrt(size)): the error of
    `got` against the oracle's `want`, relative to how far the oracle moved
    from `start` (or to the noise floor, per element, when it moved less).
    Returns 0 when got == want, 1 when got == start (and the change is above
    the floor), and inf when nothing moved, no floor is given and got differs."""
    g = np.asarray(got, np.float64)
    w = np.asarray(want, np.float64)
    s = np.asarray(start, np.float64)
    num = float(np.linalg.norm(g - w))
    den = max(float(np.linalg.norm(w - s)), floor * np.sqrt(w.size))
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return num / den


def start_state(batch, dx: float | None = None, dt: float | None = None) -> dict:
    """The fields of a ParticleBatch (or a Scene) that a step changes, as a
    run's start, with the per-field noise floors of the scene's dx and dt."""
    if hasattr(batch, "particles"):
        dx, dt, batch = batch.dx, batch.dt, batch.particles
    out = {k: np.array(getattr(batch, k), np.float32, copy=True) for k in STATE_KEYS}
    if dx is not None and dt is not None:
        m = float(np.mean(batch.mass)) if batch.n else 0.0
        xmax = float(np.abs(batch.pos).max()) if batch.n else 0.0
        u = 100.0 * float(np.finfo(np.float32).eps)
        out["_floor"] = {"pos": u * xmax, "vel": u * dx / dt, "aff": u * m / dt, "def_grad": u}
    return out


def state_errors(got: dict, want: dict, start: dict) -> dict:
    fl = start.get("_floor", {})
    return {k: change_rel_l2(got[k], want[k], start[k], fl.get(k, 0.0)) for k in STATE_KEYS}


def moved_fields(want: dict, start: dict) -> list:
    """Fields whose change exceeds its noise floor (an unmoved result must fail these)."""
    fl = start.get("_floor", {})
    return [k for k in STATE_KEYS if np.linalg.norm(np.asarray(want[k], np.float64) - start[k]) >
            fl.get(k, 0.0) * np.sqrt(np.asarray(want[k]).size)]


def check_state(got: dict, want: dict, start: dict, bounds: dict):
    """Errors of `got` against `want` per field (change_rel_l2) and the list of
    fields over their bound (empty = within tolerance)."""
    err = state_errors(got, want, start)
    bad = [f"{k}: {err[k]:.3e} > {bounds[k]:.0e}" for k in STATE_KEYS if not err[k] <= bounds[k]]
    return err, bad


def format_errors(err: dict) -> str:
    return ", ".join(f"{k} {v:.3e}" for k, v in err.items())


def noise_bounds(bounds: dict, o32: dict, o64: dict, start: dict) -> dict:
    """Per field: max(bound, NOISE_FACTOR x the FP32 oracle's error against
    the FP64 oracle), the precision floor of single-precision state."""
    noise = state_errors(o32, o64, start)
    return {k: max(bounds[k], NOISE_FACTOR * noise[k]) for k in STATE_KEYS}


def assert_run_matches(label, g, o, o64, start, bounds):
    """The run's state against the FP32 oracle within `bounds` raised to the
    FP32 precision floor of the scene (noise_bounds; change_rel_l2 per field),
    the same particles disabled; FP64-oracle errors printed beside them.
    Negative control: the same check on the unmoved input must fail."""
    bounds = noise_bounds(bounds, o, o64, start)
    err, bad = check_state(g, o, start, bounds)
    err64 = state_errors(g, o64, start)
    print(f"{label}: vs f32 [{format_errors(err)}]; vs f64 [{format_errors(err64)}]; "
          f"bounds [{format_errors(bounds)}]")
    assert np.array_equal(g["enabled"], o["enabled"])
    assert not bad, f"{label}: " + "; ".join(bad)
    moved = moved_fields(o, start)
    _, bad0 = check_state({k: start[k] for k in STATE_KEYS}, o, start, bounds)
    failed = {b.split(":")[0] for b in bad0}
    assert "pos" in moved and set(moved) <= failed, \
        f"{label}: the unmoved input passes the check for {sorted(set(moved) - failed)}"
    return err
