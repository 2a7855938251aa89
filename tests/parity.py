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
