"""Autotuner of the batched step's tile shapes.

Tunable per size bin (grids binned by cell count and dimensionality):

* ``seg`` -- cells one thread marches in the y/z sweeps.  Longer segments
  recompute fewer segment-boundary faces (1/seg extra Riemann solves) but
  give fewer, longer tiles.
* ``cells_per_thread`` -- cells per thread of an edge-EMF or finish tile
  (tile = 128 x cells_per_thread cells): fewer queue operations and
  dependency checks per cell against coarser load balance.

and, for the whole batch, the number of blocks of the persistent launch.

The search is coordinate descent on the live batch: every trial times a few
graph-replayed steps of all slots (host clock around advance + wait, best of
``reps``), one parameter of one bin at a time, starting from the defaults.
Results do not depend on the tile shapes (the batch tests check this), so
tuning on the grids that will be run is safe; the steps it takes count
against the slots' budgets, so tune a copy or a sample.

The table is a plain dict (JSON-serialisable)::

    {"bins": [[ndim, lo_cells, hi_cells], ...],
     "shapes": [[seg, cells_per_thread], ...],
     "ctas_per_sm": k}
"""
from __future__ import annotations

import json
import time

from . import batch as gb

SEGS = (8, 16, 32, 64)
CPTS = (1, 2, 4, 8)
CTAS_PER_SM = (1, 2, 3)
NUM_SMS = 148

# cell-count bin edges (2-D and 3-D separately)
EDGES = (0, 1 << 13, 1 << 15, 1 << 17, 1 << 62)


def default_table() -> dict:
    bins, shapes = [], []
    for ndim in (2, 3):
        for lo, hi in zip(EDGES[:-1], EDGES[1:]):
            bins.append([ndim, lo, hi])
            shapes.append([32, 2])
    return {"bins": bins, "shapes": shapes, "ctas_per_sm": 0}


def bin_of(table: dict, ndim: int, ncells: int) -> int:
    for i, (d, lo, hi) in enumerate(table["bins"]):
        if d == ndim and lo <= ncells < hi:
            return i
    raise ValueError(f"no bin for ndim={ndim} cells={ncells}")


def shape_for(table: dict, ndim: int, ncells: int) -> gb.TileShape:
    seg, cpt = table["shapes"][bin_of(table, ndim, ncells)]
    return gb.TileShape(seg, cpt)


def apply(b: gb.Batch, table: dict, slot_info: dict) -> None:
    """Set every slot's shape from the table; slot_info: slot -> (ndim, cells)."""
    for slot, (ndim, cells) in slot_info.items():
        b.set_shape(slot, shape_for(table, ndim, cells))
    k = table.get("ctas_per_sm", 0)
    b.set_ctas(k * NUM_SMS if k else 0)


def _time(b: gb.Batch, steps: int, reps: int) -> float:
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        b.advance(steps)
        b.wait()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(b: gb.Batch, slot_info: dict, steps: int = 4, reps: int = 2,
         table: dict | None = None, log=None) -> dict:
    """Coordinate descent over (seg, cells_per_thread) per occupied bin, then
    the block count.  Returns the tuned table (a copy)."""
    table = json.loads(json.dumps(table or default_table()))
    used = sorted({bin_of(table, nd, c) for nd, c in slot_info.values()})
    apply(b, table, slot_info)
    b.advance(steps)            # capture the graph and warm up
    b.wait()
    best = _time(b, steps, reps)
    trials = [("start", None, best)]
    for bi in used:
        for which, values in ((0, SEGS), (1, CPTS)):
            cur = list(table["shapes"][bi])
            for v in values:
                if v == cur[which]:
                    continue
                cand = list(cur)
                cand[which] = v
                table["shapes"][bi] = cand
                apply(b, table, slot_info)
                t = _time(b, steps, reps)
                trials.append((f"bin{bi}", cand, t))
                if t < best:
                    best, cur = t, cand
            table["shapes"][bi] = cur
    apply(b, table, slot_info)
    cur = table.get("ctas_per_sm", 0)
    for k in CTAS_PER_SM:
        table["ctas_per_sm"] = k
        apply(b, table, slot_info)
        b.advance(steps)        # new block count: new graph
        b.wait()
        t = _time(b, steps, reps)
        trials.append(("ctas_per_sm", k, t))
        if t < best:
            best, cur = t, k
    table["ctas_per_sm"] = cur
    apply(b, table, slot_info)
    table["seconds_per_step"] = best / steps
    if log is not None:
        log.extend(trials)
    return table


def save(table: dict, path: str) -> None:
    with open(path, "w") as f:
        json.dump(table, f, indent=1)


def load(path: str) -> dict:
    with open(path) as f:
        return json.load(f)
