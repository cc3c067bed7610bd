"""Autotuner of the batched form.

The batched kernel has three knobs: the image split S (lanes sharing one
atom's images, which sets the tile of atoms per work item: 256 / S), the
shared-memory stage size (how the loop tables are cut into chunks) and the
pipeline depth (stages in flight per CTA; deeper pipelines hide the copies
better but take more shared memory, hence fewer resident CTAs).  tune() times
every candidate on a reduced copy of the batch (its most expensive samples, a
contiguous slice of their atoms) with CUDA events, picks the fastest per
evaluation, and persists the choice to a JSON file keyed by GPU name,
precision and method, so later runs reuse it.
"""
import json
import os
import time

import numpy as np

from . import _capi as C
from . import backend as B

CANDIDATES = [(s, kb, d) for s in (1, 2, 4, 8) for kb in (24, 48) for d in (2, 3)]
DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "tuning.json")


def _key(precision, method):
    import torch
    return f"{torch.cuda.get_device_name(0)}|{'fp32c' if precision == C.DISCO_FP32C else 'fp64'}|{method}"


def reduced(batch, max_samples=16, atoms=16384):
    """The most expensive samples, each cut to a contiguous slice of atoms."""
    order = sorted(range(len(batch)), key=lambda i: -batch[i].n * batch[i].evals_per_atom())
    out = []
    for i in order[:max_samples]:
        w = batch[i]
        k = min(w.n, atoms)
        out.append(w.subset(np.arange(k)))
    return out


def _time(batch, precision, split, stage_kb, stages, reps=2):
    import torch
    pos = [torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda") for w in batch]
    u = [torch.zeros_like(p) for p in pos]
    ptrs = [(p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(), q[0].data_ptr(), q[1].data_ptr(),
             q[2].data_ptr()) for p, q in zip(pos, u)]
    plan = B.BatchPlan(batch, ptrs, precision=precision, image_split=split, stage_kb=stage_kb, stages=stages)
    s = torch.cuda.current_stream()
    plan.execute(s.cuda_stream)                       # builds and replays the graph once
    plan.sync(s.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        plan.execute(s.cuda_stream)
    e1.record(s)
    plan.sync(s.cuda_stream)
    plan.close()
    return e0.elapsed_time(e1) * 1e-3 / reps


def tune(batch, precision=C.DISCO_FP32C, path=None, force=False, candidates=None, log=None):
    """Returns {"image_split": S, "stage_kb": kb, "stages": d, "evals_per_s": {...}} for this GPU."""
    path = path or os.environ.get("DISCO_B200_TUNING", DEFAULT_PATH)
    method = batch[0].method if batch else "line"
    key = _key(precision, method)
    table = {}
    if os.path.exists(path):
        try:
            table = json.load(open(path))
        except (OSError, ValueError):
            table = {}
    if not force and key in table and "stages" in table[key]:
        return table[key]
    small = reduced(batch)
    evals = sum(w.n * w.evals_per_atom() for w in small)
    times = {}
    t0 = time.time()
    for split, kb, d in (candidates or CANDIDATES):
        dt = _time(small, precision, split, kb, d)
        times[f"{split}x{kb}x{d}"] = evals / dt
        if log:
            log(f"autotune S={split} stage={kb}KB depth={d}: {evals / dt:.3e} evals/s")
    best = max(times, key=times.get)
    split, kb, d = (int(v) for v in best.split("x"))
    entry = {"image_split": split, "stage_kb": kb, "stages": d, "evals_per_s": times,
             "tune_seconds": time.time() - t0,
             "reduced_batch": f"{len(small)} samples, {sum(w.n for w in small)} atoms"}
    table[key] = entry
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(table, f, indent=1)
    return entry
