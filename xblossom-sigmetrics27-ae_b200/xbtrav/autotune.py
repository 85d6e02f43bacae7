"""Autotuner for the traversal engine's tunables.

Searches sources-per-word (32/64), words traversed together (1/2/4), the
degree cutoff between the tile path and the per-vertex (heavy) path, and the
push/pull switch factor alpha, by timing the engine's own calls (device-side
CUDA events of xb_traverse) on a sample of the workload's sources.  The
reference has no tuner; its only knobs are compile-time buffer ratios and a
hybrid per-node/per-edge threshold (apps/xb/src/include/xbsm_gpu/xblossom_gpu_engine_hybrid.h:119).

    best, table = autotune(ctx, graph, sources)
    save(best, "tuning.json"); ctx.set_tuning(**load("tuning.json"))
"""
from __future__ import annotations

import itertools
import json

DEFAULT_SPACE = {
    "word_bits": [64, 32],
    "words": [1, 2, 4],
    "heavy_degree": [128, 256, 512, 1024],
    "pull_alpha": [4.0, 32.0, 128.0],
}


def _time_config(ctx, graph, sources, cfg: dict, reps: int) -> float:
    import torch

    ctx.set_tuning(timing=0, **cfg)
    dev = torch.device("cuda", ctx.device)
    src = torch.as_tensor(sources, dtype=torch.int32, device=dev)
    k, n = int(src.numel()), graph.n
    lv = torch.empty((k, n), dtype=torch.int32, device=dev)
    pr = torch.empty((k, n), dtype=torch.int32, device=dev)
    ctx.traverse(graph, src, out="device", level=lv, parent=pr)  # warm-up (workspace, heavy lists)
    best = float("inf")
    for _ in range(reps):
        r = ctx.traverse(graph, src, out="device", level=lv, parent=pr)
        best = min(best, r.stats["device_ms"])
    return best


def autotune(ctx, graph, sources, space: dict | None = None, reps: int = 2, staged: bool = True):
    """Returns (best tuning dict, list of (cfg, ms)).

    staged=True searches coordinate-wise (word layout first with the default
    cutoffs, then the cutoffs for the winning layout) instead of the full grid.
    """
    space = dict(DEFAULT_SPACE if space is None else space)
    base = ctx.tuning()
    table = []
    if not staged:
        keys = list(space)
        for vals in itertools.product(*(space[k] for k in keys)):
            cfg = dict(zip(keys, vals))
            table.append((cfg, _time_config(ctx, graph, sources, cfg, reps)))
    else:
        fixed = {"heavy_degree": base["heavy_degree"], "pull_alpha": base["pull_alpha"]}
        for wb, nw in itertools.product(space["word_bits"], space["words"]):
            cfg = dict(fixed, word_bits=wb, words=nw)
            table.append((cfg, _time_config(ctx, graph, sources, cfg, reps)))
        layout = min(table, key=lambda x: x[1])[0]
        for h, a in itertools.product(space["heavy_degree"], space["pull_alpha"]):
            cfg = dict(word_bits=layout["word_bits"], words=layout["words"], heavy_degree=h, pull_alpha=a)
            table.append((cfg, _time_config(ctx, graph, sources, cfg, reps)))
    best = dict(min(table, key=lambda x: x[1])[0])
    ctx.set_tuning(**best)
    return best, table


def save(cfg: dict, path: str) -> None:
    with open(path, "w") as f:
        json.dump(cfg, f, indent=1, sort_keys=True)


def load(path: str) -> dict:
    with open(path) as f:
        d = json.load(f)
    return {k: d[k] for k in ("word_bits", "words", "heavy_degree", "pull_alpha") if k in d}
