"""Autotuner for the traversal engine's tunables.

Searches sources-per-word (32/64), words traversed together (1/2/4), the
degree cutoff between the per-lane light pull and the per-warp heavy pull,
the push/pull switch factor alpha, the tail push threshold push_beta (push
after a pull once the frontier holds fewer than n/push_beta vertices; 0 =
off), the launch tile of the pull and table
kernels (xb_tuning.tile: rounds in flight per heavy-pull warp, warps per
table block), the grouping of sources into passes (xb_tuning.source_order:
by out-degree or as given) and, for the batched path, the number of concurrent chains, by
timing the engine's own calls (device-side CUDA events of xb_traverse or
xb_traverse_batched, median of `reps` runs) on the workload's sources.  The
reference has no tuner; its only knobs are compile-time buffer ratios and a
hybrid per-node/per-edge threshold (apps/xb/src/include/xbsm_gpu/xblossom_gpu_engine_hybrid.h:119).

    best, table = autotune(ctx, graph, sources, path="batched")
    save(best, "tuning.json"); ctx.set_tuning(**load("tuning.json"))
"""
from __future__ import annotations

import itertools
import json

DEFAULT_SPACE = {
    "word_bits": [64, 32],
    "words": [1, 2, 4],
    "heavy_degree": [128, 256, 512],
    "pull_alpha": [16.0, 64.0, 256.0, 1024.0],
    "push_beta": [0.0, 24.0],
    "tile": [0, 1],
    "source_order": [0, 1],
    "chains": [1, 2, 4, 8],
}
KEYS = ("word_bits", "words", "heavy_degree", "pull_alpha", "push_beta", "tile", "source_order", "chains")


def _time_config(ctx, graph, sources, cfg: dict, reps: int, path: str) -> float:
    import torch

    ctx.set_tuning(timing=0, **cfg)
    dev = torch.device("cuda", ctx.device)
    src = torch.as_tensor(sources, dtype=torch.int32, device=dev)
    k, n = int(src.numel()), graph.n
    lv = torch.empty((k, n), dtype=torch.int32, device=dev)
    pr = torch.empty((k, n), dtype=torch.int32, device=dev)

    def once():
        if path == "batched":
            return ctx.traverse_batched([(graph, src)], outputs=[(lv, pr)])[1]["device_ms"]
        return ctx.traverse(graph, src, out="device", level=lv, parent=pr).stats["device_ms"]

    once()  # warm-up (workspaces, heavy lists, the captured launch)
    times = sorted(once() for _ in range(max(1, reps)))
    return times[len(times) // 2]  # median: one slow or fast outlier does not pick the winner


def autotune(ctx, graph, sources, space: dict | None = None, reps: int = 5, staged: bool = True,
             path: str = "plain"):
    """Returns (best tuning dict, list of (cfg, ms)); path "plain" times
    xb_traverse, "batched" xb_traverse_batched (which also uses chains).

    staged=True searches coordinate-wise (word layout first with the current
    cutoffs, then cutoffs and alpha for the winning layout, then the launch
    tail push threshold, then the launch tile, then the source grouping,
    then chains) instead of the full grid.
    """
    space = dict(DEFAULT_SPACE if space is None else space)
    if path != "batched":
        space["chains"] = [ctx.tuning()["chains"]]
    base = {k: v for k, v in ctx.tuning().items() if k in KEYS}
    table = []

    def run(cfg):
        table.append((dict(cfg), _time_config(ctx, graph, sources, cfg, reps, path)))

    if not staged:
        keys = [k for k in KEYS if k in space]
        for vals in itertools.product(*(space[k] for k in keys)):
            run(dict(base, **dict(zip(keys, vals))))
    else:
        for wb, nw in itertools.product(space["word_bits"], space["words"]):
            run(dict(base, word_bits=wb, words=nw))
        best = min(table, key=lambda x: x[1])[0]
        for h, a in itertools.product(space["heavy_degree"], space["pull_alpha"]):
            run(dict(best, heavy_degree=h, pull_alpha=a))
        best = min(table, key=lambda x: x[1])[0]
        for pb in space.get("push_beta", [best.get("push_beta", 0.0)]):
            run(dict(best, push_beta=pb))
        best = min(table, key=lambda x: x[1])[0]
        for tl in space.get("tile", [best.get("tile", 0)]):
            run(dict(best, tile=tl))
        best = min(table, key=lambda x: x[1])[0]
        for so in space.get("source_order", [best.get("source_order", 0)]):
            run(dict(best, source_order=so))
        best = min(table, key=lambda x: x[1])[0]
        for ch in space["chains"]:
            run(dict(best, chains=ch))
    best = dict(min(table, key=lambda x: x[1])[0])
    ctx.set_tuning(**best)
    return best, table


def save(cfg: dict, path: str) -> None:
    with open(path, "w") as f:
        json.dump(cfg, f, indent=1, sort_keys=True)


def load(path: str) -> dict:
    with open(path) as f:
        d = json.load(f)
    return {k: d[k] for k in KEYS if k in d}
