"""Autotuner of the stage launch shape, with an on-disk cache.

The stage kernels run one CTA per (block, z-slab).  How many slabs a block
is cut into trades parallelism (small meshes leave SMs idle) against
redundant halo planes (each slab reloads two planes on either side).  With
whole blocks the corrector can also carry the viscous step, which saves a
pass over the state but needs more shared memory per CTA (fewer CTAs per
SM for the passive-scalar equation sets).  The best shape depends on the
block count, the levels and the equation set, so it is measured on the live
mesh (wx3d_autotune) and cached by a workload signature in a JSON file.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

DEFAULT_CACHE = Path(os.environ.get("WX3D_TUNE_CACHE", Path.home() / ".cache" / "wx3d" / "tuning.json"))


def signature(cfg, nblocks: int, levels) -> str:
    """Workload key: equation set, solver, limiter and the mesh's histogram
    of blocks per level (the launch shape depends on how many blocks there
    are and on the share of coarse/fine faces the levels bring)."""
    hist = {}
    for l in levels:
        hist[int(l)] = hist.get(int(l), 0) + 1
    lv = ",".join(f"{l}:{hist[l]}" for l in sorted(hist))
    return f"neq{cfg.neqtot}-s{cfg.solver_type}-l{cfg.limiter_type}-mhd{int(cfg.mhd)}-nb{nblocks}-lev{lv}"


def tune(w, prob, cache: Path | None = DEFAULT_CACHE, reps: int = 3, force: bool = False) -> dict:
    """Picks the launch shape for w's mesh; returns a record of the choice."""
    levels = [prob.tree.level(int(b)) for b in prob.local_blocks]
    key = signature(prob.cfg, prob.nblocks, levels)
    table = {}
    if cache is not None and cache.exists():
        try:
            table = json.loads(cache.read_text())
        except ValueError:
            table = {}
    if key in table and not force and "fused" in table[key]:
        w.set_zsplit(int(table[key]["zsplit"]))
        w.set_fusion(bool(table[key]["fused"]))
        return dict(table[key], cached=True, key=key)
    best, fused, ms = w.autotune(reps)
    rec = {"zsplit": best, "fused": fused, "ms_per_pass": {str(k): v for k, v in ms.items()}}
    if cache is not None:
        cache.parent.mkdir(parents=True, exist_ok=True)
        table[key] = rec
        tmp = cache.with_suffix(".tmp")
        tmp.write_text(json.dumps(table, indent=1, sort_keys=True))
        tmp.replace(cache)
    return dict(rec, cached=False, key=key)
