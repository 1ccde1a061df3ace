"""Per-workload launch shapes chosen by the autotuner (World.autotune), kept in a JSON file.

`tuned(world, workload, dt, path)` applies the shapes stored for `workload` in the file at `path`,
or, when it has none, runs the tuner on the world as it stands and stores its choice. The shapes
change no result, only a step's time (dyn_set_launch_config).
"""
from __future__ import annotations

import json
from pathlib import Path


def recall(path, workload: str) -> dict | None:
    p = Path(path)
    if not p.exists():
        return None
    return json.loads(p.read_text()).get(workload)


def remember(path, workload: str, config: dict, ms_per_step: float) -> None:
    p = Path(path)
    table = json.loads(p.read_text()) if p.exists() else {}
    table[workload] = {**config, "ms_per_step": ms_per_step}
    p.write_text(json.dumps(table, indent=1, sort_keys=True))


def tuned(world, workload: str, dt: float, path=None, steps: int = 3) -> tuple[dict, float | None, bool]:
    """The launch shapes for `workload` (stored, or tuned now and stored): (shapes, the tuner's
    ms per step or None when stored ones were applied, whether the tuner ran)."""
    if path is not None:
        stored = recall(path, workload)
        if stored is not None:
            shapes = {k: v for k, v in stored.items() if k != "ms_per_step"}
            world.set_launch_config(**shapes)
            return shapes, None, False
    shapes, ms = world.autotune(dt, steps)
    if path is not None:
        remember(path, workload, shapes, ms)
    return shapes, ms, True
