"""Per-device cache of the kernel variants chosen by ``KMM.autotune``.

The choice (``jfb_kmm_autotune``: the fastest of the plan's kernel variants
by CUDA-event timing of graph-replayed steps) depends on the GPU model, the
grid, the wall-normal family, the nonlinear form and the precision form; it
is stored as JSON keyed by those, in the
file named by JFB200_AUTOTUNE_CACHE (default
``~/.cache/jaxfun_b200/autotune.json``).
"""

from __future__ import annotations

import json
import os

import torch


def cache_path() -> str:
    return os.environ.get("JFB200_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "jaxfun_b200", "autotune.json")


def cache_key(solver) -> str:
    name = torch.cuda.get_device_name(solver.device).replace(" ", "_")
    nx, ny, nz = solver.N
    pad = "x".join(f"{p:g}" for p in solver.padding_factor[1:])
    form = getattr(solver, "nonlinear_form", "rotational")
    fam = getattr(solver, "family", "C")
    return f"{name}/{nx}x{ny}x{nz}/pad{pad}/{fam}/{form}/{solver.precision}"


def _read() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(key: str):
    return _read().get(key)


def store(key: str, record: dict) -> None:
    path = cache_path()
    data = _read()
    data[key] = {k: v for k, v in record.items() if k != "cached"}
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache only costs a re-tune
