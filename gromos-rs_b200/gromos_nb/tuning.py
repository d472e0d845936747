"""Persistent cache of autotuning results (solvent kernel variant per system shape and GPU).

``gr_autotune`` / ``gr_batch_autotune`` time whole pairlist periods of every solvent kernel
variant (lane layout x i-cluster width) on the systems themselves; that costs a few
periods per variant.  The choice depends on the GPU and on the shape of the work (atom
counts, box, cutoffs, rebuild interval), not on the coordinates, so it is kept in a small
JSON file and reused: a later run of the same shape on the same kind of GPU applies the
cached variant without timing anything.

The cache is a plain JSON object ``{key: entry}``; ``key`` is the GPU name and SM count plus
the system signature, ``entry`` the chosen ``water_layout`` / ``cluster_size`` with the
candidates' measured device ms per step.  Writes go to a temporary file that replaces the
cache atomically, so concurrent runs never leave a half-written file.
"""
from __future__ import annotations

import json
import os
import tempfile
from typing import Callable, Dict, Iterable, Optional

from .system import System


def system_signature(s: System) -> Dict:
    """What the kernel choice depends on: sizes, box (to 0.01 nm), cutoffs, NSNB, kernel shape."""
    t = s.topo
    p = s.params
    return {"n_atoms": int(t.n_atoms), "n_solute_atoms": int(t.n_solute_atoms),
            "n_cg": int(len(t.cg_offsets) - 1), "box": [round(float(b), 2) for b in s.box],
            "rcutp": round(float(p.rcutp), 4), "rcutl": round(float(p.rcutl), 4), "nsnb": int(p.nsnb),
            "boundary": int(p.boundary), "perturbed": bool(t.pert_idx is not None and (t.pert_idx >= 0).any())}


def cache_key(device: Dict, signatures: Iterable[Dict]) -> str:
    """One key per GPU kind and set of systems (a batch's members in order)."""
    return json.dumps({"device": device, "systems": list(signatures)}, sort_keys=True, separators=(",", ":"))


def device_signature(device: int = 0) -> Dict:
    import torch
    prop = torch.cuda.get_device_properties(device)
    return {"name": prop.name, "sms": int(prop.multi_processor_count)}


class TuningCache:
    """JSON file of autotuning results; missing or unreadable files read as empty."""

    def __init__(self, path: str):
        self.path = path

    def load(self) -> Dict[str, Dict]:
        try:
            with open(self.path) as fh:
                data = json.load(fh)
            return data if isinstance(data, dict) else {}
        except (OSError, ValueError):
            return {}

    def get(self, key: str) -> Optional[Dict]:
        e = self.load().get(key)
        if isinstance(e, dict) and "water_layout" in e and "cluster_size" in e:
            return e
        return None

    def put(self, key: str, entry: Dict) -> None:
        data = self.load()
        data[key] = entry
        d = os.path.dirname(os.path.abspath(self.path))
        os.makedirs(d, exist_ok=True)
        fd, tmp = tempfile.mkstemp(prefix=".tuning-", suffix=".json", dir=d)
        try:
            with os.fdopen(fd, "w") as fh:
                json.dump(data, fh, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except BaseException:
            try:
                os.unlink(tmp)
            except OSError:
                pass
            raise


def tune_cached(cache: Optional[TuningCache], key: str, tune: Callable[[], Dict],
                apply: Callable[[int, int], None]) -> Dict:
    """A cached choice is applied (``apply(layout, width)``) without timing; otherwise ``tune()``
    runs, and its result is stored.  Returns the entry with ``"cached": True/False``."""
    if cache is not None:
        e = cache.get(key)
        if e is not None:
            apply(int(e["water_layout"]), int(e["cluster_size"]))
            return dict(e, cached=True)
    r = tune()
    if cache is not None:
        cache.put(key, {k: v for k, v in r.items() if k != "cached"})
    return dict(r, cached=False)
