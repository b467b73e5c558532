"""Checkpoints of the RBM parameters and training metadata.

Mirrors the interface of ``NQSCheckpointManager`` (``QES/NQS/src/nqs_checkpoint_manager.py:58-514``):
``save(step, params, metadata)``, ``load(step)``, ``load_metadata(step)``, ``list_checkpoints()``,
``latest_step()``, files named ``checkpoint_<step>``.  The reference writes HDF5 or Orbax; neither
h5py nor Orbax is part of this stack, so a checkpoint here is a NumPy ``.npz`` holding the flat
parameter vector ([a, b, W], float64 / complex128) and the per-leaf shapes, plus a JSON file with
the metadata (step, model, sampler settings, energy history).  Only host memory is involved: the
caller moves parameters off the device (``NQS.get_params(unravel=True)``).
"""

from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Any, Dict, Optional, Union

import numpy as np


def _jsonable(x):
    if isinstance(x, dict):
        return {str(k): _jsonable(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_jsonable(v) for v in x]
    if isinstance(x, complex) or np.iscomplexobj(x):
        z = complex(np.asarray(x).item()) if np.ndim(x) == 0 else None
        if z is not None:
            return {"re": z.real, "im": z.imag}
        return [_jsonable(v) for v in np.asarray(x).tolist()]
    if isinstance(x, np.ndarray):
        return x.tolist()
    if isinstance(x, (np.floating, np.integer, np.bool_)):
        return x.item()
    return x


class NQSCheckpointManager:
    def __init__(self, directory: Union[str, Path], use_orbax: bool = False, max_to_keep: int = 3, logger=None):
        self.directory = Path(directory)
        self.max_to_keep = int(max_to_keep)
        self.directory.mkdir(parents=True, exist_ok=True)

    def _path(self, step, ext):
        return self.directory / f"checkpoint_{step}.{ext}"

    def save(self, step: Union[int, str], params: Any, metadata: Optional[Dict[str, Any]] = None,
             filename: Optional[str] = None, **kwargs) -> Path:
        """Write params (a flat array, or the RBM dict of visible_bias / hidden_bias / W) and metadata."""
        metadata = dict(metadata or {})
        metadata["step"] = step
        if isinstance(params, dict):
            leaves = {k: np.asarray(params[k]) for k in ("visible_bias", "hidden_bias", "W")}
            flat = np.concatenate([v.reshape(-1) for v in leaves.values()])
            shapes = {k: list(v.shape) for k, v in leaves.items()}
        else:
            flat = np.asarray(params).reshape(-1)
            shapes = {}
        path = self.directory / filename if filename else self._path(step, "npz")
        tmp = str(path) + ".tmp.npz"
        np.savez(tmp, params=flat, shapes=json.dumps(shapes))
        os.replace(tmp, path)
        with open(self._path(step, "json"), "w") as f:
            json.dump(_jsonable(metadata), f, indent=1)
        self._prune()
        return path

    def load(self, step: Optional[Union[int, str]] = None, filename: Optional[str] = None, **kwargs):
        """Flat parameter vector of ``step`` (default: the latest)."""
        if step is None and filename is None:
            step = self.latest_step()
            if step is None:
                raise FileNotFoundError(f"no checkpoint in {self.directory}")
        path = self.directory / filename if filename else self._path(step, "npz")
        with np.load(path) as z:
            return z["params"].copy()

    def load_metadata(self, step: Optional[Union[int, str]] = None) -> Dict[str, Any]:
        if step is None:
            step = self.latest_step()
        p = self._path(step, "json")
        if not p.exists():
            return {}
        with open(p) as f:
            return json.load(f)

    def list_checkpoints(self) -> list:
        out = []
        for p in self.directory.glob("checkpoint_*.npz"):
            tag = p.stem[len("checkpoint_"):]
            out.append(int(tag) if tag.isdigit() else tag)
        ints = sorted(s for s in out if isinstance(s, int))
        return ints + sorted(s for s in out if not isinstance(s, int))

    def latest_step(self):
        steps = self.list_checkpoints()
        ints = [s for s in steps if isinstance(s, int)]
        if ints:
            return ints[-1]
        return "latest" if "latest" in steps else (steps[-1] if steps else None)

    def _prune(self):
        if self.max_to_keep <= 0:
            return
        ints = [s for s in self.list_checkpoints() if isinstance(s, int)]
        for s in ints[:-self.max_to_keep]:
            for ext in ("npz", "json"):
                p = self._path(s, ext)
                if p.exists():
                    p.unlink()
