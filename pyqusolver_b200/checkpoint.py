"""Checkpoints of the RBM parameters and training metadata, in the reference's file layout.

Mirrors ``NQSCheckpointManager`` (``QES/NQS/src/nqs_checkpoint_manager.py:58-514``) on its
HDF5-less path, which is the one this stack takes (neither h5py nor Orbax is part of it):

* ``save(step, params, metadata, filename)`` writes ``checkpoint_<step>.npz`` whose keys are the
  parameter tree flattened with "/" (``_save_npz`` / ``_flatten_dict`` ``:456-473``), e.g.
  ``visible_bias``, ``VisibleToHidden/kernel``, ``VisibleToHidden/bias`` for the RBM, and the
  metadata as JSON beside it, ``checkpoint_<step>.json`` (``_save_hdf5_wrapper`` ``:239-250``),
  complex numbers as ``{"__complex__": true, "real": .., "imag": ..}``
  (``_make_json_serializable`` ``:495-510``).  The same JSON is also written as
  ``metadata_<step>.json``, the name the reference's ``load_metadata`` reads (``:376-393``), so
  either side reads the other's files.  A custom ``filename`` keeps its JSON beside it (same stem).
* ``load(step, filename)`` returns the flattened dict of arrays (``_load_npz``, no pickles);
  ``load_metadata``, ``list_checkpoints``, the ``latest_step`` property and ``max_to_keep``
  pruning behave as the reference's.

Every file is written to a temporary name and moved into place, so a crash leaves either the old
file or the complete new one.  Only host memory is involved.
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
    if isinstance(x, np.ndarray):
        if np.iscomplexobj(x):
            return [_jsonable(complex(v)) for v in x.reshape(-1)] if x.ndim else _jsonable(complex(x))
        return x.tolist()
    if isinstance(x, (complex, np.complexfloating)):
        z = complex(x)
        return {"__complex__": True, "real": z.real, "imag": z.imag}
    if isinstance(x, (np.floating, np.integer, np.bool_)):
        return x.item()
    if hasattr(x, "__dict__") and not isinstance(x, (str, int, float, bool)):
        return str(x)
    return x


def flatten_tree(d: dict, parent_key: str = "", sep: str = "/") -> dict:
    """Nested dict -> {"a/b": leaf} (the reference's ``_flatten_dict``)."""
    out = {}
    for k, v in d.items():
        key = f"{parent_key}{sep}{k}" if parent_key else str(k)
        if isinstance(v, dict):
            out.update(flatten_tree(v, key, sep))
        else:
            out[key] = v
    return out


def _atomic_write(path: Path, write):
    tmp = path.with_name(path.name + ".tmp")
    write(tmp)
    os.replace(tmp, path)


class NQSCheckpointManager:
    TAG_MAP = {"latest": 999999, "best": 999998, "final": 999997}

    def __init__(self, directory: Union[str, Path], use_orbax: bool = False, max_to_keep: int = 3, logger=None,
                 **kwargs):
        if use_orbax:
            raise NotImplementedError("Orbax is not part of this stack; use_orbax=False writes the npz layout")
        self.directory = Path(directory)
        self.use_orbax = False
        self.max_to_keep = int(max_to_keep)
        self.directory.mkdir(parents=True, exist_ok=True)

    # ------------------------------------------------------------------ paths
    def _resolve_path(self, filename: Optional[str], step, extension: str = "npz") -> Path:
        if filename is not None:
            p = Path(filename)
            p = p if p.is_absolute() else self.directory / p
            return p.with_suffix("." + extension)
        return self.directory / f"checkpoint_{'latest' if step is None else step}.{extension}"

    # ------------------------------------------------------------------ save / load
    def save(self, step: Union[int, str], params: Any, metadata: Optional[Dict[str, Any]] = None,
             filename: Optional[str] = None, **kwargs) -> Path:
        """Write the parameter tree (a dict, nested or already flattened; a bare array is stored under
        the key ``params``) and the metadata (with ``step`` added)."""
        metadata = dict(metadata or {})
        metadata["step"] = step
        tree = params if isinstance(params, dict) else {"params": np.asarray(params)}
        flat = {k: np.asarray(v.detach().cpu().numpy() if hasattr(v, "detach") else v)
                for k, v in flatten_tree(tree).items()}
        npz = self._resolve_path(filename, step, "npz")
        npz.parent.mkdir(parents=True, exist_ok=True)

        def write_npz(tmp):
            with open(tmp, "wb") as f:
                np.savez(f, **flat)
        _atomic_write(npz, write_npz)
        text = json.dumps(_jsonable(metadata), indent=2)
        jsons = [npz.with_suffix(".json")]
        if filename is None:
            jsons.append(self.directory / f"metadata_{step}.json")
        for jp in jsons:
            _atomic_write(jp, lambda tmp: Path(tmp).write_text(text))
        self._prune()
        return npz

    def load(self, step: Optional[Union[int, str]] = None, filename: Optional[str] = None, **kwargs) -> dict:
        """Flattened parameter dict of ``step`` (default: the latest checkpoint)."""
        if filename is None and step is None:
            step = self.latest_step
            if step is None:
                raise FileNotFoundError(f"no checkpoint in {self.directory}")
        path = self._resolve_path(filename, step, "npz")
        if not path.exists():
            raise FileNotFoundError(f"Checkpoint not found: {path}")
        with np.load(path, allow_pickle=False) as z:
            return {k: z[k].copy() for k in z.files}

    def load_metadata(self, step: Optional[Union[int, str]] = None, filename: Optional[str] = None) -> Dict[str, Any]:
        if filename is not None:
            cands = [self._resolve_path(filename, 0, "json")]
        else:
            if step is None:
                step = self.latest_step
            cands = [self.directory / f"metadata_{step}.json", self.directory / f"checkpoint_{step}.json"]
        for p in cands:
            if p.exists():
                with open(p) as f:
                    return json.load(f)
        return {}

    def list_checkpoints(self) -> list:
        out = []
        for p in self.directory.glob("checkpoint_*.npz"):
            tag = p.stem[len("checkpoint_"):]
            out.append(int(tag) if tag.isdigit() else tag)
        ints = sorted(s for s in out if isinstance(s, int))
        return ints + sorted(s for s in out if not isinstance(s, int))

    @property
    def latest_step(self):
        steps = self.list_checkpoints()
        ints = [s for s in steps if isinstance(s, int)]
        if ints:
            return ints[-1]
        return "latest" if "latest" in steps else (steps[-1] if steps else None)

    def wait_until_finished(self):
        """Saves are synchronous here (the reference waits for Orbax's asynchronous saves)."""

    def _prune(self):
        if self.max_to_keep <= 0:
            return
        ints = [s for s in self.list_checkpoints() if isinstance(s, int)]
        for s in ints[:-self.max_to_keep]:
            for name in (f"checkpoint_{s}.npz", f"checkpoint_{s}.json", f"metadata_{s}.json"):
                p = self.directory / name
                if p.exists():
                    p.unlink()

