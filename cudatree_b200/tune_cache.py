"""Autotuned fit options, kept across processes in a JSON file.

The reference fits its depth-first/breadth-first switch offline
(``estimate_threshold.py:29-96``) and ships the regression in the package
(``random_forest.py:278-289``).  Here ``ct_autotune`` times candidate option
sets on the device at hand; this module keeps each choice per device and
data shape, so a later process fitting the same shape reuses it without
timing again.  Options never change the trees a fit grows, only its speed,
so a stale entry costs time, not correctness.

File: ``$CUDATREE_B200_TUNE_CACHE`` if set (``off`` or an empty value keeps
the cache in the process only), else ``~/.cache/cudatree_b200/autotune.json``.
Layout: ``{"format": 1, "entries": {key: options}}``, where key is the JSON
text of ``[device name, shape key]`` and options the dict that
``RandomForestClassifier.autotune`` returns.  Writes go to a temporary file
that replaces the old one, so a reader never sees a half-written file; a
file that does not parse is treated as empty.
"""
from __future__ import annotations

import json
import os
import tempfile
from pathlib import Path

FORMAT = 1
ENV = "CUDATREE_B200_TUNE_CACHE"
_MEMORY: dict = {}  # key -> options, this process


def path() -> Path | None:
    """The cache file, or None when the cache is kept in memory only."""
    v = os.environ.get(ENV)
    if v is not None:
        return None if v.strip() in ("", "off") else Path(v).expanduser()
    return Path("~/.cache/cudatree_b200/autotune.json").expanduser()


def key(device: str, shape: tuple) -> str:
    return json.dumps([device, list(shape)])


def _read(p: Path) -> dict:
    try:
        with open(p) as fh:
            data = json.load(fh)
    except (OSError, ValueError):
        return {}
    if not isinstance(data, dict) or data.get("format") != FORMAT or not isinstance(data.get("entries"), dict):
        return {}
    return data["entries"]


def get(k: str) -> dict | None:
    """Options stored under k: this process's first, then the file's."""
    if k in _MEMORY:
        return dict(_MEMORY[k])
    p = path()
    if p is None:
        return None
    v = _read(p).get(k)
    if isinstance(v, dict):
        _MEMORY[k] = dict(v)
        return dict(v)
    return None


def put(k: str, options: dict) -> None:
    """Store options under k in this process and, when enabled, in the file."""
    _MEMORY[k] = dict(options)
    p = path()
    if p is None:
        return
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        entries = _read(p)
        entries[k] = dict(options)
        fd, tmp = tempfile.mkstemp(prefix=".autotune.", dir=p.parent)
        with os.fdopen(fd, "w") as fh:
            json.dump({"format": FORMAT, "entries": entries}, fh, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only home keeps the choice in this process


def clear_memory() -> None:
    _MEMORY.clear()
