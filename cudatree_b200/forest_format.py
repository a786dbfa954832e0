"""Versioned flat forest format: a fitted forest as one byte string or file.

The reference pickles its trees (``random_forest.py:18-23``,
``random_tree.py:21-36``), and a restored forest cannot predict: its predict
kernel and label table are only set by ``fit`` (``random_forest.py:94``,
``:453-457``).  Here a forest serializes to a flat, versioned layout whose
node section is exactly the ``ct_packed_node`` array that ``ct_predict`` and
``ct_server_add_forest`` take, so a stored forest is loaded by viewing the
bytes, checking them with ``ct_check_forest`` (no device work) and, for
serving, copying them into a server's forest pool.  Pickling a fitted forest
writes this format too.

Layout (little-endian; every section starts on a 16-byte boundary):

    offset  bytes   field
    0       8       magic b"CTFOREST"
    8       4       format version (uint32), currently 1
    12      4       header length H (uint32)
    16      H       header, UTF-8 JSON: n_trees, n_nodes, n_features,
                    n_classes, label_dtype, params (constructor arguments),
                    node_layout
    A       4 T     tree offsets (uint32): first node of each tree
    B       16 N    nodes {float32 threshold, uint32 feature, uint32 left,
                    uint32 value}; left 0 marks a leaf, else the local index
                    of the left child and the right child is left + 1
                    (breadth-first numbering); value is the leaf's class id
    D       L       label table: the class id -> label map as an .npy blob
                    (numeric or fixed-width string dtypes)
    end-4   4       CRC-32 of every byte before it

A reader refuses other magics, versions it does not know, a bad CRC and
forests that fail the node check, with ValueError.
"""
from __future__ import annotations

import io
import json
import struct
import zlib

import numpy as np

from . import _lib

MAGIC = b"CTFOREST"
VERSION = 1
NODE_LAYOUT = "threshold:f32,feature:u32,left:u32,value:u32"
PACKED_DTYPE = np.dtype([("threshold", "<f4"), ("feature", "<u4"), ("left", "<u4"), ("value", "<u4")])


def _pad16(n: int) -> int:
    return (n + 15) & ~15


def _json_safe(v):
    return v.item() if isinstance(v, np.generic) else v


def encode(packed: np.ndarray, offsets: np.ndarray, n_features: int, n_classes: int, table, params: dict) -> bytes:
    """The flat format of a packed forest (see the module docstring)."""
    params = {k: _json_safe(v) for k, v in params.items()}
    packed = np.ascontiguousarray(packed, dtype=PACKED_DTYPE)
    offsets = np.ascontiguousarray(offsets, dtype="<u4")
    table = np.asarray(table)
    if table.dtype.hasobject:
        raise ValueError("labels of dtype object cannot be stored in the flat forest format")
    header = json.dumps({
        "n_trees": int(offsets.shape[0]), "n_nodes": int(packed.shape[0]), "n_features": int(n_features),
        "n_classes": int(n_classes), "label_dtype": np.dtype(np.uint8 if n_classes <= 0xFF else np.uint16).str,
        "params": params, "node_layout": NODE_LAYOUT}, sort_keys=True).encode()
    lab = io.BytesIO()
    np.save(lab, table, allow_pickle=False)
    out = bytearray(MAGIC + struct.pack("<II", VERSION, len(header)) + header)
    out += b"\0" * (_pad16(len(out)) - len(out))
    out += offsets.tobytes()
    out += b"\0" * (_pad16(len(out)) - len(out))
    out += packed.tobytes()
    out += lab.getvalue()
    out += struct.pack("<I", zlib.crc32(out) & 0xFFFFFFFF)
    return bytes(out)


def decode(data: bytes):
    """(packed nodes, tree offsets, header, label table) of a flat forest,
    checked: magic, version, CRC, section sizes, and the node check of
    ct_check_forest (children after their node inside its tree, features
    and leaf classes in range)."""
    data = bytes(data)
    if len(data) < 20 or data[:8] != MAGIC:
        raise ValueError("not a cudatree_b200 flat forest (bad magic)")
    version, hlen = struct.unpack_from("<II", data, 8)
    if version != VERSION:
        raise ValueError(f"flat forest format version {version} is not supported (this reader knows {VERSION})")
    (crc,) = struct.unpack_from("<I", data, len(data) - 4)
    if zlib.crc32(data[:-4]) & 0xFFFFFFFF != crc:
        raise ValueError("flat forest is corrupt (CRC mismatch)")
    try:
        hdr = json.loads(data[16:16 + hlen].decode())
        t, n = int(hdr["n_trees"]), int(hdr["n_nodes"])
        nf, nc = int(hdr["n_features"]), int(hdr["n_classes"])
    except (ValueError, KeyError, UnicodeDecodeError) as e:
        raise ValueError(f"flat forest header is malformed: {e}") from None
    if hdr.get("node_layout") != NODE_LAYOUT:
        raise ValueError("flat forest has an unknown node layout")
    a = _pad16(16 + hlen)
    b = _pad16(a + 4 * t)
    d = b + 16 * n
    if t < 1 or n < t or d > len(data) - 4:
        raise ValueError("flat forest sections are truncated or empty")
    offsets = np.frombuffer(data, dtype="<u4", count=t, offset=a).copy()
    packed = np.frombuffer(data, dtype=PACKED_DTYPE, count=n, offset=b).copy()
    try:
        table = np.load(io.BytesIO(data[d:-4]), allow_pickle=False)
    except (ValueError, EOFError, OSError) as e:
        raise ValueError(f"flat forest label table is malformed: {e}") from None
    if table.shape != (nc,):
        raise ValueError("flat forest label table does not hold one label per class")
    st = _lib.load().ct_check_forest(packed.ctypes.data, n, offsets.ctypes.data, t, nf, nc)
    if st != 0:
        raise ValueError(_lib.last_error())
    return packed, offsets, hdr, table


def dumps(forest) -> bytes:
    """Flat format of a fitted RandomForestClassifier."""
    from .random_forest import pack_trees
    if not forest._trees:
        raise ValueError("forest is not fitted")
    packed, offsets = pack_trees(forest._trees)
    return encode(packed, offsets, forest.n_features, forest.n_labels, forest.compt_table, forest._params())


def loads(data: bytes):
    """A RandomForestClassifier that predicts as the stored one did."""
    from .random_forest import restore_forest, unpack_trees
    packed, offsets, hdr, table = decode(data)
    trees = unpack_trees(packed, offsets, hdr["n_features"], np.dtype(hdr["label_dtype"]))
    return restore_forest(trees, hdr["label_dtype"], table, hdr["n_features"], hdr.get("params"))


def save(forest, path) -> None:
    with open(path, "wb") as fh:
        fh.write(dumps(forest))


def load(path):
    with open(path, "rb") as fh:
        return loads(fh.read())


def restore_forest_flat(data: bytes):
    """Unpickle hook of forests pickled in the flat format."""
    return loads(data)
