"""Depthmap files in OpenSfM's layout.

OpenSfM keeps one file per view and stage under ``<data>/depthmaps/``:
``<image>.raw.npz`` (fields depth, plane, score, nghbr, nghbrs and an
optional confidence) and ``<image>.clean.npz`` (depth, plane, score and an
optional confidence).  Each is an ``np.savez`` archive wrapped in one LZ4
frame (``opensfm/dataset.py:1063-1149``).  This module writes and reads that
layout with the library's own LZ4 frame code (``dn_lz4f_*``), so neither
``lz4`` nor OpenSfM is needed; files written here decode with
``lz4.frame.decompress`` and files written by OpenSfM decode here.
"""
from __future__ import annotations

import ctypes
import io
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib


def _io_check(st: int) -> None:
    if st != _lib.DN_OK:
        msg = _lib.load().dn_io_last_error().decode(errors="replace")
        raise ValueError(msg)


def xxh32(data: bytes, seed: int = 0) -> int:
    """xxHash32 of ``data`` (the LZ4 frame checksum)."""
    return int(_lib.load().dn_xxh32(data, len(data), seed))


def lz4_frame_compress(data: bytes) -> bytes:
    """One LZ4 frame holding ``data`` (content size stored)."""
    L = _lib.load()
    n = ctypes.c_int64()
    cap = int(L.dn_lz4f_compress_bound(len(data)))
    out = ctypes.create_string_buffer(cap)
    _io_check(L.dn_lz4f_compress(data, len(data), out, cap, ctypes.byref(n)))
    return out.raw[: n.value]


def lz4_frame_decompress(data: bytes) -> bytes:
    """The content of one or more concatenated LZ4 frames."""
    L = _lib.load()
    src = ctypes.create_string_buffer(data, len(data))
    n = ctypes.c_int64()
    _io_check(L.dn_lz4f_decompress(src, len(data), None, 0, ctypes.byref(n)))
    out = ctypes.create_string_buffer(max(n.value, 1))
    _io_check(L.dn_lz4f_decompress(src, len(data), out, n.value, ctypes.byref(n)))
    return out.raw[: n.value]


def depthmap_file(data_path: str, image: str, suffix: str) -> str:
    """``<data_path>/depthmaps/<image>.<suffix>`` (``dataset.py:958-963``)."""
    return os.path.join(data_path, "depthmaps", image + "." + suffix)


def _write(path: str, arrays: dict) -> None:
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    buf = io.BytesIO()
    np.savez(buf, **arrays)
    with open(path, "wb") as f:
        f.write(lz4_frame_compress(buf.getvalue()))


def _read(path: str) -> dict:
    with open(path, "rb") as f:
        raw = lz4_frame_decompress(f.read())
    with np.load(io.BytesIO(raw)) as o:
        return {k: o[k] for k in o.files}


def save_raw_depthmap(data_path: str, image: str, depth: np.ndarray, plane: np.ndarray,
                      score: np.ndarray, nghbr: np.ndarray, nghbrs: Sequence[str],
                      confidence: Optional[np.ndarray] = None) -> str:
    """``DataSet.save_raw_depthmap`` (``dataset.py:1066-1098``)."""
    arrays = dict(depth=depth, plane=plane, score=score, nghbr=nghbr, nghbrs=list(nghbrs))
    if confidence is not None:
        arrays["confidence"] = confidence
    path = depthmap_file(data_path, image, "raw.npz")
    _write(path, arrays)
    return path


def load_raw_depthmap(data_path: str, image: str
                      ) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray, List[str],
                                 Optional[np.ndarray]]:
    """``DataSet.load_raw_depthmap`` (``dataset.py:1100-1112``)."""
    o = _read(depthmap_file(data_path, image, "raw.npz"))
    return (o["depth"], o["plane"], o["score"], o["nghbr"], o["nghbrs"],
            o.get("confidence"))


def save_clean_depthmap(data_path: str, image: str, depth: np.ndarray, plane: np.ndarray,
                        score: np.ndarray, confidence: Optional[np.ndarray] = None) -> str:
    """``DataSet.save_clean_depthmap`` (``dataset.py:1117-1135``)."""
    arrays = dict(depth=depth, plane=plane, score=score)
    if confidence is not None:
        arrays["confidence"] = confidence
    path = depthmap_file(data_path, image, "clean.npz")
    _write(path, arrays)
    return path


def load_clean_depthmap(data_path: str, image: str
                        ) -> Tuple[np.ndarray, np.ndarray, np.ndarray, Optional[np.ndarray]]:
    """``DataSet.load_clean_depthmap`` (``dataset.py:1137-1149``)."""
    o = _read(depthmap_file(data_path, image, "clean.npz"))
    return o["depth"], o["plane"], o["score"], o.get("confidence")
