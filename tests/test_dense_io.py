"""Depthmap files in OpenSfM's layout (an .npz inside one LZ4 frame,
opensfm/dataset.py:1063-1149) through the library's own LZ4 frame and
xxHash32 code: published known answers, frames built by hand from the
format description, round trips, and the raw/clean file fields.  Host code
only: these run without a GPU."""
import os
import struct

import numpy as np
import pytest

from opensfm_b200 import dense_io


def test_xxh32_known_answers():
    assert dense_io.xxh32(b"") == 0x02CC5D05
    assert dense_io.xxh32(b"a") == 0x550D7456
    assert dense_io.xxh32(b"abc") == 0x32D153FF
    # Longer than one 16-byte stripe.
    assert dense_io.xxh32(b"Nobody inspects the spammish repetition") == 0xE2293B2F


def _frame(flg, bd, blocks, content=None, size=None):
    """An LZ4 frame from raw block payloads [(bytes, stored)]."""
    desc = bytes([flg, bd]) + (struct.pack("<Q", size) if size is not None else b"")
    out = struct.pack("<I", 0x184D2204) + desc + bytes([(dense_io.xxh32(desc) >> 8) & 0xFF])
    for data, stored in blocks:
        out += struct.pack("<I", len(data) | (0x80000000 if stored else 0)) + data
        if flg & 0x10:
            out += struct.pack("<I", dense_io.xxh32(data))
    out += struct.pack("<I", 0)
    if flg & 0x04:
        out += struct.pack("<I", dense_io.xxh32(content))
    return out


def test_hand_built_frames_decode():
    # "abc" + a 12-byte overlapping match at offset 3 + final literals.
    blk = bytes([0x38]) + b"abc" + bytes([3, 0]) + bytes([0x50]) + b"12345"
    want = b"abcabcabcabcabc12345"
    assert dense_io.lz4_frame_decompress(_frame(0x60, 0x40, [(blk, False)])) == want
    # Content checksum, content size and a block checksum.
    f = _frame(0x60 | 0x04 | 0x08 | 0x10, 0x40, [(blk, False)], content=want, size=len(want))
    assert dense_io.lz4_frame_decompress(f) == want
    # Linked blocks: the second block's match reaches into the first block.
    blk2 = bytes([0x04]) + bytes([20, 0]) + bytes([0x10]) + b"!"  # 8 bytes from 20 back, "!"
    f = _frame(0x40, 0x40, [(blk, False), (blk2, False)])
    assert dense_io.lz4_frame_decompress(f) == want + b"abcabcab" + b"!"
    # A stored block, then a skippable frame, then a second frame.
    f = _frame(0x60, 0x40, [(b"plain bytes", True)])
    skip = struct.pack("<II", 0x184D2A51, 3) + b"xyz"
    assert dense_io.lz4_frame_decompress(f + skip + f) == b"plain bytes" * 2


@pytest.mark.parametrize("bad", ["magic", "header", "content", "offset"])
def test_corrupt_frames_raise(bad):
    blk = bytes([0x38]) + b"abc" + bytes([3, 0]) + bytes([0x50]) + b"12345"
    want = b"abcabcabcabcabc12345"
    f = bytearray(_frame(0x64, 0x40, [(blk, False)], content=want))
    if bad == "magic":
        f[0] ^= 1
    elif bad == "header":
        f[6] ^= 1  # the header checksum byte
    elif bad == "content":
        f[-1] ^= 1
    else:
        f[7 + 4 + 4] = 9  # match offset 9 reaches before the frame's output
    with pytest.raises(ValueError):
        dense_io.lz4_frame_decompress(bytes(f))


@pytest.mark.parametrize("n", [0, 1, 12, 13, 17, 1000, (4 << 20) + 12345])
def test_round_trip(n):
    rng = np.random.default_rng(n)
    noise = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
    runs = (b"depthmap" * (n // 8 + 1))[:n]
    for data in (noise, runs):
        comp = dense_io.lz4_frame_compress(data)
        assert comp[:4] == struct.pack("<I", 0x184D2204)
        assert dense_io.lz4_frame_decompress(comp) == data
    if n >= 1000:
        assert len(dense_io.lz4_frame_compress(runs)) < n // 10


def test_raw_and_clean_files(tmp_path):
    rng = np.random.default_rng(0)
    H, W = 48, 64
    depth = rng.uniform(5, 20, (H, W)).astype(np.float32)
    depth[rng.random((H, W)) < 0.3] = 0
    plane = rng.standard_normal((H, W, 3)).astype(np.float32)
    score = rng.uniform(-1, 1, (H, W)).astype(np.float32)
    nghbr = rng.integers(0, 5, (H, W)).astype(np.int32)
    conf = rng.uniform(0, 1, (H, W)).astype(np.float32)
    d = str(tmp_path)
    p = dense_io.save_raw_depthmap(d, "img_01.jpg", depth, plane, score, nghbr,
                                   ["img_02.jpg", "img_03.jpg"], confidence=conf)
    assert p == os.path.join(d, "depthmaps", "img_01.jpg.raw.npz")
    got = dense_io.load_raw_depthmap(d, "img_01.jpg")
    for a, b in zip(got[:4], (depth, plane, score, nghbr)):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    assert list(got[4]) == ["img_02.jpg", "img_03.jpg"]
    assert np.array_equal(got[5], conf)
    dense_io.save_clean_depthmap(d, "img_01.jpg", depth, plane, score)
    c = dense_io.load_clean_depthmap(d, "img_01.jpg")
    assert np.array_equal(c[0], depth) and np.array_equal(c[1], plane)
    assert c[3] is None
