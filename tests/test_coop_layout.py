"""CPU test of the cooperative patch layouts (opensfm_b200/csrc/common.cuh,
coop_slot and CoopPatch), compiled for the host with nvcc.

For 2, 4 and 8 lanes per pixel the lanes of a group together hold every tap
of the 7 x 7 patch exactly once:
  * 2 lanes: 25 slots each (25 and 24 taps, one padding slot), no padding
    column;
  * 4 and 8 lanes: the patch padded to 8 columns, the padding slots sampling
    column 6 with weight 0.
The fast walk pairs slots (2k, 2k + 1); for 2 lanes the pairs are checked to
be the positions the walk forms: two columns of a row, two rows of a column.
"""
import os
import shutil
import subprocess

import pytest

from opensfm_b200 import build as B

SRC = r"""
#include <cstdio>
#include "common.cuh"
template <int L>
void dump() {
  for (int lane = 0; lane < L; ++lane)
    for (int t = 0; t < dn::CoopPatch<L>::S; ++t) {
      int dx = -1, dy = -1;
      const bool real = dn::coop_slot<L>(lane, t, dx, dy);
      std::printf("%d %d %d %d %d %d\n", L, lane, t, dx, dy, real ? 1 : 0);
    }
}
int main() {
  dump<2>();
  dump<4>();
  dump<8>();
  return 0;
}
"""


@pytest.fixture(scope="module")
def slots(tmp_path_factory):
    if not (shutil.which(B.NVCC) or os.path.exists(B.NVCC)):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("layout")
    src, exe = d / "layout.cu", d / "layout"
    src.write_text(SRC)
    subprocess.check_call([B.NVCC, "-std=c++17", "-I", B.CSRC, str(src), "-o", str(exe)])
    rows = [tuple(int(v) for v in line.split())
            for line in subprocess.check_output([str(exe)], text=True).splitlines()]
    out = {}
    for L, lane, t, dx, dy, real in rows:
        out.setdefault(L, {}).setdefault(lane, []).append((t, dx, dy, bool(real)))
    return out


@pytest.mark.parametrize("L", [2, 4, 8])
def test_lane_groups_cover_every_tap_once(slots, L):
    seen = {}
    for lane in range(L):
        for t, dx, dy, real in slots[L][lane]:
            assert 0 <= dx <= 6 and 0 <= dy <= 6
            if real:
                seen[(dx, dy)] = seen.get((dx, dy), 0) + 1
    assert len(seen) == 49 and set(seen.values()) == {1}


def test_two_lanes_hold_25_and_24_taps_in_walk_pairs(slots):
    lanes = slots[2]
    assert [len(lanes[l]) for l in (0, 1)] == [25, 25]
    assert [sum(r for *_, r in lanes[l]) for l in (0, 1)] == [25, 24]
    for lane in (0, 1):
        s = {t: (dx, dy) for t, dx, dy, _ in lanes[lane]}
        for k in range(7):  # columns lane and lane + 2 of row k
            assert s[2 * k] == (lane, k) and s[2 * k + 1] == (lane + 2, k)
        for k in range(3):  # column lane + 4, rows 2k and 2k + 1
            assert s[14 + 2 * k] == (lane + 4, 2 * k) and s[15 + 2 * k] == (lane + 4, 2 * k + 1)
        first = 4 * lane  # column 6: rows 0-3, or 4-6 and row 6 again
        assert [s[t] for t in range(20, 24)] == [(6, min(first + k, 6)) for k in range(4)]
        assert s[24] == (lane + 4, 6)


@pytest.mark.parametrize("L", [4, 8])
def test_wide_groups_pad_column_seven_onto_six(slots, L):
    pads = [(lane, t) for lane in range(L) for t, dx, dy, real in slots[L][lane] if not real]
    assert len(pads) == 7  # one padding column of 7 rows
    for lane, t in pads:
        _, dx, dy, _ = slots[L][lane][t]
        assert dx == 6
