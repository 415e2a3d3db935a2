"""CPU tests of the schedule host logic: what ``learned.Schedule.apply``
sets on a batch, and the bench's learned-schedule list (its order, and the
launch count it reports)."""
import bench
from opensfm_b200 import learned


class RecordingBatch:
    """Stands in for pydense.Batch: records every setter call."""

    def __init__(self):
        self.calls = {}

    def __getattr__(self, name):
        if not name.startswith("set_"):
            raise AttributeError(name)

        def rec(*args, **kw):
            self.calls[name] = (args, kw)

        return rec


def test_schedule_apply_sets_every_switch():
    b = RecordingBatch()
    learned.Schedule("s", "learned", 4, {"n_refine": 2}, sample=2, active=0.01, seed=0.9,
                     fallback=True).apply(b)
    assert b.calls["set_schedule"] == ((), {"half_passes": 4, "n_refine": 2})
    assert b.calls["set_candidate_views"] == ((2,), {})
    assert b.calls["set_active_pixels"] == ((True, 0.01), {})
    assert b.calls["set_active_seed"] == ((0.9,), {})
    assert b.calls["set_init_fallback"] == ((True,), {})
    assert b.calls["set_knight_moves"] == ((False,), {})


def test_plain_schedule_leaves_the_learned_switches_off():
    b = RecordingBatch()
    plain, _ = bench.schedules()
    plain.apply(b)
    assert plain.init == "plain" and plain.half_passes == 2 * bench.ITERS
    assert b.calls["set_candidate_views"] == ((0,), {})
    assert b.calls["set_active_pixels"] == ((False, 0.0), {})
    assert b.calls["set_active_seed"] == ((0.0,), {})
    assert b.calls["set_init_fallback"] == ((False,), {})


def test_bench_learned_schedules_are_ordered_by_kind():
    """Settled-start schedules first, then the ones without it, then the
    random-initialisation fallbacks; every one learned, with active pixels,
    and a unique name."""
    _, scheds = bench.schedules()
    assert len({s.name for s in scheds}) == len(scheds)
    kinds = [0 if s.seed > 0 else (2 if s.fallback else 1) for s in scheds]
    assert kinds == sorted(kinds) and kinds[0] == 0 and kinds[-1] == 2
    for s in scheds:
        assert s.init == "learned" and s.active > 0 and s.sample in (0, 1, 2)
        assert 0 <= s.seed <= 1
