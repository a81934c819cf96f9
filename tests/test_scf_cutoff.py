"""QUICK's integral-cutoff schedule during the SCF (adjust_Cutoff,
src/modules/quick_method_module.f90:1107-1129) on the host: the rule itself and
what the schedule does to an engine (a fake here; the GPU tests run it for real)."""
import pytest

from quick_b200.scf import FINAL_CUTOFF, CutoffSchedule, adjust_cutoff


@pytest.mark.parametrize("prms,cut,prim,want", [
    (1e-4, 1e-7, 1e-8, (1e-7, 1e-8)),       # PRMS above 1e-5: unchanged
    (1e-5, 1e-7, 1e-8, (1e-9, 1e-9)),       # at 1e-5: 1e-9, primLimit follows it down
    (9e-6, 1e-8, 1e-9, (1e-9, 1e-9)),
    (1e-6, 1e-7, 1e-8, (1e-10, 1e-10)),     # the tests run in turn: two steps in one call
    (1e-7, 1e-7, 1e-8, (1e-11, 1e-11)),     # three steps
    (1e-6, 1e-9, 1e-12, (1e-10, 1e-12)),    # a tighter primLimit is kept
    (1e-5, 1e-9, 1e-10, (1e-9, 1e-10)),     # 1e-9 is not looser than 10^-8.5
    (1e-7, 3e-11, 1e-12, (3e-11, 1e-12)),   # 3e-11 is not looser than 10^-10.5
    (1e-9, 1e-12, 1e-13, (1e-12, 1e-13)),   # never loosens
])
def test_adjust_cutoff_rule(prms, cut, prim, want):
    assert adjust_cutoff(prms, cut, prim) == want


class FakeEngine:
    def __init__(self, cut, prim):
        self.integral_cutoff, self.prim_limit = cut, prim
        self.calls = []

    def set_cutoffs(self, cut, prim):
        self.integral_cutoff, self.prim_limit = cut, prim
        self.calls.append(("set", cut, prim))

    def prepare(self):
        self.calls.append(("prepare", self.integral_cutoff))


def test_schedule_builds_lists_once_at_the_final_cutoff_and_restores():
    eng = FakeEngine(1e-7, 1e-8)
    s = CutoffSchedule(eng, True)
    # lists at the final cutoff, then back to the starting one
    assert eng.calls == [("set", FINAL_CUTOFF, 1e-8), ("prepare", FINAL_CUTOFF), ("set", 1e-7, 1e-8)]
    eng.calls.clear()
    assert not s.update(1, 1e-3)
    assert s.update(2, 5e-6) and (eng.integral_cutoff, eng.prim_limit) == (1e-9, 1e-9)
    assert not s.update(3, 4e-6)
    assert s.update(4, 5e-8) and eng.integral_cutoff == 1e-11
    assert s.changes == [(2, 1e-9, 1e-9), (4, 1e-11, 1e-11)]
    assert [c[0] for c in eng.calls] == ["set", "set"]      # no further list builds
    assert s.restore() and (eng.integral_cutoff, eng.prim_limit) == (1e-7, 1e-8)
    assert not s.restore()


def test_schedule_disabled_or_already_tight_leaves_the_engine_alone():
    eng = FakeEngine(1e-10, 1e-11)
    s = CutoffSchedule(eng, False)
    assert not s.update(5, 1e-8) and eng.calls == [] and not s.restore()
    tight = FakeEngine(1e-12, 1e-13)
    s = CutoffSchedule(tight, True)
    assert tight.calls == []                  # already at or below the final cutoff
    assert not s.update(9, 1e-9) and not s.restore()
