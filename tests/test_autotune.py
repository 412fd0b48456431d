"""The autotuner's selection rule (kgpu_tune_select), on the CPU: the
fastest candidate replaces the incumbent only when it beats it by the
required fraction; failed trials (negative or non-finite timings) never win;
a failed incumbent is replaced by any finished candidate."""
import numpy as np
import pytest


def test_fastest_wins_beyond_the_margin(kgpu):
    assert kgpu.tune_select([10.0, 8.0, 9.0], 0, 0.02) == 1
    assert kgpu.tune_select([10.0, 9.9, 9.95], 0, 0.02) == 0      # within 2%: keep the incumbent
    assert kgpu.tune_select([10.0, 9.9, 9.95], 0, 0.0) == 1
    assert kgpu.tune_select([7.0, 8.0, 9.0], 2, 0.02) == 0
    assert kgpu.tune_select([5.0], 0, 0.5) == 0


def test_failed_trials_never_win(kgpu):
    assert kgpu.tune_select([10.0, -1.0, np.nan, np.inf], 0, 0.02) == 0
    assert kgpu.tune_select([-1.0, 12.0, 11.0], 0, 0.02) == 2     # the incumbent failed
    assert kgpu.tune_select([-1.0, np.nan], 0, 0.02) == 0         # nothing finished: keep it


def test_bad_arguments_rejected(kgpu):
    for ms, inc, gain in (([1.0, 2.0], 2, 0.0), ([1.0], -1, 0.0), ([1.0, 2.0], 0, -0.1)):
        with pytest.raises(kgpu.KgpuError):
            kgpu.tune_select(ms, inc, gain)
