"""The autotuner on the GPU: it picks launch shapes and solver settings by
timing them on the context's own state, restores that state, and the tuned
context computes the same bits as an untuned one (every candidate performs
the same arithmetic).  The choice is cached for the process and reused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_pair(kgpu, make, steps, graph):
    a, b = make(), make()
    for s in (a, b):
        s.rk2imex_steps(2) if a.cfg.nv == 13 else s.rk2_steps(2)
    t, ms = a.autotune(steps=2)
    print("chosen", t.as_dict(), "ms per step before/after", ms)
    assert ms[0] > 0 and ms[1] > 0
    ua, pa = a.download_state()
    ub, pb = b.download_state()
    assert np.array_equal(ua, ub) and np.array_equal(pa, pb)   # the state the trials started from
    for s in (a, b):
        s.rk2imex_steps(steps, graph=graph) if s.cfg.nv == 13 else s.rk2_steps(steps, graph=graph)
    ua, pa = a.download_state()
    ub, pb = b.download_state()
    assert np.array_equal(ua, ub) and np.array_equal(pa, pb)
    assert a.tstepdenmax == b.tstepdenmax
    return t


def test_autotune_torus_same_bits(kgpu):
    t = run_pair(kgpu, lambda: kgpu.fm_torus(32, 16, 8), 5, True)
    c = kgpu.fm_torus(32, 16, 8)
    t2, ms = c.autotune(reuse=True)
    assert ms == (-1.0, -1.0) and t2.as_dict() == t.as_dict()


def test_autotune_radiative_torus_same_bits(kgpu):
    run_pair(kgpu, lambda: kgpu.radtorus(32, 16, 8), 3, True)
