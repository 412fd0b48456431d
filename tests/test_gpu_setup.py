"""Device set-up of the torus problems: the MKS2 metric tables and the
Fishbone-Moncrief state computed by kernels (kgpu_init_fm_torus,
kgpu_init_fm_radtorus) against the host functions that tests/test_setup.py
holds to the reference (kgpu_init_fm_torus_host, ..._radtorus_host).

Both paths run the same source for every point and cell; they differ only
in the math library behind sin, cos, tan, exp, log and pow (CUDA's are
within two units in the last place, glibc's within one).  The bounds:
 - metric tables: per point, the largest difference over the row's largest
   entry below 1e-12 (the trace-corrected Christoffels divide a difference
   of neighbouring sqrt(-g) by the cell size, which turns a last-place
   difference of sqrt(-g) into ~1e-14 of the row);
 - state: per variable |device - host| <= 1e-12 |host| + 1e-12 max|host|
   (the density near the torus surface is a power 2.25 of ln h - ln h_in,
   so its relative difference grows where that difference goes to zero,
   while its absolute difference shrinks);
 - ghost cells: both paths fill them with the same boundary kernels.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (48, 32, 16)


def metric_errors(a_tabs, b_tabs):
    out = {}
    for name, a, b in zip(("g", "G", "gKr", "gbx", "gby", "gbz", "Gbx", "Gby", "Gbz"), a_tabs, b_tabs):
        k = 64 if name == "gKr" else 20
        a, b = a.reshape(-1, k), b.reshape(-1, k)
        scale = np.abs(b).max(axis=1, keepdims=True) + 1e-300
        out[name] = float((np.abs(a - b) / scale).max())
    return out


def state_check(ud, pd, uh, ph, nv):
    worst = {}
    for name, d, h in (("p", pd, ph), ("u", ud, uh)):
        for v in range(nv):
            a, b = d[..., v], h[..., v]
            scale = np.abs(b).max()
            bound = 1e-12 * np.abs(b) + 1e-12 * scale
            assert (np.abs(a - b) <= bound).all(), (name, v, float(np.abs(a - b).max()), float(scale))
            nz = np.abs(b) > 1e-3 * scale
            worst[(name, v)] = float((np.abs(a - b)[nz] / np.abs(b)[nz]).max()) if nz.any() else 0.
    return worst


@pytest.mark.parametrize("radiation", [False, True])
def test_device_setup_matches_host_setup(kgpu, radiation):
    if radiation:
        dev, host = kgpu.radtorus(*SHAPE), kgpu.radtorus(*SHAPE, on_host=True)
    else:
        dev, host = kgpu.fm_torus(*SHAPE), kgpu.fm_torus(*SHAPE, on_host=True)
    err = metric_errors(dev.download_metric(), host.download_metric())
    print("metric, largest row-relative difference:", {k: f"{v:.1e}" for k, v in err.items()})
    for name, e in err.items():
        assert e < 1e-12, (name, e)
    ud, pd = dev.download_state()
    uh, ph = host.download_state()
    nv = 13 if radiation else 9
    # (a cell on different branches, torus or atmosphere, would differ by
    # the atmosphere's density, far above the bound)
    worst = state_check(ud, pd, uh, ph, nv)
    print("state, largest relative difference (|x| > 1e-3 max):", {f"{k[0]}{k[1]}": f"{v:.1e}" for k, v in worst.items()})
    # the first time step is a reduction of the wave speeds of that state
    assert abs(dev.tstepdenmax - host.tstepdenmax) <= 1e-12 * host.tstepdenmax
    dev.close()
    host.close()


def test_device_setup_time_full_torus(kgpu):
    """The 192x96x64 torus set up on the device in well under the time the
    host set-up takes (printed; the bound only guards against a host
    fallback)."""
    t0 = time.perf_counter()
    s = kgpu.fm_torus(192, 96, 64)
    t_dev = time.perf_counter() - t0
    s.close()
    print(f"device set-up of the 192x96x64 torus (context included): {t_dev:.3f} s")
    assert t_dev < 3.0
