"""The radiation constants of the product (unit conversions for the
black-hole mass, KORAL's solver defaults) equal those of the reference
build bit for bit: the implicit solve's arithmetic depends on them.  The
product's Kerr-Schild metric agrees with the reference's to rounding."""
import numpy as np
import pytest

from conftest import ref_lib_available

pytestmark = pytest.mark.skipif(not ref_lib_available("libkref_radcells.so"),
                                reason="reference radiating-cells build not present")


def test_rad_params_equal_reference(kgpu, oracle):
    c = oracle.RefRadCells().consts
    rp = kgpu.rad_params(mass=10.0, gamma=13.0 / 9.0)
    pairs = [(rp.kb, c[0]), (rp.mp, c[1]), (rp.sigma, c[2]), (rp.mu, c[3]), (rp.ggg, c[4]), (rp.ccc, c[5]),
             (rp.masscm, c[6]), (rp.gammamaxrad, c[7]), (rp.eradfloor, c[8]), (rp.eps, c[9]), (rp.conv, c[10]),
             (rp.entrconv, c[11]), (rp.maxiter, c[12]), (rp.dampfac, c[13]), (rp.maxdown, c[14]),
             (rp.maxup, c[15]), (rp.maxdamping, c[16]), (rp.threshold, c[17]), (rp.gammasmalllimit, c[18]),
             (rp.numepsilon, c[19]), (rp.eerhoratiomin, c[20]), (rp.eerhoratiomax, c[21]),
             (rp.eeuuratiomin, c[22]), (rp.eeuuratiomax, c[23])]
    for i, (a, b) in enumerate(pairs):
        assert a == b, (i, a, b)


def test_ks_metric_close_to_reference(kgpu, oracle):
    ref = oracle.RefRadCells()
    rng = np.random.default_rng(3)
    for _ in range(50):
        r, th = np.exp(rng.uniform(np.log(2.), np.log(100.))), rng.uniform(0.1, np.pi - 0.1)
        g, G = kgpu.ks_metric(0.9, r, th)
        gr, Gr = ref.metric(r, th)
        assert np.allclose(g, gr, rtol=1e-13, atol=1e-13 * np.abs(gr).max())
        assert np.allclose(G, Gr, rtol=1e-13, atol=1e-13 * np.abs(Gr).max())
