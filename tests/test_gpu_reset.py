"""Restarting training from a written model (B200 required).

gs_write_gaussians + gs_reset_moments + the iteration counter put a trainer
back in the state setup() leaves: the same steps then give the same
parameters, SH coefficients and Adam moments, bit for bit.  The benchmark
starts every timed segment this way."""
import numpy as np
import pytest

from test_gpu_parity import assert_bits, config0, make

pytestmark = pytest.mark.gpu


def test_write_and_reset_moments_restart_training_exactly():
    params, sh, cams, rgbs = config0()
    t, _, _ = make(params, sh, cams, rgbs, dict(shDeg=2), radius=1.0)

    def run():
        t.iter = 2000
        for _ in range(3):
            t.stepBatch([0])
        g = t.readGaussians()
        return g["data"].copy(), g["sh"].copy(), [x.copy() for x in t.readMoments()]

    p1, s1, m1 = run()
    assert not np.array_equal(p1, params)
    assert np.any(m1[0] != 0)
    # training on from here leaves other moments; the reset returns to setup's
    t.stepBatch([0])
    t.writeGaussians(params, sh)
    t.resetMoments()
    assert all(not np.any(x) for x in t.readMoments())
    p2, s2, m2 = run()
    assert_bits(p2, p1, "params after the restart")
    assert_bits(s2, s1, "SH after the restart")
    for a, b, name in zip(m2, m1, ("m", "v", "SH m", "SH v")):
        assert_bits(a, b, f"Adam {name} after the restart")
