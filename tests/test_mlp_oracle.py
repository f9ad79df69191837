"""The NumPy oracle of the learned-guess network: analytic gradient against central finite
differences (CPU), so that it can judge the GPU training kernels."""
import numpy as np

import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = np.zeros(mo.NPAR)
    w[:mo.NTRAIN] = rng.normal(0, 0.4, mo.NTRAIN)
    w[mo.OMU:mo.OSD] = [40.0, -3.0, -2.0, 0.015]
    w[mo.OSD:mo.OYMU] = [10.0, 2.0, 1.5, 0.003]
    w[mo.OYMU], w[mo.OYSD] = -0.5, 0.8
    x = np.stack([rng.uniform(20, 60, 64), rng.uniform(-8, 1, 64), rng.uniform(-4, 0, 64),
                  rng.uniform(0.01, 0.02, 64)], 1)
    y = rng.normal(-0.5, 0.8, 64)
    loss, g = mo.loss_grad(w, x, y)
    idx = list(range(0, 128, 9)) + list(range(128, 160, 5)) + list(range(160, 1184, 37)) + \
        list(range(1184, 1249, 7)) + [1248]
    for p in idx:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[p] += h
        wm[p] -= h
        fd = (mo.loss_grad(wp, x, y)[0] - mo.loss_grad(wm, x, y)[0]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 + 1e-5 * abs(g[p]), (p, fd, g[p])
    assert loss > 0
