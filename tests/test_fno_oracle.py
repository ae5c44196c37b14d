"""The FNO oracle (CPU): analytic gradients against central finite
differences, and the truncated transforms against numpy's FFT."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import fno_oracle  # noqa: E402


class Spec:
    def __init__(self, n, width, modes, layers, cin=3, cout=2):
        self.n, self.width, self.layers, self.cin, self.cout = n, width, layers, cin, cout
        self.mx, self.my, self.mz = modes
        self.M = self.mx * self.my * self.mz
        self.P = n ** 3


def params_for(pkg, s, seed):
    spec = pkg.fno.FnoSpec(n=s.n, width=s.width, modes=(s.mx, s.my, s.mz), layers=s.layers, cin=s.cin,
                           cout=s.cout)
    p = pkg.fno.init_params(spec, seed)
    # spectral weights larger than the default so the spectral branch
    # carries a visible share of the gradient
    for k in p:
        if k.startswith("R"):
            p[k] = p[k] * 40.0
    return p


def test_dft_matrices_match_package(pkg):
    a = fno_oracle.dft_matrices(16, 4, 6, 4)
    b = pkg.fno.dft_matrices(16, 4, 6, 4)
    for k in a:
        assert np.array_equal(a[k], b[k])


def test_truncated_transform_against_numpy():
    n, mx, my, mz = 8, 3, 4, 4
    s = Spec(n, 1, (mx, my, mz), 1)
    o = fno_oracle.FnoOracle(s, {})
    rng = np.random.default_rng(0)
    h = rng.standard_normal((1, 1, n ** 3))
    V = o._fwd_spec(h).reshape(mz, my, mx)
    full = np.fft.rfftn(h.reshape(n, n, n))
    kz = fno_oracle.mode_freqs(mz, n)
    ky = fno_oracle.mode_freqs(my, n)
    assert np.allclose(V, full[np.ix_(kz, ky, np.arange(mx))], atol=1e-12)
    # a field made of retained modes (and their conjugates) survives the
    # truncated round trip exactly
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    f = np.cos(2 * np.pi * (2 * x + 1 * y - 1 * z) / n) + 0.5 * np.sin(2 * np.pi * (1 * x - 2 * y) / n) + 0.25
    g = f.reshape(1, 1, -1)
    back = o._inv_spec(o._fwd_spec(g))
    assert np.allclose(back, g, atol=1e-12)


def test_oracle_gradient_finite_differences(pkg):
    s = Spec(6, 4, (2, 2, 2), 2)
    p = params_for(pkg, s, 3)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, s.cin, s.P))
    t = rng.standard_normal((2, s.cout, s.P))
    o = fno_oracle.FnoOracle(s, p)
    y = o.forward(x)
    L0, gy = o.loss(y, t)
    g = o.backward(gy)

    def loss_at(pp):
        oo = fno_oracle.FnoOracle(s, pp)
        return oo.loss(oo.forward(x), t)[0]

    checked = 0
    for name in p:
        flat = p[name].reshape(-1)
        for idx in rng.choice(flat.size, size=min(3, flat.size), replace=False):
            eps = 1e-6
            pp = {k: v.copy() for k, v in p.items()}
            pp[name].reshape(-1)[idx] += eps
            lp = loss_at(pp)
            pp[name].reshape(-1)[idx] -= 2 * eps
            lm = loss_at(pp)
            fd = (lp - lm) / (2 * eps)
            an = g[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 + 1e-5 * abs(fd), (name, idx, fd, an)
            checked += 1
    assert checked > 20
