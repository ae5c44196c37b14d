"""CPU oracle of the FNO coarse propagator (test infrastructure only).

A float64 numpy restatement of the network that the CUDA kernels of
csrc/fno.cu evaluate (see fno.py for the architecture), with an analytic
backward pass.  The GPU forward and backward passes are checked against it
on the same (BF16-rounded) weights; the analytic gradients here are checked
against central finite differences.  The reference solver has no learned
component, so nothing of the reference is restated here: the truncated
transforms are the DFT matrices of fno.dft_matrices, rebuilt below.

Complex gradients follow the convention g = dL/dRe + i dL/dIm, for which a
complex-linear map y = A x has the adjoint g_x = A^H g_y, and a spectral
weight R in y = R x has g_R = conj(x) g_y.
"""
import math

import numpy as np
from scipy.special import erf


def mode_freqs(m, n):
    h = m // 2
    return np.array(list(range(h)) + list(range(n - (m - h), n)))


def dft_matrices(n, mx, my, mz):
    j = np.arange(n)
    kx = np.arange(mx)
    ky = mode_freqs(my, n)
    kz = mode_freqs(mz, n)
    wx = np.where(kx == 0, 1.0, 2.0)
    return {
        "Fx": np.exp(-2j * np.pi * np.outer(kx, j) / n),
        "Fy": np.exp(-2j * np.pi * np.outer(ky, j) / n),
        "Fz": np.exp(-2j * np.pi * np.outer(kz, j) / n),
        "Gz": np.exp(2j * np.pi * np.outer(j, kz) / n),
        "Gy": np.exp(2j * np.pi * np.outer(j, ky) / n),
        "Gx": np.exp(2j * np.pi * np.outer(j, kx) / n) * wx[None, :] / float(n) ** 3,
    }


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


class FnoOracle:
    """spec: n, width, mx, my, mz, layers, cin, cout (same meaning as
    fno.FnoSpec); params: dict of float64 arrays with fno's names/shapes."""

    def __init__(self, spec, params):
        self.s = spec
        self.p = params
        self.A = dft_matrices(spec.n, spec.mx, spec.my, spec.mz)

    def _R(self, l):
        r = self.p[f"R{l}"]
        return r[..., 0] + 1j * r[..., 1]  # [cin][cout][M]

    @staticmethod
    def _pw(W, b, x):
        # x [B][ci][P] -> [B][co][P]
        return np.einsum("oi,bip->bop", W, x) + b[None, :, None]

    def _fwd_spec(self, h):
        s, A = self.s, self.A
        B, Cw = h.shape[:2]
        n = s.n
        h5 = h.reshape(B, Cw, n, n, n)
        s1 = np.einsum("kx,bczyx->bczyk", A["Fx"], h5)
        s2 = np.einsum("jy,bczyk->bczjk", A["Fy"], s1)
        V = np.einsum("iz,bczjk->bcijk", A["Fz"], s2)
        return V.reshape(B, Cw, -1)

    def _inv_spec(self, W):
        s, A = self.s, self.A
        B, Cw = W.shape[:2]
        n = s.n
        W5 = W.reshape(B, Cw, s.mz, s.my, s.mx)
        t2 = np.einsum("zi,bcijk->bczjk", A["Gz"], W5)
        t1 = np.einsum("yj,bczjk->bczyk", A["Gy"], t2)
        u = np.einsum("xk,bczyk->bczyx", A["Gx"], t1).real
        return u.reshape(B, Cw, -1)

    def _fwd_spec_adj(self, gV):
        """adjoint of _fwd_spec (complex spectrum gradient -> real field)"""
        s, A = self.s, self.A
        B, Cw = gV.shape[:2]
        n = s.n
        g5 = gV.reshape(B, Cw, s.mz, s.my, s.mx)
        g2 = np.einsum("iz,bcijk->bczjk", A["Fz"].conj(), g5)
        g1 = np.einsum("jy,bczjk->bczyk", A["Fy"].conj(), g2)
        gh = np.einsum("kx,bczyk->bczyx", A["Fx"].conj(), g1).real
        return gh.reshape(B, Cw, -1)

    def _inv_spec_adj(self, gu):
        """adjoint of _inv_spec (real field gradient -> complex spectrum)"""
        s, A = self.s, self.A
        B, Cw = gu.shape[:2]
        n = s.n
        g5 = gu.reshape(B, Cw, n, n, n)
        g1 = np.einsum("xk,bczyx->bczyk", A["Gx"].conj(), g5)
        g2 = np.einsum("yj,bczyk->bczjk", A["Gy"].conj(), g1)
        gW = np.einsum("zi,bczjk->bcijk", A["Gz"].conj(), g2)
        return gW.reshape(B, Cw, -1)

    def forward(self, x):
        """x [B][cin][n^3] -> y [B][cout][n^3]; keeps the activations."""
        p, s = self.p, self.s
        c = {"x": x}
        h = self._pw(p["P_W"], p["P_b"], x)
        c["h"], c["pre"], c["V"] = [h], [], []
        for l in range(s.layers):
            V = self._fwd_spec(h)
            Wm = np.einsum("bim,iom->bom", V, self._R(l))
            u = self._inv_spec(Wm)
            pre = self._pw(p[f"W{l}"], p[f"b{l}"], h) + u
            h = gelu(pre) if l < s.layers - 1 else pre
            c["V"].append(V)
            c["pre"].append(pre)
            c["h"].append(h)
        qpre = self._pw(p["Q1_W"], p["Q1_b"], h)
        q = gelu(qpre)
        y = self._pw(p["Q2_W"], p["Q2_b"], q)
        c.update(qpre=qpre, q=q, y=y)
        self.c = c
        return y

    def backward(self, gy):
        """parameter gradients (dict) from dL/dy of the last forward"""
        p, s, c = self.p, self.s, self.c
        g = {}
        g["Q2_W"] = np.einsum("bop,bip->oi", gy, c["q"])
        g["Q2_b"] = gy.sum(axis=(0, 2))
        gq = np.einsum("oi,bop->bip", p["Q2_W"], gy) * gelu_grad(c["qpre"])
        g["Q1_W"] = np.einsum("bop,bip->oi", gq, c["h"][s.layers])
        g["Q1_b"] = gq.sum(axis=(0, 2))
        gh = np.einsum("oi,bop->bip", p["Q1_W"], gq)
        for l in reversed(range(s.layers)):
            gpre = gh * gelu_grad(c["pre"][l]) if l < s.layers - 1 else gh
            hl = c["h"][l]
            g[f"W{l}"] = np.einsum("bop,bip->oi", gpre, hl)
            g[f"b{l}"] = gpre.sum(axis=(0, 2))
            gnext = np.einsum("oi,bop->bip", p[f"W{l}"], gpre)
            gWm = self._inv_spec_adj(gpre)
            V = c["V"][l]
            gR = np.einsum("bim,bom->iom", V.conj(), gWm)
            g[f"R{l}"] = np.stack([gR.real, gR.imag], axis=-1)
            gV = np.einsum("bom,iom->bim", gWm, self._R(l).conj())
            gnext = gnext + self._fwd_spec_adj(gV)
            gh = gnext
        g["P_W"] = np.einsum("bop,bip->oi", gh, c["x"])
        g["P_b"] = gh.sum(axis=(0, 2))
        return g

    def loss(self, y, t):
        """relative squared error and its gradient"""
        t2 = float(np.sum(t * t))
        d = y - t
        return float(np.sum(d * d)) / t2, 2.0 * d / t2
