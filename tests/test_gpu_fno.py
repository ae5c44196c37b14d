"""FNO kernels (csrc/fno.cu through include/he4_fno.h) against the float64
CPU oracle on the same BF16-rounded weights.

Tolerances: the GPU computes in FP32 (BF16 weights, FP32 activations and
accumulation), the oracle in float64 with the identical weight values, so
the forward output agrees to 1e-5 of its largest value and every parameter
gradient to 1e-4 of its largest entry.  Training is run-to-run identical
(fixed-order reductions)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import fno_oracle  # noqa: E402


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-30))


def make(pkg, seed=3, width=8):
    spec = pkg.fno.FnoSpec(n=16, width=width, modes=(4, 4, 4), layers=3)
    p = pkg.fno.init_params(spec, seed)
    for k in p:
        if k.startswith("R"):
            p[k] = p[k] * 40.0
    return spec, p


def oracle_params(net):
    """the values the kernels use: BF16 weights, FP32 biases"""
    wb, wm = net.get_params("bf16"), net.get_params("master")
    return {k: (wm[k] if k.endswith("_b") or (k.startswith("b") and k[1:].isdigit()) else wb[k]) for k in wb}


@pytest.mark.parametrize("width", [8, 16, 32])
def test_fno_forward_backward_against_oracle(pkg, width):
    """width 8: CUDA-core pointwise layers; 16 and 32: the tensor-core
    layers (BF16 mma.sync with three-piece BF16 activations)."""
    import torch
    spec, p = make(pkg, width=width)
    net = pkg.fno.Fno(spec, p)
    rng = np.random.default_rng(5)
    B = 2
    x = rng.standard_normal((B, spec.cin, spec.P)).astype(np.float32)
    t = rng.standard_normal((B, spec.cout, spec.P)).astype(np.float32)
    xd = torch.from_numpy(x).cuda().reshape(-1)
    td = torch.from_numpy(t).cuda().reshape(-1)
    y = net.forward(xd, B)
    gy = torch.empty_like(y)
    loss = net.loss(y, td, gy)
    yh = y.cpu().numpy().reshape(B, spec.cout, spec.P)
    gyh = gy.cpu().numpy().reshape(B, spec.cout, spec.P)
    net.backward(gy)
    torch.cuda.synchronize()
    o = fno_oracle.FnoOracle(spec, oracle_params(net))
    yo = o.forward(x.astype(np.float64))
    assert rel(yh, yo) < 1e-5
    lo, go = o.loss(yo, t.astype(np.float64))
    assert abs(float(loss[0].item()) - lo) <= 1e-5 * lo
    assert rel(gyh, go) < 1e-5
    g_or = o.backward(go)
    g_gpu = net.get_params("grad")
    for k in g_or:
        e = rel(g_gpu[k], g_or[k])
        assert e < 1e-4, (k, e)


def test_fno_training_reduces_loss_and_is_reproducible(pkg):
    import torch
    spec, p = make(pkg, seed=7)
    rng = np.random.default_rng(9)
    B = 2
    x = torch.from_numpy(rng.standard_normal((B, spec.cin, spec.P)).astype(np.float32)).cuda().reshape(-1)
    # a smooth target the network can fit: a fixed linear map of the input
    t = (0.5 * x.reshape(B, spec.cin, spec.P)[:, :2] - 0.2 * x.reshape(B, spec.cin, spec.P)[:, 2:3]).contiguous()
    t = t.reshape(-1)
    losses = []
    for run in range(2):
        net = pkg.fno.Fno(spec, p)
        ls = [float(net.train_step(x, t, B, lr=3e-3)[0].item()) for _ in range(80)]
        losses.append(ls)
    assert losses[0] == losses[1]
    assert losses[0][-1] < 0.4 * losses[0][0]


def test_grid_transfer_kernels(pkg):
    import torch
    net_lib = pkg.fno._fno_lib()
    import ctypes as C
    nf, f = 32, 4
    nc = nf // f
    rng = np.random.default_rng(2)
    psi = rng.standard_normal((nf, nf, nf)) + 1j * rng.standard_normal((nf, nf, nf))
    src = torch.from_numpy(psi.view(np.float64).reshape(-1).copy()).cuda()
    dst = torch.zeros(2 * nc ** 3, dtype=torch.float32, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert net_lib.he4_fno_restrict(C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()), nf, f, 1, 2.0, s) == 0
    want = psi.reshape(nc, f, nc, f, nc, f).mean(axis=(1, 3, 5)) * 2.0
    got = dst.cpu().numpy().reshape(2, nc, nc, nc)
    assert np.allclose(got[0], want.real, atol=1e-5) and np.allclose(got[1], want.imag, atol=1e-5)
    # prolongation of a constant coarse field adds that constant everywhere
    cst = torch.ones(2 * nc ** 3, dtype=torch.float32, device="cuda")
    out = torch.zeros(2 * nf ** 3, dtype=torch.float64, device="cuda")
    assert net_lib.he4_fno_prolong_add(C.c_void_p(cst.data_ptr()), C.c_void_p(out.data_ptr()), nf, f, 0.5, s) == 0
    assert np.allclose(out.cpu().numpy(), 0.5)
    # coarse deposit: every particle inside the box is counted once
    npar = 1000
    r = rng.uniform(-9.9, 9.9, (3, npar))
    rd = torch.from_numpy(r.reshape(-1).copy()).cuda()
    den = torch.zeros(nc ** 3, dtype=torch.float32, device="cuda")
    assert net_lib.he4_fno_deposit(C.c_void_p(rd.data_ptr()), npar, C.c_void_p(den.data_ptr()), nc, 10.0, 1.0,
                                   s) == 0
    hc = 20.0 / nc
    assert abs(float(den.sum().item()) * hc ** 3 - 1.0) < 1e-5
