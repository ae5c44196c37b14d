"""Fourier neural operator coarse propagator (host side of include/he4_fno.h).

The network maps the restricted state of a droplet + impurity system on an
n^3 grid -- channels (Re psi, Im psi, impurity density) -- to the change of
(Re psi, Im psi) over one coarse step:

    h0      = P a                          (lifting, cin -> width)
    h_{l+1} = act(W_l h_l + b_l + K_l h_l)  l = 0..L-1, no act after the last
    q       = GELU(Q1 h_L + c1)
    y       = Q2 q + c2                    (width -> 2)

with K_l h = F^-1 (R_l . F h) restricted to mx * my * mz modes.  Every step
of the forward and backward passes is a kernel of libhe4b200.so; torch
tensors only hold device memory.  Weights: FP32 master copies (updated by
the Adam kernel) and the BF16 copies the kernels read.
"""
import ctypes as C
import math

import numpy as np

from .host import load_library, _check


def _fno_lib():
    L = load_library()
    if getattr(L, "_fno_ready", False):
        return L
    vp, i32, i64, f32 = C.c_void_p, C.c_int32, C.c_int64, C.c_float
    L.he4_fno_contract.argtypes = [vp, vp, vp, i32, i32, i32, i32, i32, i32, i32, vp]
    L.he4_fno_mix.argtypes = [vp, vp, vp, i32, i32, i32, i32, vp]
    L.he4_fno_mix_bwd.argtypes = [vp, vp, vp, vp, vp, i32, i32, i32, i32, vp]
    L.he4_fno_pointwise.argtypes = [vp, vp, vp, vp, vp, vp, i32, i32, i32, i64, i32, vp]
    L.he4_fno_pointwise_bwd.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, i32, i64, i32, vp]
    L.he4_fno_pointwise_work.argtypes = [i32, i32, i32, i64]
    L.he4_fno_pointwise_work.restype = i64
    L.he4_fno_loss.argtypes = [vp, vp, vp, vp, i64, vp, vp]
    L.he4_fno_adam.argtypes = [vp, vp, vp, vp, vp, i64, f32, f32, f32, f32, i32, vp]
    L.he4_fno_to_bf16.argtypes = [vp, vp, i64, vp]
    L.he4_fno_restrict.argtypes = [vp, vp, i32, i32, i32, f32, vp]
    L.he4_fno_prolong_add.argtypes = [vp, vp, i32, i32, f32, vp]
    L.he4_fno_deposit.argtypes = [vp, i32, vp, i32, C.c_double, f32, vp]
    L.he4_parareal_correct.argtypes = [vp, vp, vp, vp, i64, i32, vp, vp, vp]
    L._fno_ready = True
    return L


LOSS_WORK = 1024


def mode_freqs(m, n):
    """Frequencies kept along a y or z axis: the m lowest |k| (0..m/2-1 and
    n-m/2..n-1)."""
    h = m // 2
    return np.array(list(range(h)) + list(range(n - (m - h), n)))


def dft_matrices(n, mx, my, mz):
    """The truncated transforms as complex matrices (numpy complex128):
    forward Fx [mx][n], Fy [my][n], Fz [mz][n] (exp(-2 pi i k j / n)),
    inverse Gz [n][mz], Gy [n][my] (exp(+...)) and Gx [n][mx] with the
    Hermitian weights (1 for kx = 0, 2 otherwise) and the 1/n^3 norm, whose
    output is taken as a real part."""
    j = np.arange(n)
    kx = np.arange(mx)
    ky = mode_freqs(my, n)
    kz = mode_freqs(mz, n)
    Fx = np.exp(-2j * np.pi * np.outer(kx, j) / n)
    Fy = np.exp(-2j * np.pi * np.outer(ky, j) / n)
    Fz = np.exp(-2j * np.pi * np.outer(kz, j) / n)
    Gz = np.exp(2j * np.pi * np.outer(j, kz) / n)
    Gy = np.exp(2j * np.pi * np.outer(j, ky) / n)
    wx = np.where(kx == 0, 1.0, 2.0)
    Gx = np.exp(2j * np.pi * np.outer(j, kx) / n) * wx[None, :] / float(n) ** 3
    return {"Fx": Fx, "Fy": Fy, "Fz": Fz, "Gz": Gz, "Gy": Gy, "Gx": Gx}


class FnoSpec:
    def __init__(self, n=64, width=32, modes=(12, 12, 12), layers=4, cin=3, cout=2):
        self.n, self.width, self.layers, self.cin, self.cout = n, width, layers, cin, cout
        self.mx, self.my, self.mz = modes
        if not (self.mx <= n // 2 and self.my <= n and self.mz <= n):
            raise ValueError("too many modes for the grid")
        self.M = self.mx * self.my * self.mz
        self.P = n ** 3

    def param_shapes(self):
        """(name, shape, is_bias) in storage order; spectral weights are
        complex [cin][cout][M] stored as 2 floats per entry."""
        C, L = self.width, self.layers
        out = [("P_W", (C, self.cin)), ("P_b", (C,))]
        for l in range(L):
            out += [(f"R{l}", (C, C, self.M, 2)), (f"W{l}", (C, C)), (f"b{l}", (C,))]
        out += [("Q1_W", (C, C)), ("Q1_b", (C,)), ("Q2_W", (self.cout, C)), ("Q2_b", (self.cout,))]
        return out


def init_params(spec, seed=0):
    """Seeded initial weights (uniform +-1/sqrt(fan_in) for pointwise layers,
    uniform [0, 1/width^2) scale for the spectral weights), as a dict of
    float64 numpy arrays."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in spec.param_shapes():
        if name.startswith("R"):
            p[name] = rng.uniform(0, 1, shape) / (spec.width * spec.width)
        elif name.endswith("_b") or (name.startswith("b") and name[1:].isdigit()):
            fan = spec.cin if name == "P_b" else spec.width
            p[name] = rng.uniform(-1, 1, shape) / math.sqrt(fan)
        else:
            p[name] = rng.uniform(-1, 1, shape) / math.sqrt(shape[1])
    return p


class Fno:
    """Device-resident FNO: parameters, Adam state, activations kept for the
    backward pass, and the forward / backward / train-step orchestration."""

    def __init__(self, spec, params=None, seed=0, device=0, stream=None):
        import torch
        self.torch = torch
        self.spec = spec
        self.dev = torch.device("cuda", device)
        self.L = _fno_lib()
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.dev)
        self.sp = C.c_void_p(self.stream.cuda_stream)
        # flat parameter storage, every entry starting at an even float offset
        self.offsets = {}
        off = 0
        for name, shape in spec.param_shapes():
            size = int(np.prod(shape))
            self.offsets[name] = (off, shape, size)
            off += size + (size & 1)
        self.nparam = off
        f32 = torch.float32
        self.master = torch.zeros(off, dtype=f32, device=self.dev)
        self.bf16 = torch.zeros(off, dtype=torch.int16, device=self.dev)
        self.grad = torch.zeros(off, dtype=f32, device=self.dev)
        self.m = torch.zeros(off, dtype=f32, device=self.dev)
        self.v = torch.zeros(off, dtype=f32, device=self.dev)
        self.step_count = 0
        self.set_params(params if params is not None else init_params(spec, seed))
        mats = dft_matrices(spec.n, spec.mx, spec.my, spec.mz)
        self.mat = {}
        for k, a in mats.items():
            self.mat[k] = self._cmat(a)
            self.mat[k + "H"] = self._cmat(a.conj().T)
        self.acts = None
        self.batch = 0
        self.launches = 1  # kernels launched by this object (the BF16 copy above)

    # -- storage helpers ----------------------------------------------------
    def _cmat(self, a):
        t = np.stack([a.real, a.imag], axis=-1).astype(np.float32)
        return self.torch.from_numpy(np.ascontiguousarray(t)).to(self.dev)

    def _p(self, t):
        return C.c_void_p(t.data_ptr())

    def _at(self, buf, name):
        off, _, _ = self.offsets[name]
        return C.c_void_p(buf.data_ptr() + off * buf.element_size())

    def set_params(self, params):
        host = np.zeros(self.nparam, dtype=np.float32)
        for name, (off, shape, size) in self.offsets.items():
            host[off:off + size] = np.asarray(params[name], dtype=np.float32).reshape(-1)
        self.master.copy_(self.torch.from_numpy(host).to(self.dev))
        if hasattr(self, "launches"):
            self.launches += 1
        _check(self.L.he4_fno_to_bf16(self._p(self.master), self._p(self.bf16), self.nparam, self.sp),
               "he4_fno_to_bf16")

    def get_params(self, which="master"):
        """Parameters as float64 numpy arrays ('master', 'bf16' (the values
        the kernels use) or 'grad')."""
        if which == "bf16":
            raw = self.bf16.cpu().numpy().view(np.uint16).astype(np.uint32) << 16
            flat = raw.view(np.float32).astype(np.float64)
        else:
            flat = (self.master if which == "master" else self.grad).cpu().numpy().astype(np.float64)
        return {n: flat[o:o + s].reshape(sh) for n, (o, sh, s) in self.offsets.items()}

    def _alloc(self, batch):
        if self.acts is not None and self.batch == batch:
            return
        t, s = self.torch, self.spec
        f = dict(dtype=t.float32, device=self.dev)
        B, Cw, P, n = batch, s.width, s.P, s.n
        self.acts = {
            "h": [t.empty(B * Cw * P, **f) for _ in range(s.layers + 1)],
            "pre": [t.empty(B * Cw * P, **f) for _ in range(s.layers)],
            "V": [t.empty(B * Cw * s.M * 2, **f) for _ in range(s.layers)],
            "qpre": t.empty(B * Cw * P, **f),
            "q": t.empty(B * Cw * P, **f),
            "y": t.empty(B * s.cout * P, **f),
            "u": t.empty(B * Cw * P, **f),
            "s1": t.empty(B * Cw * n * n * s.mx * 2, **f),
            "s2": t.empty(B * Cw * n * s.my * s.mx * 2, **f),
            "s3": t.empty(B * Cw * s.M * 2, **f),
            "g1": t.empty(B * Cw * P, **f),
            "g2": t.empty(B * Cw * P, **f),
            "gy": t.empty(B * s.cout * P, **f),
            "gR": t.empty(Cw * Cw * s.M * 2, **f),
            "work": t.empty(max(self.L.he4_fno_pointwise_work(B, Cw, Cw, P),
                                self.L.he4_fno_pointwise_work(B, s.cin, Cw, P)), **f),
            "loss_work": t.empty(LOSS_WORK, dtype=t.float64, device=self.dev),
            "loss": t.zeros(2, dtype=t.float64, device=self.dev),
        }
        self.batch = batch

    def _contract(self, x, y, mat, outer, J, K, inner, in_real=0, out_real=0, acc=0):
        self.launches += 1
        _check(self.L.he4_fno_contract(self._p(x), self._p(y), self._p(self.mat[mat]), outer, J, K, inner, in_real,
                                       out_real, acc, self.sp), "he4_fno_contract")

    def _spectral(self, h, V, R, out):
        """out = K h: truncated forward transform (V keeps the spectrum),
        mixing with R, truncated inverse."""
        s, B, a = self.spec, self.batch, self.acts
        n, Cw = s.n, s.width
        self._contract(h, a["s1"], "Fx", B * Cw * n * n, n, s.mx, 1, in_real=1)
        self._contract(a["s1"], a["s2"], "Fy", B * Cw * n, n, s.my, s.mx)
        self._contract(a["s2"], V, "Fz", B * Cw, n, s.mz, s.my * s.mx)
        _check(self.L.he4_fno_mix(self._p(V), R, self._p(a["s3"]), B, Cw, Cw, s.M, self.sp), "he4_fno_mix")
        self.launches += 1
        self._contract(a["s3"], a["s2"], "Gz", B * Cw, s.mz, n, s.my * s.mx)
        self._contract(a["s2"], a["s1"], "Gy", B * Cw * n, s.my, n, s.mx)
        self._contract(a["s1"], out, "Gx", B * Cw * n * n, s.mx, n, 1, out_real=1)

    def forward(self, x, batch):
        """x: float32 device tensor [batch][cin][n^3]; returns the
        [batch][cout][n^3] output (a view of internal storage)."""
        self._alloc(batch)
        s, a, L, B = self.spec, self.acts, self.L, batch
        self._x = x
        bf, ms = self.bf16, self.master
        self.launches += 3 + s.layers  # lift, layers, Q1, Q2 pointwise kernels
        _check(L.he4_fno_pointwise(self._p(x), self._at(bf, "P_W"), self._at(ms, "P_b"), None, None,
                                   self._p(a["h"][0]), B, s.cin, s.width, s.P, 0, self.sp), "lift")
        for l in range(s.layers):
            self._spectral(a["h"][l], a["V"][l], self._at(bf, f"R{l}"), a["u"])
            act = 1 if l < s.layers - 1 else 0
            _check(L.he4_fno_pointwise(self._p(a["h"][l]), self._at(bf, f"W{l}"), self._at(ms, f"b{l}"),
                                       self._p(a["u"]), self._p(a["pre"][l]), self._p(a["h"][l + 1]), B, s.width,
                                       s.width, s.P, act, self.sp), "fourier layer")
        _check(L.he4_fno_pointwise(self._p(a["h"][s.layers]), self._at(bf, "Q1_W"), self._at(ms, "Q1_b"), None,
                                   self._p(a["qpre"]), self._p(a["q"]), B, s.width, s.width, s.P, 1, self.sp), "Q1")
        _check(L.he4_fno_pointwise(self._p(a["q"]), self._at(bf, "Q2_W"), self._at(ms, "Q2_b"), None, None,
                                   self._p(a["y"]), B, s.width, s.cout, s.P, 0, self.sp), "Q2")
        return a["y"]

    def backward(self, gy):
        """Gradients of every parameter (into self.grad) from dL/dy
        (float32 device tensor shaped like the forward output; overwritten)."""
        s, a, L, B = self.spec, self.acts, self.L, self.batch
        bf, g, n, Cw = self.bf16, self.grad, s.n, s.width
        w = self._p(a["work"])
        # pointwise backward: act' (hidden layers and Q1), W^T g, weight-grad
        # partials and their sum; mixing backward: 2 kernels per layer
        self.launches += (3 + 4) + (s.layers - 1) * 4 + 3 + 2 * s.layers + 2
        _check(L.he4_fno_pointwise_bwd(self._p(gy), None, self._p(a["q"]), self._at(bf, "Q2_W"), self._p(a["g1"]),
                                       self._at(g, "Q2_W"), self._at(g, "Q2_b"), w, B, Cw, s.cout, s.P, 0, self.sp),
               "Q2 bwd")
        _check(L.he4_fno_pointwise_bwd(self._p(a["g1"]), self._p(a["qpre"]), self._p(a["h"][s.layers]),
                                       self._at(bf, "Q1_W"), self._p(a["g2"]), self._at(g, "Q1_W"),
                                       self._at(g, "Q1_b"), w, B, Cw, Cw, s.P, 1, self.sp), "Q1 bwd")
        gh, gnext = a["g2"], a["g1"]
        for l in reversed(range(s.layers)):
            act = 1 if l < s.layers - 1 else 0
            # gh -> gpre (also the gradient of the spectral branch); gnext = W^T gpre
            _check(L.he4_fno_pointwise_bwd(self._p(gh), self._p(a["pre"][l]), self._p(a["h"][l]),
                                           self._at(bf, f"W{l}"), self._p(gnext), self._at(g, f"W{l}"),
                                           self._at(g, f"b{l}"), w, B, Cw, Cw, s.P, act, self.sp), "layer bwd")
            # spectral branch: adjoint contractions in reverse order
            self._contract(gh, a["s1"], "GxH", B * Cw * n * n, n, s.mx, 1, in_real=1)
            self._contract(a["s1"], a["s2"], "GyH", B * Cw * n, n, s.my, s.mx)
            self._contract(a["s2"], a["s3"], "GzH", B * Cw, n, s.mz, s.my * s.mx)
            gV = a["s3"]
            # mixing: gradient of V into the spectrum buffer of layer l (no
            # longer needed), gradient of R into gR
            _check(L.he4_fno_mix_bwd(self._p(gV), self._p(a["V"][l]), self._at(bf, f"R{l}"), self._p(a["V"][l]),
                                     self._at(g, f"R{l}"), B, Cw, Cw, s.M, self.sp), "mix bwd")
            self._contract(a["V"][l], a["s2"], "FzH", B * Cw, s.mz, n, s.my * s.mx)
            self._contract(a["s2"], a["s1"], "FyH", B * Cw * n, s.my, n, s.mx)
            self._contract(a["s1"], gnext, "FxH", B * Cw * n * n, s.mx, n, 1, out_real=1, acc=1)
            gh, gnext = gnext, gh
        _check(L.he4_fno_pointwise_bwd(self._p(gh), None, self._p(self._x), self._at(bf, "P_W"), None,
                                       self._at(g, "P_W"), self._at(g, "P_b"), w, B, s.cin, Cw, s.P, 0, self.sp),
               "lift bwd")

    def loss(self, pred, target, grad=None):
        """Relative squared error sum (pred-target)^2 / sum target^2 on the
        device (a float64 tensor of 2: loss, sum target^2)."""
        a = self.acts
        self.launches += 3 if grad is not None else 2
        _check(self.L.he4_fno_loss(self._p(pred), self._p(target), self._p(grad) if grad is not None else None,
                                   self._p(a["loss"]), pred.numel(), self._p(a["loss_work"]), self.sp), "loss")
        return a["loss"]

    def train_step(self, x, target, batch, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        y = self.forward(x, batch)
        a = self.acts
        loss = self.loss(y, target, a["gy"])
        self.backward(a["gy"])
        self.step_count += 1
        self.launches += 1
        _check(self.L.he4_fno_adam(self._p(self.master), self._p(self.grad), self._p(self.m), self._p(self.v),
                                   self._p(self.bf16), self.nparam, lr, beta1, beta2, eps, self.step_count, self.sp),
               "adam")
        return loss

    def predict(self, x, batch=1):
        return self.forward(x, batch)
