"""Parareal time integration with a learned coarse propagator.

Fine propagator F: the predictor-corrector integrator of the library
(he4_run on a He4Step handle: 3 RK-Gill starter steps, then Hamming PC
steps) over one time slice.  The slices of one parareal iteration run as a
batch: one handle per slice, each on its own CUDA stream, driven from host
threads (ctypes releases the GIL), so their kernels share the GPU.

Coarse propagator G: the Fourier neural operator of fno.py on the state
restricted to an n^3 grid (f^3 block averages of psi; the test particles
deposited on that grid) predicts the change of psi over one slice; the
change is interpolated back (trilinear) and added to psi.  The test
particles move ballistically under G (r += v dt).

Iteration k (Gander and Vandewalle's form of Lions-Maday-Turinici):
    U_{n+1}^{k} = G(U_n^{k}) + F(U_n^{k-1}) - G(U_n^{k-1}),
slice n's fine run being skipped once slices 0..n are converged.  The
corrected psi is rescaled to the norm of its fine term, a projection on the
atom number the fine propagator conserves (in the spirit of the projected
parareal schemes for Hamiltonian problems of Dai, Le Bris, Legoll and
Maday); it leaves the fixed point unchanged and keeps the iterates
physical, without it G = identity drives psi out of the range the fine
solver integrates stably.  It stops
when the largest relative change of psi at the slice boundaries is below
`tol`, and at most after as many iterations as there are slices (then the
iterate equals the sequential fine solution).  With G = identity
(IdentityCoarse) it is the plain method the network is compared against.
"""
import threading
import time

import numpy as np

from . import fno as fno_mod
from . import abi
from .host import He4Error, He4Step, _check

PSI_SCALE = 1.0 / np.sqrt(0.0218)  # psi of the bulk liquid -> 1
OUT_GAIN = 20.0                      # one coarse step changes psi by a few %


class State:
    """psi (complex128 [nz][ny][nx]), rimp, vimp ([3][npar]) on the device."""

    def __init__(self, torch, shape, npar, dev):
        self.psi = torch.zeros(shape + (2,), dtype=torch.float64, device=dev)
        self.r = torch.zeros((3, npar), dtype=torch.float64, device=dev)
        self.v = torch.zeros((3, npar), dtype=torch.float64, device=dev)

    def copy_(self, o):
        self.psi.copy_(o.psi)
        self.r.copy_(o.r)
        self.v.copy_(o.v)
        return self

    def ptrs(self):
        return self.psi.data_ptr(), self.r.data_ptr(), self.v.data_ptr()


class FnoCoarse:
    """G(U) with the FNO on the (nf/f)^3 grid; dt_slice in internal units."""

    def __init__(self, net, params, f, dt_slice):
        import torch
        self.torch = torch
        self.net = net
        self.nf = params.nx
        self.f = f
        self.nc = self.nf // f
        if net.spec.n != self.nc or params.ny != self.nf or params.nz != self.nf:
            raise ValueError("FNO grid does not match the restricted solver grid")
        self.xmax = params.xmax
        self.hc = 2.0 * params.xmax / self.nc
        self.dt = dt_slice
        self.L = fno_mod._fno_lib()
        self.x = torch.empty(3 * self.nc ** 3, dtype=torch.float32, device=net.dev)

    def encode(self, psi_ptr, r_ptr, npar, out=None):
        """FNO input channels (Re psi, Im psi, particle density) of a state."""
        C = fno_mod.C
        x = self.x if out is None else out
        sp = self.net.sp
        nc3 = self.nc ** 3
        self.net.launches += 3  # restrict, deposit, deposit scaling
        _check(self.L.he4_fno_restrict(C.c_void_p(psi_ptr), C.c_void_p(x.data_ptr()), self.nf, self.f, 1,
                                       PSI_SCALE, sp), "he4_fno_restrict")
        _check(self.L.he4_fno_deposit(C.c_void_p(r_ptr), npar, C.c_void_p(x.data_ptr() + 8 * nc3), self.nc,
                                      self.xmax, self.hc ** 3, sp), "he4_fno_deposit")
        return x

    def __call__(self, src, dst):
        """dst = G(src) (States), on the network's stream."""
        C = fno_mod.C
        npar = src.r.shape[1]
        x = self.encode(src.psi.data_ptr(), src.r.data_ptr(), npar)
        y = self.net.predict(x, 1)
        dst.psi.copy_(src.psi)
        self.net.launches += 1
        _check(self.L.he4_fno_prolong_add(C.c_void_p(y.data_ptr()), C.c_void_p(dst.psi.data_ptr()), self.nf,
                                          self.f, 1.0 / (PSI_SCALE * OUT_GAIN), self.net.sp), "he4_fno_prolong_add")
        dst.r.copy_(src.r).add_(src.v, alpha=self.dt)
        dst.v.copy_(src.v)


class IdentityCoarse:
    """G = identity for psi, ballistic particles: the method without the
    network."""

    def __init__(self, dt_slice):
        self.dt = dt_slice

    def __call__(self, src, dst):
        dst.psi.copy_(src.psi)
        dst.r.copy_(src.r).add_(src.v, alpha=self.dt)
        dst.v.copy_(src.v)


# ---------------------------------------------------------------------------
# training data from the solver
# ---------------------------------------------------------------------------
def trajectory_pairs(pkg_workloads, params, psi0, r0, v0, coarse_steps, steps_per_coarse, dt, enc, net_dev,
                     form_params=None, handle=None):
    """Runs one trajectory and returns (inputs, targets) of its coarse steps
    as float32 device tensors [k][3][nc^3] and [k][2][nc^3].  handle: an
    existing He4Step of the same grid to run it on (its captured step
    graphs are reused across trajectories); otherwise one is created."""
    import torch
    p = form_params if form_params is not None else params
    own = handle is None
    g = He4Step(p) if own else handle
    try:
        g.set_state(psi0, r0, v0)
        nc3 = enc.nc ** 3
        xs, ys = [], []
        prev = None
        s = torch.cuda.ExternalStream(g.stream())
        for c in range(coarse_steps + 1):
            if c > 0:
                g.run(steps_per_coarse, dt)
            torch.cuda.current_stream().wait_stream(s)
            x = torch.empty(3 * nc3, dtype=torch.float32, device=net_dev)
            enc.encode(g.device_ptr("psi"), g.device_ptr("rimp"), g.npar, out=x)
            if prev is not None:
                xs.append(prev)
                ys.append(((x[:2 * nc3] - prev[:2 * nc3]) * OUT_GAIN).clone())
            prev = x
            s.wait_stream(torch.cuda.current_stream())
        torch.cuda.synchronize()
        return xs, ys
    finally:
        if own:
            g.close()


def train(net, xs, ys, steps, batch=2, lr=1e-3, lr_min=1e-5, seed=0, log=None):
    """Adam with a cosine learning-rate schedule over shuffled mini-batches;
    returns the per-step training losses (host floats, read every 10 steps)."""
    import torch
    rng = np.random.default_rng(seed)
    nc3 = net.spec.P
    xb = torch.empty(batch * 3 * nc3, dtype=torch.float32, device=net.dev)
    yb = torch.empty(batch * 2 * nc3, dtype=torch.float32, device=net.dev)
    losses = []
    order = []
    for it in range(steps):
        if len(order) < batch:
            order = list(rng.permutation(len(xs)))
        idx = [order.pop() for _ in range(batch)]
        for j, i in enumerate(idx):
            xb[j * 3 * nc3:(j + 1) * 3 * nc3].copy_(xs[i])
            yb[j * 2 * nc3:(j + 1) * 2 * nc3].copy_(ys[i])
        cur = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * it / max(1, steps)))
        loss = net.train_step(xb, yb, batch, lr=float(cur))
        if it % 10 == 0 or it == steps - 1:
            losses.append((it, float(loss[0].item())))
            if log:
                log(f"train step {it}: loss {losses[-1][1]:.4e} lr {cur:.2e}")
    return losses


def evaluate(net, xs, ys):
    """mean relative squared error of the network on (xs, ys)"""
    import torch
    vals = []
    for x, y in zip(xs, ys):
        pred = net.predict(x, 1)
        vals.append(float(net.loss(pred, y)[0].item()))
    return float(np.mean(vals))


# ---------------------------------------------------------------------------
# the parareal driver
# ---------------------------------------------------------------------------
class Parareal:
    """nslices slices of steps_per_slice fine steps each.  params: the fine
    solver's parameters (precision form included); coarse: FnoCoarse,
    IdentityCoarse or any callable G(src, dst)."""

    def __init__(self, params, nslices, steps_per_slice, dt, coarse, concurrent=None, renorm=True):
        import torch
        self.torch = torch
        self.p = params
        self.S = nslices
        self.steps = steps_per_slice
        self.dt = dt
        self.G = coarse
        self.renorm = renorm
        self.dev = torch.device("cuda", params.device)
        self.nconc = min(concurrent or nslices, nslices)
        self.handles = [He4Step(params) for _ in range(self.nconc)]
        self.L = fno_mod._fno_lib()
        shape = (params.nz, params.ny, params.nx)
        mk = lambda: State(torch, shape, params.n_par, self.dev)
        self.U = [mk() for _ in range(self.S + 1)]
        self.Gold = [mk() for _ in range(self.S + 1)]
        self.F = [mk() for _ in range(self.S + 1)]
        self.gtmp = mk()
        self.work = torch.empty(fno_mod.LOSS_WORK, dtype=torch.float64, device=self.dev)
        self.norms = torch.zeros((self.S + 1, 3, 4), dtype=torch.float64, device=self.dev)
        self.fine_steps = 0

    def close(self):
        for h in self.handles:
            h.close()
        self.handles = []

    def warm(self, psi0, r0, v0):
        """Captures the step graphs of every fine-propagator handle (the
        starter plus one PC step of each of the 30 buffer states) from the
        given state; he4_set_state puts the buffers back in allocation
        order, so the runs that follow replay these graphs.  Like an FFT
        plan, this is set-up work done once per handle."""
        torch = self.torch
        psi = torch.from_numpy(np.ascontiguousarray(psi0).view(np.float64).reshape(self.U[0].psi.shape)).to(self.dev)
        r = torch.from_numpy(np.ascontiguousarray(r0)).to(self.dev)
        v = torch.from_numpy(np.ascontiguousarray(v0)).to(self.dev)
        torch.cuda.synchronize(self.dev)
        for h in self.handles:
            h.set_state_device(psi.data_ptr(), r.data_ptr(), v.data_ptr())
            h.run(3 + 30, self.dt)
        torch.cuda.synchronize(self.dev)

    def _fine(self, slices):
        """F(U_n) -> F[n+1] for the given slices, concurrently."""
        torch = self.torch
        torch.cuda.synchronize(self.dev)
        errors = []

        def worker(w):
            try:
                h = self.handles[w]
                for n in slices[w::self.nconc]:
                    h.set_state_device(*self.U[n].ptrs())
                    h.run(self.steps, self.dt)
                    h.get_state_device(*self.F[n + 1].ptrs())
            except Exception as e:  # surfaced after the join
                errors.append(e)

        threads = [threading.Thread(target=worker, args=(w,)) for w in range(min(self.nconc, len(slices)))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        self.fine_steps += self.steps * len(slices)
        torch.cuda.synchronize(self.dev)

    def _correct(self, n):
        """U[n+1] = gtmp + F[n+1] - Gold[n+1]; norms of the change."""
        C = fno_mod.C
        sp = C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)
        for a, (gn, fi, go, u) in enumerate([(self.gtmp.psi, self.F[n + 1].psi, self.Gold[n + 1].psi,
                                              self.U[n + 1].psi),
                                             (self.gtmp.r, self.F[n + 1].r, self.Gold[n + 1].r, self.U[n + 1].r),
                                             (self.gtmp.v, self.F[n + 1].v, self.Gold[n + 1].v, self.U[n + 1].v)]):
            out = self.norms[n + 1, a]
            renorm = 1 if (a == 0 and self.renorm) else 0
            _check(self.L.he4_parareal_correct(C.c_void_p(gn.data_ptr()), C.c_void_p(fi.data_ptr()),
                                               C.c_void_p(go.data_ptr()), C.c_void_p(u.data_ptr()), u.numel(),
                                               renorm, C.c_void_p(out.data_ptr()),
                                               C.c_void_p(self.work.data_ptr()), sp), "he4_parareal_correct")

    def _sequential(self, start, resume=False):
        """Fallback: U[n+1] = F(U[n]) for n = start..S-1, one slice after
        the other on the first handle.  resume: the first handle has just
        integrated slice start-1 and still holds U[start] with its
        predictor-corrector histories; the slices then continue that run
        (one continuous integration, no starter steps at the boundaries)."""
        torch = self.torch
        torch.cuda.synchronize(self.dev)
        h = self.handles[0]
        for n in range(start, self.S):
            if not resume:
                h.set_state_device(*self.U[n].ptrs())
            h.run(self.steps, self.dt)
            h.get_state_device(*self.U[n + 1].ptrs())
            self.fine_steps += self.steps
        torch.cuda.synchronize(self.dev)

    def _rel_psi(self, a, b):
        """||a.psi - b.psi|| / ||a.psi|| on the device."""
        torch = self.torch
        num = torch.linalg.vector_norm(a.psi - b.psi)
        den = torch.linalg.vector_norm(a.psi)
        return float((num / torch.clamp(den, min=1e-300)).item())

    def run(self, psi0, r0, v0, tol=1e-6, max_iter=None, fallback=True, contraction=0.5, first_change_max=0.1,
            judge_first=True, judge_max=None, log=None):
        """Returns a dict: iterations, per-iteration max relative psi change,
        wall seconds (device-synchronised), fine steps executed, whether the
        iteration converged (change <= tol), and where the sequential
        fallback took over (exact_by_fallback: the result is the sequential
        fine solution because the fallback ran).  fallback: when an iteration does not
        shrink the change by `contraction`, or a fine run leaves the range
        the solver integrates, the remaining slices are integrated one after
        the other from the last exact boundary (the plain integrator is both
        the fallback and the judge of the coarse propagator).  The first
        iteration's change is the coarse propagator's error over one slice as
        the fine propagator judges it; above first_change_max the remaining
        iterations cannot reach `tol` in fewer fine sweeps than the slices
        left, so the fallback starts right away.  judge_first (with fallback):
        the first iteration integrates slice 0 alone and compares its end with
        the coarse prediction before integrating slices 1.. from predicted
        states; the coarse predictions of slices 1.. are made only once the
        judge accepts, so a rejected coarse step costs one coarse step and no
        speculative fine sweep: the run is the sequential integration.
        judge_max is the largest accepted coarse error over that slice; its
        default is tol, because the slices share one GPU here: a second
        iteration would already cost more fine steps than the sequential
        run, so speculation only pays when one iteration converges."""
        torch = self.torch
        max_iter = self.S if max_iter is None else max_iter
        self.fine_steps = 0  # counted per run
        t0 = time.perf_counter()
        self.U[0].psi.copy_(torch.from_numpy(np.ascontiguousarray(psi0).view(np.float64).reshape(
            self.U[0].psi.shape)))
        self.U[0].r.copy_(torch.from_numpy(np.ascontiguousarray(r0)))
        self.U[0].v.copy_(torch.from_numpy(np.ascontiguousarray(v0)))
        torch.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        # initial coarse sweep; with the judge first, only the prediction of
        # slice 0 is needed before the judge, the rest only if it accepts
        lazy = judge_first and fallback and self.S > 1
        for n in range(1 if lazy else self.S):
            self.G(self.U[n], self.U[n + 1])
            self.Gold[n + 1].copy_(self.U[n + 1])
        history = []
        k = 0
        converged = False
        diverged = False
        fallback_at = None
        while k < max_iter:
            k += 1
            try:
                if k == 1 and judge_first and fallback and self.S > 1:
                    self._fine([0])
                    err = self._rel_psi(self.F[1], self.Gold[1])
                    if log:
                        log(f"parareal judge: coarse step error over slice 0 {err:.3e}")
                    if err > (tol if judge_max is None else judge_max):
                        history.append(err)
                        self.U[1].copy_(self.F[1])
                        fallback_at = 1
                        self._sequential(1, resume=True)
                        break
                    for n in range(1, self.S):  # the rest of the coarse sweep
                        self.G(self.U[n], self.U[n + 1])
                        self.Gold[n + 1].copy_(self.U[n + 1])
                    self._fine(list(range(1, self.S)))
                else:
                    self._fine(list(range(k - 1, self.S)))
            except He4Error as e:
                if e.code != abi.HE4_E_NONFINITE:
                    raise
                diverged = True  # an iterate left the range the fine solver integrates
                if fallback:
                    fallback_at = k - 1
                    self._sequential(k - 1)
                break
            # slice k-1's boundary is now exact
            self.U[k].copy_(self.F[k])
            for n in range(k, self.S):
                self.G(self.U[n], self.gtmp)
                self._correct(n)
                self.Gold[n + 1].copy_(self.gtmp)
            if k < self.S:
                nrm = self.norms[k + 1:, 0].cpu().numpy()
                change = float(np.sqrt(np.max(nrm[:, 0] / np.maximum(nrm[:, 1], 1e-300))))
            else:
                change = 0.0
            history.append(change)
            if log:
                log(f"parareal iteration {k}: max relative psi change {change:.3e}")
            if change <= tol:
                converged = True
                break
            if fallback and k < self.S and ((k == 1 and change > first_change_max) or
                                            (k >= 2 and change > contraction * history[-2])):
                fallback_at = k
                self._sequential(k)
                break
        # every stream is idle here, so the interval between the two events
        # on the current stream spans all device work of the run
        torch.cuda.synchronize(self.dev)
        ev1.record()
        ev1.synchronize()
        wall = time.perf_counter() - t0
        device_s = ev0.elapsed_time(ev1) * 1e-3
        # converged: the iteration itself met tol.  A run that fell back to
        # the sequential integrator also ends on the exact fine solution,
        # but did not converge; exact_by_fallback says so.
        return {"iterations": k, "converged": converged, "exact_by_fallback": fallback_at is not None,
                "diverged": diverged,
                "fallback_at": fallback_at, "changes": history, "wall_s": wall, "device_s": device_s,
                "fine_steps": self.fine_steps}

    def final_state(self):
        return self.U[self.S]
