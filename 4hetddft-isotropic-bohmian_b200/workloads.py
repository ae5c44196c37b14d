"""Synthetic droplet + impurity workloads (host-side input preparation).

The reference starts either from a density file and an unseeded rejection
sampler (readenc mode 0 + sorteo.f90:19-30) or from a wave function and
particle file (readenc mode 2, readenc.f90:96-114).  No input files ship with
it, so the workloads here build the mode-2 inputs synthetically and
reproducibly: a Fermi-profile droplet psi = sqrt(rho) and Gaussian-distributed
test particles drawn with numpy's PCG64 generator.

Configurations (sizes from the project's benchmark definition):
  c1  64^3, h=0.6 A, N=300 He, 256 particles, 100 m/s, 3 RK + 200 PC steps
  c2  128^3, h=0.4 A, N=1000 He, 4096 particles, 100 m/s, 2000 PC steps
  c3  256^3, h=0.4 A, N=5000 He, 16384 particles, 200 m/s, 5000 PC steps
All use core4='OTC', npd=7, icon=8 (periodic), ironx=1, Lambdah=0, impurity
mass 4.002602 amu and the Morse pair potential D=10 K, alpha=1.2/A,
r_e=5.5 A, capped below r_cutoff as Select_Pot does (V_impur.f90:84-935).
"""
import math

import numpy as np

from . import abi

KTOPS = 7.63822291          # 1 K^-1 in ps (DFT4He3d.f90:104)
RHO0 = 0.0218               # Fermi-profile saturation density, A^-3
AFERMI = 0.6                # Fermi-profile surface width, A
MORSE_D, MORSE_ALPHA, MORSE_RE = 10.0, 1.2, 5.5
MORSE_RCUT = 3.0


def morse(r, d=MORSE_D, a=MORSE_ALPHA, re=MORSE_RE):
    e = 1.0 - math.exp(-a * (r - re))
    return d * (e * e - 1.0)


CONFIGS = {
    "c1": dict(n=64, h=0.6, n4=300, npar=256, speed_ms=100.0, steps=203),
    "c2": dict(n=128, h=0.4, n4=1000, npar=4096, speed_ms=100.0, steps=2000),
    "c3": dict(n=256, h=0.4, n4=5000, npar=16384, speed_ms=200.0, steps=5000),
}


def make_params(n, h, npar, core4=abi.HE4_CORE_OTC, npd=7, pot=abi.HE4_POT_MORSE,
                nq=1000, ny=None, nz=None):
    p = abi.default_params()
    p.nx = n
    p.ny = ny or n
    p.nz = nz or n
    p.xmax = p.nx * h / 2.0
    p.ymax = p.ny * h / 2.0
    p.zmax = p.nz * h / 2.0
    p.npd = npd
    p.icon = 8
    p.core4 = core4
    p.n_par = npar
    p.ironx = 1
    p.mimpur = 4.002602
    p.pot_kind = pot
    p.morse_d, p.morse_alpha, p.morse_re = MORSE_D, MORSE_ALPHA, MORSE_RE
    p.r_cutoff = MORSE_RCUT
    p.umax = morse(MORSE_RCUT)
    p.nq = nq
    p.lambdah = 0.0
    return p


def grid_axes(p):
    hx = 2.0 * abs(p.xmax) / p.nx
    hy = 2.0 * abs(p.ymax) / p.ny
    hz = 2.0 * abs(p.zmax) / p.nz
    x = -p.xmax + hx * np.arange(p.nx)
    y = -p.ymax + hy * np.arange(p.ny)
    z = -p.zmax + hz * np.arange(p.nz)
    return x, y, z


def droplet_psi(p, n4):
    """psi = sqrt(rho), rho = RHO0/(1+exp((r-R)/AFERMI)), R = 2.22 n4^(1/3);
    complex128 array [nz][ny][nx]."""
    x, y, z = grid_axes(p)
    rr = np.sqrt(z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2)
    R = 2.22 * n4 ** (1.0 / 3.0)
    rho = RHO0 / (1.0 + np.exp((rr - R) / AFERMI))
    return np.sqrt(rho).astype(np.complex128)


def bubble_psi(p, n4, center, rb, wall=0.5, bump=0.3):
    """Droplet psi with a spherical cavity of radius rb around `center`:
    rho = drop(r) * g(|r - center|), g rising through 1/2 at rb over `wall`
    A with a `bump` overshoot (the density shell that forms around a
    solvated impurity).  complex128 array [nz][ny][nx]."""
    x, y, z = grid_axes(p)
    rr = np.sqrt(z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2)
    R = 2.22 * n4 ** (1.0 / 3.0)
    rho = RHO0 / (1.0 + np.exp((rr - R) / AFERMI))
    c = np.asarray(center, dtype=np.float64)
    s = np.sqrt((z[:, None, None] - c[2]) ** 2 + (y[None, :, None] - c[1]) ** 2 + (x[None, None, :] - c[0]) ** 2)
    g = (1.0 + bump * np.exp(-((s - rb - 4.0 * wall) / (2.0 * wall)) ** 2)) / (1.0 + np.exp(-(s - rb) / wall))
    return np.sqrt(rho * g).astype(np.complex128)


def particles(npar, seed, speed_ms, center=(0.0, 0.0, 2.0), width=0.3):
    """Test particles from an isotropic Gaussian of the given width around
    `center`, all moving toward the droplet centre (the origin) at speed_ms.
    Returns rimp, vimp as [3][npar] in internal units (A, A*K)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = np.asarray(center, dtype=np.float64)
    rimp = c[:, None] + width * rng.standard_normal((3, npar))
    direction = -c / np.linalg.norm(c)
    v = speed_ms / 100.0 * KTOPS            # m/s -> A/ps -> internal A*K
    vimp = np.repeat((direction * v)[:, None], npar, axis=1)
    return np.ascontiguousarray(rimp), np.ascontiguousarray(vimp)


def deltat_fs(fs=1.0):
    """Time step in internal units for `fs` femtoseconds (deltatps/7.63822291,
    DFT4He3d.f90:235)."""
    return fs * 1e-3 / KTOPS


def workload(name, seed=1234, **overrides):
    """(params, psi, rimp, vimp, steps) for a named configuration."""
    cfg = dict(CONFIGS[name])
    cfg.update(overrides)
    p = make_params(cfg["n"], cfg["h"], cfg["npar"])
    psi = droplet_psi(p, cfg["n4"])
    rimp, vimp = particles(cfg["npar"], seed, cfg["speed_ms"])
    return p, psi, rimp, vimp, cfg["steps"]


def family_member(name, seed):
    """One seeded member of a configuration's family (the training
    trajectories of the FNO coarse propagator): the same droplet and grid,
    the impurity cloud started at a random point 1.5-3 A off centre (random
    direction) with a speed drawn uniformly from [50, 200] m/s toward the
    centre.  Returns (params, psi, rimp, vimp)."""
    cfg = CONFIGS[name]
    rng = np.random.Generator(np.random.PCG64(seed))
    d = rng.standard_normal(3)
    d /= np.linalg.norm(d)
    center = d * rng.uniform(1.5, 3.0)
    speed = rng.uniform(50.0, 200.0)
    p = make_params(cfg["n"], cfg["h"], cfg["npar"])
    psi = droplet_psi(p, cfg["n4"])
    rimp, vimp = particles(cfg["npar"], seed, speed, center=tuple(center))
    return p, psi, rimp, vimp


def ensemble_member(i, seed0=0, npar=1024):
    """Member i of the batched ensemble: N log-uniform in [200, 3000], the
    smallest grid of 64^3, 96^3, 128^3 whose spacing 2.5 R / n stays within
    [0.4, 0.6] A (the spacing clamped to that range), impurity speed uniform
    in [50, 300] m/s, npar test particles 2 A off centre.  Returns (params,
    psi, rimp, vimp, n4)."""
    rng = np.random.Generator(np.random.PCG64(seed0 + i))
    n4 = int(round(math.exp(rng.uniform(math.log(200.0), math.log(3000.0)))))
    R = 2.22 * n4 ** (1.0 / 3.0)
    n = 128
    for cand in (64, 96, 128):
        if 2.5 * R / cand <= 0.6:
            n = cand
            break
    h = min(0.6, max(0.4, 2.5 * R / n))
    speed = rng.uniform(50.0, 300.0)
    p = make_params(n, h, npar)
    psi = droplet_psi(p, n4)
    rimp, vimp = particles(npar, seed0 + i, speed)
    return p, psi, rimp, vimp, n4
