"""The spherical bubble radius of the oracle (CPU): the search half of
Bubble_Radius_esferic (bubble_radius_esferic.f90:63-132) on analytic radial
profiles, its Lcontrol flags, and the binning half on a small grid against
an independent numpy histogram."""
import numpy as np
import pytest
from scipy.optimize import brentq


def shell(r, rb=4.0, wall=0.5, bump=0.3, rho0=0.0218):
    """A cavity of radius rb with a density overshoot past the wall."""
    return rho0 * (1.0 + bump * np.exp(-((r - rb - 2.0) / 1.0) ** 2)) / (1.0 + np.exp(-(r - rb) / wall))


def test_search_matches_analytic_half_maximum(ora):
    nr, rmax = 501, 30.0
    dr = rmax / (nr - 1)
    r = np.arange(nr) * dr
    f = shell(r)
    xms = np.array([0.4, 0.5, 1.2])
    xnorm = 4 * np.pi * np.sum(r ** 2 * f) * dr * 0.97  # normalisation away from 1
    rb, flags, ir, rr, d = ora.bubble_search(f, dr, xnorm, xms)
    assert flags == (True, True)
    assert np.allclose(rr, r)
    # normalised by xnorm / (4 pi sum r^2 denr dr)
    assert np.allclose(d, f * 0.97, rtol=1e-12)
    # the bin of the first maximum past max(xms), r >= 2, denr >= 0.75 max
    j = int(np.argmax(f))
    assert ir == j + 1
    half = f[j] * 0.5
    want = brentq(lambda x: shell(x) - half, 1.0, r[j])
    assert abs(rb - want) < 1e-5


def test_search_flags(ora):
    nr, dr = 201, 0.1
    r = np.arange(nr) * dr
    xms = np.array([0.3, 0.3, 0.3])

    def search(f, xms=xms, scale=1.0):
        # xnorm equal to the radial integral times `scale`
        return ora.bubble_search(f, dr, scale * 4 * np.pi * np.sum(r ** 2 * f) * dr, xms)

    # monotone density: no maximum -> (False, False)
    rb, flags, ir, _, _ = search(0.02 * r / r[-1])
    assert flags == (False, False) and ir == 0
    # the only maximum lies inside max(xms): skipped -> (False, False)
    f = shell(r, rb=4.0)
    assert search(f)[1] == (True, True)
    assert search(f, xms=np.array([9.0, 0.0, 0.0]))[1] == (False, False)
    # a maximum below 0.75 of the largest value is skipped; the later one is taken
    g = shell(r, rb=4.0) + 0.05 * np.exp(-((r - 15.0) / 0.8) ** 2)
    _, flags, ir, _, _ = search(g)
    assert flags[0] and abs(r[ir - 1] - 15.0) < 0.5
    # 0.75 of the maximum is taken before the normalisation (:66 then :75):
    # a density normalised to half its integral finds no maximum at all
    assert search(f, scale=0.5)[1] == (False, False)
    # a maximum in bin nr-1 counts as not found (bubble_radius_esferic.f90:87)
    h = np.exp(-((r - r[-2]) / 0.3) ** 2) + 1e-3
    assert search(h)[1] == (False, False)
    # a maximum but no half-maximum crossing above max(xms): (True, False)
    k = 0.02 * (1.0 + 0.1 * np.exp(-((r - 8.0) / 1.0) ** 2))
    _, flags, ir, _, _ = search(k)
    assert flags == (True, False) and ir > 0


@pytest.fixture(scope="module")
def small(pkg, ora):
    p = pkg.workloads.make_params(48, 0.6, 128)
    center = (-0.5, -0.7, -1.6)
    # a drop of 100 atoms (R = 10.3 A) inside the 28.8 A box
    psi = pkg.workloads.bubble_psi(p, 100, center, 3.5)
    r, v = pkg.workloads.particles(128, 5, 100.0, center=center)
    o = ora.Oracle(p)
    o.set_state(psi, r, v)
    return p, psi, r, o


def test_binning_against_numpy(pkg, small):
    p, psi, r, o = small
    nr = 301
    out = o.bubble_radius(nr)
    x, y, z = pkg.workloads.grid_axes(p)
    hx = 2 * p.xmax / p.nx
    ip = [int(1.5 + (np.mean(r[c]) + p.xmax) / hx) for c in range(3)]
    xp, yp, zp = x[ip[0] - 1], y[ip[1] - 1], z[ip[2] - 1]
    rmax = np.sqrt((p.xmax - xp) ** 2 + (p.ymax - yp) ** 2 + (p.zmax - zp) ** 2)
    dr = rmax / (nr - 1)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rad = np.sqrt((X - xp) ** 2 + (Y - yp) ** 2 + (Z - zp) ** 2)
    b = (rad / dr + 1.5).astype(int) - 1
    den = np.abs(psi) ** 2
    s = np.bincount(b.ravel(), den.ravel(), nr)
    n = np.bincount(b.ravel(), None, nr)
    mean = np.where(n > 0, s / np.maximum(n, 1), 0.0)
    rr = np.arange(nr) * dr
    xnorm = den.sum() * hx ** 3
    mean *= xnorm / (4 * np.pi * np.sum(rr ** 2 * mean) * dr)
    assert np.allclose(out["rr"], rr, rtol=1e-14, atol=1e-14)
    assert np.max(np.abs(out["denr"] - mean)) < 1e-12 * np.max(mean)
    # impurity mean-square radii about the origin (DFT4He3d.f90:933-947)
    denx = o.get_field("denx")
    want = [np.sqrt(np.sum(denx * X ** 2) * hx ** 3), np.sqrt(np.sum(denx * Y ** 2) * hx ** 3),
            np.sqrt(np.sum(denx * Z ** 2) * hx ** 3)]
    assert np.allclose(out["xms"], want, rtol=1e-12)
    # the cavity built at 3.5 A: the half-maximum radius lies within a grid step
    assert out["lcontrol"] == (True, True)
    assert abs(out["rb"] - 3.5) < 0.6


def test_point_past_rmax_is_an_error(pkg, ora):
    """An impurity at positive coordinates leaves grid points past rmax,
    where the reference stops ('0001'): an error code here."""
    p = pkg.workloads.make_params(32, 0.6, 64)
    center = (3.0, 0.0, 0.0)
    psi = pkg.workloads.bubble_psi(p, 300, center, 3.5)
    r, v = pkg.workloads.particles(64, 5, 100.0, center=center)
    o = ora.Oracle(p)
    o.set_state(psi, r, v)
    with pytest.raises(ora.OracleError):
        o.bubble_radius(101)
    o.close()
