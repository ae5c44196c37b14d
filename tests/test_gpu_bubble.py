"""GPU parity of the spherical bubble radius (he4_bubble_radius: the
Lspherical_bubble diagnostic, DFT4He3d.f90:893-986 with
bubble_radius_esferic.f90:1-134) against the oracle, through the C ABI.

Tolerances: the device bins den as integers of den*2^S (S chosen so no bin
can overflow; one unit is below 1e-11 of max den at these sizes), so the
radial density agrees with the oracle's FP64 sums within 1e-10 of its
largest value; rb within 1e-8 A; the flags and the bin of the maximum
exactly; the impurity mean-square radii within 1e-12 relative; the bin radii
to rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gpu_with_table(pkg, p, vq):
    import ctypes as C
    q = pkg.abi.He4Params.from_buffer_copy(p)
    q.pot_kind = pkg.abi.HE4_POT_TABLE
    vq = np.ascontiguousarray(vq)
    q.vq_table = vq.ctypes.data_as(C.POINTER(C.c_double))
    return pkg.He4Step(q), vq


def assert_same(g, o):
    assert g["lcontrol"] == o["lcontrol"]
    assert g["ir"] == o["ir"]
    assert np.allclose(g["xms"], o["xms"], rtol=1e-12, atol=0)
    assert np.allclose(g["rr"], o["rr"], rtol=1e-15, atol=1e-15)
    assert np.max(np.abs(g["denr"] - o["denr"])) <= 1e-10 * np.max(np.abs(o["denr"]))
    if all(o["lcontrol"]):
        assert abs(g["rb"] - o["rb"]) <= 1e-8


@pytest.fixture(scope="module")
def cavity(pkg, ora):
    """64^3 droplet of 300 atoms with a 4 A cavity around 256 particles at
    negative coordinates (every grid point then lies within rmax)."""
    p = pkg.workloads.make_params(64, 0.6, 256)
    center = (-0.5, -0.7, -2.0)
    psi = pkg.workloads.bubble_psi(p, 300, center, 4.0)
    r, v = pkg.workloads.particles(256, 7, 100.0, center=center)
    o = ora.Oracle(p)
    vq = o.get_kernel("vq")
    return p, psi, r, v, o, vq


@pytest.mark.parametrize("nr", [501, 97])
def test_bubble_radius_parity(pkg, cavity, nr):
    p, psi, r, v, o, vq = cavity
    o.set_state(psi, r, v)
    want = o.bubble_radius(nr)
    assert want["lcontrol"] == (True, True)
    g, keep = gpu_with_table(pkg, p, vq)
    with g:
        g.set_state(psi, r, v)
        got = g.bubble_radius(nr)
        assert_same(got, want)
        # deterministic: the integer bins do not depend on the atomics' order
        again = g.bubble_radius(nr)
        assert np.array_equal(again["denr"], got["denr"]) and again["rb"] == got["rb"]


def test_bubble_radius_after_steps(pkg, cavity):
    """After 3 RK + 2 PC steps the merged (time-step) evaluation's den and
    denx feed the diagnostic."""
    p, psi, r, v, o, vq = cavity
    dt = pkg.workloads.deltat_fs(1.0)
    o.set_state(psi, r, v)
    o.run(5, dt)
    want = o.bubble_radius(501)
    g, keep = gpu_with_table(pkg, p, vq)
    with g:
        g.set_state(psi, r, v)
        g.run(5, dt)
        got = g.bubble_radius(501)
    assert_same(got, want)


def test_bubble_radius_ragged_grid(pkg, ora):
    p = pkg.workloads.make_params(48, 0.6, 64, ny=40, nz=36)
    center = (-0.4, -0.3, -0.9)
    psi = pkg.workloads.bubble_psi(p, 40, center, 3.0)
    r, v = pkg.workloads.particles(64, 3, 100.0, center=center)
    o = ora.Oracle(p)
    o.set_state(psi, r, v)
    want = o.bubble_radius(211)
    with pkg.He4Step(p) as g:
        g.set_state(psi, r, v)
        got = g.bubble_radius(211)
    o.close()
    assert_same(got, want)


def test_bubble_radius_errors(pkg, ora):
    p = pkg.workloads.make_params(32, 0.6, 64)
    center = (3.0, 0.0, 0.0)
    psi = pkg.workloads.bubble_psi(p, 60, center, 3.0)
    r, v = pkg.workloads.particles(64, 5, 100.0, center=center)
    o = ora.Oracle(p)
    o.set_state(psi, r, v)
    with pytest.raises(ora.OracleError):
        o.bubble_radius(101)
    o.close()
    with pkg.He4Step(p) as g:
        g.set_state(psi, r, v)
        # grid points past rmax: the reference stops ('0001'), here an error
        with pytest.raises(pkg.He4Error) as e:
            g.bubble_radius(101)
        assert e.value.code == -1
        for nr in (3, 9000):
            with pytest.raises(pkg.He4Error):
                g.bubble_radius(nr)
        # the handle stays usable
        g.field()
