"""The C++ host driver end to end on the GPU: namelist + readenc mode-2
files in, time loop through the C ABI, printoutc files and the trajectory
files out; the final state equals the Python mirror's run bit for bit."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "4hetddft-isotropic-bohmian_b200")


def write_inputs(d, p, psi, rimp, vimp):
    pf, jf = os.path.join(d, "he4.input.density"), os.path.join(d, "X.input.wf")
    with open(pf, "w") as f:
        h = 2 * p.xmax / p.nx
        f.write("# synthetic droplet\n")
        f.write(f" {p.xmax:.17E} {p.ymax:.17E} {p.zmax:.17E} {h:.17E} {h:.17E} {h:.17E} {p.nx} {p.ny} {p.nz}\n")
        f.write("\n".join(f" ({c.real:.17E},{c.imag:.17E})" for c in psi.reshape(-1)))
        f.write("\n")
    with open(jf, "w") as f:
        f.write(f"# particles\n {rimp.shape[1]}\n")
        f.write("\n".join(f" {x:.17E}" for x in np.concatenate([rimp.reshape(-1), vimp.reshape(-1)])))
        f.write("\n")
    return pf, jf


def read_psi(path, shape):
    body = [l for l in open(path).read().splitlines() if not l.startswith("#")]
    vals = np.array([complex(*map(float, l.strip()[1:-1].split(","))) for l in body[1:]])
    return vals.reshape(shape)


def test_driver_run_matches_library(pkg, tmp_path):
    w = pkg.workloads
    p, psi, r, v, _ = w.workload("c1")
    d = str(tmp_path)
    write_inputs(d, p, psi, r, v)
    nml = f""" &input nx={p.nx}, ny={p.ny}, nz={p.nz}, xmax={p.xmax!r}, ymax={p.ymax!r}, zmax={p.zmax!r},
   n4=300, mode=2, core4='OTC', npd=7, icon=8, N_par={p.n_par}, mimpur={p.mimpur!r},
   deltatps=1.d-3, niter=13, pener=5, pcurr=10, ironx=1,
   selec_gs='morse', morse_d={w.MORSE_D}, morse_alpha={w.MORSE_ALPHA}, morse_re={w.MORSE_RE},
   r_cutoff_gs={p.r_cutoff!r}, umax_gs={p.umax!r}, nq={p.nq} /
"""
    res = subprocess.run([os.path.join(PKG, "he4run")], input=nml, capture_output=True, text=True, cwd=d)
    assert res.returncode == 0, res.stderr[-2000:]
    out = res.stdout
    assert out.count("Err(He, rimp, vimp)") == 10 and "TOTAL energy (He+X)" in out
    for f in ("rimp.out", "vimp.out", "aimp.out", "density.001.dat", "densityx.001.dat", "he4.output.density",
              "X.output.wf", "denx-x.dat"):
        assert os.path.exists(os.path.join(d, f)), f
    assert len(open(os.path.join(d, "rimp.out")).read().splitlines()) == 1 + 1 + 13
    got = read_psi(os.path.join(d, "he4.output.density"), psi.shape)
    # the same call sequence through the Python mirror: the first field
    # evaluation (he4_field, split form), energies every pener steps
    dt = w.deltat_fs(1.0)
    with pkg.He4Step(p) as g:
        g.set_state(psi, r, v)
        g.field()
        g.energy()
        for it in range(1, 14):
            if it <= 3:
                g.steprk(dt)
            else:
                g.steppc(dt)
            if it % 5 == 0:
                e = g.energy()  # the driver prints these (iterations 5 and 10)
            if it == 10:
                at10 = g.get_state()[0]
        want = g.get_state()[0]
    assert np.array_equal(got, want)
    # the pcurr backup (snapshot copied while the loop went on) holds the
    # state of iteration 10
    assert np.array_equal(read_psi(os.path.join(d, "density.001.dat"), psi.shape), at10)
    last_tot = [l for l in out.splitlines() if "TOTAL energy" in l][-1]
    assert float(last_tot.split()[-2]) == pytest.approx(e["etot"], abs=2e-6)


def test_driver_spherical_bubble(pkg, tmp_path):
    """Lbubble_radius: the driver writes the spherical bubble radius at the
    start and every pener steps (DFT4He3d.f90:698-760,929-986); the values
    equal he4_bubble_radius after the same call sequence."""
    w = pkg.workloads
    p = w.make_params(64, 0.6, 256)
    center = (-0.5, -0.7, -2.0)
    psi = w.bubble_psi(p, 300, center, 4.0)
    r, v = w.particles(256, 7, 100.0, center=center)
    d = str(tmp_path)
    write_inputs(d, p, psi, r, v)
    nml = f""" &input nx={p.nx}, ny={p.ny}, nz={p.nz}, xmax={p.xmax!r}, ymax={p.ymax!r}, zmax={p.zmax!r},
   n4=300, mode=2, core4='OTC', npd=7, icon=8, N_par={p.n_par}, mimpur={p.mimpur!r},
   deltatps=1.d-3, niter=6, pener=3, pcurr=0, ironx=1, lbubble_radius=.true., nr=97,
   selec_gs='morse', morse_d={w.MORSE_D}, morse_alpha={w.MORSE_ALPHA}, morse_re={w.MORSE_RE},
   r_cutoff_gs={p.r_cutoff!r}, umax_gs={p.umax!r}, nq={p.nq} /
"""
    res = subprocess.run([os.path.join(PKG, "he4run")], input=nml, capture_output=True, text=True, cwd=d)
    assert res.returncode == 0, res.stderr[-2000:]
    assert res.stdout.count("Impurity mean square radius") == 3
    lines = open(os.path.join(d, "spherical_bubble.out")).read().splitlines()
    dt = w.deltat_fs(1.0)
    want = []
    with pkg.He4Step(p) as g:
        g.set_state(psi, r, v)
        g.field()
        g.energy()
        want.append((0.0, g.bubble_radius(97)))
        for it in range(1, 7):
            if it <= 3:
                g.steprk(dt)
            else:
                g.steppc(dt)
            if it % 3 == 0:
                g.energy()
                want.append((it * 1e-3, g.bubble_radius(97)))
    want = [(t, b["rb"]) for t, b in want if all(b["lcontrol"])]
    assert len(want) >= 2 and len(lines) == len(want)
    for l, (t, rb) in zip(lines, want):
        tt, rr = map(float, l.split())
        assert tt == pytest.approx(t, abs=1e-9)
        assert rr == pytest.approx(rb, rel=1e-9)


def read_particles(path):
    body = [l for l in open(path).read().splitlines() if not l.startswith("#")]
    n = int(body[0])
    vals = np.array([float(l) for l in body[1:1 + 6 * n]])
    return n, vals[:3 * n].reshape(3, n), vals[3 * n:].reshape(3, n)


def test_driver_shipped_style_start(pkg, tmp_path):
    """The options of the shipped inputs (data_files/input_He2S.*) on a small
    grid: mode=0 start from density files, icon=13, npd=13, ironx=3, an
    absorbing layer, a non-power-of-two axis (generic FFT path), and a pair
    potential given as sampled V(r) (vrfile).  The driver's run equals the
    library's run from the start it wrote (density.000.dat / densityx.000.dat)."""
    import ctypes as C
    w = pkg.workloads
    d = str(tmp_path)
    nx, nz, h = 48, 40, 0.6
    p = w.make_params(nx, h, 400, npd=13, nz=nz)
    p.icon = 13
    p.ironx = 3
    p.lambdah, p.tzmean, p.tzsurf = 2.0, 10.0, 1.0
    x, y, z = w.grid_axes(p)
    den = np.abs(w.droplet_psi(p, 300)) ** 2
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    denx = np.exp(-((X - 0.3) ** 2 + Y ** 2 + (Z - 1.0) ** 2) / 0.5)
    for name, f in (("den.inp", den), ("denx.inp", denx)):
        with open(os.path.join(d, name), "w") as fh:
            fh.write(f"# start\n {p.xmax!r} {p.ymax!r} {p.zmax!r} {h!r} {h!r} {h!r} {p.nx} {p.ny} {p.nz} T 0. 0. 0.\n")
            fh.write("\n".join(f" {v:.17E}" for v in f.reshape(-1)) + "\n")
    dr = 0.01
    r = p.r_cutoff + dr * np.arange(int((60.0 - p.r_cutoff) / dr) + 1)
    v = p.morse_d * ((1.0 - np.exp(-p.morse_alpha * (r - p.morse_re))) ** 2 - 1.0)
    with open(os.path.join(d, "vr.dat"), "w") as fh:
        fh.write("".join(f" {a:.17E} {b:.17E}\n" for a, b in zip(r, v)))
    nml = f""" &input nx={p.nx}, ny={p.ny}, nz={p.nz}, xmax={p.xmax!r}, ymax={p.ymax!r}, zmax={p.zmax!r},
   n4=300, mode=0, filedenin='den.inp', fileimpin='denx.inp', core4='OTC', npd=13, icon=13,
   N_par={p.n_par}, mimpur={p.mimpur!r}, ironx=3, Lambdah=2.d0, tzmean=10.d0, tzsurf=1.d0,
   xi=-1.5d0, xf=2.d0, yi=-1.5d0, yf=1.5d0, zi=-0.5d0, zf=2.5d0, v0z=-1.d0, seed=3,
   deltatps=1.d-3, niter=6, pener=3, pcurr=0, selec_gs='He2S_fci', vrfile='vr.dat',
   r_cutoff_gs={p.r_cutoff!r}, umax_gs={p.umax!r}, nq={p.nq} /
"""
    res = subprocess.run([os.path.join(PKG, "he4run")], input=nml, capture_output=True, text=True, cwd=d)
    assert res.returncode == 0, res.stderr[-2000:]
    assert "TOTAL energy (He+X)" in res.stdout
    psi0 = read_psi(os.path.join(d, "density.000.dat"), den.shape)
    assert np.allclose(np.abs(psi0) ** 2, den, rtol=1e-14, atol=1e-30)
    n, r0, v0 = read_particles(os.path.join(d, "densityx.000.dat"))
    assert n == p.n_par and np.all(v0[2] == -7.63822291) and np.all(v0[:2] == 0)
    got = read_psi(os.path.join(d, "he4.output.density"), den.shape)
    q = pkg.abi.He4Params.from_buffer_copy(p)
    q.pot_kind = pkg.abi.HE4_POT_RTABLE
    vv = np.ascontiguousarray(v)
    q.vr_table = vv.ctypes.data_as(C.POINTER(C.c_double))
    q.n_vr, q.vr_r0, q.vr_dr = vv.size, float(r[0]), (r[-1] - r[0]) / (r.size - 1)
    dt = w.deltat_fs(1.0)
    with pkg.He4Step(q) as g:
        g.set_state(psi0, r0, v0)
        g.field()
        g.energy()
        for it in range(1, 7):
            if it <= 3:
                g.steprk(dt)
            else:
                g.steppc(dt)
            if it % 3 == 0:
                g.energy()
        want = g.get_state()[0]
    # the files hold 17 significant digits, so the start differs from the
    # driver's in the last place
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_driver_shipped_namelist_without_host_potential(pkg, ora, tmp_path):
    """The shipped namelist's potential entry (Selec_gs='He2S_fci',
    r_cutoff_gs, umax_gs; data_files/input_He2S.0:2) runs with no vrfile or
    vqfile: the library evaluates Select_Pot on the device.  A 32x32x40 grid,
    mode 0 start, icon=13, npd=13, ironx=3 and the absorbing layer as in the
    shipped inputs; the driver's final state equals the oracle's run from
    the start the driver wrote, and its Vq the oracle's to one FP32 ulp."""
    w = pkg.workloads
    d = str(tmp_path)
    nx, nz, h = 32, 40, 0.6
    p = w.make_params(nx, h, 200, npd=13, nz=nz, pot=pkg.abi.HE4_POT_HE2S_FCI, nq=1500)
    p.icon = 13
    p.ironx = 3
    p.r_cutoff, p.umax = 3.17502, 580.0065
    p.lambdah, p.tzmean, p.tzsurf = 2.0, 10.0, 1.0
    x, y, z = w.grid_axes(p)
    den = np.abs(w.droplet_psi(p, 150)) ** 2
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    denx = np.exp(-((X - 0.3) ** 2 + Y ** 2 + (Z - 1.0) ** 2) / 0.5)
    for name, f in (("den.inp", den), ("denx.inp", denx)):
        with open(os.path.join(d, name), "w") as fh:
            fh.write(f"# start\n {p.xmax!r} {p.ymax!r} {p.zmax!r} {h!r} {h!r} {h!r} {p.nx} {p.ny} {p.nz} T 0. 0. 0.\n")
            fh.write("\n".join(f" {v:.17E}" for v in f.reshape(-1)) + "\n")
    nml = f""" &input
 Selec_gs='He2S_fci', r_cutoff_gs=3.17502d0, umax_gs=5.800065d2
 nx={p.nx}, ny={p.ny}, nz={p.nz}, xmax={p.xmax!r}, ymax={p.ymax!r}, zmax={p.zmax!r},
 n4=150, mode=0, filedenin='den.inp', fileimpin='denx.inp', core4='OTC', npd=13, icon=13,
 N_par={p.n_par}, mimpur=4.002602d0, ironx=3, Lambdah=2.d0, tzmean=10.d0, tzsurf=1.d0,
 xi=-1.5d0, xf=2.d0, yi=-1.5d0, yf=1.5d0, zi=-0.5d0, zf=2.5d0, v0z=-1.d0, seed=5,
 deltatps=1.d-3, niter=5, pener=5, pcurr=0, Nq=1500 /
"""
    res = subprocess.run([os.path.join(PKG, "he4run")], input=nml, capture_output=True, text=True, cwd=d)
    assert res.returncode == 0, res.stderr[-2000:]
    psi0 = read_psi(os.path.join(d, "density.000.dat"), den.shape)
    _, r0, v0 = read_particles(os.path.join(d, "densityx.000.dat"))
    got = read_psi(os.path.join(d, "he4.output.density"), den.shape)
    o = ora.Oracle(p)
    with pkg.He4Step(p) as g:
        gv, ov = g.get_kernel("vq"), o.get_kernel("vq")
        # one FP32 ulp, or the FP64 rounding of the radial integrals (summed
        # in another order on the device, ~1e-14 of the scale) where Vq is
        # near zero and its FP32 ulp is smaller than that
        ulp = np.spacing(np.abs(ov).astype(np.float32)).astype(np.float64)
        assert np.all(np.abs(gv - ov) <= ulp + 1e-13 * np.max(np.abs(ov)))
        assert np.mean(gv == ov) > 0.99
    o.set_state(psi0, r0, v0)
    o.run(5, w.deltat_fs(1.0))
    want = o.get_state()[0]
    o.close()
    # the oracle builds its own Vq (1-ulp FP32 flips possible) and the start
    # files hold 17 significant digits
    assert np.max(np.abs(got - want)) <= 1e-9 * np.max(np.abs(want))
