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
