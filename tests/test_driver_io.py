"""The C++ host driver's input and output (driver/he4io.cpp, he4run): the
&input namelist (DFT4He3d.f90:147-187), readenc mode 2 (readenc.f90:96-114
with titols.f90) and printoutc (printoutc.f90:13-131), formatted and binary.
No GPU: --print-input stops before he4_create, --roundtrip only reads and
writes."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "4hetddft-isotropic-bohmian_b200")


@pytest.fixture(scope="module")
def he4run(pkg):
    exe = os.path.join(PKG, "he4run")
    if not os.path.exists(exe):
        import importlib.util
        spec = importlib.util.spec_from_file_location("he4_build", os.path.join(PKG, "build.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    return exe


def fortran_e(x):
    return f"{x:.16E}".replace("E", "D") if x < 0 else f"{x:.16E}"


def write_reference_style(tmp, nx, ny, nz, psi, rimp, vimp):
    """Files laid out the way list-directed Fortran writes them: comment
    lines, several values per line, D exponents, a repeat count."""
    pf = os.path.join(tmp, "psi.in")
    with open(pf, "w") as f:
        f.write("#  Density after               5 iterations.\n#  Actual delatatps....:  1.0000000000E-03\n")
        f.write("#  Backup copy.\n")
        h = 0.6
        f.write(f"  {nx*h/2:.16E}  {ny*h/2:.16E}  {nz*h/2:.16E}  {h:.16E}  {h:.16E}\n  {h:.16E}"
                f"  {nx} {ny} {nz}\n")
        vals = [f"({fortran_e(c.real)},{fortran_e(c.imag)})" for c in psi.reshape(-1)]
        # a repeat count as Fortran may write it for equal values
        vals[:2] = ["2*(0.0,0.0)"] if psi.reshape(-1)[0] == 0 and psi.reshape(-1)[1] == 0 else vals[:2]
        for i in range(0, len(vals), 3):
            f.write("  " + " , ".join(vals[i:i + 3]) + "\n")
    jf = os.path.join(tmp, "imp.in")
    with open(jf, "w") as f:
        f.write("#  Density after               5 iterations.\n")
        f.write(f"  {rimp.shape[1]}\n")
        for a in (rimp, vimp):
            flat = a.reshape(-1)
            for i in range(0, flat.size, 4):
                f.write("  " + "  ".join(fortran_e(x) for x in flat[i:i + 4]) + "\n")
    return pf, jf


def read_binary(path):
    out = []
    with open(path, "rb") as f:
        while True:
            m = f.read(4)
            if not m:
                break
            n = struct.unpack("<i", m)[0]
            out.append(f.read(n))
            assert struct.unpack("<i", f.read(4))[0] == n
    return out


def test_roundtrip_formatted_and_binary(he4run, tmp_path):
    rng = np.random.default_rng(4)
    nx, ny, nz, npar = 4, 3, 2, 5
    psi = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
    psi.reshape(-1)[:2] = 0
    rimp = rng.standard_normal((3, npar))
    vimp = rng.standard_normal((3, npar))
    pf, jf = write_reference_style(str(tmp_path), nx, ny, nz, psi, rimp, vimp)
    out_p, out_j = str(tmp_path / "psi.out"), str(tmp_path / "imp.out")
    r = subprocess.run([he4run, "--roundtrip", pf, jf, out_p, out_j], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["4", "3", "2", "5"]
    # formatted output: comment header, grid line, one complex per line
    lines = open(out_p).read().splitlines()
    assert lines[0].startswith("#  Density after") and lines[4] == "#  Backup copy."
    body = [l for l in lines if not l.startswith("#")]
    assert body[0].split()[6:] == ["4", "3", "2"]
    got = np.array([complex(*map(float, l.strip()[1:-1].split(","))) for l in body[1:]])
    assert np.array_equal(got, psi.reshape(-1))
    # the formatted output reads back to the same bits, and so does binary
    bp, bj = str(tmp_path / "psi.bin"), str(tmp_path / "imp.bin")
    r = subprocess.run([he4run, "--roundtrip", "--binary", out_p, out_j, bp, bj], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    recs = read_binary(bp)
    hdr = struct.unpack("<6d3i", recs[0])
    assert hdr[6:] == (4, 3, 2) and hdr[3] == 0.6
    assert np.array_equal(np.frombuffer(recs[1], dtype=np.complex128), psi.reshape(-1))
    recj = read_binary(bj)
    assert struct.unpack("<i", recj[0])[0] == npar
    assert np.array_equal(np.frombuffer(recj[1]).reshape(3, npar), rimp)
    assert np.array_equal(np.frombuffer(recj[2]).reshape(3, npar), vimp)
    # and binary reads back (readenc accepts both forms)
    r = subprocess.run([he4run, "--roundtrip", bp, bj, str(tmp_path / "p2"), str(tmp_path / "j2")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_namelist_and_readenc(he4run, tmp_path):
    rng = np.random.default_rng(5)
    nx = ny = nz = 4
    npar = 3
    psi = rng.standard_normal((nz, ny, nx)) + 0j
    rimp = rng.standard_normal((3, npar))
    vimp = rng.standard_normal((3, npar))
    pf, jf = write_reference_style(str(tmp_path), nx, ny, nz, psi, rimp, vimp)
    nml = f"""! comment line
 &INPUT title='test run', nx={nx}, ny={ny}, nz={nz},
   xmax=1.2d0, ymax=1.2d0, zmax=1.2d0   ! inline comment
   core4='OTC', npd=7, icon=8, N_par={npar}, mode=2,
   filedenin='{pf}', fileimpin='{jf}',
   deltatps=1.d-3, niter=20, pener=10, pcurr=5,
   selec_gs='morse', r_cutoff_gs=3.0, umax_gs=3633.0, precision='fp32conv',
   lbubble_radius=.false. /
"""
    r = subprocess.run([he4run, "--print-input"], input=nml, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    kv = dict(t.split("=") for t in r.stdout.split())
    assert kv["nx"] == "4" and kv["core4"] == "1" and kv["n_par"] == "3" and kv["pot_kind"] == "1"
    assert float(kv["xmax"]) == 1.2 and float(kv["r_cutoff"]) == 3.0 and kv["precision"] == "1"
    assert float(kv["deltat"]) == pytest.approx(1e-3 / 7.63822291, rel=1e-15)
    assert float(kv["psi_norm2"]) == pytest.approx(float(np.sum(np.abs(psi) ** 2)), rel=1e-15)
    assert float(kv["rimp0"]) == rimp[0, 0] and float(kv["vimp_last"]) == vimp[-1, -1]
    # N_par mismatch stops as readenc does
    bad = nml.replace(f"N_par={npar}", "N_par=7")
    r = subprocess.run([he4run, "--print-input"], input=bad, capture_output=True, text=True)
    assert r.returncode != 0 and "N_par" in r.stderr
    # unsupported Select_Pot entries ask for a table
    bad = nml.replace("selec_gs='morse'", "selec_gs='Ba_plus'")
    r = subprocess.run([he4run, "--print-input"], input=bad, capture_output=True, text=True)
    assert r.returncode != 0 and "vqfile" in r.stderr and "vrfile" in r.stderr
    # any entry sampled on a uniform r grid (HE4_POT_RTABLE), and the
    # spherical-bubble keys of the pener block
    vr = tmp_path / "vr.dat"
    rr = 3.0 + 0.01 * np.arange(500)
    vr.write_text("".join(f" {a:.17E} {b:.17E}\n" for a, b in zip(rr, 10.0 * np.exp(-rr))))
    good = nml.replace("selec_gs='morse',", f"selec_gs='He2S_fci', vrfile='{vr}',").replace(
        "lbubble_radius=.false.", "lbubble_radius=.true., nr=301")
    r = subprocess.run([he4run, "--print-input"], input=good, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    kv = dict(t.split("=") for t in r.stdout.split())
    assert kv["pot_kind"] == "3" and kv["n_vr"] == "500"
    assert float(kv["vr_r0"]) == 3.0 and float(kv["vr_dr"]) == pytest.approx(0.01, rel=1e-12)
    assert kv["lbubble"] == "1" and kv["lspherical"] == "1" and kv["nr"] == "301"
    # a table whose r values are not evenly spaced is refused
    vr.write_text(" 3.0 1.0\n 3.1 0.5\n 3.3 0.2\n 3.4 0.1\n")
    r = subprocess.run([he4run, "--print-input"], input=good, capture_output=True, text=True)
    assert r.returncode != 0 and "uniformly" in r.stderr


def write_density(path, xmax, h, n, den):
    """A readenc mode-0 density file: '#' comment lines (titols), the header
    xmax,ymax,zmax,hx,hy,hz,nx,ny,nz,limp,ximp,yimp,zimp, then den(nx,ny,nz)."""
    with open(path, "w") as f:
        f.write("# synthetic density\n")
        f.write(f" {xmax!r} {xmax!r} {xmax!r} {h!r} {h!r} {h!r} {n} {n} {n} T 0.0 0.0 0.0\n")
        f.write("\n".join(f" {v:.17E}" for v in den.reshape(-1)))
        f.write("\n")


def test_readenc_mode0_start(he4run, tmp_path):
    """mode=0 (the shipped inputs): psi = sqrt(den) times the constraint phase,
    test particles drawn from denx inside [xi,xf]x[yi,yf]x[zi,zf], all at v0
    (DFT4He3d.f90:585-617, readenc.f90:78-92, sorteo.f90:1-28); the draw is
    seeded here, the reference's is not."""
    n, h = 16, 0.5
    xmax = n * h / 2
    x = -xmax + h * np.arange(n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    den = 0.0218 / (1 + np.exp((np.sqrt(X ** 2 + Y ** 2 + Z ** 2) - 3.0) / 0.5))
    denx = np.where((np.abs(X - 1.0) < 0.6) & (np.abs(Y) < 0.6) & (np.abs(Z + 0.5) < 0.6), 1.0, 0.0)
    d = str(tmp_path)
    write_density(os.path.join(d, "den.inp"), xmax, h, n, den)
    write_density(os.path.join(d, "denx.inp"), xmax, h, n, denx)
    nml = f""" &input nx={n}, ny={n}, nz={n}, xmax={xmax!r}, ymax={xmax!r}, zmax={xmax!r},
   mode=0, filedenin='den.inp', fileimpin='denx.inp', N_par=200, npd=7, icon=13,
   xi=-2.d0, xf=3.d0, yi=-2.d0, yf=2.d0, zi=-2.d0, zf=2.d0, v0z=1.5d0, xlamda=0.3d0,
   deltatps=1.d-3, niter=0, seed=7 /
"""
    r = subprocess.run([he4run, "--print-input"], input=nml, capture_output=True, text=True, cwd=d)
    assert r.returncode == 0, r.stderr
    kv = dict(t.split("=") for t in r.stdout.split())
    assert kv["icon"] == "13" and kv["n_par"] == "200"
    # |psi|^2 = den whatever the phase
    assert float(kv["psi_norm2"]) == pytest.approx(float(np.sum(den)), rel=1e-13)
    # every particle at v0 (A/ps -> A*K), drawn where denx > 0 and inside the box
    assert float(kv["vimp_last"]) == pytest.approx(1.5 * 7.63822291, rel=1e-15)
    r0 = float(kv["rimp0"])
    assert 0.4 - h <= r0 <= 1.6 + h
    # the start's density.000.dat holds that psi
    assert os.path.exists(os.path.join(d, "density.000.dat"))
    # the draw is reproducible for a seed and changes with it
    again = subprocess.run([he4run, "--print-input"], input=nml, capture_output=True, text=True, cwd=d)
    assert dict(t.split("=") for t in again.stdout.split())["rimp0"] == kv["rimp0"]
    other = subprocess.run([he4run, "--print-input"], input=nml.replace("seed=7", "seed=8"), capture_output=True,
                           text=True, cwd=d)
    assert dict(t.split("=") for t in other.stdout.split())["rimp0"] != kv["rimp0"]
    # mode 0 needs the particle box; mode 1 does not exist in the reference either
    bad = nml.replace("xi=-2.d0, ", "")
    r = subprocess.run([he4run, "--print-input"], input=bad, capture_output=True, text=True, cwd=d)
    assert r.returncode != 0 and "xi" in r.stderr
    r = subprocess.run([he4run, "--print-input"], input=nml.replace("mode=0", "mode=1"), capture_output=True,
                       text=True, cwd=d)
    assert r.returncode != 0 and "not programmed" in r.stderr
