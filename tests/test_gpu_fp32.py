"""The FP32-convolution form (HE4_PREC_FP32CONV) against the FP64 oracle and
the plain FP64 form on the same seeded inputs.

Only the convolution spectra, their twiddles, the k-space kernels and the
derivative symbol are FP32; real grids, the psi update, the reductions and
the particle integration stay FP64.  The FP32 transforms round at every
butterfly stage, so the convolution outputs carry about 1e-7..1e-6 relative
error.  Stated tolerances:
  * 3D R2C / C2R transforms: 2e-6 of the largest coefficient;
  * every field after one evaluation: 5e-6 of its largest value (convolution
    outputs; fields that involve no FFT keep the plain form's 1e-11);
  * each energy term after one evaluation: 1e-5 relative (measured at 64^3:
    ecor4 7e-7, every other term below 1e-7); the total energy 1e-7;
  * 3 RK + 50 PC steps at 64^3: density relative L2 1e-6 against the plain
    FP64 form, atom number 1e-8 relative, psi 1e-5 of its largest value.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def fp32_params(pkg, p):
    q = pkg.abi.He4Params.from_buffer_copy(p)
    q.precision = pkg.abi.HE4_PREC_FP32CONV
    return q


@pytest.fixture(scope="module")
def c1(pkg):
    return pkg.workloads.workload("c1")


@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 128, 16), (128, 256, 16)])
def test_fp32_fft_against_numpy(pkg, shape):
    import ctypes as C
    nx, ny, nz = shape
    p = pkg.workloads.make_params(nx, 0.5, 8, pot=pkg.abi.HE4_POT_NULL, ny=ny, nz=nz)
    rng = np.random.default_rng(3)
    a = rng.standard_normal((nz, ny, nx))
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    L = pkg.load_library()
    with pkg.He4Step(fp32_params(pkg, p)) as g:
        out = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
        assert L.he4_fft_r2c(g._h, dp(a), dp(out.view(np.float64))) == 0
        want = np.fft.rfftn(a)
        e = rel(out, want)
        assert 1e-10 < e < 2e-6  # FP32 arithmetic, not a silent FP64 path
        back = np.zeros_like(a)
        assert L.he4_fft_c2r(g._h, dp(want.view(np.float64)), dp(back)) == 0
        assert rel(back / a.size, a) < 2e-6


def test_fp32_field_and_energy_terms(pkg, ora, c1):
    p, psi, r, v, _ = c1
    o = ora.Oracle(p)
    o.set_state(psi, r, v)
    o.field()
    report = {}
    with pkg.He4Step(fp32_params(pkg, p)) as g:
        g.set_state(psi, r, v)
        g.field()
        # no FFT involved: the FP64 tolerance of the plain form
        for name in ("den", "denx", "psix", "hpsix", "dxden", "dyden", "dzden", "penalty"):
            assert rel(g.get_field(name), o.get_field(name)) < 1e-11, name
        for name in pkg.abi.FIELDS:
            e = rel(g.get_field(name), o.get_field(name))
            report[name] = e
            assert e < 5e-6, (name, e)
        assert max(report[n] for n in ("pot4", "dencg", "delj4", "uimp", "fx")) > 1e-9
        eg, eo = g.energy(), o.energy()
        for k in eo:
            err = abs(eg[k] - eo[k]) / max(abs(eo[k]), 1e-30)
            print(f"fp32 energy term {k}: {eg[k]:.12g} vs {eo[k]:.12g} rel {err:.2e}")
            assert err < 1e-5, (k, eg[k], eo[k])
        assert abs(eg["etot"] - eo["etot"]) <= 1e-7 * abs(eo["etot"])
    o.close()


def test_fp32_icon13_against_oracle(pkg, ora):
    """The FP32 form with zero-padded stencils (icon=13: FP64 intermediate
    grids, the force from transformed gradients) against the FP64 oracle:
    the tolerances of the periodic case."""
    w = pkg.workloads
    p = w.make_params(64, 0.6, 256)
    p.icon = 13
    psi = w.droplet_psi(p, 600)
    r, v = w.particles(256, 1234, 100.0)
    o = ora.Oracle(p)
    o.set_state(psi, r, v)
    o.field()
    with pkg.He4Step(fp32_params(pkg, p)) as g:
        g.set_state(psi, r, v)
        g.field()
        for name in ("den", "denx", "dxden", "dzden", "penalty"):
            assert rel(g.get_field(name), o.get_field(name)) < 1e-11, name
        for name in pkg.abi.FIELDS:
            assert rel(g.get_field(name), o.get_field(name)) < 5e-6, name
        assert rel(g.get_state()[3], o.get_state()[3]) < 5e-6
        eg, eo = g.energy(), o.energy()
        assert abs(eg["etot"] - eo["etot"]) <= 1e-7 * abs(eo["etot"])
    o.close()


def test_fp32_steps_against_fp64(pkg, c1):
    p, psi, r, v, _ = c1
    dt = pkg.workloads.deltat_fs(1.0)
    with pkg.He4Step(p) as g64, pkg.He4Step(fp32_params(pkg, p)) as g32:
        for g in (g64, g32):
            g.set_state(psi, r, v)
        e64, m64 = g64.run(53, dt)
        e32, m32 = g32.run(53, dt)
        assert np.all(np.isfinite(e32)) and np.all(np.isfinite(m32))
        s64, s32 = g64.get_state(), g32.get_state()
        d64, d32 = np.abs(s64[0]) ** 2, np.abs(s32[0]) ** 2
        assert np.linalg.norm(d32 - d64) / np.linalg.norm(d64) < 1e-6
        assert rel(s32[0], s64[0]) < 1e-5
        n64, n32 = g64.diagnostics(1)[0], g32.diagnostics(1)[0]
        assert abs(n32 - n64) <= 1e-8 * n64
        E64, E32 = g64.energy(), g32.energy()
        for k in E64:
            assert abs(E32[k] - E64[k]) <= 1e-5 * max(abs(E64[k]), 1e-30), (k, E32[k], E64[k])


def test_fp32_run_deterministic(pkg, c1):
    p, psi, r, v, _ = c1
    dt = pkg.workloads.deltat_fs(1.0)
    with pkg.He4Step(fp32_params(pkg, p)) as g:
        g.set_state(psi, r, v)
        e1, m1 = g.run(8, dt)
        s1 = g.get_state()[0]
        g.set_state(psi, r, v)
        e2, m2 = g.run(8, dt)
        assert np.array_equal(s1, g.get_state()[0])
        assert np.array_equal(e1, e2) and np.array_equal(m1, m2)


def test_fp32_rejects_generic_lengths(pkg):
    p = pkg.workloads.make_params(48, 0.6, 16, pot=pkg.abi.HE4_POT_NULL)
    with pytest.raises(pkg.He4Error) as ei:
        pkg.He4Step(fp32_params(pkg, p))
    assert ei.value.code == pkg.abi.HE4_E_UNSUPPORTED


def test_pot4_split_weights_match_fp64_sums(pkg, monkeypatch):
    """The streamed float-grid pot4 (128^3 and up) assembles pot4 in FP32 with
    split first-derivative weights; HE4_POT4_SPLIT=0 selects the same kernel
    with FP64 sums.  After the same steps both pot4 agree to the FP32 form's
    field tolerance (measured: ~1e-8 of the largest value)."""
    w = pkg.workloads
    p, psi, r, v, _ = w.workload("c2")
    dt = w.deltat_fs(1.0)
    out = {}
    for split in ("1", "0"):
        monkeypatch.setenv("HE4_POT4_SPLIT", split)
        with pkg.He4Step(fp32_params(pkg, p)) as g:
            g.set_state(psi, r, v)
            g.run(5, dt)
            out[split] = (g.get_field("pot4"), g.get_state()[0])
    e = rel(out["1"][0], out["0"][0])
    assert 0.0 < e < 5e-7, e
    assert rel(out["1"][1], out["0"][1]) < 1e-6  # measured 7.9e-8 after 5 steps
