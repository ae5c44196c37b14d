"""GPU parity tests: the CUDA library (through its C ABI) against the CPU
oracle on the same seeded inputs.

Tolerances (FP64 everywhere):
  * k-space kernels: pmod bit-identical; wcgk, kalfs 1e-14 and fvlj4 1e-8
    relative to the largest value (different sin/cos/exp implementations,
    amplified by the cancellation inside the reference's sinx11);
    Vq (single-precision values) within one FP32 ulp.
  * one field evaluation: every field within 1e-11 of its largest value.
  * energies after a field evaluation: 1e-10 relative per component.
  * 3 RK + 10 PC steps: energy components and the norm 1e-10 relative, psi
    and the pot4 of the merged (time-step) evaluation within 1e-10 of their
    largest values, trajectory means 1e-9 relative.
Integer work (the NGP deposit counts) must match exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    s = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / s)


@pytest.fixture(scope="module")
def c1(pkg, ora):
    """64^3 droplet + 256 particles (the small benchmark configuration)."""
    p, psi, r, v, _ = pkg.workloads.workload("c1")
    o = ora.Oracle(p)
    vq = o.get_kernel("vq")
    return p, psi, r, v, o, vq


def gpu_with_table(pkg, p, vq):
    import ctypes as C
    q = pkg.abi.He4Params.from_buffer_copy(p)
    q.pot_kind = pkg.abi.HE4_POT_TABLE
    vq = np.ascontiguousarray(vq)
    q.vq_table = vq.ctypes.data_as(C.POINTER(C.c_double))
    g = pkg.He4Step(q)
    return g


def test_kspace_kernels(pkg, c1):
    p, psi, r, v, o, vq = c1
    with pkg.He4Step(p) as g:
        assert np.array_equal(g.get_kernel("pmod"), o.get_kernel("pmod"))
        assert rel(g.get_kernel("wcgk"), o.get_kernel("wcgk")) < 1e-14
        assert rel(g.get_kernel("kalfs"), o.get_kernel("kalfs")) < 1e-14
        # sinx11 (fforma.f90:96-100) subtracts two terms that agree to ~6
        # digits at the largest |p|, so 1-ulp differences between libm's and
        # CUDA's sin/cos become ~1e-9 relative there
        assert rel(g.get_kernel("fvlj4"), o.get_kernel("fvlj4")) < 1e-8
        gv = g.get_kernel("vq")
        # both are single-precision numbers; at most one FP32 ulp apart
        ulp = np.spacing(np.abs(vq).astype(np.float32)).astype(np.float64)
        assert np.all(np.abs(gv - vq) <= ulp)
        assert np.mean(gv == vq) > 0.99


def test_vq_from_sampled_potential(pkg, ora):
    """HE4_POT_RTABLE: FT_V_spline on the device from a caller-sampled V(r)
    equals the oracle's to one FP32 ulp, and the analytic entry it samples."""
    import test_oracle_pins as pins
    p = pkg.workloads.make_params(32, 0.6, 8, nq=400)
    q, keep = pins.rtable_params(pkg, p)
    o = ora.Oracle(q)
    want = o.get_kernel("vq")
    o.close()
    with pkg.He4Step(q) as g:
        got = g.get_kernel("vq")
    with pkg.He4Step(p) as g:
        morse = g.get_kernel("vq")
    ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
    assert np.all(np.abs(got - want) <= ulp)
    assert np.max(np.abs(got - morse)) <= 2e-6 * np.max(np.abs(morse))
    q.vr_r0 = p.r_cutoff + 0.5
    with pytest.raises(pkg.He4Error):
        pkg.He4Step(q)


def test_vq_of_the_he2s_fci_entry(pkg, ora):
    """HE4_POT_HE2S_FCI: Select_Pot's 'He2S_fci' potential evaluated on the
    device (double-double sums) and transformed by FT_V_spline, against the
    oracle (binary128 sums) to one FP32 ulp, with the shipped inputs'
    r_cutoff_gs and umax_gs (data_files/input_He2S.0:2)."""
    p = pkg.workloads.make_params(48, 0.5, 8, pot=pkg.abi.HE4_POT_HE2S_FCI, nq=1500)
    p.r_cutoff, p.umax = 3.17502, 580.0065
    o = ora.Oracle(p)
    want = o.get_kernel("vq")
    o.close()
    with pkg.He4Step(p) as g:
        got = g.get_kernel("vq")
    # one FP32 ulp, or the FP64 rounding of the radial integrals (summed in
    # another order on the device, ~1e-14 of the scale) where Vq is near zero
    ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
    assert np.all(np.abs(got - want) <= ulp + 1e-13 * np.max(np.abs(want)))
    assert np.mean(got == want) > 0.99
    # not the Morse kernel by accident
    with pkg.He4Step(pkg.workloads.make_params(48, 0.5, 8, nq=1500)) as g:
        assert np.max(np.abs(g.get_kernel("vq") - got)) > 1e-3 * np.max(np.abs(got))


@pytest.mark.parametrize("shape", [(64, 64, 64), (96, 64, 80), (48, 40, 30), (128, 256, 16), (256, 128, 8)])
def test_fft_against_numpy_and_cufft(pkg, shape):
    import ctypes as C
    import torch
    nx, ny, nz = shape
    p = pkg.workloads.make_params(nx, 0.5, 8, pot=pkg.abi.HE4_POT_NULL, ny=ny, nz=nz)
    rng = np.random.default_rng(11)
    a = rng.standard_normal((nz, ny, nx))
    with pkg.He4Step(p) as g:
        L = pkg.load_library()
        out = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
        dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
        assert L.he4_fft_r2c(g._h, dp(a), dp(out.view(np.float64))) == 0
        want = np.fft.rfftn(a)
        assert rel(out, want) < 1e-14
        cufft = torch.fft.rfftn(torch.from_numpy(a).cuda()).cpu().numpy()
        assert rel(out, cufft) < 1e-14
        back = np.zeros_like(a)
        assert L.he4_fft_c2r(g._h, dp(want.view(np.float64)), dp(back)) == 0
        assert rel(back / a.size, a) < 1e-14


def test_field_parity(pkg, c1):
    p, psi, r, v, o, vq = c1
    o.set_state(psi, r, v)
    o.field()
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        g.field()
        # integer deposit: identical impurity density
        assert np.array_equal(g.get_field("denx"), o.get_field("denx"))
        for name in pkg.abi.FIELDS:
            assert rel(g.get_field(name), o.get_field(name)) < 1e-11, name
        _, _, _, ag = g.get_state()
        _, _, _, ao = o.get_state()
        assert rel(ag, ao) < 1e-11
        eg, eo = g.energy(), o.energy()
        for k in eo:
            assert abs(eg[k] - eo[k]) <= 1e-10 * max(abs(eo[k]), 1e-30), (k, eg[k], eo[k])


@pytest.fixture(scope="module")
def c1_icon13(pkg, ora):
    """64^3 with icon=13 (zero-padded stencils, the shipped inputs' mode) and a
    droplet of 600 atoms (R = 18.7 A) whose density reaches the box faces, so
    the boundary rows matter."""
    w = pkg.workloads
    p = w.make_params(64, 0.6, 256)
    p.icon = 13
    psi = w.droplet_psi(p, 600)
    r, v = w.particles(256, 1234, 100.0)
    o = ora.Oracle(p)
    return p, psi, r, v, o, o.get_kernel("vq")


def test_field_and_steps_parity_icon13(pkg, c1_icon13):
    p, psi, r, v, o, vq = c1_icon13
    o.set_state(psi, r, v)
    o.field()
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        g.field()
        for name in pkg.abi.FIELDS:
            assert rel(g.get_field(name), o.get_field(name)) < 1e-11, name
        assert rel(g.get_state()[3], o.get_state()[3]) < 1e-11
        # the boundary mode is live: the periodic stencils give other fields
        q = pkg.abi.He4Params.from_buffer_copy(p)
        q.icon = 8
        with gpu_with_table(pkg, q, vq) as g8:
            g8.set_state(psi, r, v)
            g8.field()
            assert rel(g8.get_field("dxden"), g.get_field("dxden")) > 1e-6
    dt = pkg.workloads.deltat_fs(1.0)
    o.set_state(psi, r, v)
    eo, mo = o.run(8, dt)
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        eg, mg = g.run(8, dt)
        assert np.allclose(eg[3:], eo[3:], rtol=1e-8, atol=0)
        assert np.allclose(mg, mo, rtol=1e-9, atol=1e-9 * np.abs(mo).max())
        assert rel(g.get_field("pot4"), o.get_field("pot4")) < 1e-10
        assert rel(g.get_state()[0], o.get_state()[0]) < 1e-10
        Eg, Eo = g.energy(), o.energy()
        for k in Eo:
            assert abs(Eg[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-30), (k, Eg[k], Eo[k])


def test_field_and_steps_parity_icon12(pkg, ora):
    """icon=12 (redef.f:133-150): zero-padded centred rows at the upper end,
    the Bickley matrix's one-sided rows for the first ko2 points; npd 7 and
    13 on a droplet that reaches the box faces.  Fields after one evaluation
    within 1e-11 of the oracle, 3 RK + 5 PC steps within 1e-10, and the
    lower-end rows are live (icon=13 gives another density gradient)."""
    w = pkg.workloads
    for npd in (7, 13):
        p = w.make_params(48, 0.6, 256, npd=npd, nz=40)
        p.icon = 12
        psi = w.droplet_psi(p, 350)
        r, v = w.particles(256, 77, 100.0)
        o = ora.Oracle(p)
        vq = o.get_kernel("vq")
        o.set_state(psi, r, v)
        o.field()
        with gpu_with_table(pkg, p, vq) as g:
            g.set_state(psi, r, v)
            g.field()
            for name in pkg.abi.FIELDS:
                assert rel(g.get_field(name), o.get_field(name)) < 1e-11, (npd, name)
            q = pkg.abi.He4Params.from_buffer_copy(p)
            q.icon = 13
            with gpu_with_table(pkg, q, vq) as g13:
                g13.set_state(psi, r, v)
                g13.field()
                assert rel(g13.get_field("dxden"), g.get_field("dxden")) > 1e-6
        dt = w.deltat_fs(1.0)
        o.set_state(psi, r, v)
        eo, mo = o.run(8, dt)
        with gpu_with_table(pkg, p, vq) as g:
            g.set_state(psi, r, v)
            eg, mg = g.run(8, dt)
            assert np.allclose(eg[3:], eo[3:], rtol=1e-8, atol=0)
            assert np.allclose(mg, mo, rtol=1e-9, atol=1e-9 * np.abs(mo).max())
            assert rel(g.get_state()[0], o.get_state()[0]) < 1e-10
            Eg, Eo = g.energy(), o.energy()
            for k in Eo:
                assert abs(Eg[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-30), (npd, k, Eg[k], Eo[k])
        o.close()


def test_steps_parity(pkg, c1):
    p, psi, r, v, o, vq = c1
    dt = pkg.workloads.deltat_fs(1.0)
    o.set_state(psi, r, v)
    eo, mo = o.run(13, dt)
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        eg, mg = g.run(13, dt)
        assert np.all(eg[:3] == 0) and np.all(eo[:3] == 0)
        assert np.allclose(eg[3:], eo[3:], rtol=1e-8, atol=0)
        assert np.allclose(mg, mo, rtol=1e-9, atol=1e-9 * np.abs(mo).max())
        # pot4 of the final state comes from the merged time-step
        # evaluation (one summed inverse FFT for the linear convolutions);
        # the named intermediates are computed on request
        assert rel(g.get_field("pot4"), o.get_field("pot4")) < 1e-10
        for name in ("uimp", "delj4", "corr", "ualphas", "penalty"):
            assert rel(g.get_field(name), o.get_field(name)) < 1e-10, name
        psg, rg, vg, ag = g.get_state()
        pso, ro, vo, ao = o.get_state()
        assert rel(psg, pso) < 1e-10
        assert rel(rg, ro) < 1e-12 and rel(vg, vo) < 1e-10
        Eg, Eo = g.energy(), o.energy()
        for k in Eo:
            assert abs(Eg[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-30), (k, Eg[k], Eo[k])
        dxyz = (2 * p.xmax / p.nx) ** 3
        ng = np.sum(g.get_field("den")) * dxyz
        no = np.sum(o.get_field("den")) * dxyz
        assert abs(ng - no) <= 1e-10 * no


def test_steps_parity_absorbing_layer(pkg, ora, c1):
    """Lambdah != 0: timec = (Lambdah (1 + tanh((z - tzmean)/tzsurf)), 1)
    (DFT4He3d.f90:773-782, real part rounded to real(4)) multiplies H psi in
    every RK stage and PC step; 3 RK + 5 PC steps against the oracle."""
    p, psi, r, v, o0, vq = c1
    q = pkg.abi.He4Params.from_buffer_copy(p)
    q.lambdah, q.tzmean, q.tzsurf = 0.05, 12.0, 2.0
    dt = pkg.workloads.deltat_fs(1.0)
    o = ora.Oracle(q)
    o.set_state(psi, r, v)
    eo, mo = o.run(8, dt)
    with gpu_with_table(pkg, q, vq) as g:
        g.set_state(psi, r, v)
        eg, mg = g.run(8, dt)
        assert np.allclose(eg[3:], eo[3:], rtol=1e-8, atol=0)
        assert np.allclose(mg, mo, rtol=1e-9, atol=1e-9 * np.abs(mo).max())
        psg = g.get_state()[0]
        pso = o.get_state()[0]
        assert rel(psg, pso) < 1e-10
        Eg, Eo = g.energy(), o.energy()
        for k in Eo:
            assert abs(Eg[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-30), (k, Eg[k], Eo[k])
    o.close()
    # the layer damps: the norm decays only where tanh is switched on
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        g.run(8, dt)
        n_plain = np.sum(np.abs(g.get_state()[0]) ** 2)
    assert np.sum(np.abs(psg) ** 2) != n_plain


def test_run_equals_single_steps_and_is_deterministic(pkg, c1):
    p, psi, r, v, o, vq = c1
    dt = pkg.workloads.deltat_fs(1.0)
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        e1, m1 = g.run(6, dt)
        s1 = g.get_state()[0]
        g.set_state(psi, r, v)
        ms = [g.steprk(dt) for _ in range(3)]
        es = []
        for _ in range(3):
            e, m = g.steppc(dt)
            es.append(e)
            ms.append(m)
        s2 = g.get_state()[0]
        assert np.array_equal(s1, s2)
        assert np.array_equal(np.array(ms), m1)
        assert np.array_equal(np.array(es), e1[3:])


def test_step_graphs_cover_the_cycle_and_survive_set_state(pkg, c1):
    """The PC step's buffer states repeat every 30 steps: he4_run captures
    30 graphs and runs no step uncaptured, and a new he4_set_state (which
    puts the buffers back in allocation order) replays them."""
    p, psi, r, v, o, vq = c1
    dt = pkg.workloads.deltat_fs(1.0)
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        g.run(3 + 45, dt)
        assert g.graph_stats() == (30, 0)
        a = g.get_state()[0]
        g.set_state(psi, r, v)
        g.run(3 + 45, dt)
        assert g.graph_stats() == (30, 0)
        assert np.array_equal(g.get_state()[0], a)


@pytest.mark.parametrize("variant", ["npd13", "ot_core", "noncubic", "edge"])
def test_field_parity_variants(pkg, ora, variant):
    """Other stencil widths, the 'OT ' core, a non-cubic grid, and particles
    next to a face of the grid (the impurity box falls back to the whole
    grid there)."""
    w = pkg.workloads
    center = (0.0, 0.0, 2.0)
    if variant == "npd13":
        p = w.make_params(48, 0.6, 64, npd=13)
    elif variant == "ot_core":
        p = w.make_params(48, 0.6, 64, core4=pkg.abi.HE4_CORE_OT)
    elif variant == "edge":
        p = w.make_params(48, 0.6, 64)
        center = (0.0, 0.0, p.zmax - 1.5)
    else:
        p = w.make_params(40, 0.6, 64, ny=48, nz=60)
    psi = w.droplet_psi(p, 150)
    r, v = w.particles(p.n_par, 5, 100.0, center=center)
    o = ora.Oracle(p)
    vq = o.get_kernel("vq")
    o.set_state(psi, r, v)
    o.field()
    dt = w.deltat_fs(1.0)
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        g.field()
        names = ["pot4", "dencg", "delj4", "uimp", "fx", "fy", "fz", "hpsix"]
        if variant != "ot_core":
            names += ["ualphas", "intxalf"]
        for name in names:
            assert rel(g.get_field(name), o.get_field(name)) < 1e-11, name
        eg, _ = g.run(5, dt)
        eo, _ = o.run(5, dt)
        assert np.allclose(eg, eo, rtol=1e-8, atol=0)
        Eg, Eo = g.energy(), o.energy()
        for k in Eo:
            assert abs(Eg[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-30), (k, Eg[k], Eo[k])
    o.close()


def test_diagnostics_parity(pkg, c1):
    """Atom number and centre of mass reduced on the device (DFT4He3d.f90:885,
    r_cm.f90) against the oracle, after a few steps."""
    p, psi, r, v, o, vq = c1
    dt = pkg.workloads.deltat_fs(1.0)
    o.set_state(psi, r, v)
    o.run(5, dt)
    with gpu_with_table(pkg, p, vq) as g:
        g.set_state(psi, r, v)
        d0 = g.diagnostics(300)
        assert d0[0] == pytest.approx(np.sum(np.abs(psi) ** 2) * (2 * p.xmax / p.nx) ** 3, rel=1e-13)
        g.run(5, dt)
        dg, do = g.diagnostics(300), o.diagnostics(300)
        assert abs(dg[0] - do[0]) <= 1e-12 * do[0]
        assert np.allclose(dg[1:], do[1:], rtol=1e-9, atol=1e-12)


def test_launch_count_and_errors(pkg, c1):
    p, psi, r, v, o, vq = c1
    with pkg.He4Step(p) as g:
        with pytest.raises(pkg.He4Error) as ei:
            g.field()  # no state yet
        assert ei.value.code == pkg.abi.HE4_E_STATE
        g.set_state(psi, r, v)
        n0 = g.launch_count()
        g.field()
        assert g.launch_count() > n0
        with pytest.raises(pkg.He4Error):
            g.steppc(float("nan"))


def test_force_xy_shared_transform(pkg, monkeypatch):
    """The force z convolution transforms i D_x and i D_y once (they are
    constant along z); HE4_ZCONV_SHARE_XY=0 transforms each output.  The
    full-grid forces agree to FP64 rounding."""
    w = pkg.workloads
    p, psi, r, v, _ = w.workload("c1")
    f = {}
    for share in ("1", "0"):
        monkeypatch.setenv("HE4_ZCONV_SHARE_XY", share)
        with pkg.He4Step(p) as g:
            g.set_state(psi, r, v)
            g.field()
            f[share] = [g.get_field(n) for n in ("fx", "fy", "fz")]
    for a, b in zip(f["1"], f["0"]):
        scale = np.max(np.abs(b))
        assert np.max(np.abs(a - b)) <= 1e-12 * scale

