"""The batched ensemble (he4_batch_*) and the tile autotuner (he4_tune).

* An ensemble of systems on different grids (register-path and generic-path
  FFT lengths) advanced with one graph launch per step gives, member by
  member, bit-identical states to running each system alone with the same
  tile shapes (the same kernels in the same order per member).
* The tuner returns valid shapes; on the generic path the tile width only
  regroups pencils (results bit-identical), on the register path another
  four-step split changes the rounding only (1e-12 relative).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def members(w):
    out = []
    for n, h, n4, seed, speed in [(32, 0.7, 60, 1, 80.0), (48, 0.6, 150, 2, 150.0), (64, 0.5, 250, 3, 250.0),
                                  (32, 0.7, 80, 4, 120.0), (48, 0.6, 120, 5, 60.0)]:
        p = w.make_params(n, h, 256)
        psi = w.droplet_psi(p, n4)
        r, v = w.particles(256, seed, speed)
        out.append((p, psi, r, v))
    return out


def test_ensemble_matches_individual_runs(pkg):
    w = pkg.workloads
    dt = w.deltat_fs(1.0)
    ms = members(w)
    with pkg.He4Batch([m[0] for m in ms]) as b:
        for mem, (p, psi, r, v) in zip(b.members, ms):
            mem.set_state(psi, r, v)
        n0 = b.launch_count()
        e, means = b.run(11, dt)
        assert b.launch_count() > n0
        e2, _ = b.run(4, dt)  # graphs replayed across calls
        e3, _ = b.run(37, dt)  # a 30-step graph, then 5, 1 and 1
        got = [mem.get_state() for mem in b.members]
        energies = [mem.energy()["etot"] for mem in b.members]
    for (p, psi, r, v), (gpsi, gr, gv, _), et in zip(ms, got, energies):
        with pkg.He4Step(p) as g:
            g.set_state(psi, r, v)
            g.run(11, dt)
            g.run(4, dt)
            g.run(37, dt)
            spsi, sr, sv, _ = g.get_state()
            assert np.array_equal(gpsi, spsi)
            assert np.array_equal(gr, sr) and np.array_equal(gv, sv)
            assert g.energy()["etot"] == et
    assert np.all(np.isfinite(e)) and np.all(np.isfinite(means))


def test_tuner_shapes_and_results(pkg):
    w = pkg.workloads
    dt = w.deltat_fs(1.0)
    for n in (48, 64):
        p = w.make_params(n, 0.6, 256)
        psi = w.droplet_psi(p, 150)
        r, v = w.particles(256, 9, 100.0)
        with pkg.He4Step(p) as g, pkg.He4Step(p) as ref:
            g.set_state(psi, r, v)
            t0 = g.tiles()
            tiles, ms = g.tune(reps=2)
            assert ms > 0
            if n == 48:
                assert tiles[:3] == [0, 0, 0] and all(x in (8, 16, 24, 32) for x in tiles[3:])
            else:
                assert all(x in (4, 8) for x in tiles[:3])
            assert g.tiles() == tiles
            g.set_state(psi, r, v)
            ref.set_state(psi, r, v)
            g.run(6, dt)
            ref.run(6, dt)
            a, b = g.get_state()[0], ref.get_state()[0]
            if n == 48:
                assert np.array_equal(a, b), (t0, tiles)
            else:
                assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
            with pytest.raises(pkg.He4Error):
                g.set_tiles([3, 0, 0, 8, 8, 8] if n == 64 else [0, 0, 0, 12, 8, 8])
