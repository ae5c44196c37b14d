"""he4_snapshot_begin / he4_snapshot_wait: the asynchronous checkpoint of the
pcurr backups (DFT4He3d.f90:992-1009).  The snapshot equals he4_get_state at
the point it was taken, however many steps run before it is collected, and
taking it changes nothing in the run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def snapshot_fns(pkg):
    L = pkg.load_library()
    pp = C.POINTER(C.POINTER(C.c_double))
    L.he4_snapshot_begin.argtypes = [C.c_void_p]
    L.he4_snapshot_wait.argtypes = [C.c_void_p, pp, pp, pp, pp]
    return L


def test_snapshot_is_the_state_it_was_taken_from(pkg):
    w = pkg.workloads
    p, psi, r, v, _ = w.workload("c1")
    dt = w.deltat_fs(1.0)
    L = snapshot_fns(pkg)
    with pkg.He4Step(p) as g, pkg.He4Step(p) as ref:
        g.set_state(psi, r, v)
        ref.set_state(psi, r, v)
        g.run(5, dt)
        ref.run(5, dt)
        want = g.get_state()
        assert L.he4_snapshot_begin(g._h) == 0
        g.run(3, dt)  # the copy overlaps these steps
        ptrs = [C.POINTER(C.c_double)() for _ in range(4)]
        assert L.he4_snapshot_wait(g._h, *[C.byref(q) for q in ptrs]) == 0
        N, P3 = psi.size, 3 * p.n_par
        got_psi = np.ctypeslib.as_array(ptrs[0], shape=(2 * N,)).copy().view(np.complex128).reshape(psi.shape)
        assert np.array_equal(got_psi, want[0])
        for q, arr in zip(ptrs[1:], want[1:]):
            assert np.array_equal(np.ctypeslib.as_array(q, shape=(P3,)).reshape(arr.shape), arr)
        # the run goes on as if no snapshot had been taken
        ref.run(3, dt)
        assert np.array_equal(g.get_state()[0], ref.get_state()[0])
        # a wait without a snapshot in flight is a state error
        assert L.he4_snapshot_wait(g._h, *[C.byref(q) for q in ptrs]) == pkg.abi.HE4_E_STATE
