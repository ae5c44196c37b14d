"""he4_diagnostics_noalloc: the handle-free, allocation-free variant of
he4_diagnostics, for hosts that cannot call cudaMalloc because their device
memory belongs to another allocator.

The test owns the device buffers (torch allocates them, as the caller's own
allocator would), calls the new entry point twice in a row on two different
densities through the C ABI, and checks each result against he4_diagnostics
on the same density with the tolerance of the parity tests (1e-12 relative
for the atom number, 1e-9 for the centre of mass).  It sits in a file of its
own so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.he4_diagnostics_noalloc
    f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                  C.c_int32, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_handle_diagnostics_twice(pkg):
    import torch
    lib = pkg.load_library()
    f = _noalloc(lib)
    w = pkg.workloads
    p, psi, r, v, _ = w.workload("c1")
    n4 = 300
    dt = w.deltat_fs(1.0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    with pkg.He4Step(p) as g:
        g.set_state(psi, r, v)
        g.field()
        dens, refs = [], []
        for _ in range(2):
            refs.append(g.diagnostics(n4))
            dens.append(torch.from_numpy(g.get_field("den")).to(dev))
            g.run(3, dt)  # a different density for the second call
        outs = [torch.full((4,), float("nan"), dtype=torch.float64, device=dev) for _ in range(2)]
        torch.cuda.synchronize(dev)
        for d, o in zip(dens, outs):  # two calls in a row
            rc = f(d.data_ptr(), p.nx, p.ny, p.nz, p.xmax, p.ymax, p.zmax, n4, o.data_ptr(), stream.cuda_stream)
            assert rc == 0, lib.he4_last_error()
        torch.cuda.synchronize(dev)
        assert not np.allclose(refs[0], refs[1], rtol=0, atol=0)
        for o, ref in zip(outs, refs):
            got = o.cpu().numpy()
            assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0])
            assert np.allclose(got[1:], ref[1:], rtol=1e-9, atol=1e-12)


def test_noalloc_rejects_grids_beyond_its_scratch(pkg):
    import torch
    lib = pkg.load_library()
    f = _noalloc(lib)
    d = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    o = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    rc = f(d.data_ptr(), 1, 2, 4097, 1.0, 1.0, 1.0, 1, o.data_ptr(), None)
    assert rc == pkg.abi.HE4_E_ARG
    assert b"4096" in lib.he4_last_error()
    assert f(None, 1, 2, 4, 1.0, 1.0, 1.0, 1, o.data_ptr(), None) == pkg.abi.HE4_E_ARG
