"""Python host mirror of the C ABI (include/he4_tddft.h).

The reference drives its time step through argument-less Fortran subroutines
operating on module arrays (DFT4He3d.f90:630-634, 848-878): potenimp, poten,
forceimp, steprk(deltat), steppc(deltat, errHe, errimp, errvimp), energy.
`He4Step` exposes the same operations, with the same names and argument
meaning, on a handle that owns the device state.  Errors raise `He4Error`
carrying the library's code and message; nothing falls back to the CPU.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhe4b200.so")

_lib = None


class He4Error(RuntimeError):
    def __init__(self, code, what, detail):
        super().__init__(f"{what}: {detail} (code {code})")
        self.code = code


def load_library():
    """Load libhe4b200.so; raises if the CUDA library has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `python {os.path.join(HERE, 'build.py')}`")
    L = C.CDLL(LIB_PATH)
    vp, dp, i32 = C.c_void_p, C.POINTER(C.c_double), C.c_int32
    L.he4_params_default.argtypes = [vp]
    L.he4_params_default.restype = None
    L.he4_create.argtypes = [vp, C.POINTER(vp)]
    L.he4_destroy.argtypes = [vp]
    L.he4_destroy.restype = None
    L.he4_set_state.argtypes = [vp, dp, dp, dp]
    L.he4_get_state.argtypes = [vp, dp, dp, dp, dp]
    for n in ("he4_potenimp", "he4_poten", "he4_forceimp", "he4_field"):
        getattr(L, n).argtypes = [vp]
    L.he4_step_rk.argtypes = [vp, C.c_double, dp]
    L.he4_step_pc.argtypes = [vp, C.c_double, dp, dp]
    L.he4_run.argtypes = [vp, i32, C.c_double, dp, dp]
    L.he4_energy.argtypes = [vp, vp]
    L.he4_get_field.argtypes = [vp, i32, dp]
    L.he4_diagnostics.argtypes = [vp, i32, dp]
    L.he4_bubble_radius.argtypes = [vp, i32, dp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), dp, dp, dp]
    L.he4_get_kernel.argtypes = [vp, i32, dp]
    L.he4_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.he4_device_ptr.argtypes = [vp, i32, C.POINTER(vp)]
    ip = C.POINTER(C.c_int32)
    L.he4_set_tiles.argtypes = [vp, ip]
    L.he4_get_tiles.argtypes = [vp, ip]
    L.he4_tune.argtypes = [vp, i32, dp, ip]
    L.he4_batch_create.argtypes = [i32, vp, C.POINTER(vp)]
    L.he4_batch_destroy.argtypes = [vp]
    L.he4_batch_destroy.restype = None
    L.he4_batch_size.argtypes = [vp]
    L.he4_batch_member.argtypes = [vp, i32]
    L.he4_batch_member.restype = vp
    L.he4_batch_tune.argtypes = [vp, i32, ip, dp]
    L.he4_batch_run.argtypes = [vp, i32, C.c_double, dp, dp]
    L.he4_batch_launch_count.argtypes = [vp]
    L.he4_batch_launch_count.restype = C.c_int64
    L.he4_launch_count.argtypes = [vp]
    L.he4_launch_count.restype = C.c_int64
    L.he4_graph_stats.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.he4_strerror.argtypes = [C.c_int]
    L.he4_strerror.restype = C.c_char_p
    L.he4_last_error.argtypes = []
    L.he4_last_error.restype = C.c_char_p
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(code, what):
    if code != 0:
        L = load_library()
        raise He4Error(code, what, (L.he4_last_error() or b"").decode() or L.he4_strerror(code).decode())


def params_default():
    """he4_params_default() from the library."""
    p = abi.He4Params()
    load_library().he4_params_default(C.byref(p))
    return p


class He4Step:
    """Device-resident time step of one droplet + impurity system."""

    def __init__(self, params, _borrowed=None):
        L = load_library()
        self.p = params
        self._owned = _borrowed is None
        if _borrowed is None:
            self._h = C.c_void_p()
            _check(L.he4_create(C.byref(params), C.byref(self._h)), "he4_create")
        else:
            self._h = C.c_void_p(_borrowed)
        self.shape = (params.nz, params.ny, params.nx)
        self.hshape = (params.nz, params.ny, params.nx // 2 + 1)
        self.npar = params.n_par

    def close(self):
        if self._h and self._owned:
            load_library().he4_destroy(self._h)
        self._h = C.c_void_p()

    def tiles(self):
        t = (C.c_int32 * 6)()
        _check(load_library().he4_get_tiles(self._h, t), "he4_get_tiles")
        return list(t)

    def set_tiles(self, tiles):
        t = (C.c_int32 * 6)(*tiles)
        _check(load_library().he4_set_tiles(self._h, t), "he4_set_tiles")

    def tune(self, reps=3):
        """he4_tune: returns (tiles, ms per field evaluation)."""
        t = (C.c_int32 * 6)()
        ms = C.c_double()
        _check(load_library().he4_tune(self._h, reps, C.byref(ms), t), "he4_tune")
        return list(t), ms.value

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def device_ptr(self, which):
        """Device address of a state array: 'psi', 'rimp', 'vimp', 'den',
        'denx' (he4_device_ptr)."""
        ids = {"psi": abi.HE4_D_PSI, "rimp": abi.HE4_D_RIMP, "vimp": abi.HE4_D_VIMP, "den": abi.HE4_D_DEN,
               "denx": abi.HE4_D_DENX}
        out = C.c_void_p()
        _check(load_library().he4_device_ptr(self._h, ids[which], C.byref(out)), "he4_device_ptr")
        return out.value

    def set_state_device(self, psi_ptr, rimp_ptr, vimp_ptr):
        """he4_set_state from device arrays (addresses as integers)."""
        dpp = lambda a: C.cast(C.c_void_p(a), C.POINTER(C.c_double))
        _check(load_library().he4_set_state(self._h, dpp(psi_ptr), dpp(rimp_ptr), dpp(vimp_ptr)),
               "he4_set_state")

    def get_state_device(self, psi_ptr, rimp_ptr, vimp_ptr):
        """he4_get_state into device arrays (addresses as integers, 0 = skip)."""
        dpp = lambda a: C.cast(C.c_void_p(a), C.POINTER(C.c_double)) if a else None
        _check(load_library().he4_get_state(self._h, dpp(psi_ptr), dpp(rimp_ptr), dpp(vimp_ptr), None),
               "he4_get_state")

    # readenc mode 2 / printoutc
    def set_state(self, psi, rimp, vimp):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        rimp = np.ascontiguousarray(rimp, dtype=np.float64)
        vimp = np.ascontiguousarray(vimp, dtype=np.float64)
        if psi.shape != self.shape or rimp.shape != (3, self.npar) or vimp.shape != (3, self.npar):
            raise ValueError("state arrays do not match the grid / n_par")
        _check(load_library().he4_set_state(self._h, _dp(psi.view(np.float64)), _dp(rimp), _dp(vimp)),
               "he4_set_state")

    def get_state(self):
        psi = np.zeros(self.shape, dtype=np.complex128)
        r, v, a = (np.zeros((3, self.npar)) for _ in range(3))
        _check(load_library().he4_get_state(self._h, _dp(psi.view(np.float64)), _dp(r), _dp(v), _dp(a)),
               "he4_get_state")
        return psi, r, v, a

    # field evaluation
    def potenimp(self):
        _check(load_library().he4_potenimp(self._h), "he4_potenimp")

    def poten(self):
        _check(load_library().he4_poten(self._h), "he4_poten")

    def forceimp(self):
        _check(load_library().he4_forceimp(self._h), "he4_forceimp")

    def field(self):
        _check(load_library().he4_field(self._h), "he4_field")

    # time steps
    def steprk(self, deltat):
        m = np.zeros(9)
        _check(load_library().he4_step_rk(self._h, deltat, _dp(m)), "he4_step_rk")
        return m

    def steppc(self, deltat):
        e, m = np.zeros(3), np.zeros(9)
        _check(load_library().he4_step_pc(self._h, deltat, _dp(e), _dp(m)), "he4_step_pc")
        return e, m

    def run(self, nsteps, deltat):
        e, m = np.zeros((nsteps, 3)), np.zeros((nsteps, 9))
        _check(load_library().he4_run(self._h, nsteps, deltat, _dp(e), _dp(m)), "he4_run")
        return e, m

    def energy(self):
        E = abi.He4Energies()
        _check(load_library().he4_energy(self._h, C.byref(E)), "he4_energy")
        return E.as_dict()

    def diagnostics(self, n4):
        """(atom number, xcm, ycm, zcm) of the current density."""
        out = np.zeros(4)
        _check(load_library().he4_diagnostics(self._h, n4, _dp(out)), "he4_diagnostics")
        return out

    def bubble_radius(self, nr=501):
        """Spherical bubble radius of the current state (Bubble_Radius_esferic,
        bubble_radius_esferic.f90:1-134, with the caller's ipx and xmsx of
        DFT4He3d.f90:893-947).  Returns a dict with rb, lcontrol (two bools),
        ir (1-based bin of the density maximum), xms (3), rr and denr (nr)."""
        rb = C.c_double(0.0)
        found = (C.c_int32 * 2)()
        ir = C.c_int32(0)
        xms, rr, denr = np.zeros(3), np.zeros(nr), np.zeros(nr)
        _check(load_library().he4_bubble_radius(self._h, nr, C.byref(rb), found, C.byref(ir), _dp(xms), _dp(rr),
                                                _dp(denr)), "he4_bubble_radius")
        return {"rb": rb.value, "lcontrol": (bool(found[0]), bool(found[1])), "ir": ir.value, "xms": xms,
                "rr": rr, "denr": denr}

    def get_field(self, name):
        out = np.zeros(self.shape)
        _check(load_library().he4_get_field(self._h, abi.FIELD_ID[name], _dp(out)), "he4_get_field")
        return out

    def get_kernel(self, name):
        out = np.zeros(self.hshape)
        _check(load_library().he4_get_kernel(self._h, abi.KERNEL_ID[name], _dp(out)), "he4_get_kernel")
        return out

    def stream(self):
        s = C.c_void_p()
        _check(load_library().he4_get_stream(self._h, C.byref(s)), "he4_get_stream")
        return s.value

    def launch_count(self):
        return int(load_library().he4_launch_count(self._h))

    def graph_stats(self):
        """(graphs captured, PC steps run uncaptured) of he4_run."""
        cap, unc = C.c_int64(), C.c_int64()
        _check(load_library().he4_graph_stats(self._h, C.byref(cap), C.byref(unc)), "he4_graph_stats")
        return cap.value, unc.value


class He4Batch:
    """Batched ensemble of independent systems (he4_batch_*): members are
    He4Step views that do not own their handles."""

    def __init__(self, params_list):
        L = load_library()
        n = len(params_list)
        arr = (abi.He4Params * n)(*params_list)
        self._b = C.c_void_p()
        _check(L.he4_batch_create(n, arr, C.byref(self._b)), "he4_batch_create")
        self.members = [He4Step(params_list[i], _borrowed=L.he4_batch_member(self._b, i)) for i in range(n)]

    def __len__(self):
        return len(self.members)

    def close(self):
        if self._b:
            for m in self.members:
                m.close()
            load_library().he4_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def tune(self, reps=3):
        n = len(self.members)
        t = (C.c_int32 * (6 * n))()
        ms = np.zeros(n)
        _check(load_library().he4_batch_tune(self._b, reps, t, _dp(ms)), "he4_batch_tune")
        return np.array(list(t), dtype=np.int32).reshape(n, 6), ms

    def run(self, nsteps, deltat):
        """Advances every member; returns (err_max [n][3], means [n][9])."""
        n = len(self.members)
        e = np.zeros((n, 3))
        m = np.zeros((n, 9))
        _check(load_library().he4_batch_run(self._b, nsteps, deltat, _dp(e), _dp(m)), "he4_batch_run")
        return e, m

    def launch_count(self):
        return load_library().he4_batch_launch_count(self._b)
