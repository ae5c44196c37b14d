"""ctypes wrapper of the CPU oracle (oracle/he4_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, as the checker or the timed CPU baseline.  The method
names mirror the product wrapper (and the reference subroutines) so parity
tests drive both with the same calls.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhe4oracle.so")


def build(force=False):
    """Compile the oracle with the committed Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "he4_oracle.c"))):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    vp, dp, i32 = C.c_void_p, C.POINTER(C.c_double), C.c_int32
    L.ora_create.argtypes = [vp, C.POINTER(vp)]
    L.ora_destroy.argtypes = [vp]
    L.ora_destroy.restype = None
    L.ora_set_state.argtypes = [vp, dp, dp, dp]
    L.ora_get_state.argtypes = [vp, dp, dp, dp, dp]
    for n in ("ora_potenimp", "ora_poten", "ora_forceimp", "ora_field"):
        getattr(L, n).argtypes = [vp]
    L.ora_step_rk.argtypes = [vp, C.c_double, dp]
    L.ora_step_pc.argtypes = [vp, C.c_double, dp, dp]
    L.ora_run.argtypes = [vp, i32, C.c_double, dp, dp]
    L.ora_energy.argtypes = [vp, vp]
    L.ora_diagnostics.argtypes = [vp, i32, dp]
    ip = C.POINTER(C.c_int32)
    L.ora_bubble_radius.argtypes = [vp, i32, dp, ip, ip, dp, dp, dp]
    L.ora_bubble_search.argtypes = [i32, C.c_double, C.c_double, dp, dp, dp, dp, ip, ip]
    L.ora_get_field.argtypes = [vp, i32, dp]
    L.ora_get_kernel.argtypes = [vp, i32, dp]
    L.ora_set_threads.argtypes = [C.c_int]
    L.ora_set_threads.restype = None
    L.ora_fd_weights.argtypes = [C.c_int, C.c_int, dp]
    L.ora_fd_rows.argtypes = [C.c_int, C.c_int, dp]
    L.ora_si.argtypes = [C.c_double]
    L.ora_si.restype = C.c_double
    L.ora_v_he2s_fci.argtypes = [C.c_double]
    L.ora_v_he2s_fci.restype = C.c_double
    L.ora_fft3_r2c.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp]
    L.ora_fft3_c2r.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp]
    L.ora_spline.argtypes = [dp, dp, dp, dp, dp, dp, C.c_double, C.c_double, C.c_int]
    L.ora_deriv.argtypes = [vp, C.c_int, C.c_int, dp, dp]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleError(RuntimeError):
    pass


def _check(code, what):
    if code != 0:
        raise OracleError(f"{what} failed with code {code}")


def set_threads(n):
    lib().ora_set_threads(int(n))


def fd_weights(npd, order):
    w = np.zeros(npd)
    _check(lib().ora_fd_weights(npd, order, _dp(w)), "ora_fd_weights")
    return w


def fd_rows(npd, order):
    """The whole npd x npd Bickley matrix (rows = nodes), no 1/h^order."""
    w = np.zeros(npd * npd)
    _check(lib().ora_fd_rows(npd, order, _dp(w)), "ora_fd_rows")
    return w.reshape(npd, npd)


def si(x):
    return lib().ora_si(float(x))


def v_he2s_fci(x):
    """V_He2s_fci(x) in K (binary128 sums, rounded to double)."""
    return lib().ora_v_he2s_fci(float(x))


def fft3_r2c(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    nz, ny, nx = a.shape
    out = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
    _check(lib().ora_fft3_r2c(nx, ny, nz, _dp(a), _dp(out.view(np.float64))), "r2c")
    return out


def fft3_c2r(s, nx):
    s = np.ascontiguousarray(s, dtype=np.complex128)
    nz, ny, _ = s.shape
    out = np.zeros((nz, ny, nx))
    _check(lib().ora_fft3_c2r(nx, ny, nz, _dp(s.view(np.float64)), _dp(out)), "c2r")
    return out


def spline(x, y, s1, sn):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = len(x)
    a, b, c, d = (np.zeros(n) for _ in range(4))
    _check(lib().ora_spline(_dp(x), _dp(y), _dp(a), _dp(b), _dp(c), _dp(d), s1, sn, n), "spline")
    return a, b, c, d


class Oracle:
    """CPU restatement of the reference step with the product's call surface."""

    def __init__(self, params):
        from ctypes import byref
        self.p = params
        self._h = C.c_void_p()
        _check(lib().ora_create(byref(params), byref(self._h)), "ora_create")
        self.shape = (params.nz, params.ny, params.nx)
        self.hshape = (params.nz, params.ny, params.nx // 2 + 1)
        self.npar = params.n_par

    def close(self):
        if self._h:
            lib().ora_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, psi, rimp, vimp):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        rimp = np.ascontiguousarray(rimp, dtype=np.float64)
        vimp = np.ascontiguousarray(vimp, dtype=np.float64)
        _check(lib().ora_set_state(self._h, _dp(psi.view(np.float64)), _dp(rimp), _dp(vimp)), "set_state")

    def get_state(self):
        psi = np.zeros(self.shape, dtype=np.complex128)
        r, v, a = (np.zeros((3, self.npar)) for _ in range(3))
        _check(lib().ora_get_state(self._h, _dp(psi.view(np.float64)), _dp(r), _dp(v), _dp(a)), "get_state")
        return psi, r, v, a

    def potenimp(self):
        _check(lib().ora_potenimp(self._h), "potenimp")

    def poten(self):
        _check(lib().ora_poten(self._h), "poten")

    def forceimp(self):
        _check(lib().ora_forceimp(self._h), "forceimp")

    def field(self):
        _check(lib().ora_field(self._h), "field")

    def steprk(self, dt):
        m = np.zeros(9)
        _check(lib().ora_step_rk(self._h, dt, _dp(m)), "steprk")
        return m

    def steppc(self, dt):
        e, m = np.zeros(3), np.zeros(9)
        _check(lib().ora_step_pc(self._h, dt, _dp(e), _dp(m)), "steppc")
        return e, m

    def run(self, nsteps, dt):
        e, m = np.zeros((nsteps, 3)), np.zeros((nsteps, 9))
        _check(lib().ora_run(self._h, nsteps, dt, _dp(e), _dp(m)), "run")
        return e, m

    def energy(self):
        import sys
        pkg = sys.modules.get("he4b200")
        from_abi = pkg.abi if pkg is not None else None
        if from_abi is None:
            raise OracleError("package he4b200 must be loaded for the energy struct")
        E = from_abi.He4Energies()
        _check(lib().ora_energy(self._h, C.byref(E)), "energy")
        return E.as_dict()

    def diagnostics(self, n4):
        out = np.zeros(4)
        _check(lib().ora_diagnostics(self._h, n4, _dp(out)), "diagnostics")
        return out

    def bubble_radius(self, nr=501):
        rb = C.c_double(0.0)
        found = (C.c_int32 * 2)()
        ir = C.c_int32(0)
        xms, rr, denr = np.zeros(3), np.zeros(nr), np.zeros(nr)
        _check(lib().ora_bubble_radius(self._h, nr, C.byref(rb), found, C.byref(ir), _dp(xms), _dp(rr), _dp(denr)),
               "bubble_radius")
        return {"rb": rb.value, "lcontrol": (bool(found[0]), bool(found[1])), "ir": ir.value, "xms": xms,
                "rr": rr, "denr": denr}

    def get_field(self, name):
        import sys
        ids = sys.modules["he4b200"].abi.FIELD_ID
        out = np.zeros(self.shape)
        _check(lib().ora_get_field(self._h, ids[name], _dp(out)), "get_field")
        return out

    def get_kernel(self, name):
        import sys
        ids = sys.modules["he4b200"].abi.KERNEL_ID
        out = np.zeros(self.hshape)
        _check(lib().ora_get_kernel(self._h, ids[name], _dp(out)), "get_kernel")
        return out

    def deriv(self, f, order, axis):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros_like(f)
        _check(lib().ora_deriv(self._h, order, axis, _dp(f), _dp(out)), "deriv")
        return out


def bubble_search(denr, dr, xnorm, xms):
    """The search half of Bubble_Radius_esferic on a binned radial density
    (bubble_radius_esferic.f90:63-132).  Returns (rb, (Lcontrol1, Lcontrol2),
    ir, rr, normalised denr)."""
    d = np.ascontiguousarray(denr, dtype=np.float64).copy()
    nr = d.size
    rr = np.zeros(nr)
    x = np.ascontiguousarray(xms, dtype=np.float64)
    rb = C.c_double(0.0)
    found = (C.c_int32 * 2)()
    ir = C.c_int32(0)
    _check(lib().ora_bubble_search(nr, dr, xnorm, _dp(x), _dp(rr), _dp(d), C.byref(rb), found, C.byref(ir)),
           "bubble_search")
    return rb.value, (bool(found[0]), bool(found[1])), ir.value, rr, d
