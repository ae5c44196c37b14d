"""ctypes mirror of include/he4_tddft.h (types and constants only).

The structure layouts must match the C header field for field; the
`test_abi_layout` test checks the sizes against the compiled library.
"""
import ctypes as C

HE4_OK = 0
HE4_E_ARG = -1
HE4_E_UNSUPPORTED = -2
HE4_E_NOMEM = -3
HE4_E_CUDA = -4
HE4_E_STATE = -5
HE4_E_NONFINITE = -6
HE4_E_NODEVICE = -7

HE4_CORE_OT = 0
HE4_CORE_OTC = 1

HE4_POT_TABLE = 0
HE4_POT_MORSE = 1
HE4_POT_NULL = 2
HE4_POT_RTABLE = 3
HE4_POT_HE2S_FCI = 4

HE4_PREC_FP64 = 0
HE4_PREC_FP32CONV = 1

HE4_D_PSI = 0
HE4_D_RIMP = 1
HE4_D_VIMP = 2
HE4_D_DEN = 3
HE4_D_DENX = 4

FIELDS = [
    "den", "pot4", "denx", "psix", "hpsix", "uimp", "dencg", "delj4", "denalf",
    "ualphas", "falfs", "intxalf", "intyalf", "intzalf", "dxden", "dyden",
    "dzden", "fx", "fy", "fz", "penalty", "corr",
]
FIELD_ID = {name: i for i, name in enumerate(FIELDS)}

KERNELS = ["wcgk", "fvlj4", "kalfs", "vq", "pmod"]
KERNEL_ID = {name: i for i, name in enumerate(KERNELS)}

ENERGY_NAMES = ["etot", "etot4", "ekin4", "elj4", "ecor4", "ealphas", "esolid",
                "ekinx", "ekinqx", "eHeX", "eimpu"]


class He4Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("npd", C.c_int32), ("icon", C.c_int32),
        ("core4", C.c_int32),
        ("cp4", C.c_double), ("cpp4", C.c_double), ("den4c", C.c_double),
        ("alphas", C.c_double), ("l_alfs", C.c_double), ("den0s", C.c_double),
        ("h2o2m4", C.c_double),
        ("c_solid", C.c_double), ("beta_solid", C.c_double), ("den_m", C.c_double),
        ("eps4", C.c_double), ("sigma4", C.c_double), ("b4", C.c_double), ("h4", C.c_double),
        ("n_par", C.c_int32), ("ironx", C.c_int32),
        ("mimpur", C.c_double),
        ("pot_kind", C.c_int32),
        ("morse_d", C.c_double), ("morse_alpha", C.c_double), ("morse_re", C.c_double),
        ("r_cutoff", C.c_double), ("umax", C.c_double),
        ("nq", C.c_int32),
        ("vq_table", C.POINTER(C.c_double)),
        ("lambdah", C.c_double), ("tzmean", C.c_double), ("tzsurf", C.c_double),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("vr_table", C.POINTER(C.c_double)),
        ("n_vr", C.c_int32),
        ("vr_r0", C.c_double), ("vr_dr", C.c_double),
    ]


class He4Energies(C.Structure):
    _fields_ = [(n, C.c_double) for n in ENERGY_NAMES]

    def as_dict(self):
        return {n: getattr(self, n) for n in ENERGY_NAMES}


def default_params():
    """Reference defaults (modules.f90:15-19,81-90,124-139,144,205-210;
    DFT4He3d.f90:184-186); same values as he4_params_default()."""
    p = He4Params()
    p.nx = p.ny = p.nz = 64
    p.xmax = p.ymax = p.zmax = 64.0
    p.npd = 7
    p.icon = 8
    p.core4 = HE4_CORE_OT
    p.cp4 = -2.41186e4
    p.cpp4 = 1.85850e6
    p.den4c = 0.062
    p.alphas = 54.31
    p.l_alfs = 1.0
    p.den0s = 0.04
    p.h2o2m4 = 6.05969638298
    p.c_solid = 3.1577504e4
    p.beta_solid = 40.0
    p.den_m = 0.37
    p.eps4 = 10.22
    p.sigma4 = 2.556
    p.b4 = -718.99
    p.h4 = 2.190323
    p.n_par = 100000
    p.ironx = 1
    p.mimpur = 4.002602
    p.pot_kind = HE4_POT_NULL
    p.morse_d = 0.0
    p.morse_alpha = 0.0
    p.morse_re = 0.0
    p.r_cutoff = 3.0
    p.umax = 400.0
    p.nq = 1000
    p.vq_table = None
    p.lambdah = 0.0
    p.tzmean = 0.0
    p.tzsurf = 1.0
    p.precision = HE4_PREC_FP64
    p.device = 0
    return p
