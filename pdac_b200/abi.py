"""ctypes mirror of include/pdac_gpu.h (the engine's C ABI).

The structures here are the exact field-for-field layout of ``pdac_cfg`` and
``pdac_state_view``; they are the host-side representation of the
reference's namelist variables (input.f:159-209) and of its module-global
state arrays (press.f, velocity.f, dens.f, temp.f, eosg.f).
"""
import ctypes as C

PDAC_OK = 0
PDAC_ERR_CONFIG = 1
PDAC_ERR_CUDA = 2
PDAC_ERR_MAXOUT = 3
PDAC_ERR_EOS = 4
PDAC_ERR_NONFINITE = 5
PDAC_ERR_ARG = 6
PDAC_ERR_BOUNDARY = 7
PDAC_ERR_TIMEOUT = 8

STATUS_NAMES = {
    0: "ok", 1: "config", 2: "cuda", 3: "maxout", 4: "eos", 5: "nonfinite",
    6: "arg", 7: "boundary", 8: "timeout",
}

# cell flags, grid.f:45-58
FLUID, SLIP_WALL, NOSLIP_WALL, FREE_IO, INLET_CELL, ZERO_GRAD, VENT_CELL = 1, 2, 4, 8, 16, 32, 64

MAX_NSOLID = 8
MAX_NGAS = 7

PREC_FP64 = 0
PREC_MIXED = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class PdacCfg(C.Structure):
    _fields_ = [
        ("job_type", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("itc", C.c_int), ("nsolid", C.c_int), ("ngas", C.c_int),
        ("gas_type", C.c_int * MAX_NGAS),
        ("dt", C.c_double), ("rungekut", C.c_int), ("time_integration", C.c_int),
        ("alpha", C.c_double), ("alphagrav", C.c_double),
        ("omega", C.c_double), ("delg", C.c_double),
        ("inmax", C.c_int), ("maxout", C.c_int), ("cstop", C.c_int),
        ("muscl", C.c_int), ("lv", C.c_int), ("lm", C.c_int),
        ("beta", C.c_double), ("flim", C.c_double), ("update_eosg", C.c_int),
        ("implicit_fluxes", C.c_int), ("implicit_enthalpy", C.c_int), ("optimization", C.c_int),
        ("pmodel", C.c_int), ("drag_model", C.c_int), ("icpc", C.c_int),
        ("tref", C.c_double),
        ("gas_viscosity", C.c_int), ("part_viscosity", C.c_int), ("repulsive_model", C.c_int),
        ("iturb", C.c_int), ("modturbo", C.c_int), ("iss", C.c_int), ("cmut", C.c_double),
        ("gravx", C.c_double), ("gravy", C.c_double), ("gravz", C.c_double),
        ("dk", C.c_double * MAX_NSOLID), ("rl", C.c_double * MAX_NSOLID),
        ("phis", C.c_double * MAX_NSOLID), ("cmus", C.c_double * MAX_NSOLID),
        ("cps", C.c_double * MAX_NSOLID), ("kap", C.c_double * MAX_NSOLID),
        ("plim", C.c_double * MAX_NSOLID),
        ("void_fraction", C.c_double), ("atm_ygc", C.c_double * MAX_NGAS),
        ("irand", C.c_int),
        ("isink", C.c_int), ("rprox", C.c_double), ("rdist", C.c_double),
        ("center_x", C.c_double), ("center_y", C.c_double),
        ("compute_mixture", C.c_int), ("formatted_output", C.c_int),
        ("precision", C.c_int),
        ("dx", _dp), ("dy", _dp), ("dz", _dp), ("flag", _ip),
        ("p_atm", _dp), ("t_atm", _dp),
        ("nvent", C.c_int), ("vent_ijk", _ip),
        ("immb", C.c_int), ("ib_faces", _ip), ("ib_ivf", _dp),
        ("ib_num", _ip * 3), ("ib_nfp", C.c_int * 3), ("ib_fp", _ip * 3), ("ib_nsl", _dp * 3),
        ("x", _dp), ("xb", _dp), ("y", _dp), ("yb", _dp), ("z", _dp), ("zb", _dp),
        ("zrough", C.c_double), ("topo_c", _dp),
    ]


class PdacStateView(C.Structure):
    _fields_ = [(n, _dp) for n in (
        "p", "ep", "rog", "rgp", "tg", "sieg", "cg",
        "ug", "vg", "wg",
        "rlk", "ts", "sies",
        "us", "vs", "ws",
        "ygc", "xgc")]


STATE_CELL = ("p", "ep", "rog", "rgp", "tg", "sieg", "cg", "ug", "vg", "wg")
STATE_SOLID = ("rlk", "ts", "sies", "us", "vs", "ws")
STATE_GAS = ("ygc", "xgc")
STATE_FIELDS = STATE_CELL + STATE_SOLID + STATE_GAS


def dptr(a):
    """Pointer to the data of a C-contiguous float64 numpy array (or NULL)."""
    if a is None:
        return C.cast(None, _dp)
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return C.cast(None, _ip)
    return a.ctypes.data_as(_ip)


def make_state_view(state):
    """Build a PdacStateView over the arrays of a ``State`` (kept alive by it)."""
    v = PdacStateView()
    for name in STATE_FIELDS:
        setattr(v, name, dptr(state.get(name)))
    return v


def declare(lib, prefix, handle_type):
    """Set argtypes/restype of the per-call entry points of ``lib``.

    ``prefix`` is ``pdac_gpu`` (the product) or ``pdac_oracle`` (the test
    oracle, which exposes the same call shape on a void* handle)."""
    h = handle_type
    sigs = {
        "boundary": [h, C.c_int],
        "fieldn": [h],
        "initialize_fieldn": [h],
        "tilde": [h, C.c_double],
        "explicit_iter": [h, C.c_double],
        "iter": [h, C.c_double, C.POINTER(C.c_int)],
        "ygas": [h, C.c_double],
        "htilde": [h, C.c_double],
        "ftem": [h, C.c_double],
        "step": [h, C.c_int, C.POINTER(C.c_int)],
        "get_array": [h, C.c_char_p, _dp, C.POINTER(C.c_long)],
        "mass_totals": [h, _dp, C.c_int],
    }
    if prefix == "pdac_gpu":
        sigs.update({
            "sgsg": [h],
            "sgss": [h],
            "write_restart": [h, C.c_char_p, C.c_double, C.c_int],
            "read_restart": [h, C.c_char_p, _dp, C.POINTER(C.c_int)],
            "write_output": [h, C.c_char_p, C.c_double],
            "compute_mixture_fields": [h],
            "mass_residuals": [h, C.c_int, C.c_double, _dp, C.c_int],
            "append_mass_check": [h, C.c_char_p, C.c_int, C.c_double],
            "write_mass_loss": [h, C.c_char_p],
            "read_mass_loss": [h, C.c_char_p],
        })
    if prefix == "pdac_oracle":
        sigs["sgs"] = [h]
    for name, args in sigs.items():
        fn = getattr(lib, f"{prefix}_{name}")
        fn.argtypes = args
        fn.restype = C.c_int
