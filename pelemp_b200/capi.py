"""ctypes mirror of include/pmp_spray.h (structs, enums, constants).

Field order and types match the C header exactly; the tests check the sizes
against the library.
"""
import ctypes as C

PMP_MAX_FUEL = 4
PMP_MAX_SPEC = 8
PMP_NAME_LEN = 32


def pstate_num(nfuel):
    """SprayComps::pstateNum (Source/PP_Spray/SprayFuelData.H:19)."""
    return 10 + nfuel


PMP_MAX_RCOMP = pstate_num(PMP_MAX_FUEL)

# particle real component offsets (SprayFuelData.H:10-19)
PSTATE_VEL = 0
PSTATE_T = 3
PSTATE_DIA = 4
PSTATE_Y = 5


def pstate_numdens(f):
    return 5 + f


def pstate_filmhght(f):
    return 9 + f


PMP_OK = 0
PMP_COUPLING_LMEX = 0
PMP_COUPLING_PELEC = 1
PMP_ERR_LEFT_DOMAIN = 1
PMP_ERR_STATE_BOX = 2
PMP_ERR_SOURCE_BOX = 3
PMP_ERR_UNSUPPORTED = 4
PMP_ERR_TIMEOUT = 5
PMP_ERR_CUDA = 6
PMP_ERR_INVALID = 7
PMP_ERR_NO_DEVICE = 8

STATUS_NAMES = {
    0: "PMP_OK", 1: "PMP_ERR_LEFT_DOMAIN", 2: "PMP_ERR_STATE_BOX",
    3: "PMP_ERR_SOURCE_BOX", 4: "PMP_ERR_UNSUPPORTED", 5: "PMP_ERR_TIMEOUT",
    6: "PMP_ERR_CUDA", 7: "PMP_ERR_INVALID", 8: "PMP_ERR_NO_DEVICE",
}

PMP_MODE_FP64 = 0
PMP_MODE_MIXED = 1
PMP_MODE_LEARNED = 2

PMP_LAYOUT_AOS = 0
PMP_LAYOUT_SOA = 1
PMP_WHERE_HOST = 0
PMP_WHERE_DEVICE = 1


class Geometry(C.Structure):
    _fields_ = [
        ("plo", C.c_double * 3), ("phi", C.c_double * 3), ("dx", C.c_double * 3),
        ("domain_lo", C.c_int * 3), ("domain_hi", C.c_int * 3),
        ("bndry_lo", C.c_int * 3), ("bndry_hi", C.c_int * 3),
    ]


class Box(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3)]


class BoxView(C.Structure):
    _fields_ = [
        ("p", C.c_void_p), ("lo", C.c_int * 3), ("hi", C.c_int * 3),
        ("jstride", C.c_longlong), ("kstride", C.c_longlong),
        ("nstride", C.c_longlong), ("ncomp", C.c_int),
    ]


class SprayComps(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "rhoIndx", "momIndx", "engIndx", "utempIndx", "specIndx",
        "rhoSrcIndx", "momSrcIndx", "engSrcIndx", "specSrcIndx")]


F4 = C.c_double * PMP_MAX_FUEL
F16 = C.c_double * (4 * PMP_MAX_FUEL)
I4 = C.c_int * PMP_MAX_FUEL


class SprayData(C.Structure):
    _fields_ = [
        ("nfuel", C.c_int), ("mass_trans", C.c_int), ("mom_trans", C.c_int),
        ("fixed_parts", C.c_int), ("do_splash", C.c_int), ("do_breakup", C.c_int),
        ("min_eb_vfrac", C.c_double), ("ref_T", C.c_double), ("sigma", C.c_double),
        ("wall_T", C.c_double), ("theta_c", C.c_double), ("dtmod", C.c_double),
        ("body_force", C.c_double * 3),
        ("critT", F4), ("boilT", F4), ("cp", F4), ("latent", F4), ("ref_latent", F4),
        ("psat_coef", F16), ("rho_coef", F16), ("lambda_coef", F16), ("mu_coef", F16),
        ("indx", I4), ("dep_indx", I4),
    ]


NAME = C.c_char * PMP_NAME_LEN
C44 = (C.c_double * 4) * PMP_MAX_FUEL


class SprayInputs(C.Structure):
    _fields_ = [
        ("nfuel", C.c_int),
        ("fuel_species", NAME * PMP_MAX_FUEL),
        ("dep_fuel_species", NAME * PMP_MAX_FUEL),
        ("mass_transfer", C.c_int), ("mom_transfer", C.c_int),
        ("fixed_parts", C.c_int), ("use_splash_model", C.c_int),
        ("use_breakup_model", C.c_int),
        ("cfl", C.c_double), ("fuel_ref_temp", C.c_double),
        ("crit_temp", F4), ("boil_temp", F4), ("cp", F4), ("latent", F4),
        ("ncoef_lambda", I4), ("ncoef_psat", I4), ("ncoef_rho", I4), ("ncoef_mu", I4),
        ("lambda_", C44), ("psat", C44), ("rho", C44), ("mu", C44),
        ("body_force", C.c_double * 3),
    ]


class Particles(C.Structure):
    _fields_ = [
        ("layout", C.c_int), ("where", C.c_int), ("n", C.c_longlong),
        ("aos", C.c_void_p), ("pos", C.c_void_p * 3),
        ("rdata", C.c_void_p * PMP_MAX_RCOMP), ("id", C.c_void_p),
    ]


class SprayConfig(C.Structure):
    _fields_ = [
        ("nfuel", C.c_int), ("nspec", C.c_int),
        ("species", NAME * PMP_MAX_SPEC), ("device", C.c_int),
    ]


class ErrorInfo(C.Structure):
    _fields_ = [
        ("code", C.c_int), ("box", C.c_int), ("particle", C.c_longlong),
        ("pos", C.c_double * 3), ("message", C.c_char * 160),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("substeps", C.c_longlong), ("killed", C.c_longlong),
        ("inner_steps", C.c_longlong), ("fallback", C.c_longlong),
        ("kernel_ms", C.c_double), ("graph", C.c_int),
    ]


PMP_LAUNCH_GRID = 0
PMP_LAUNCH_PERSISTENT = 1
PMP_LAUNCH_PER_BOX = 2


class LaunchConfig(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("kind", "block", "regs", "chunk", "ctas_per_sm", "use_graph")]


class TuneReport(C.Structure):
    _fields_ = [
        ("cached", C.c_int), ("ncandidates", C.c_int), ("best_ms", C.c_double),
        ("default_ms", C.c_double), ("per_box_ms", C.c_double), ("best", LaunchConfig),
    ]


class LearnConfig(C.Structure):
    _fields_ = [
        ("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_double),
        ("gate_margin", C.c_double), ("audit_fraction", C.c_double),
        ("no_quant", C.c_int), ("seed", C.c_ulonglong),
    ]


class LearnReport(C.Structure):
    _fields_ = [
        ("tuples", C.c_longlong), ("steps", C.c_longlong),
        ("loss_first", C.c_double), ("loss_last", C.c_double),
        ("val_rel_rms", C.c_double * 5), ("train_ms", C.c_double),
        ("base_resid_frac", C.c_double * 5),
    ]


LEARN_IN = 10
LEARN_OUT = 5


# pmp_mech of pelemp_b200/csrc/phys/pmp_thermo.h (opaque blob of the right size
# for the oracle bindings; the layout is checked in the tests)
class Mech(C.Structure):
    _fields_ = [
        ("nspec", C.c_int), ("db_index", C.c_int * PMP_MAX_SPEC),
        ("mw", C.c_double * PMP_MAX_SPEC),
        ("cp", (C.c_double * 5) * PMP_MAX_SPEC),
        ("hc", (C.c_double * 6) * PMP_MAX_SPEC),
        ("mu", (C.c_double * 4) * PMP_MAX_SPEC),
        ("lam", (C.c_double * 4) * PMP_MAX_SPEC),
        ("dbin", ((C.c_double * 4) * PMP_MAX_SPEC) * PMP_MAX_SPEC),
    ]


def names_array(names, count=PMP_MAX_SPEC):
    arr = (NAME * count)()
    for i, n in enumerate(names):
        arr[i].value = n.encode()
    return arr
