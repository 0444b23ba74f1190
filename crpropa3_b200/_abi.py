"""ctypes mirror of include/crp_gpu.h and the loader of the engine library.

The engine is the shared library ``crpropa3_b200/lib/libcrp_b200.so`` built by
``__graft_entry__.build()`` (nvcc, sm_100a).  Loading fails loudly when the
library is missing: there is no CPU fallback for the stepping path.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libcrp_b200.so")

ABI_VERSION = 9

# crp_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_TIMEOUT = 5
ERR_CANCELLED = 6
ERR_CAPACITY = 7
ERR_NO_DEVICE = 8

STATUS_NAMES = {
    OK: "CRP_OK", ERR_INVALID_ARGUMENT: "CRP_ERR_INVALID_ARGUMENT",
    ERR_UNSUPPORTED: "CRP_ERR_UNSUPPORTED", ERR_CUDA: "CRP_ERR_CUDA",
    ERR_OUT_OF_MEMORY: "CRP_ERR_OUT_OF_MEMORY", ERR_TIMEOUT: "CRP_ERR_TIMEOUT",
    ERR_CANCELLED: "CRP_ERR_CANCELLED", ERR_CAPACITY: "CRP_ERR_CAPACITY",
    ERR_NO_DEVICE: "CRP_ERR_NO_DEVICE",
}

FIELD_GRID, FIELD_PLANE_WAVE, FIELD_UNIFORM, FIELD_TOROIDAL, FIELD_MODULATED_GRID, FIELD_JF12, FIELD_UF23, \
    FIELD_PT11, FIELD_ARCHIMEDEAN_SPIRAL, FIELD_TF17, FIELD_SINGLE_MODE, FIELD_KST24, FIELD_CMZ = \
    1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13
PT11_ASS, PT11_BSS, PT11_HALO = 0, 1, 2
TF17_AD1, TF17_BD1, TF17_DD1 = 0, 1, 2
TF17_C0, TF17_C1 = 0, 1
SINGLE_MODE_AMPLITUDE, SINGLE_MODE_RMS = 0, 1
SINGLE_MODE_POLARIZATION, SINGLE_MODE_HELICITY = 0, 1
SINGLE_MODE_ELLIPTICAL, SINGLE_MODE_CIRCULAR, SINGLE_MODE_LINEAR = 0, 1, 2
UF23_BASE, UF23_NECL, UF23_EXPX, UF23_SPUR, UF23_CRE10, UF23_SYNCG, UF23_TWISTX, UF23_NEBCOR = range(8)
JF12_VARIANT_JF12, JF12_VARIANT_PLANCK, JF12_VARIANT_SOLENOIDAL = 0, 1, 2
INTERPOLATION_TRILINEAR, INTERPOLATION_TRICUBIC, INTERPOLATION_NEAREST_NEIGHBOUR = 0, 1, 2
MODULE_PROPAGATION, MODULE_MAX_TRAJECTORY_LENGTH, MODULE_OBSERVER, MODULE_BOUNDARY = 1, 2, 3, 4
PROP_CK, PROP_BP, PROP_SDE = 1, 2, 3
OBSERVER_SURFACE_SPHERE, OBSERVER_DETECT_ALL, OBSERVER_SURFACE_PLANE, OBSERVER_SURFACE_BOX = 1, 2, 3, 4
OBSERVER_TRACKING, OBSERVER_1D, OBSERVER_INACTIVE_VETO, OBSERVER_NUCLEUS_VETO = 5, 6, 7, 8
OBSERVER_NEUTRINO_VETO, OBSERVER_PHOTON_VETO, OBSERVER_ELECTRON_VETO, OBSERVER_PARTICLE_ID_VETO = 9, 10, 11, 12
MAX_OBSERVER_FEATURES = 4
BOUNDARY_SPHERICAL, BOUNDARY_CUBIC, BOUNDARY_ELLIPSOIDAL, BOUNDARY_CYLINDRICAL = 1, 2, 3, 4
PRECISION_FP64, PRECISION_MIXED = 0, 1
FLAG_REJECTED, FLAG_DETECTED, FLAG_NAN = 1, 2, 4
MODE_AUTO, MODE_CHUNKED, MODE_PERSISTENT = 0, 1, 2

_d = C.c_double
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)


class GridDesc(C.Structure):
    _fields_ = [("values", _fp), ("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64),
                ("origin", _d * 3), ("spacing", _d * 3), ("reflective", C.c_int32),
                ("clip_volume", C.c_int32), ("interpolation", C.c_int32), ("_pad", C.c_int32)]


class PlaneWaveDesc(C.Structure):
    _fields_ = [("n_modes", C.c_int32), ("seed", C.c_int32), ("xi", _dp), ("kappa", _dp),
                ("k", _dp), ("beta", _dp), ("ak", _dp), ("brms", _d), ("lmin", _d),
                ("lmax", _d), ("lbendover", _d), ("sindex", _d), ("qindex", _d)]


TURBULENCE_GRID, TURBULENCE_SIMPLE, TURBULENCE_HELICAL = 0, 1, 2


class TurbulenceDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("seed", C.c_int32), ("n", C.c_uint64), ("spacing", _d), ("brms", _d),
                ("lmin", _d), ("lmax", _d), ("lbendover", _d), ("sindex", _d), ("qindex", _d),
                ("helicity", _d)]


class JF12Desc(C.Structure):
    _fields_ = [("use_regular", C.c_int32), ("use_disk", C.c_int32), ("use_toroidal_halo", C.c_int32),
                ("use_x", C.c_int32), ("use_striated", C.c_int32), ("use_turbulent", C.c_int32),
                ("variant", C.c_int32), ("_pad", C.c_int32), ("kpc", _d), ("sin_pitch", _d), ("cos_pitch", _d), ("tan90_minus_pitch", _d),
                ("r_arms", _d * 8), ("b_ring", _d), ("h_disk", _d), ("w_disk", _d), ("b_disk", _d * 8),
                ("b_north", _d), ("b_south", _d), ("r_north", _d), ("r_south", _d), ("w_halo", _d),
                ("z0", _d), ("b_x", _d), ("sin_theta_x0", _d), ("cos_theta_x0", _d), ("tan_theta_x0", _d),
                ("r_xc", _d), ("r_x", _d), ("sqrt_beta", _d), ("b_disk_turb", _d * 8),
                ("b_disk_turb5", _d), ("z_disk_turb", _d), ("b_halo_turb", _d), ("r_halo_turb", _d),
                ("z_halo_turb", _d), ("cot_pitch", _d), ("cot_theta_x0", _d), ("z_s", _d), ("delta", _d),
                ("r1", _d), ("r2", _d), ("r1s", _d), ("r2s", _d), ("phi0_arms", _d * 11), ("b_arms", _d * 11),
                ("phi_coeff", _d * 10)]


class UF23Desc(C.Structure):
    _fields_ = [("model", C.c_int32), ("_pad", C.c_int32)] + [
        (n, _d) for n in ("disk_b1", "disk_b2", "disk_b3", "disk_h", "disk_phase1", "disk_phase2", "disk_phase3",
                          "disk_pitch", "disk_w", "poloidal_a", "poloidal_b", "poloidal_p", "poloidal_r",
                          "poloidal_w", "poloidal_z", "poloidal_xi", "spur_center", "spur_length", "spur_width",
                          "striation", "toroidal_bn", "toroidal_bs", "toroidal_r", "toroidal_w", "toroidal_z",
                          "twisting_time", "sin_pitch", "cos_pitch", "tan_pitch", "max_radius_squared", "kpc",
                          "microgauss")]


class PT11Desc(C.Structure):
    _fields_ = [("use_ass", C.c_int32), ("use_bss", C.c_int32), ("use_halo", C.c_int32), ("_pad", C.c_int32)] + [
        (n, _d) for n in ("d", "r_sun", "r_c", "z0_d", "b0_d", "z0_h", "r0_h", "b0_hn", "b0_hs", "z11_h", "z12_h",
                          "pitch", "cos_pitch", "sin_pitch", "phi", "cos_phi")]


class ArchimedeanDesc(C.Structure):
    _fields_ = [("b0", _d), ("r0", _d), ("omega", _d), ("vw", _d)]


class TF17Desc(C.Structure):
    _fields_ = [("disk_model", C.c_int32), ("halo_model", C.c_int32), ("use_disk", C.c_int32),
                ("use_halo", C.c_int32)] + [
        (n, _d) for n in ("a_disk", "z1_disk", "r1_disk", "b1_disk", "l_disk", "phi_star_disk", "h_disk",
                          "a_halo", "z1_halo", "b1_halo", "l_halo", "phi_star_halo",
                          "p0", "cot_p0", "h_p", "l_p", "epsilon")]


class SingleModeDesc(C.Structure):
    _fields_ = [("b_max", _d), ("sigma", _d), ("r0", _d * 3), ("u1", _d * 3), ("u2", _d * 3), ("k", _d * 3),
                ("b0", _d), ("wavelength", _d), ("e1", _d * 3), ("e2", _d * 3),
                ("amplitude_rms", C.c_int32), ("polarization_helicity", C.c_int32), ("mode", C.c_int32),
                ("_pad", C.c_int32)]


class KST24Arm(C.Structure):
    _fields_ = [(n, _d) for n in ("b", "pitch_deg", "phi0_deg", "x_shift", "y_shift", "arc_radius1", "arc_radius2",
                                  "arc_eps", "arc_div_deg", "rmin", "rmax", "zmin", "zmax")]


class KST24Desc(C.Structure):
    _fields_ = [(n, _d) for n in ("north_b", "north_zmin", "north_zmax", "north_rmin", "north_rmax",
                                  "south_b", "south_zmin", "south_zmax", "south_rmin", "south_rmax",
                                  "x_b", "x_rmin", "x_rmax", "x_theta_rad",
                                  "lb_b", "lb_rmin", "lb_dr", "lb_x0", "lb_y0", "lb_z0")] + [
        ("lb_dir", _d * 3), ("arms", KST24Arm * 5), ("kpc", _d), ("gauss", _d)]


class CMZCloud(C.Structure):
    _fields_ = [("mid", _d * 3), ("b1", _d), ("eta", _d), ("r", _d)]


class CMZPoloidal(C.Structure):
    _fields_ = [("mid", _d * 3), ("b", _d), ("a", _d), ("l", _d)]


class CMZDesc(C.Structure):
    _fields_ = [("use_mc", C.c_int32), ("use_ic", C.c_int32), ("use_ntf", C.c_int32), ("use_radio_arc", C.c_int32),
                ("clouds", CMZCloud * 12), ("sgra_shift", _d * 3), ("sgra_r", _d), ("sgra_b1", _d),
                ("ic", CMZPoloidal), ("ntf", CMZPoloidal * 7), ("radio_arc", CMZPoloidal), ("gauss", _d)]


class FieldComponent(C.Structure):
    _fields_ = [("kind", C.c_int32), ("periodic", C.c_int32), ("periodic_reflective", C.c_int32),
                ("_pad0", C.c_int32), ("periodic_origin", _d * 3), ("periodic_extends", _d * 3),
                ("grid", GridDesc), ("plane_wave", PlaneWaveDesc), ("uniform", _d * 3),
                ("toroidal_b0", _d), ("modulation", GridDesc), ("jf12", JF12Desc),
                ("uf23", UF23Desc), ("pt11", PT11Desc),
                ("archimedean", ArchimedeanDesc), ("tf17", TF17Desc), ("single_mode", SingleModeDesc),
                ("kst24", KST24Desc), ("cmz", CMZDesc)]


class FeatureDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("particle_id", C.c_int32), ("a", _d * 3), ("b", _d * 3),
                ("r", _d), ("step", _d)]


ADVECTION_UNIFORM, ADVECTION_CONSTANT_SPHERICAL, ADVECTION_SPHERICAL, ADVECTION_CARTESIAN_SHOCK, \
    ADVECTION_SPHERICAL_SHOCK_1D, ADVECTION_OBLIQUE_SHOCK, ADVECTION_SPHERICAL_SHOCK, ADVECTION_TIME_SHOCK, \
    ADVECTION_SEDOV_TAYLOR = 1, 2, 3, 4, 5, 6, 7, 8, 9
MAX_ADVECTION = 4


class AdvectionDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("cool_upstream", C.c_int32), ("value", _d * 3), ("origin", _d * 3)] + [
        (n, _d) for n in ("v", "radius", "tau", "alpha", "compression", "length", "vy", "r_rot", "v_phi",
                          "v1", "v0", "x0", "t0", "energy", "density")]


class ModuleDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("propagator", C.c_int32), ("tolerance", _d),
                ("min_step", _d), ("max_step", _d), ("sde_epsilon", _d), ("sde_alpha", _d),
                ("sde_scale", _d), ("n_advection", C.c_int32), ("_pad_adv", C.c_int32),
                ("advection", AdvectionDesc * MAX_ADVECTION),
                ("max_length", _d), ("per_candidate_length", C.c_int32),
                ("observer_feature", C.c_int32), ("sphere_center", _d * 3),
                ("sphere_radius", _d), ("deactivate_on_detection", C.c_int32),
                ("record", C.c_int32), ("n_features", C.c_int32), ("boundary", C.c_int32),
                ("features", FeatureDesc * 4), ("boundary_a", _d * 3), ("boundary_b", _d * 3),
                ("boundary_size", _d), ("boundary_radius", _d), ("boundary_margin", _d),
                ("boundary_limit_step", C.c_int32), ("_pad1", C.c_int32)]


class PlanDesc(C.Structure):
    _fields_ = [("abi_version", C.c_uint32), ("precision", C.c_int32),
                ("fields", C.POINTER(FieldComponent)), ("n_fields", C.c_int32),
                ("n_modules", C.c_int32), ("modules", C.POINTER(ModuleDesc)),
                ("seed", C.c_uint64)]


CANDIDATE_FIELDS = [
    ("id", C.c_int32), ("charge", _d), ("energy", _d), ("x", _d), ("y", _d), ("z", _d),
    ("dx", _d), ("dy", _d), ("dz", _d), ("px", _d), ("py", _d), ("pz", _d),
    ("trajectory_length", _d), ("time", _d), ("current_step", _d), ("next_step", _d),
    ("active", C.c_uint8), ("flags", C.c_uint32), ("max_length", _d),
    ("step_count", C.c_uint64),
]


class SourceDesc(C.Structure):
    _fields_ = [("n_types", C.c_int32), ("spectrum", C.c_int32), ("ids", C.POINTER(C.c_int32)),
                ("abundances", _dp), ("emin", _d), ("emax", _d), ("index", _d), ("energy", _d),
                ("isotropic", C.c_int32), ("_pad0", C.c_int32), ("direction", _d * 3)]


class OutputDesc(C.Structure):
    _fields_ = [("columns", C.c_uint32), ("one_dimensional", C.c_int32), ("length_scale", _d),
                ("time_scale", _d), ("energy_scale", _d), ("version", C.c_char_p)]


class OutputRows(C.Structure):
    _fields_ = [("serial", C.POINTER(C.c_uint64)), ("trajectory_length", _dp), ("time", _dp),
                ("id", C.POINTER(C.c_int32)), ("energy", _dp), ("position", _dp),
                ("direction", _dp), ("source_id", C.POINTER(C.c_int32)), ("source_energy", _dp),
                ("source_position", _dp), ("source_direction", _dp), ("weight", _dp)]


class NoAllocGridBpDesc(C.Structure):
    _fields_ = [("grid_values", C.c_void_p), ("nx", C.c_uint64), ("ny", C.c_uint64),
                ("nz", C.c_uint64), ("origin", _d * 3), ("spacing", _d * 3),
                ("reflective", C.c_int32), ("clip_volume", C.c_int32), ("step", _d),
                ("max_length", _d), ("precision", C.c_int32), ("steps_per_launch", C.c_int32)]


NOALLOC_MAX_CANDIDATES = 1 << 20


class Candidates(C.Structure):
    _fields_ = [(name, C.POINTER(t)) for name, t in CANDIDATE_FIELDS]


RECORD_FIELDS = [
    ("index", C.c_uint64), ("module", C.c_int32), ("trajectory_length", _d), ("time", _d),
    ("x", _d), ("y", _d), ("z", _d), ("dx", _d), ("dy", _d), ("dz", _d), ("energy", _d),
    ("id", C.c_int32),
]


class Records(C.Structure):
    _fields_ = [("capacity", C.c_uint64), ("count", C.POINTER(C.c_uint64))] + \
               [(name, C.POINTER(t)) for name, t in RECORD_FIELDS]


class RunOpts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("block_size", C.c_int32), ("ctas_per_sm", C.c_int32),
                ("steps_per_launch", C.c_int32), ("refill_threshold", C.c_int32),
                ("budget_us", C.c_int32), ("max_steps", C.c_uint64),
                ("cancel", C.POINTER(C.c_int32)), ("stream", C.c_void_p),
                ("records", C.POINTER(Records))]


class AdjointDesc(C.Structure):
    _fields_ = [("grid_values", C.c_void_p), ("nx", C.c_uint64), ("ny", C.c_uint64),
                ("nz", C.c_uint64), ("origin", _d * 3), ("spacing", _d * 3), ("step", _d),
                ("n_steps", C.c_int32), ("checkpoint_every", C.c_int32)]


class AdjointIO(C.Structure):
    _fields_ = [("n", C.c_uint64)] + [(k, C.c_void_p) for k in (
        "x", "y", "z", "dx", "dy", "dz", "energy", "charge", "tx", "ty", "tz", "loss", "ux", "uy",
        "uz", "grad_dx", "grad_dy", "grad_dz", "grad_energy", "grad_grid")]


class AutotuneResult(C.Structure):
    _fields_ = [("mode", C.c_int32), ("ctas_per_sm", C.c_int32), ("refill_threshold", C.c_int32),
                ("burst", C.c_int32), ("trials", C.c_int32), ("_pad0", C.c_int32),
                ("steps_per_second", _d), ("chunked_steps_per_second", _d)]


class RunStats(C.Structure):
    _fields_ = [("particle_steps", C.c_uint64), ("tries", C.c_uint64),
                ("field_evaluations", C.c_uint64), ("launches", C.c_uint64),
                ("active_left", C.c_uint64), ("device_ms", _d)]


_lib = None


class CrpError(RuntimeError):
    """A non-zero crp_status, carrying the status code and the library message."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load():
    """Load libcrp_b200.so; raises if it is absent (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"crpropa3_b200: engine library {LIB_PATH} is missing; run "
            "__graft_entry__.build() (nvcc, sm_100a) first")
    lib = C.CDLL(LIB_PATH)
    from . import _signatures
    _signatures.declare(lib)
    if lib.crp_abi_version() != ABI_VERSION:
        raise RuntimeError("crpropa3_b200: ABI version mismatch between Python and the library")
    _lib = lib
    return lib


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(4096)
    lib.crp_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(status):
    if status != OK:
        raise CrpError(status, last_error())
