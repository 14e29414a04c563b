"""ctypes binding of liboscars_b200.so (the C ABI declared in include/oscars_b200.h).

The library is the CUDA extension: importing this module fails loudly if it is missing or does not
load; there is no CPU fallback for the radiation calls.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboscars_b200.so")

OSC_OK = 0
STATUS_NAMES = {1: "invalid argument", 2: "out of range", 3: "length error", 4: "call order",
                5: "CUDA error", 6: "no usable GPU", 7: "allocation failed", 8: "device wait timeout"}

D = ctypes.c_double
I = ctypes.c_int
LL = ctypes.c_longlong
VP = ctypes.c_void_p
DP = ctypes.POINTER(D)
I32P = ctypes.POINTER(ctypes.c_int32)
LLP = ctypes.POINTER(LL)


class FieldDesc(ctypes.Structure):
    _fields_ = [("kind", I), ("bfield", D * 3), ("bfield_b", D * 3), ("period", D * 3), ("nperiods", I),
                ("center", D * 3), ("phase", D), ("taper", D), ("frequency", D), ("frequency_phase", D),
                ("time_offset", D), ("half_period_scale", DP), ("n_half_periods", I), ("grid_n", LL * 3),
                ("grid_start", D * 3), ("grid_step", D * 3), ("grid_values", DP), ("rotations", D * 3)]


class BeamDesc(ctypes.Structure):
    _fields_ = [("particle", I), ("charge", D), ("mass", D), ("energy_GeV", D), ("x0", D * 3), ("d0", D * 3),
                ("horizontal", D * 3), ("t0", D), ("current", D), ("sigma_energy_GeV", D), ("emittance", D * 2),
                ("has_emittance", I), ("beta", D * 2), ("alpha", D * 2), ("has_beta", I), ("has_alpha", I),
                ("eta", D * 2), ("distribution", I), ("ctstartstop", D * 2), ("has_ctstartstop", I),
                ("gamma", D * 2), ("has_gamma", I), ("lattice_reference", D * 3), ("has_lattice_reference", I),
                ("predefined", I), ("has_d0", I), ("weight", D)]


class RadOpts(ctypes.Structure):
    _fields_ = [("polarization", I), ("angle", D), ("horizontal", D * 3), ("propagation", D * 3),
                ("precision", D), ("max_level", I), ("max_level_extended", I), ("nparticles", I),
                ("quantity", I), ("precision_mode", I), ("shard_rank", I), ("shard_count", I)]


class JobDesc(ctypes.Structure):
    _fields_ = [("field_begin", I), ("field_count", I), ("particle", I), ("charge", D), ("mass", D),
                ("energy_GeV", D), ("x0", D * 3), ("d0", D * 3), ("t0", D), ("current", D), ("ctstart", D),
                ("ctstop", D), ("npoints", LL), ("obs_begin", LL), ("n_obs", LL), ("energy_begin", LL),
                ("n_energies", LL), ("spectrum", I)]


# name -> (restype, argtypes); this table is also the list of exported symbols the tests check
SIGNATURES = {
    "osc_get_device_count": (I, [ctypes.POINTER(I)]),
    "osc_ctx_create": (I, [I, ctypes.POINTER(VP)]),
    "osc_ctx_destroy": (None, [VP]),
    "osc_last_error": (ctypes.c_char_p, [VP]),
    "osc_version": (ctypes.c_char_p, []),
    "osc_clear_fields": (I, [VP]),
    "osc_add_field": (I, [VP, ctypes.POINTER(FieldDesc)]),
    "osc_get_bfield": (I, [VP, DP, D, DP]),
    "osc_add_field_file": (I, [VP, ctypes.c_char_p, ctypes.c_char_p, DP, DP, DP, I, D, D, D]),
    "osc_set_beam": (I, [VP, ctypes.POINTER(BeamDesc)]),
    "osc_add_beam": (I, [VP, ctypes.POINTER(BeamDesc), ctypes.c_char_p]),
    "osc_clear_beams": (I, [VP]),
    "osc_set_new_particle_of_beam": (I, [VP, ctypes.c_char_p, I]),
    "osc_set_seed": (I, [VP, I]),
    "osc_set_new_particle": (I, [VP, I]),
    "osc_get_particle": (I, [VP, DP, DP, DP, DP]),
    "osc_beam_particles": (I, [VP, LL, I, I, DP, LLP]),
    "osc_set_ctstartstop": (I, [VP, D, D]),
    "osc_get_ctstartstop": (I, [VP, DP, DP]),
    "osc_set_npoints_trajectory": (I, [VP, LL]),
    "osc_set_trajectory_calculation": (I, [VP, ctypes.c_char_p, D]),
    "osc_get_trajectory_calculation": (I, [VP, ctypes.POINTER(ctypes.c_int), DP]),
    "osc_get_npoints_trajectory": (I, [VP, LLP]),
    "osc_calculate_trajectory": (I, [VP]),
    "osc_get_trajectory": (I, [VP, DP, LL, LLP]),
    "osc_surface_rectangle": (I, [ctypes.c_char_p, I, I, D, D, DP, DP, I, DP, DP, DP]),
    "osc_surface_x0x1x2": (I, [I, I, DP, DP, DP, I, DP, DP, DP]),
    "osc_surface_points": (I, [LL, DP, DP, DP, DP, I, DP, DP]),
    "osc_flux": (I, [VP, DP, LL, D, ctypes.POINTER(RadOpts), DP, I32P, LLP]),
    "osc_spectrum": (I, [VP, DP, DP, LL, ctypes.POINTER(RadOpts), DP, I32P, LLP]),
    "osc_flux_multi": (I, [VP, DP, LL, DP, LL, ctypes.POINTER(RadOpts), I, DP, I32P, LLP]),
    "osc_power_density": (I, [VP, DP, DP, LL, I, ctypes.POINTER(RadOpts), DP, I32P, LLP]),
    "osc_power_density_stl": (I, [VP, DP, DP, LL, ctypes.POINTER(RadOpts), DP, I32P, LLP]),
    "osc_flux_device": (I, [VP, VP, LL, D, ctypes.POINTER(RadOpts), VP, VP, VP]),
    "osc_power_density_device": (I, [VP, VP, VP, LL, I, ctypes.POINTER(RadOpts), VP, VP, VP]),
    "osc_batch_flux": (I, [VP, ctypes.POINTER(FieldDesc), I, ctypes.POINTER(JobDesc), I, DP, LL, DP, LL,
                           ctypes.POINTER(RadOpts), I, DP, I32P, LLP]),
    "osc_set_particle_trajectory": (I, [VP, I, D, D, D, DP, DP, D, DP, LL]),
    "osc_get_device_properties": (I, [I, ctypes.c_char_p, LL]),
    "osc_batch_trajectories": (I, [VP, ctypes.POINTER(FieldDesc), I, ctypes.POINTER(JobDesc), I, DP, LL, LLP]),
    "osc_set_half_period_scale": (I, [VP, I, DP, LL]),
    "osc_trajectory_vjp": (I, [VP, DP, LL, DP, LL]),
    "osc_flux_vjp": (I, [VP, DP, LL, DP, LL, I, ctypes.POINTER(RadOpts), I, DP, DP, DP, LL, DP]),
    "osc_last_stats": (I, [VP, LLP, LLP]),
    "osc_set_profiling": (I, [VP, I]),
    "osc_set_beam_batch_threshold": (I, [VP, I]),
    "osc_set_batch_spline_kernel": (I, [VP, I]),
    "osc_get_profile": (I, [VP, DP, LLP, LLP, I]),
    "osc_set_variant": (I, [VP, I, I]),
    "osc_get_variant": (I, [VP, I, ctypes.POINTER(I), ctypes.POINTER(I)]),
    "osc_variant_name": (I, [I, I, ctypes.c_char_p, ctypes.c_longlong]),
    "osc_drop_level_cache": (I, [VP]),
    "osc_measure_fma_peak": (I, [VP, I, DP]),
    "osc_flux_fixed_level_noalloc": (I, [I, DP, LL, DP, LL, D, I, D, D, DP, DP, ctypes.c_char_p, LL]),
}

_lib = None


def lib():
    """Load liboscars_b200.so once; raise ImportError with the reason when it cannot load."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("oscars_b200: %s is missing; build it with `python -m oscars_b200.build`" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def dptr(a):
    return a.ctypes.data_as(DP)


def i32ptr(a):
    return a.ctypes.data_as(I32P)


class Context:
    """Owns one osc_ctx."""

    def __init__(self, device: int = 0):
        L = lib()
        h = VP()
        rc = L.osc_ctx_create(int(device), ctypes.byref(h))
        if rc != OSC_OK:
            raise RuntimeError("oscars_b200: cannot create a context on device %d: %s"
                               % (device, L.osc_last_error(None).decode()))
        self.h = h
        self.L = L
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.L.osc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        rc = getattr(self.L, name)(self.h, *args)
        if rc != OSC_OK:
            msg = self.L.osc_last_error(self.h).decode()
            if rc in (5, 6, 7, 8):
                raise RuntimeError("oscars_b200 %s (%s): %s" % (name, STATUS_NAMES.get(rc, rc), msg))
            raise ValueError(msg)
        return rc


def variant_name(kind: int, variant: int) -> str:
    """Kernel and template arguments of compiled variant `variant` of kind 0 (FP64 flux), 2 (mixed)
    or 3 (batched mixed)."""
    buf = ctypes.create_string_buffer(96)
    rc = lib().osc_variant_name(int(kind), int(variant), buf, len(buf))
    if rc != OSC_OK:
        raise ValueError(lib().osc_last_error(None).decode())
    return buf.value.decode()


def device_count() -> int:
    n = I(0)
    lib().osc_get_device_count(ctypes.byref(n))
    return n.value
