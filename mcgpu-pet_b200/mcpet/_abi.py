"""ctypes declarations of the C ABI in include/mcpet.h.

The library is loaded from the package's ``lib/`` directory.  There is no
fallback: when ``libmcpet.so`` is missing the import fails with an error that
says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

MAX_MATERIALS = 15
MAX_SHELLS = 30
NP_RAYLEIGH = 128
MAX_ENERGY_BINS = 25005
PSF_RECORD_BYTES = 44

LANES_REFERENCE = 0
LANES_BALANCED = 1

ALGORITHM_AUTO = 0
ALGORITHM_HISTORIES = 1
ALGORITHM_EVENTS = 2

STATUS_NAMES = {
    0: "MCPET_OK",
    1: "MCPET_ERR_ARG",
    2: "MCPET_ERR_IO",
    3: "MCPET_ERR_FORMAT",
    4: "MCPET_ERR_CUDA",
    5: "MCPET_ERR_NOMEM",
    6: "MCPET_ERR_LIMIT",
    7: "MCPET_ERR_DEVICE",
}

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libmcpet.so")


class Config(C.Structure):
    _fields_ = [
        ("seed", C.c_int),
        ("gpu_id", C.c_int),
        ("threads_per_block", C.c_int),
        ("density_factor", C.c_float),
        ("acquisition_time_ps", C.c_ulonglong),
        ("mean_life", C.c_float),
        ("material_activity", C.c_float * MAX_MATERIALS),
        ("psf_file", C.c_char * 250),
        ("detector_center", C.c_float * 3),
        ("detector_height", C.c_float),
        ("detector_radius", C.c_float),
        ("psf_size", C.c_int),
        ("tally_type", C.c_int),
        ("tally_psf_sinogram", C.c_int),
        ("detector_auto_center", C.c_int),
        ("tally_material_dose", C.c_int),
        ("tally_voxel_dose", C.c_int),
        ("dose_file", C.c_char * 250),
        ("dose_roi", C.c_short * 6),
        ("energy_resolution", C.c_float),
        ("energy_window_low", C.c_float),
        ("energy_window_high", C.c_float),
        ("fov_z", C.c_float),
        ("n_rows", C.c_int),
        ("n_crystals", C.c_int),
        ("n_angles", C.c_int),
        ("n_radial", C.c_int),
        ("n_z_slices", C.c_int),
        ("image_res", C.c_int),
        ("n_energy_bins", C.c_int),
        ("max_ring_difference", C.c_int),
        ("span", C.c_int),
        ("n_segments", C.c_int),
        ("n_sinograms", C.c_int),
        ("n_bins", C.c_longlong),
        ("voxel_file", C.c_char * 250),
        ("material_files", (C.c_char * 250) * MAX_MATERIALS),
        ("prompt_gamma_energy", C.c_float),
        ("prompt_gamma_yield", C.c_float),
    ]


class SceneInfo(C.Structure):
    _fields_ = [
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("nz", C.c_int),
        ("voxel_size", C.c_float * 3),
        ("bbox", C.c_float * 3),
        ("n_voxels", C.c_longlong),
        ("n_emitting_voxels", C.c_longlong),
        ("total_activity_bq", C.c_double),
        ("n_energy", C.c_int),
        ("e0", C.c_float),
        ("inv_de", C.c_float),
        ("n_materials_used", C.c_int),
        ("n_palette", C.c_int),
        ("density_max", C.c_float * MAX_MATERIALS),
        ("density_nominal", C.c_float * MAX_MATERIALS),
        ("n_bins", C.c_longlong),
        ("n_energy_spectrum", C.c_int),
        ("n_emitters", C.c_int),
        ("n_lanes", C.c_longlong),
        ("last_h2d_bytes", C.c_longlong),
        ("n_dose_voxels", C.c_longlong),
    ]


class RunOpts(C.Structure):
    _fields_ = [
        ("lane_mode", C.c_int),
        ("background_mode", C.c_int),
        ("histories_per_lane", C.c_int),
        ("block_threads", C.c_int),
        ("blocks_per_sm", C.c_int),
        ("collect_counters", C.c_int),
        ("seed_override", C.c_int),
        ("stream", C.c_void_p),
        ("algorithm", C.c_int),
        ("max_woodcock_steps", C.c_int),
        ("max_rejections", C.c_int),
    ]


class Counters(C.Structure):
    _fields_ = [
        ("woodcock_steps_inside", C.c_ulonglong),
        ("table_refreshes", C.c_ulonglong),
        ("majorant_refreshes", C.c_ulonglong),
        ("tally_increments", C.c_ulonglong),
        ("photons", C.c_ulonglong),
        ("compton", C.c_ulonglong),
        ("rayleigh", C.c_ulonglong),
        ("photoelectric", C.c_ulonglong),
        ("lanes", C.c_ulonglong),
        ("guard_trips", C.c_ulonglong),
    ]


class Tallies(C.Structure):
    _fields_ = [
        ("trues", C.c_void_p),
        ("scatter", C.c_void_p),
        ("image_trues", C.c_void_p),
        ("image_scatter", C.c_void_p),
        ("spectrum", C.c_void_p),
        ("psf", C.c_void_p),
        ("psf_capacity", C.c_longlong),
        ("psf_count", C.c_void_p),
        ("total_histories", C.c_void_p),
        ("coincidences", C.c_void_p),
        ("counters", C.c_void_p),
        ("transport_ms", C.c_void_p),
        ("material_dose", C.c_void_p),
        ("voxel_dose", C.c_void_p),
    ]


class GradArgs(C.Structure):
    _fields_ = [
        ("measured", C.c_void_p),
        ("background", C.c_void_p),
        ("grad_activity", C.c_void_p),
        ("grad_density_scale", C.c_void_p),
        ("event_buffer", C.c_void_p),
        ("event_capacity", C.c_longlong),
        ("loglik", C.c_double),
        ("events", C.c_ulonglong),
        ("replayed", C.c_ulonglong),
        ("mismatches", C.c_ulonglong),
        ("forward_ms", C.c_double),
        ("gradient_ms", C.c_double),
    ]


class TuneResult(C.Structure):
    _fields_ = [
        ("block_threads", C.c_int),
        ("histories_per_lane", C.c_int),
        ("best_ms", C.c_double),
        ("auto_ms", C.c_double),
        ("sample_fraction", C.c_double),
        ("candidates", C.c_int),
    ]


EVENT_RECORD_BYTES = 24

PSF_SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_longlong, C.c_void_p)

P = C.c_void_p
_SIGNATURES = {
    "mcpet_config_read": (C.c_int, [C.c_char_p, C.POINTER(Config)]),
    "mcpet_scene_load": (C.c_int, [C.c_char_p, C.POINTER(P)]),
    "mcpet_scene_from_arrays": (C.c_int, [C.POINTER(Config), C.c_int, C.c_int, C.c_int, P, P, P, P, C.POINTER(P)]),
    "mcpet_scene_set_activity": (C.c_int, [P, P]),
    "mcpet_scene_get_config": (C.c_int, [P, C.POINTER(Config)]),
    "mcpet_scene_get_info": (C.c_int, [P, C.POINTER(SceneInfo)]),
    "mcpet_scene_export_tables": (C.c_int, [P] + [P] * 15),
    "mcpet_scene_free": (None, [P]),
    "mcpet_scene_to_device": (C.c_int, [P, C.c_int]),
    "mcpet_run": (C.c_int, [P, C.POINTER(RunOpts), C.POINTER(Tallies)]),
    "mcpet_run_device": (C.c_int, [P, C.POINTER(RunOpts), C.POINTER(Tallies)]),
    "mcpet_run_batch": (C.c_int, [P, C.c_int, C.POINTER(RunOpts), C.POINTER(Tallies)]),
    "mcpet_grad": (C.c_int, [P, C.POINTER(RunOpts), C.POINTER(Tallies), C.POINTER(GradArgs)]),
    "mcpet_run_psf_stream": (C.c_int, [P, C.POINTER(RunOpts), C.c_longlong, P, P, C.POINTER(Tallies)]),
    "mcpet_run_batch_device": (C.c_int, [P, C.c_int, C.POINTER(RunOpts), C.POINTER(Tallies)]),
    "mcpet_run_device_noalloc": (C.c_int, [P, P, C.POINTER(RunOpts), C.POINTER(Tallies)]),
    "mcpet_last_run_guard": (C.c_int, [P, C.POINTER(C.c_ulonglong)]),
    "mcpet_scene_lane_plan": (C.c_int, [P, C.c_int, C.c_int, C.c_longlong, P, P, P, P, P,
                                        C.POINTER(C.c_longlong), C.POINTER(C.c_ulonglong)]),
    "mcpet_run_async": (C.c_int, [P, C.POINTER(RunOpts), C.POINTER(Tallies)]),
    "mcpet_run_wait": (C.c_int, [P]),
    "mcpet_autotune": (C.c_int, [P, C.c_int, C.POINTER(RunOpts), C.POINTER(Tallies), C.c_double,
                                 C.POINTER(TuneResult)]),
    "mcpet_batch_graph_create": (C.c_int, [P, C.c_int, C.POINTER(RunOpts), C.POINTER(Tallies), C.c_int,
                                           C.POINTER(P)]),
    "mcpet_batch_graph_launch": (C.c_int, [P, P]),
    "mcpet_batch_graph_set_seeds": (C.c_int, [P, P, P]),
    "mcpet_batch_graph_guard_trips": (C.c_int, [P, C.POINTER(C.c_ulonglong)]),
    "mcpet_batch_graph_destroy": (None, [P]),
    "mcpet_write_outputs": (C.c_int, [P, C.POINTER(Tallies), C.c_char_p, C.c_int, C.c_double]),
    "mcpet_probe_rng": (C.c_int, [C.c_int, C.c_int, P, C.c_int, P, P, P]),
    "mcpet_probe_detector": (C.c_int, [P, C.c_int] + [P] * 10),
    "mcpet_probe_compton": (C.c_int, [P, C.c_int, P, P, P, P, P, P]),
    "mcpet_probe_rayleigh": (C.c_int, [P, C.c_int, P, P, P, P, P, P]),
    "mcpet_probe_source": (C.c_int, [C.c_int, C.c_int, C.c_int, P, C.c_int, P, P, P]),
    "mcpet_last_error": (C.c_char_p, []),
    "mcpet_version": (C.c_char_p, []),
}

EXPORTED = tuple(_SIGNATURES)

_lib = None


def lib() -> C.CDLL:
    """Load libmcpet.so once (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class McpetError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int) -> None:
    if status != 0:
        raise McpetError(status, lib().mcpet_last_error().decode(errors="replace"))
