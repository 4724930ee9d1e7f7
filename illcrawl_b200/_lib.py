"""ctypes binding of ``libilcuda.so`` (the C ABI declared in ``include/ilc.h``).

The library is built in-tree by ``illcrawl_b200.build``. There is no CPU
fallback: if the library is missing or no CUDA device is usable, every entry
point raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libilcuda.so")

ILC_OK = 0
STATUS_NAMES = {
    0: "ILC_OK", 1: "ILC_ERR_INVALID_ARGUMENT", 2: "ILC_ERR_CUDA", 3: "ILC_ERR_OUT_OF_MEMORY",
    4: "ILC_ERR_NO_PARTICLES", 5: "ILC_ERR_NO_GAUNT_TABLE", 6: "ILC_ERR_STEP_LIMIT",
    7: "ILC_ERR_NONFINITE_INPUT", 8: "ILC_ERR_GRID_TOO_LARGE", 9: "ILC_ERR_INTERNAL",
    10: "ILC_ERR_NO_ARF_TABLE",
}
CONTROLLER_REF32 = 0
CONTROLLER_FP64 = 1
DA_PIXEL_AREA, DA_UNIT, DA_INVERSE_RANGE = 0, 1, 2
DV_VOLUME, DV_MEAN = 0, 1
ENGINE_GRID, ENGINE_PERSISTENT = 0, 1


class IlcError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Camera(ctypes.Structure):
    _fields_ = [("position", ctypes.c_double * 3), ("look_at", ctypes.c_double * 3),
                ("roll", ctypes.c_double), ("screen_width", ctypes.c_double),
                ("num_pix_x", ctypes.c_int32), ("num_pix_y", ctypes.c_int32)]


class Tolerance(ctypes.Structure):
    _fields_ = [("absolute", ctypes.c_double), ("relative", ctypes.c_double)]


class LosScaling(ctypes.Structure):
    _fields_ = [("length_conversion", ctypes.c_double), ("area_conversion", ctypes.c_double),
                ("dA_mode", ctypes.c_int32)]


class GridDesc(ctypes.Structure):
    _fields_ = [("min_corner", ctypes.c_float * 3), ("cell_sizes", ctypes.c_float * 3),
                ("num_cells", ctypes.c_int32 * 3), ("total_cells", ctypes.c_uint64),
                ("num_particles", ctypes.c_uint64)]


class RenderStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_uint64), ("accepted_steps", ctypes.c_uint64),
                ("queries", ctypes.c_uint64), ("cells_visited", ctypes.c_uint64),
                ("candidates", ctypes.c_uint64), ("max_steps_per_ray", ctypes.c_uint64),
                ("rays_at_step_limit", ctypes.c_uint64), ("kernel_ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class AdjointStats(ctypes.Structure):
    _fields_ = [("loss", ctypes.c_double), ("quantity_ms", ctypes.c_float),
                ("forward_ms", ctypes.c_float), ("adjoint_ms", ctypes.c_float),
                ("forward_steps", ctypes.c_uint64), ("adjoint_steps", ctypes.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


ADJOINT_CHECKPOINT, ADJOINT_RECOMPUTE = 0, 1


class FitsCard(ctypes.Structure):
    _fields_ = [("key", ctypes.c_char_p), ("type", ctypes.c_int32), ("number", ctypes.c_double),
                ("integer", ctypes.c_int64), ("text", ctypes.c_char_p),
                ("comment", ctypes.c_char_p)]


class Job(ctypes.Structure):
    """ilc_job: one camera of a batched render."""
    _fields_ = [("camera", Camera), ("z_range", ctypes.c_double),
                ("aperture_radius", ctypes.c_double), ("sphere_center", ctypes.c_double * 3),
                ("sphere_radius", ctypes.c_double), ("min_chord", ctypes.c_double),
                ("scale", ctypes.c_float), ("reserved", ctypes.c_int32),
                ("out_offset", ctypes.c_uint64)]

_P = ctypes.c_void_p
_u64, _i64, _i32, _f32, _f64, _int = (ctypes.c_uint64, ctypes.c_int64, ctypes.c_int32,
                                      ctypes.c_float, ctypes.c_double, ctypes.c_int)

# name -> (restype, argtypes); mirrors include/ilc.h
SIGNATURES = {
    "ilc_create": (_P, [_int]),
    "ilc_destroy": (None, [_P]),
    "ilc_last_error": (ctypes.c_char_p, [_P]),
    "ilc_set_step_limit": (_int, [_P, _i64]),
    "ilc_get_stream": (_P, [_P]),
    "ilc_set_z_window": (_int, [_P, _f32]),
    "ilc_nn8_setup_particles": (_int, [_P, _P, _u64, _int]),
    "ilc_grid_describe": (_int, [_P, _P]),
    "ilc_grid_export": (_int, [_P, _P, _P, _P, _int]),
    "ilc_nn8_query": (_int, [_P, _P, _u64, _int, _P, _P, _P, _int]),
    "ilc_gaunt_load": (_int, [_P, _P, _i32, _i32, _f32, _f32, _f32, _f32]),
    "ilc_quantity_xray_flux": (_int, [_P, _P, _P, _P, _u64, _f32, _f32, _f32, _f32, _i32, _P,
                                      _int]),
    "ilc_quantity_xray_spectral_flux": (_int, [_P, _P, _P, _P, _u64, _f32, _f32, _f32, _f32,
                                               _P, _int]),
    "ilc_quantity_temperature": (_int, [_P, _P, _P, _u64, _P, _int]),
    "ilc_camera_plane": (_int, [_P, _P]),
    "ilc_render_adaptive": (_int, [_P, _P, _f64, Tolerance, _i32, _P, _P, _int, _P]),
    "ilc_render_fixed": (_int, [_P, _P, _f64, _i64, _P, _P, _int, _P]),
    "ilc_render_record": (_int, [_P, _P, _f64, Tolerance, _i32, _P, _P, _i64, _int, _P, _int, _P]),
    "ilc_render_frozen": (_int, [_P, _P, _f64, _P, _P, _i64, _int, _P, _P, _int, _P]),
    "ilc_render_ray_stats": (_int, [_P, _P, _f64, Tolerance, _i32, _P, _P, _P, _int, _P]),
    "ilc_set_checkpoint_budget": (_int, [_P, _u64]),
    "ilc_set_query_engine": (_int, [_P, _i32]),
    "ilc_nn8_query_stats": (_int, [_P, _P, _P]),
    "ilc_render_frozen_f64": (_int, [_P, _P, _f64, _P, _P, _i64, _int, _P, _P, _int, _P]),
    "ilc_los_scale": (_f32, [_P, _f64, _P]),
    "ilc_project_xray_flux": (_int, [_P, _P, _P, _P, _P, _u64, _f32, _f32, _f32, _f32, _i32, _P,
                                     _f64, Tolerance, _i32, _P, _P, _int, _P]),
    "ilc_kernel_launches": (_u64, [_P]),
    "ilc_grid_build_noalloc": (_int, [_P, _u64, _P, _P, _u64, _P, _P, _P]),
    "ilc_device_alloc": (_int, [_P, _u64, _P]),
    "ilc_device_free": (_int, [_P, _P]),
    "ilc_copy": (_int, [_P, _P, _P, _u64]),
    "ilc_autotune_render": (_int, [_P, _P, _f64, Tolerance, _i32, _P, _i32, _P, _i32, _i32, _P,
                                   _P, _P]),
    "ilc_set_render_occupancy": (_int, [_P, _i32]),
    "ilc_set_render_engine": (_int, [_P, _i32]),
    "ilc_quantity_xray_spectrum": (_int, [_P, _P, _P, _P, _u64, _f32, _f32, _P, _P, _i32, _P,
                                          _int]),
    "ilc_quantity_xray_photon_flux": (_int, [_P, _P, _P, _P, _u64, _f32, _f32, _f32, _f32, _i32,
                                             _P, _int]),
    "ilc_arf_load": (_int, [_P, _P, _i32, _f32, _f32]),
    "ilc_mc_profile_shells": (_int, [_f64, _i32, _f64, _P, _P]),
    "ilc_mc_profile_points": (_int, [_P, _f64, _i32, _f64, _u64, _u64, _u64, _P]),
    "ilc_mc_radial_profile": (_int, [_P, _P, _f64, _i32, _f64, _u64, _i32, _f64, _P, _P, _P]),
    "ilc_quantity_chandra_count_rate": (_int, [_P, _P, _P, _P, _u64, _f32, _f32, _P, _int]),
    "ilc_quantity_chandra_spectral_count_rate": (_int, [_P, _P, _P, _P, _u64, _f32, _f32, _f32,
                                                        _f32, _P, _int]),
    "ilc_quantity_chandra_spectrum": (_int, [_P, _P, _P, _P, _u64, _f32, _f32, _P, _P, _i32, _P,
                                             _int]),
    "ilc_volumetric_slice": (_int, [_P, _P, _f64, _i32, _u64, _P, _int]),
    "ilc_volumetric_tomography": (_int, [_P, _P, _f64, _i64, _i64, _P, _int]),
    "ilc_fits_write_image": (_int, [ctypes.c_char_p, _P, _i32, _P, _P, _i32]),
    "ilc_ingest_cells": (_int, [_P, _P, _P, _u64, _P, _P, _P, _f64, _P, _P, _P, _int]),
    "ilc_render_batched": (_int, [_P, _P, _i32, _int, _P, _i32, Tolerance, _P, _u64, _int, _P]),
    "ilc_set_batch_schedule": (_int, [_P, _i32, _i32, _f32, _i32]),
    "ilc_autotune_batched": (_int, [_P, _P, _i32, _int, _P, _i32, Tolerance, _P, _i32, _P, _i32,
                                    _P, _i32, _P, _P, _P, _P]),
    "ilc_adjoint_xray_flux": (_int, [_P, _P, _P, _P, _P, _u64, _f32, _f32, _f32, _f32, _i32, _P,
                                     _f64, Tolerance, _i32, _P, _P, _i32, _P, _P, _P, _int, _P]),
}

_lib = None


def load(path=LIB_PATH):
    """Loads the CUDA library (raises if it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build the CUDA extension (python -m illcrawl_b200.build)")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
