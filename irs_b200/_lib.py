"""ctypes bindings of the irs_b200 C ABI.

Four shared libraries are built into irs_b200/lib/ (see irs_b200/build.py):
lib_ipm.so / lib_ipm_double.so export the symbol set of the reference's
src/lib_ipm.cu, lib_irs.so / lib_irs_double.so the same conventions for IRS.
Loading fails loudly when a library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

LIBDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

_FLOAT_FIELDS = [
    "kappa_tot", "shear", "kappa_star", "theta_star", "m_solar", "m_lower", "m_upper",
    "light_loss", "safety_scale", "center_y1", "center_y2", "half_length_y1", "half_length_y2",
]
_INT_FIELDS = [
    "rectangular", "approx", "num_pixels_y1", "num_pixels_y2", "num_rays_y", "random_seed",
    "write_stars", "write_maps", "write_parities", "write_histograms",
]
_STR_FIELDS = ["mass_function", "starfile", "outfile_prefix"]

# Symbols of the reference ABI (src/lib_ipm.cu:15-81), in order.
REFERENCE_IPM_SYMBOLS = (
    ["init"]
    + [f"set_{f}" for f in ["kappa_tot", "shear", "kappa_star", "theta_star", "mass_function", "m_solar",
                            "m_lower", "m_upper", "light_loss", "rectangular", "approx", "safety_scale",
                            "starfile", "center_y1", "center_y2", "half_length_y1", "half_length_y2",
                            "num_pixels_y1", "num_pixels_y2", "num_rays_y", "random_seed", "write_stars",
                            "write_maps", "write_parities", "write_histograms", "outfile_prefix"]]
    + [f"get_{f}" for f in ["kappa_tot", "shear", "kappa_star", "theta_star", "mass_function", "m_solar",
                            "m_lower", "m_upper", "light_loss", "rectangular", "approx", "safety_scale",
                            "starfile", "center_y1", "center_y2", "half_length_y1", "half_length_y2",
                            "num_pixels_y1", "num_pixels_y2", "num_rays_y", "random_seed", "write_stars",
                            "write_maps", "write_parities", "write_histograms", "outfile_prefix"]]
    + ["get_num_stars", "get_corner_x1", "get_corner_x2", "get_stars", "get_pixels",
       "get_pixels_minima", "get_pixels_saddles", "get_t_shoot_cells", "run", "save"]
)
EXTENSION_SYMBOLS = [
    "destroy", "set_expansion_order", "get_expansion_order", "set_precision", "get_precision",
    "set_stars", "get_t_pipeline", "rerun", "set_band", "set_shoot_launch", "get_shoot_threads",
    "get_shoot_ctas_per_sm", "copy_maps_device", "derive", "get_value", "get_tree_num_nodes", "copy_tree",
    "copy_coeffs", "get_num_vertices", "copy_vertices", "copy_fixed_maps",
]
IRS_ONLY_SYMBOLS = ["get_t_shoot_rays", "get_num_rays_shot", "get_num_rays_received"]
IPM_ONLY_SYMBOLS = ["ipm_deposit_noalloc", "batch_init", "batch_destroy", "batch_add", "batch_size",
                    "batch_set_expansion_order", "batch_set_corner_capacity", "batch_run", "batch_rerun",
                    "batch_copy_maps", "batch_maps_device", "batch_copy_stars", "batch_get_value",
                    "ada_init", "ada_destroy", "ada_base", "ada_set_policy", "ada_set_levels", "ada_set_tolerance", "ada_set_quantile", "ada_set_error_mode",
                    "ada_set_max_level",
                    "ada_set_audit", "ada_set_audit_bound", "ada_set_refine_capacity", "ada_set_tiled_min", "ada_set_network", "ada_run", "ada_num_tiles",
                    "ada_copy_features", "ada_copy_levels", "ada_labels", "ada_copy_map", "ada_get_value",
                    "mlp_num_params", "mlp_train", "mlp_gradients", "mlp_predict"]

LIB_NAMES = {
    ("ipm", False): "lib_ipm.so",
    ("ipm", True): "lib_ipm_double.so",
    ("irs", False): "lib_irs.so",
    ("irs", True): "lib_irs_double.so",
}

_cache: dict = {}


def lib_path(kind: str, is_double: bool) -> str:
    return os.path.join(LIBDIR, LIB_NAMES[(kind, is_double)])


def _bind(lib, kind: str, is_double: bool):
    T = C.c_double if is_double else C.c_float
    vp = C.c_void_p
    lib.init.argtypes = []
    lib.init.restype = vp
    for f in _FLOAT_FIELDS:
        getattr(lib, f"set_{f}").argtypes = [vp, T]
        getattr(lib, f"set_{f}").restype = None
        getattr(lib, f"get_{f}").argtypes = [vp]
        getattr(lib, f"get_{f}").restype = T
    for f in _INT_FIELDS:
        getattr(lib, f"set_{f}").argtypes = [vp, C.c_int]
        getattr(lib, f"set_{f}").restype = None
        getattr(lib, f"get_{f}").argtypes = [vp]
        getattr(lib, f"get_{f}").restype = C.c_int
    for f in _STR_FIELDS:
        getattr(lib, f"set_{f}").argtypes = [vp, C.c_char_p]
        getattr(lib, f"set_{f}").restype = None
        getattr(lib, f"get_{f}").argtypes = [vp]
        getattr(lib, f"get_{f}").restype = C.c_char_p
    PixT = C.c_int if kind == "irs" else T
    lib.get_num_stars.argtypes = [vp]
    lib.get_num_stars.restype = C.c_int
    lib.get_corner_x1.argtypes = [vp]
    lib.get_corner_x1.restype = T
    lib.get_corner_x2.argtypes = [vp]
    lib.get_corner_x2.restype = T
    lib.get_stars.argtypes = [vp]
    lib.get_stars.restype = C.POINTER(T)
    for f in ["get_pixels", "get_pixels_minima", "get_pixels_saddles"]:
        getattr(lib, f).argtypes = [vp]
        getattr(lib, f).restype = C.POINTER(PixT)
    if kind == "irs":
        lib.get_t_shoot_rays.argtypes = [vp]
        lib.get_t_shoot_rays.restype = C.c_double
        lib.get_num_rays_shot.argtypes = [vp]
        lib.get_num_rays_shot.restype = C.c_ulonglong
        lib.get_num_rays_received.argtypes = [vp]
        lib.get_num_rays_received.restype = C.c_ulonglong
    else:
        lib.get_t_shoot_cells.argtypes = [vp]
        lib.get_t_shoot_cells.restype = C.c_double
    lib.run.argtypes = [vp, C.c_int]
    lib.run.restype = C.c_bool
    lib.save.argtypes = [vp, C.c_int]
    lib.save.restype = C.c_bool
    # extensions
    lib.destroy.argtypes = [vp]
    lib.destroy.restype = None
    lib.set_expansion_order.argtypes = [vp, C.c_int]
    lib.set_expansion_order.restype = None
    lib.get_expansion_order.argtypes = [vp]
    lib.get_expansion_order.restype = C.c_int
    lib.set_precision.argtypes = [vp, C.c_int]
    lib.set_precision.restype = None
    lib.get_precision.argtypes = [vp]
    lib.get_precision.restype = C.c_int
    lib.set_stars.argtypes = [vp, C.POINTER(T), C.c_int, C.c_int, T, T, T]
    lib.set_stars.restype = None
    lib.get_t_pipeline.argtypes = [vp]
    lib.get_t_pipeline.restype = C.c_double
    lib.rerun.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
    lib.rerun.restype = C.c_bool
    lib.copy_pixels.argtypes = [vp, C.c_int, C.POINTER(PixT)]
    lib.copy_pixels.restype = C.c_bool
    lib.set_pixels_out.argtypes = [vp, C.POINTER(PixT)]
    lib.set_pixels_out.restype = None
    lib.set_band.argtypes = [vp, C.c_longlong, C.c_longlong]
    lib.set_band.restype = None
    lib.set_shoot_launch.argtypes = [vp, C.c_int, C.c_int]
    lib.set_shoot_launch.restype = None
    lib.get_shoot_threads.argtypes = [vp]
    lib.get_shoot_threads.restype = C.c_int
    lib.get_shoot_ctas_per_sm.argtypes = [vp]
    lib.get_shoot_ctas_per_sm.restype = C.c_int
    lib.copy_maps_device.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.copy_maps_device.restype = C.c_bool
    lib.derive.argtypes = [vp]
    lib.derive.restype = C.c_bool
    lib.get_value.argtypes = [vp, C.c_char_p]
    lib.get_value.restype = C.c_double
    lib.get_tree_num_nodes.argtypes = [vp]
    lib.get_tree_num_nodes.restype = C.c_int
    lib.copy_tree.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.copy_tree.restype = C.c_bool
    lib.copy_coeffs.argtypes = [vp, C.c_void_p, C.c_void_p]
    lib.copy_coeffs.restype = C.c_bool
    lib.get_num_vertices.argtypes = [vp]
    lib.get_num_vertices.restype = C.c_longlong
    lib.copy_vertices.argtypes = [vp, C.c_void_p]
    lib.copy_vertices.restype = C.c_bool
    lib.copy_fixed_maps.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.copy_fixed_maps.restype = C.c_bool
    if kind == "ipm":
        lib.batch_init.argtypes = []
        lib.batch_init.restype = vp
        lib.batch_destroy.argtypes = [vp]
        lib.batch_destroy.restype = None
        lib.batch_add.argtypes = [vp, vp]
        lib.batch_add.restype = C.c_int
        lib.batch_size.argtypes = [vp]
        lib.batch_size.restype = C.c_int
        lib.batch_set_expansion_order.argtypes = [vp, C.c_int]
        lib.batch_set_expansion_order.restype = None
        lib.batch_set_corner_capacity.argtypes = [vp, C.c_longlong]
        lib.batch_set_corner_capacity.restype = None
        lib.batch_run.argtypes = [vp, C.c_int]
        lib.batch_run.restype = C.c_bool
        lib.batch_rerun.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
        lib.batch_rerun.restype = C.c_bool
        lib.batch_copy_maps.argtypes = [vp, C.c_void_p]
        lib.batch_copy_maps.restype = C.c_bool
        lib.batch_maps_device.argtypes = [vp]
        lib.batch_maps_device.restype = C.c_void_p
        lib.batch_copy_stars.argtypes = [vp, C.c_void_p]
        lib.batch_copy_stars.restype = C.c_bool
        lib.batch_get_value.argtypes = [vp, C.c_int, C.c_char_p]
        lib.batch_get_value.restype = C.c_double
        fp, ip = C.c_void_p, C.c_void_p
        for name, args, res in [
                ("ada_init", [], vp), ("ada_destroy", [vp], None), ("ada_base", [vp], vp),
                ("ada_set_policy", [vp, C.c_int, C.c_int], None), ("ada_set_levels", [vp, ip, C.c_int], None),
                ("ada_set_tolerance", [vp, C.c_double], None), ("ada_set_quantile", [vp, C.c_float], None),
                ("ada_set_error_mode", [vp, C.c_int], None), ("ada_set_max_level", [vp, C.c_int], None),
                ("ada_set_audit", [vp, C.c_double, C.c_uint], None), ("ada_set_audit_bound", [vp, C.c_double], None),
                ("ada_set_refine_capacity", [vp, C.c_longlong], None), ("ada_set_tiled_min", [vp, C.c_int], None), ("ada_set_network", [vp, fp, fp, fp], None),
                ("ada_run", [vp, C.c_int], C.c_bool), ("ada_num_tiles", [vp], C.c_int),
                ("ada_copy_features", [vp, fp], C.c_bool), ("ada_copy_levels", [vp, ip, C.c_int], C.c_bool),
                ("ada_labels", [vp, ip, C.c_int, ip, fp], C.c_bool), ("ada_copy_map", [vp, C.c_void_p], C.c_bool),
                ("ada_get_value", [vp, C.c_char_p], C.c_double), ("mlp_num_params", [], C.c_int),
                ("mlp_train", [fp, ip, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint, fp, fp, fp, fp], C.c_bool),
                ("mlp_gradients", [fp, fp, fp, fp, ip, C.c_int, fp, fp], C.c_bool),
                ("mlp_predict", [fp, fp, fp, fp, C.c_int, ip], C.c_bool)]:
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
    return lib


def load(kind: str = "ipm", is_double: bool = False):
    """Load (once) and bind one of the four libraries; raises if it is missing."""
    key = (kind, bool(is_double))
    if key in _cache:
        return _cache[key]
    path = lib_path(kind, is_double)
    if not os.path.exists(path):
        raise RuntimeError(
            f"irs_b200: CUDA library {path} is missing; build it with `python -m irs_b200.build` "
            "(there is no CPU fallback)")
    lib = _bind(C.CDLL(path), kind, bool(is_double))
    _cache[key] = lib
    return lib
