"""ctypes mirror of include/patchstereo.h and the loader of libpatchstereo.so.

The loader fails loudly when the library is missing: there is no CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes as C
import pathlib

HERE = pathlib.Path(__file__).resolve().parent
ENGINE_PATH = HERE / "libpatchstereo.so"
SYNTH_PATH = HERE / "libps_synth.so"

PS_OK, PS_EINVAL, PS_ECUDA, PS_ENODEV, PS_ECOMPILE, PS_ETIMEOUT, PS_EFAULT, PS_ENOMEM, PS_EBUSY = range(9)
STATUS_NAMES = {0: "PS_OK", 1: "PS_EINVAL", 2: "PS_ECUDA", 3: "PS_ENODEV", 4: "PS_ECOMPILE", 5: "PS_ETIMEOUT",
                6: "PS_EFAULT", 7: "PS_ENOMEM", 8: "PS_EBUSY"}
PS_IMAGE_U8, PS_IMAGE_F32 = 0, 1
PS_MATH_PARITY, PS_MATH_FAST = 0, 1
PS_MAX_SOURCES = 32
PS_NOALLOC_MAX_PIXELS = 1 << 21  # capacity of the allocation-free median filter's static device array
PS_INIT_RANDOM, PS_INIT_PROPOSAL = 1, 2  # ps_run_params.random_init / ps_schedule.init
PS_SWEEP_PLANES, PS_NET_CH_IN, PS_NET_CH_OUT = 32, 48, 8


class Options(C.Structure):
    _fields_ = [("math_mode", C.c_uint32), ("max_batch", C.c_uint32), ("batch_pixels", C.c_uint64),
                ("checked", C.c_uint32), ("tuning", C.c_uint32)]


PS_TUNE_NO_WEIGHT_CACHE, PS_TUNE_TEX_GATHER, PS_TUNE_ONE_LANE = 0x1, 0x2, 0x4
PS_TUNE_ROW_PAIRS, PS_TUNE_STAGED, PS_TUNE_PERSISTENT, PS_TUNE_TMA = 0x8, 0x10, 0x20, 0x40
PS_INJECT_NONE, PS_INJECT_DEVICE_ALLOC, PS_INJECT_UPLOAD, PS_INJECT_CHECK_PROBE, PS_INJECT_QUEUE_STALL = 0, 1, 2, 3, 4
PS_KERNEL_HALF, PS_KERNEL_EVAL, PS_KERNEL_FILTER, PS_KERNEL_OTHER, PS_KERNEL_SWEEP, PS_KERNEL_NET = range(6)
PS_KERNEL_KINDS = 6


class PmParams(C.Structure):
    """PmParams (crates/dense/src/params.rs:76-124)."""
    _fields_ = [("window_radius", C.c_int32), ("window_step", C.c_int32), ("sigma_spatial", C.c_float),
                ("sigma_color", C.c_float), ("tau0", C.c_float), ("tau_alpha", C.c_float), ("tau1", C.c_float),
                ("beta", C.c_float), ("n1", C.c_uint32), ("n2", C.c_uint32), ("prev_view_weight", C.c_float),
                ("min_triangulation_angle_deg", C.c_float), ("incident_angle_sigma", C.c_float),
                ("geom_lambda", C.c_float), ("geom_max_cost", C.c_float), ("top_k", C.c_uint32),
                ("eps0_photometric", C.c_float), ("eps0_geometric", C.c_float), ("phi0_photometric_deg", C.c_float),
                ("phi0_geometric_deg", C.c_float), ("eps_min", C.c_float), ("phi_min_deg", C.c_float),
                ("weak_texture_var", C.c_float)]


class FilterParams(C.Structure):
    """FilterParams (crates/dense/src/params.rs:180-207)."""
    _fields_ = [("min_ncc", C.c_float), ("min_triangulation_angle_deg", C.c_float), ("min_num_consistent", C.c_uint32),
                ("geom_max_cost", C.c_float), ("ncc_sigma", C.c_float), ("median_filter", C.c_uint32)]


class LevelImage(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("format", C.c_uint32), ("stride", C.c_uint32),
                ("pixels", C.c_void_p), ("k", C.c_float * 4)]


class PairGeometry(C.Structure):
    _fields_ = [("r", C.c_float * 9), ("t", C.c_float * 3), ("center", C.c_float * 3)]


class KernelView(C.Structure):
    _fields_ = [("key", C.c_uint64), ("levels", C.POINTER(LevelImage)), ("sources", C.POINTER(C.c_uint32)),
                ("num_sources", C.c_uint32), ("reserved", C.c_uint32), ("pairs", C.POINTER(PairGeometry)),
                ("pairs_f64", C.POINTER(C.c_double)), ("depth_min", C.c_float), ("depth_max", C.c_float)]


class KernelInput(C.Structure):
    _fields_ = [("views", C.POINTER(KernelView)), ("num_views", C.c_uint32), ("num_levels", C.c_uint32),
                ("pm", PmParams), ("filter", FilterParams), ("seed", C.c_uint64)]


class ViewState(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("depth", C.POINTER(C.c_float)),
                ("normal", C.POINTER(C.c_float)), ("cost", C.POINTER(C.c_float)), ("prior", C.POINTER(C.c_float))]


class RunParams(C.Structure):
    _fields_ = [("level", C.c_uint32), ("geometric", C.c_uint32), ("random_init", C.c_uint32),
                ("iterations", C.c_uint32), ("run_id", C.c_uint32), ("use_prior", C.c_uint32)]


class Schedule(C.Structure):
    _fields_ = [("level", C.c_uint32), ("photometric_iters", C.c_uint32), ("geometric_rounds", C.c_uint32),
                ("geometric_iters", C.c_uint32), ("run_id_base", C.c_uint32), ("use_graph", C.c_uint32),
                ("init", C.c_uint32)]


class PostParams(C.Structure):
    """PostParams (crates/dense/src/postproc.rs:41-74)."""
    _fields_ = [("remove_speckles", C.c_uint32), ("speckle_rel_depth", C.c_float), ("speckle_min_area_frac", C.c_double),
                ("speckle_keep_cost", C.c_float), ("fill_holes", C.c_uint32), ("fill_max_frac", C.c_double),
                ("fill_edge_step", C.c_float), ("fill_max_cost", C.c_float)]


PS_FUSION_RESIDUAL_NONE, PS_FUSION_RESIDUAL_RELEASE, PS_FUSION_RESIDUAL_SECOND_PASS = 0, 1, 2


class FusionParams(C.Structure):
    """FusionParams of consistency fusion (crates/dense/src/params.rs:264-351), with the residual handling."""
    _fields_ = [("min_consistent_views", C.c_uint32), ("consistency_num_images", C.c_uint32), ("mark_used", C.c_uint32),
                ("mark_radius", C.c_uint32), ("inverse_variance", C.c_uint32), ("residual", C.c_uint32),
                ("sigma_px0", C.c_double), ("sigma_px_slope", C.c_double), ("max_reproj_error", C.c_double),
                ("max_depth_error", C.c_double), ("max_normal_error_deg", C.c_double),
                ("residual_min_views", C.c_uint32), ("reserved", C.c_uint32), ("residual_depth_error", C.c_double),
                ("residual_normal_error_deg", C.c_double), ("residual_min_dist_gsd", C.c_double),
                ("visibility_check_views", C.c_uint32), ("visibility_min_violations", C.c_uint32),
                ("visibility_tau", C.c_double), ("smooth_iterations", C.c_uint32), ("reserved2", C.c_uint32),
                ("smooth_radius_gsd", C.c_double), ("smooth_sigma_range_gsd", C.c_double),
                ("smooth_normal_deg", C.c_double)]


class ScoreFusionParams(C.Structure):
    """ScoreFusionOptions of score fusion (crates/dense/src/fusion_score.rs:56-103)."""
    _fields_ = [("sigma_e_px", C.c_double), ("sigma_theta_deg", C.c_double), ("lambda", C.c_double),
                ("tau", C.c_double), ("depth_error", C.c_double), ("normal_error_deg", C.c_double),
                ("num_neighbors", C.c_uint32), ("mark_used", C.c_uint32), ("inverse_variance", C.c_uint32),
                ("reserved", C.c_uint32), ("sigma_px0", C.c_double), ("sigma_px_slope", C.c_double)]


class FusionView(C.Structure):
    _fields_ = [("k", C.c_double * 4), ("r", C.c_double * 9), ("t", C.c_double * 3), ("baseline", C.c_double),
                ("image_id", C.c_uint32), ("num_overlap", C.c_uint32), ("overlap", C.POINTER(C.c_uint32))]


class MultiscaleSchedule(C.Structure):
    _fields_ = [("photometric_iters", C.c_uint32), ("photometric_iters_upper", C.c_uint32),
                ("geometric_rounds", C.c_uint32), ("geometric_iters", C.c_uint32), ("jbu_sigma_spatial", C.c_float),
                ("jbu_sigma_color", C.c_float), ("restorer_threshold", C.c_float), ("weak_texture_prior", C.c_uint32),
                ("run_id_base", C.c_uint32), ("use_graph", C.c_uint32)]


class SparseView(C.Structure):
    _fields_ = [("r", C.c_double * 9), ("t", C.c_double * 3)]


class NeighborParams(C.Structure):
    _fields_ = [("num_views", C.c_uint32), ("direction_bins", C.c_uint32), ("min_triangulation_angle_deg", C.c_double),
                ("diversity_decay", C.c_double)]


class DepthSnapshot(C.Structure):
    _fields_ = [("id", C.c_uint64), ("level", C.c_uint32), ("num_maps", C.c_uint32),
                ("maps", C.POINTER(C.POINTER(C.c_float))), ("map_lengths", C.POINTER(C.c_uint64))]


# Every exported symbol of include/patchstereo.h with (restype, argtypes).
_P = C.c_void_p
_U32P = C.POINTER(C.c_uint32)
SIGNATURES = {
    "ps_abi_version": (C.c_int, []),
    "ps_pm_params_default": (None, [C.POINTER(PmParams)]),
    "ps_filter_params_default": (None, [C.POINTER(FilterParams)]),
    "ps_options_default": (None, [C.POINTER(Options)]),
    "ps_backend_create": (C.c_int, [C.c_int, C.POINTER(Options), C.POINTER(_P)]),
    "ps_backend_destroy": (None, [_P]),
    "ps_backend_name": (C.c_char_p, [_P]),
    "ps_backend_last_error": (C.c_char_p, [_P]),
    "ps_begin": (C.c_int, [_P, C.POINTER(KernelInput), C.POINTER(_P)]),
    "ps_end": (C.c_int, [_P]),
    "ps_last_error": (C.c_char_p, [_P]),
    "ps_run": (C.c_int, [_P, _U32P, C.c_size_t, C.POINTER(ViewState), C.POINTER(RunParams), C.POINTER(DepthSnapshot)]),
    "ps_evaluate": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(ViewState), C.c_uint32,
                              C.POINTER(DepthSnapshot), C.POINTER(C.POINTER(C.c_float))]),
    "ps_filter": (C.c_int, [_P, _U32P, C.c_size_t, C.POINTER(ViewState), C.POINTER(DepthSnapshot),
                            C.POINTER(C.POINTER(C.c_uint8))]),
    "ps_upsample": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(ViewState), C.c_float, C.c_float,
                              C.POINTER(ViewState)]),
    "ps_median_filter": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(ViewState), C.POINTER(ViewState)]),
    "ps_state_upload": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(ViewState)]),
    "ps_state_download": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(ViewState)]),
    "ps_run_resident": (C.c_int, [_P, _U32P, C.c_size_t, C.POINTER(RunParams)]),
    "ps_snapshot_capture": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.c_uint64, C.c_uint32]),
    "ps_snapshot_buffer": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    "ps_snapshot_mark": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.c_uint64]),
    "ps_filter_resident": (C.c_int, [_P, _U32P, C.c_size_t, C.POINTER(C.POINTER(C.c_uint8))]),
    "ps_readout_resident": (C.c_int, [_P, _U32P, C.c_size_t, C.POINTER(ViewState)]),
    "ps_schedule_resident": (C.c_int, [_P, _U32P, C.c_size_t, C.POINTER(Schedule)]),
    "ps_multiscale_schedule_default": (None, [C.POINTER(MultiscaleSchedule)]),
    "ps_schedule_multiscale": (C.c_int, [_P, _U32P, C.c_size_t, C.POINTER(MultiscaleSchedule)]),
    "ps_median_filter_inplace_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_uint32, C.c_uint32,
                                                    C.POINTER(C.c_float), C.c_void_p]),
    "ps_synchronize": (C.c_int, [_P]),
    "ps_launch_count": (C.c_uint64, [_P]),
    "ps_session_stream": (C.c_void_p, [_P]),
    "ps_set_profiling": (C.c_int, [_P, C.c_uint32]),
    "ps_kernel_stats": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint64)]),
    "ps_reset_stats": (C.c_int, [_P]),
    "ps_backend_inject_failure": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "ps_kernel_staged_stats": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint64)]),
    "ps_measure_fp32_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "ps_check_reciprocal": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    # post-processing, fusion, output
    "ps_post_params_default": (None, [C.POINTER(PostParams)]),
    "ps_fusion_params_default": (None, [C.POINTER(FusionParams)]),
    "ps_postprocess_resident": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(PostParams),
                                          C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "ps_readout_download": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(ViewState)]),
    "ps_fuse_resident": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(FusionView), C.POINTER(FusionParams),
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "ps_fused_visibility_removed": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "ps_score_fusion_params_default": (None, [C.POINTER(ScoreFusionParams)]),
    "ps_fuse_scored_resident": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(FusionView),
                                          C.POINTER(ScoreFusionParams), C.POINTER(FusionParams),
                                          C.POINTER(C.c_uint64)]),
    "ps_fused_points": (C.c_int, [_P, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_uint32]),
    "ps_build_pyramid": (C.c_int, [C.c_int, C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_double), C.c_uint32,
                                   C.POINTER(C.c_void_p), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_double)]),
    "ps_write_ply": (C.c_int, [C.c_char_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]),
    # neighbour views and depth ranges
    "ps_neighbor_params_default": (None, [C.POINTER(NeighborParams)]),
    "ps_select_neighbors": (C.c_int, [C.c_int, C.POINTER(SparseView), C.c_uint32, _P, _P, _P, C.c_uint64,
                                      C.POINTER(NeighborParams), _P, _P, _P, _P, _P, _P]),
    # learned proposal
    "ps_net_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_P)]),
    "ps_net_destroy": (None, [_P]),
    "ps_net_last_error": (C.c_char_p, [_P]),
    "ps_net_num_params": (C.c_uint64, [_P]),
    "ps_net_step": (C.c_uint32, [_P]),
    "ps_net_get_params": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "ps_net_set_params": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "ps_net_forward": (C.c_int, [_P, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    "ps_net_train_step": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                    C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "ps_net_set_conv_path": (C.c_int, [C.c_int]),
    "ps_net_conv_timeouts": (C.c_int, [C.c_int, C.POINTER(C.c_uint32), C.c_int]),
    "ps_net_test_stall_convolutions": (C.c_int, [C.c_int, C.c_int]),
    "ps_net_conv_check": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ps_sweep_volume": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32]),
    "ps_set_sweep_normals": (C.c_int, [_P, C.c_void_p]),
    "ps_propose": (C.c_int, [_P, _P, C.c_uint32, _U32P, C.c_size_t, C.c_float, C.POINTER(C.c_uint64)]),
    "ps_proposal_upload": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(C.POINTER(C.c_float))]),
    "ps_proposal_download": (C.c_int, [_P, C.c_uint32, _U32P, C.c_size_t, C.POINTER(C.POINTER(C.c_float)),
                                       C.POINTER(C.POINTER(C.c_float))]),
}

_engine = None


def engine() -> C.CDLL:
    """Loads libpatchstereo.so (built in-tree by cumulus3d_b200.build); raises if it is missing."""
    global _engine
    if _engine is None:
        if not ENGINE_PATH.exists():
            raise RuntimeError(f"{ENGINE_PATH} is not built; run `python -m cumulus3d_b200.build` "
                               "(the engine has no CPU fallback)")
        lib = C.CDLL(str(ENGINE_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _engine = lib
    return _engine


# PmParams::default() (crates/dense/src/params.rs:126-154) and FilterParams::default() (:209-220), the values
# ps_pm_params_default / ps_filter_params_default return (a CPU test keeps them equal).  Plain Python, so that building
# an input never loads the engine library (the CPU oracle's users, such as the benchmark's reference arm, rely on it).
_PM_DEFAULTS = dict(window_radius=5, window_step=2, sigma_spatial=-1.0, sigma_color=0.2, tau0=0.8, tau_alpha=90.0,
                    tau1=1.2, beta=0.3, n1=2, n2=3, prev_view_weight=0.2, min_triangulation_angle_deg=1.0,
                    incident_angle_sigma=0.9, geom_lambda=0.2, geom_max_cost=3.0, top_k=3, eps0_photometric=0.2,
                    eps0_geometric=0.05, phi0_photometric_deg=30.0, phi0_geometric_deg=10.0, eps_min=0.005,
                    phi_min_deg=1.0, weak_texture_var=0.0)
_FILTER_DEFAULTS = dict(min_ncc=0.1, min_triangulation_angle_deg=3.0, min_num_consistent=2, geom_max_cost=1.0,
                        ncc_sigma=0.6, median_filter=1)


def default_pm() -> PmParams:
    return PmParams(**_PM_DEFAULTS)


def default_filter() -> FilterParams:
    return FilterParams(**_FILTER_DEFAULTS)


class PsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code
