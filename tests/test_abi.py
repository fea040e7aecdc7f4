"""The C ABI library (CPU only: no compute calls).

* libpatchstereo.so loads and exports every function declared in include/patchstereo.h, and the integration guide
  names each of them;
* the ctypes mirror has the same struct sizes and field offsets as a C compilation of the header;
* without a GPU, backend creation fails with PS_ENODEV (no CPU fallback exists);
* parameter defaults equal the reference's PmParams::default / FilterParams::default
  (crates/dense/src/params.rs:126-154, :196-207).
"""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from cumulus3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "patchstereo.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(ps_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_lib.ENGINE_PATH))
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes table covers the same set
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_integration_guide_names_every_declared_function():
    """The integration guide is where a maintainer writing the binding looks each entry point up."""
    guide = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    missing = [n for n in declared_functions() if not re.search(r"\b" + n + r"\b", guide)]
    assert not missing, missing


STRUCTS = {
    "ps_options": _lib.Options, "ps_pm_params": _lib.PmParams, "ps_filter_params": _lib.FilterParams,
    "ps_level_image": _lib.LevelImage, "ps_pair_geometry": _lib.PairGeometry, "ps_kernel_view": _lib.KernelView,
    "ps_kernel_input": _lib.KernelInput, "ps_view_state": _lib.ViewState, "ps_run_params": _lib.RunParams,
    "ps_depth_snapshot": _lib.DepthSnapshot, "ps_schedule": _lib.Schedule,
    "ps_multiscale_schedule": _lib.MultiscaleSchedule, "ps_post_params": _lib.PostParams,
    "ps_fusion_params": _lib.FusionParams, "ps_fusion_view": _lib.FusionView, "ps_sparse_view": _lib.SparseView,
    "ps_neighbor_params": _lib.NeighborParams, "ps_score_fusion_params": _lib.ScoreFusionParams,
}


def test_struct_layout_matches_c():
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-o", exe, c], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(l.rsplit(" ", 1) for l in out if l)
    for cname, py in STRUCTS.items():
        assert int(got[f"{cname} size"]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def test_no_gpu_means_enodev():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.engine()
    h = C.c_void_p()
    rc = lib.ps_backend_create(0, None, C.byref(h))
    assert rc == _lib.PS_ENODEV and not h.value
    from cumulus3d_b200.patchstereo import PatchMatchBackend, PsError
    with pytest.raises(PsError) as e:
        PatchMatchBackend(0)
    assert e.value.code == _lib.PS_ENODEV


def test_null_arguments_rejected_without_device():
    lib = _lib.engine()
    assert lib.ps_backend_create(0, None, None) == _lib.PS_EINVAL
    assert lib.ps_begin(None, None, None) == _lib.PS_EINVAL
    assert lib.ps_end(None) == _lib.PS_EINVAL
    assert lib.ps_run(None, None, 0, None, None, None) == _lib.PS_EINVAL
    assert lib.ps_last_error(None) == b"session is NULL"
    assert lib.ps_abi_version() == 5
    # learned-proposal entry points
    assert lib.ps_net_create(0, 1, None) == _lib.PS_EINVAL
    assert lib.ps_net_num_params(None) == 0
    assert lib.ps_net_last_error(None) == b"net is NULL"
    assert lib.ps_net_forward(None, None, 1, 8, 8, None, None) == _lib.PS_EINVAL
    assert lib.ps_net_train_step(None, None, None, 1, 8, 8, 25.0, 60.0, 0.0, 0.0, None, None) == _lib.PS_EINVAL
    assert lib.ps_sweep_volume(None, 0, 0, None, 0) == _lib.PS_EINVAL
    assert lib.ps_propose(None, None, 0, None, 0, 0.5, None) == _lib.PS_EINVAL
    # post-processing and fusion entry points
    assert lib.ps_postprocess_resident(None, 0, None, 0, None, None, None, None) == _lib.PS_EINVAL
    assert lib.ps_fuse_resident(None, 0, None, 0, None, None, None, None) == _lib.PS_EINVAL
    assert lib.ps_fuse_scored_resident(None, 0, None, 0, None, None, None, None) == _lib.PS_EINVAL
    assert lib.ps_fused_points(None, 0, None, None, None, None, None, None, 0) == _lib.PS_EINVAL
    assert lib.ps_fused_visibility_removed(None, None) == _lib.PS_EINVAL
    lib.ps_score_fusion_params_default(None)  # NULL is ignored, as by the other *_default functions


def test_defaults_match_reference():
    pm = _lib.default_pm()
    assert (pm.window_radius, pm.window_step, pm.sigma_spatial, pm.top_k, pm.n1, pm.n2) == (5, 2, -1.0, 3, 2, 3)
    for name, want in [("sigma_color", 0.2), ("tau0", 0.8), ("tau_alpha", 90.0), ("tau1", 1.2), ("beta", 0.3),
                       ("prev_view_weight", 0.2), ("min_triangulation_angle_deg", 1.0), ("incident_angle_sigma", 0.9),
                       ("geom_lambda", 0.2), ("geom_max_cost", 3.0), ("eps0_photometric", 0.2),
                       ("eps0_geometric", 0.05), ("phi0_photometric_deg", 30.0), ("phi0_geometric_deg", 10.0),
                       ("eps_min", 0.005), ("phi_min_deg", 1.0), ("weak_texture_var", 0.0)]:
        assert abs(getattr(pm, name) - want) < 1e-7, name
    fl = _lib.default_filter()
    assert (fl.min_num_consistent, fl.median_filter) == (2, 1)
    for name, want in [("min_ncc", 0.1), ("min_triangulation_angle_deg", 3.0), ("geom_max_cost", 1.0),
                       ("ncc_sigma", 0.6)]:
        assert abs(getattr(fl, name) - want) < 1e-7, name
    o = _lib.Options()
    _lib.engine().ps_options_default(C.byref(o))
    assert (o.math_mode, o.max_batch, o.batch_pixels, o.checked, o.tuning) == (0, 64, 0, 0, 0)
    # the Python defaults (which never load the engine) are the engine's exported defaults, field for field
    epm, efl = _lib.PmParams(), _lib.FilterParams()
    _lib.engine().ps_pm_params_default(C.byref(epm))
    _lib.engine().ps_filter_params_default(C.byref(efl))
    assert bytes(epm) == bytes(pm) and bytes(efl) == bytes(fl)


def test_post_fusion_and_neighbour_defaults_match_reference():
    """PostParams (crates/dense/src/postproc.rs:61-74), FusionParams with ResidualParams / VisibilityParams /
    SmoothParams (crates/dense/src/params.rs:278-351, visibility.rs:60-64, smooth.rs:67-71) and NeighborOptions
    (params.rs:366-369) defaults."""
    import math
    lib = _lib.engine()
    post = _lib.PostParams()
    lib.ps_post_params_default(C.byref(post))
    assert (post.remove_speckles, post.fill_holes) == (1, 0)
    for name, want in [("speckle_rel_depth", 0.02), ("speckle_min_area_frac", 2e-4), ("speckle_keep_cost", 0.2),
                       ("fill_max_frac", 0.01), ("fill_edge_step", 0.06), ("fill_max_cost", 1.0)]:
        assert abs(getattr(post, name) - want) < 1e-7, name
    f = _lib.FusionParams()
    lib.ps_fusion_params_default(C.byref(f))
    assert (f.min_consistent_views, f.consistency_num_images, f.mark_used, f.mark_radius, f.inverse_variance,
            f.residual, f.residual_min_views) == (5, 12, 1, 0, 1, _lib.PS_FUSION_RESIDUAL_NONE, 2)
    assert math.isnan(f.residual_depth_error) and math.isnan(f.residual_normal_error_deg)
    assert f.residual_min_dist_gsd == 0.5
    assert (f.visibility_check_views, f.visibility_min_violations, f.visibility_tau) == (0, 2, 0.01)
    assert (f.smooth_iterations, f.smooth_radius_gsd, f.smooth_sigma_range_gsd, f.smooth_normal_deg) == \
        (0, 1.0, 0.25, 30.0)
    nb = _lib.NeighborParams()
    lib.ps_neighbor_params_default(C.byref(nb))
    assert (nb.num_views, nb.direction_bins, nb.min_triangulation_angle_deg, nb.diversity_decay) == (10, 8, 1.0, 1.0)
    sf = _lib.ScoreFusionParams()
    lib.ps_score_fusion_params_default(C.byref(sf))  # ScoreFusionOptions (crates/dense/src/fusion_score.rs:81-97)
    assert (sf.sigma_e_px, sf.sigma_theta_deg, getattr(sf, "lambda"), sf.tau, sf.depth_error, sf.normal_error_deg,
            sf.num_neighbors, sf.mark_used, sf.inverse_variance, sf.sigma_px0, sf.sigma_px_slope) == \
        (1.0, 2.0, 1.0, 2.0, 0.01, 10.0, 12, 1, 1, 0.25, 1.0)


def test_reciprocal_check_validates_its_range_without_device():
    lib = _lib.engine()
    bad = C.c_uint64()
    assert lib.ps_check_reciprocal(0, -127, 0, C.byref(bad), None) == _lib.PS_EINVAL
    assert lib.ps_check_reciprocal(0, 0, 128, C.byref(bad), None) == _lib.PS_EINVAL
    assert lib.ps_check_reciprocal(0, 5, 4, C.byref(bad), None) == _lib.PS_EINVAL
    assert lib.ps_check_reciprocal(0, 0, 1, None, None) == _lib.PS_EINVAL
    assert lib.ps_fused_visibility_removed(None, C.byref(bad)) == _lib.PS_EINVAL
