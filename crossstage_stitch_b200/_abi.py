"""ctypes mirror of include/stitch_b200.h and loader of libstitch_b200.so.

The structs here have the layouts of the reference's stage structs
(src/common/types.hpp:16-70, src/s2_s3/s2.hpp:19-23, src/s4/s4.hpp:8-21,
src/s5/s5.hpp:11-19). Importing this module loads the native library and
raises if it is missing: there is no Python or CPU fallback for any stage.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libstitch_b200.so"


class Status(IntEnum):
    """src/common/status.hpp:6-13."""
    OK = 0
    INVALID_ARGUMENT = 1
    INSUFFICIENT_WORKSPACE = 2
    CUDA_ERROR = 3
    NOT_ENOUGH_POINTS = 4
    DEGENERATE = 5


class StageError(RuntimeError):
    def __init__(self, where: str, status: int):
        super().__init__(f"{where}: {Status(status).name if status in Status._value2member_map_ else status}")
        self.status = status


GRAY8 = 1
RGB8 = 0
BINARY_U8 = 0
FLOAT32 = 1


class ImageView(C.Structure):
    _fields_ = [("data", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("pitch_bytes", C.c_int), ("format", C.c_int)]


class ScaleInfo(C.Structure):
    _fields_ = [("orig_w", C.c_int), ("orig_h", C.c_int), ("work_w", C.c_int), ("work_h", C.c_int),
                ("sx", C.c_double), ("sy", C.c_double), ("D", C.c_double * 9)]


class Keypoints(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("response", C.c_void_p),
                ("capacity", C.c_int), ("d_count", C.c_void_p)]


class Descriptors(C.Structure):
    _fields_ = [("type", C.c_int), ("dim", C.c_int), ("row_stride_bytes", C.c_int), ("data", C.c_void_p)]


class Matches(C.Structure):
    _fields_ = [("idx_a", C.c_void_p), ("idx_b", C.c_void_p), ("distance", C.c_void_p),
                ("capacity", C.c_int), ("d_count", C.c_void_p)]


class HomographyResult(C.Structure):
    _fields_ = [("H", C.c_double * 9), ("H_s", C.c_double * 9), ("num_matches", C.c_int),
                ("num_inliers", C.c_int), ("inlier_ratio", C.c_double), ("inlier_coverage", C.c_double),
                ("reproj_residual", C.c_double), ("status", C.c_int)]


class S2Config(C.Structure):
    _fields_ = [("fast_threshold", C.c_int), ("max_keypoints", C.c_int), ("harris_k", C.c_float)]


class S4Config(C.Structure):
    _fields_ = [("ratio_threshold", C.c_double), ("cross_check", C.c_uint8), ("reserved", C.c_uint8 * 7)]


class Top2(C.Structure):
    _fields_ = [("first_distance", C.c_double), ("second_distance", C.c_double),
                ("first_index", C.c_int), ("second_index", C.c_int)]


class S5Config(C.Structure):
    _fields_ = [("hypotheses", C.c_int), ("previous_hypotheses", C.c_int), ("batch_size", C.c_int),
                ("refinement_steps", C.c_int), ("threshold", C.c_double), ("seed", C.c_uint64),
                ("generation", C.c_uint64)]


class PyramidConfig(C.Structure):
    """stitch_pyramid_config: levels 1 (or 0) is the single-level path."""
    _fields_ = [("levels", C.c_int), ("scale_factor", C.c_float)]


class PairDesc(C.Structure):
    """stitch_pair_desc: one pair of the batched form."""
    _fields_ = [("image_a", ImageView), ("image_b", ImageView), ("scale_a", ScaleInfo), ("scale_b", ScaleInfo),
                ("s2", S2Config), ("s4", S4Config), ("s5", S5Config), ("pyramid", PyramidConfig)]


class BatchTuning(C.Structure):
    """stitch_batch_tuning: launch shapes of a batch plan (0: default)."""
    _fields_ = [("fast_ctas_per_sm", C.c_int), ("blur_ctas_per_sm", C.c_int), ("matcher", C.c_int),
                ("search_hpw", C.c_int), ("resize_tile_h", C.c_int)]


class ServerConfig(C.Structure):
    """stitch_server_config."""
    _fields_ = [("arena", C.c_void_p), ("arena_bytes", C.c_size_t), ("device", C.c_int), ("max_batch", C.c_int),
                ("streams", C.c_int)]


class Request(C.Structure):
    """stitch_request: one pair for the served form (host images)."""
    _fields_ = [("host_a", C.c_void_p), ("host_b", C.c_void_p),
                ("width_a", C.c_int), ("height_a", C.c_int), ("pitch_a", C.c_int),
                ("width_b", C.c_int), ("height_b", C.c_int), ("pitch_b", C.c_int),
                ("scale_a", ScaleInfo), ("scale_b", ScaleInfo), ("s2", S2Config), ("s4", S4Config),
                ("s5", S5Config), ("pyramid", PyramidConfig), ("rgb", C.c_int), ("scale", C.c_double),
                ("retry_hypotheses", C.c_int), ("retry_min_inliers", C.c_int), ("tag", C.c_uint64),
                ("host_panorama", C.c_void_p), ("host_mask", C.c_void_p), ("panorama_capacity", C.c_size_t)]


class ServerResult(C.Structure):
    """stitch_server_result."""
    _fields_ = [("tag", C.c_uint64), ("submit_ms", C.c_double), ("launch_ms", C.c_double),
                ("done_ms", C.c_double), ("batch_pairs", C.c_int), ("status", C.c_int), ("attempts", C.c_int),
                ("result", HomographyResult), ("render_status", C.c_int), ("canvas_width", C.c_int),
                ("canvas_height", C.c_int), ("origin_x", C.c_int), ("origin_y", C.c_int),
                ("union_pixels", C.c_uint64), ("overlap_pixels", C.c_uint64)]


class S6Policy(C.Structure):
    """stitch_s6_policy (src/s6/geometry.hpp:10-16)."""
    _fields_ = [("denominator_tolerance", C.c_double), ("inverse_tolerance", C.c_double),
                ("snap_tolerance", C.c_double), ("max_canvas_pixels", C.c_size_t)]


class S6Geometry(C.Structure):
    """stitch_s6_geometry (src/s6/geometry.hpp:18-34)."""
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("origin_x", C.c_int), ("origin_y", C.c_int),
                ("width_a", C.c_int), ("height_a", C.c_int), ("width_b", C.c_int), ("height_b", C.c_int),
                ("denominator_tolerance", C.c_double), ("snap_tolerance", C.c_double),
                ("inverse", C.c_double * 9)]


S6_FEATHER, S6_MULTIBAND3, S6_MULTIBAND5 = 0, 1, 2

P = C.POINTER
_size_p = P(C.c_size_t)

# name -> (restype, argtypes); every entry point of include/stitch_b200.h.
PROTOTYPES: dict[str, tuple] = {
    "stitch_abi_version": (C.c_int, []),
    "stitch_status_name": (C.c_char_p, [C.c_int]),
    "stitch_launch_count": (C.c_longlong, []),
    "stitch_make_scale_info": (C.c_int, [C.c_int, C.c_int, C.c_double, P(ScaleInfo)]),
    "stitch_to_original": (C.c_int, [P(C.c_double)] * 4),
    "stitch_s1_preprocess": (C.c_int, [P(ImageView), P(ImageView), C.c_double, P(ImageView), P(ImageView),
                                       P(ScaleInfo), P(ScaleInfo), C.c_void_p]),
    "stitch_s1_preprocess_single": (C.c_int, [P(ImageView), C.c_double, P(ImageView), P(ScaleInfo), C.c_void_p]),
    "stitch_s1_compute_gradient": (C.c_int, [P(ImageView), P(ImageView), C.c_void_p, P(C.c_double),
                                             P(C.c_double), C.c_void_p]),
    "stitch_s2_workspace_bytes": (C.c_int, [C.c_int, C.c_int, P(S2Config), _size_p]),
    "stitch_s2_detect": (C.c_int, [P(ImageView), P(S2Config), P(Keypoints), C.c_void_p, C.c_size_t, C.c_void_p]),
    "stitch_s2_detect_marked": (C.c_int, [P(ImageView), P(S2Config), P(Keypoints), C.c_void_p, C.c_size_t,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "stitch_s3_workspace_bytes": (C.c_int, [C.c_int, C.c_int, _size_p]),
    "stitch_s3_describe": (C.c_int, [P(ImageView), P(Keypoints), P(Descriptors), C.c_void_p, C.c_size_t,
                                     C.c_void_p]),
    "stitch_s3_describe_marked": (C.c_int, [P(ImageView), P(Keypoints), P(Descriptors), C.c_void_p,
                                            C.c_size_t, C.c_void_p, C.c_void_p]),
    "stitch_pyramid_workspace_bytes": (C.c_int, [C.c_int, C.c_int, P(S2Config), P(PyramidConfig), _size_p]),
    "stitch_pyramid_detect_describe": (C.c_int, [P(ImageView), P(S2Config), P(PyramidConfig), P(Keypoints),
                                                 P(Descriptors), C.c_void_p, C.c_size_t, C.c_void_p]),
    "stitch_s4_set_matcher": (C.c_int, [C.c_int]),
    "stitch_s4_matcher": (C.c_int, []),
    "stitch_s4_tc_errors": (C.c_int, []),
    "stitch_s4_workspace_bytes": (C.c_int, [C.c_int, C.c_int, P(S4Config), _size_p]),
    "stitch_s4_knn_top2": (C.c_int, [P(Keypoints), P(Descriptors), P(Keypoints), P(Descriptors), C.c_void_p,
                                     C.c_void_p]),
    "stitch_s4_match": (C.c_int, [P(Keypoints), P(Descriptors), P(Keypoints), P(Descriptors), P(S4Config),
                                  P(Matches), C.c_void_p, C.c_size_t, C.c_void_p]),
    "stitch_s4_forward_neighbors": (C.c_int, [C.c_int, C.c_int, P(S4Config), C.c_void_p, C.c_size_t,
                                              P(C.c_void_p)]),
    "stitch_s4_match_static": (C.c_int, [P(Keypoints), P(Descriptors), P(Keypoints), P(Descriptors), P(S4Config),
                                         P(Matches), C.c_void_p]),
    "stitch_s5_workspace_bytes": (C.c_int, [P(S5Config), _size_p]),
    "stitch_s5_estimate": (C.c_int, [P(Keypoints), P(Keypoints), P(Matches), P(ScaleInfo), P(ScaleInfo),
                                     P(S5Config), C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "stitch_s6_default_policy": (None, [P(S6Policy)]),
    "stitch_s6_prepare_geometry": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_double), P(S6Policy),
                                             P(S6Geometry)]),
    "stitch_s6_workspace_bytes": (C.c_int, [P(S6Geometry), C.c_int, _size_p]),
    "stitch_s6_render": (C.c_int, [P(ImageView), P(ImageView), P(S6Geometry), C.c_int, P(ImageView), P(ImageView),
                                   C.c_void_p, C.c_size_t, C.c_void_p, P(C.c_uint64)]),
    "stitch_batch_create": (C.c_int, [C.c_int, P(PairDesc), P(C.c_void_p), _size_p, P(C.c_int)]),
    "stitch_batch_create_tuned": (C.c_int, [C.c_int, P(PairDesc), P(BatchTuning), P(C.c_void_p), _size_p,
                                            P(C.c_int)]),
    "stitch_batch_enqueue": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "stitch_batch_capture": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "stitch_batch_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "stitch_batch_pair_outputs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, P(Keypoints), P(Keypoints),
                                            P(Descriptors), P(Descriptors), P(Matches), P(C.c_void_p),
                                            P(C.c_void_p)]),
    "stitch_batch_destroy": (None, [C.c_void_p]),
    "stitch_batch_set_matcher": (C.c_int, [C.c_void_p, C.c_int]),
    "stitch_batch_set_marks": (C.c_int, [C.c_void_p, P(C.c_void_p), C.c_int]),
    "stitch_server_create": (C.c_int, [P(ServerConfig), P(C.c_void_p)]),
    "stitch_server_request_bytes": (C.c_int, [P(Request), _size_p]),
    "stitch_server_submit": (C.c_int, [C.c_void_p, P(Request)]),
    "stitch_server_poll": (C.c_int, [C.c_void_p, P(ServerResult), C.c_int, P(C.c_int)]),
    "stitch_server_outstanding": (C.c_int, [C.c_void_p]),
    "stitch_server_destroy": (None, [C.c_void_p]),
}

BATCH_MARKS = ("tables", "pyramid", "fast_nms", "select_scatter", "harris", "sort_topk", "blur", "describe", "knn",
               "knn_merge", "accept", "prepare", "search", "finish")

_LIB: C.CDLL | None = None


def load(path: Path | None = None) -> C.CDLL:
    """Loads the native library once and binds every prototype."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"native library {p} is missing: run `python -m crossstage_stitch_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib
