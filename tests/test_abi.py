"""The native library loads without a GPU, exports every C entry point of
include/stitch_b200.h and the reference's C++ stage symbols, and its
host-only checks behave as the reference's (no device work is queued)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from crossstage_stitch_b200 import _abi
from crossstage_stitch_b200._abi import S2Config, S4Config, S5Config, ScaleInfo, Status

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "stitch_b200.h"
REF_STAGES = ROOT / "oracle" / "_ref" / "libref_stages.so"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(stitch_[a-z0-9_]+)\s*\(", text)))


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}


def test_every_header_function_is_exported_and_bound():
    lib = _abi.load()
    names = header_functions()
    assert names, "no declarations parsed"
    syms = exported(_abi.LIB_PATH)
    for n in names:
        assert n in syms, n
        assert n in _abi.PROTOTYPES, f"{n} missing from the ctypes mirror"
        getattr(lib, n)


def test_reference_cpp_symbols_are_exported():
    """Code compiled against the reference headers links against this library."""
    if not REF_STAGES.exists():
        pytest.skip("reference stage build not present (oracle/_ref)")
    ref = {s for s in exported(REF_STAGES) if s.startswith("_ZN6stitch2s") or s.startswith("_ZN6stitch5s2_s3")}
    public = {s for s in ref if "detail" not in s or "marked" in s}
    ours = exported(_abi.LIB_PATH)
    missing = sorted(public - ours)
    assert not missing, missing


def test_struct_sizes():
    assert C.sizeof(_abi.HomographyResult) == 184
    assert C.sizeof(_abi.ScaleInfo) == 104
    assert C.sizeof(_abi.S4Config) == 16
    assert C.sizeof(_abi.S5Config) == 40
    assert C.sizeof(_abi.Top2) == 24


def test_workspace_queries():
    L = _abi.load()
    b = C.c_size_t(123)
    assert L.stitch_s2_workspace_bytes(640, 480, C.byref(S2Config(20, 0, 0.04)), C.byref(b)) == 0 and b.value == 0
    assert L.stitch_s2_workspace_bytes(640, 480, C.byref(S2Config(0, 10, 0.04)), C.byref(b)) == Status.INVALID_ARGUMENT
    assert L.stitch_s2_workspace_bytes(640, 480, C.byref(S2Config(20, 10, -1.0)), C.byref(b)) == Status.INVALID_ARGUMENT
    assert L.stitch_s2_workspace_bytes(640, 480, C.byref(S2Config(20, 1000, 0.04)), C.byref(b)) == 0
    small = b.value
    assert L.stitch_s2_workspace_bytes(677, 480, C.byref(S2Config(20, 1000, 0.04)), C.byref(b)) == 0
    assert b.value > small   # a wider image needs more workspace
    assert L.stitch_s3_workspace_bytes(0, 5, C.byref(b)) == Status.INVALID_ARGUMENT
    c4 = S4Config()
    c4.ratio_threshold = 1.0
    assert L.stitch_s4_workspace_bytes(10, 10, C.byref(c4), C.byref(b)) == Status.INVALID_ARGUMENT
    c4.ratio_threshold = 0.8
    assert L.stitch_s4_workspace_bytes(0, 10, C.byref(c4), C.byref(b)) == 0 and b.value == 0
    assert L.stitch_s4_workspace_bytes(-1, 10, C.byref(c4), C.byref(b)) == Status.INVALID_ARGUMENT
    c5 = S5Config(129, 0, 32, 2, 3.0, 20261022, 1)
    e = C.c_size_t()
    assert L.stitch_s5_workspace_bytes(C.byref(c5), C.byref(b)) == 0 and b.value > 0
    c5.hypotheses, c5.previous_hypotheses = 1000, 129
    assert L.stitch_s5_workspace_bytes(C.byref(c5), C.byref(e)) == 0 and e.value == b.value
    for field, value in (("previous_hypotheses", 1001), ("threshold", float("nan")), ("threshold", 0.0),
                         ("batch_size", 65536), ("refinement_steps", -1)):
        bad = S5Config(1000, 0, 32, 2, 3.0, 1, 1)
        setattr(bad, field, value)
        assert L.stitch_s5_workspace_bytes(C.byref(bad), C.byref(b)) == Status.INVALID_ARGUMENT, field
    assert L.stitch_s5_workspace_bytes(C.byref(c5), None) == Status.INVALID_ARGUMENT


def test_scale_info_and_to_original():
    L = _abi.load()
    s = ScaleInfo()
    assert L.stitch_make_scale_info(1281, 961, 0.5, C.byref(s)) == 0
    assert (s.work_w, s.work_h) == (641, 481)
    assert L.stitch_make_scale_info(10, 10, 1.5, C.byref(s)) == Status.INVALID_ARGUMENT
    import numpy as np
    from oracle import c_oracle
    a = c_oracle.make_scale_info(641, 479, 0.5)
    bb = c_oracle.make_scale_info(803, 601, 0.75)
    hs = np.array([1, 0.01, 5, -0.02, 1, 9, 0.0001, 0.0002, 1.0])
    out = np.zeros(9)
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    assert L.stitch_to_original(dp(hs), dp(a["D"]), dp(bb["D"]), dp(out)) == 0
    rec = np.linalg.inv(np.diag([1, 1, 1.0])) @ (a["D"].reshape(3, 3) @ out.reshape(3, 3)
                                                @ np.linalg.inv(bb["D"].reshape(3, 3)))
    assert np.max(np.abs(rec / rec[2, 2] - hs.reshape(3, 3))) < 1e-12


def test_host_validation_needs_no_device():
    """Invalid arguments are rejected before any CUDA call."""
    L = _abi.load()
    iv = _abi.ImageView(0, 64, 64, 64, 1)
    kp = _abi.Keypoints(0, 0, 0, 10, 0)
    assert L.stitch_s2_detect(C.byref(iv), C.byref(S2Config(20, 10, 0.04)), C.byref(kp), None, 0, None) \
        == Status.INVALID_ARGUMENT


def test_pyramid_workspace_and_validation():
    """The pyramid knob's checks and workspace query are host-only."""
    L = _abi.load()
    b = C.c_size_t()
    cfg = S2Config(20, 1000, 0.04)
    for levels, factor in ((17, 1.2), (8, 1.0), (8, float("nan")), (8, 16.5), (-1, 1.2)):
        assert L.stitch_pyramid_workspace_bytes(512, 512, C.byref(cfg), C.byref(_abi.PyramidConfig(levels, factor)),
                                                C.byref(b)) == Status.INVALID_ARGUMENT, (levels, factor)
    sizes = []
    for levels in (1, 2, 8):
        assert L.stitch_pyramid_workspace_bytes(512, 512, C.byref(cfg), C.byref(_abi.PyramidConfig(levels, 1.2)),
                                                C.byref(b)) == 0
        sizes.append(b.value)
    assert sizes[0] < sizes[1] < sizes[2]
    # levels 0 means one level; a factor is not needed then
    assert L.stitch_pyramid_workspace_bytes(512, 512, C.byref(cfg), C.byref(_abi.PyramidConfig(0, 0.0)),
                                            C.byref(b)) == 0 and b.value == sizes[0]
    iv = _abi.ImageView(0, 64, 64, 64, 1)
    kp = _abi.Keypoints(0, 0, 0, 10, 0)
    ds = _abi.Descriptors(0, 32, 32, 0)
    assert L.stitch_pyramid_detect_describe(C.byref(iv), C.byref(S2Config(20, 10, 0.04)),
                                            C.byref(_abi.PyramidConfig(8, 1.2)), C.byref(kp), C.byref(ds), None, 0,
                                            None) == Status.INVALID_ARGUMENT


def test_server_request_bytes_is_host_only():
    """The served form's footprint query (no device work): a request's arena
    bytes grow with its images, K and a panorama buffer, and requests the
    server would reject are rejected the same way."""
    import numpy as np

    from crossstage_stitch_b200._abi import Request
    from crossstage_stitch_b200.stages import Knobs

    L = _abi.load()
    host = np.zeros((1080, 1920 * 3), np.uint8)

    def request(w, h, rgb=False, k=1000, pano=0, mask=False):
        r = Request()
        r.host_a = r.host_b = host.ctypes.data
        r.width_a = r.width_b = w
        r.height_a = r.height_b = h
        r.pitch_a = r.pitch_b = host.strides[0]
        r.rgb = 1 if rgb else 0
        r.scale = 1.0 if rgb else 0.0
        kn = Knobs(max_keypoints=k, levels=8)
        r.s2, r.s4, r.s5, r.pyramid = kn.s2(), kn.s4(), kn.s5(), kn.pyramid()
        if pano:
            r.host_panorama, r.panorama_capacity = host.ctypes.data, pano
        if mask:
            r.host_mask = host.ctypes.data
        return r

    def nbytes(r):
        b = C.c_size_t(123)
        st = L.stitch_server_request_bytes(C.byref(r), C.byref(b))
        return st, b.value

    st_small, small = nbytes(request(512, 512))
    st_big, big = nbytes(request(1920, 1080))
    st_k, more_k = nbytes(request(512, 512, k=8000))
    assert st_small == st_big == st_k == Status.OK and 0 < small < big and small < more_k
    st_rgb, rgb = nbytes(request(512, 512, rgb=True))
    st_pano, pano = nbytes(request(512, 512, rgb=True, pano=1 << 20))
    assert st_rgb == st_pano == Status.OK and rgb > small and pano >= rgb + 4 * (1 << 20)
    assert nbytes(request(512, 512, pano=1 << 20))[0] == Status.INVALID_ARGUMENT   # panoramas need RGB
    assert nbytes(request(512, 512, rgb=True, mask=True))[0] == Status.INVALID_ARGUMENT  # mask without panorama
    bad = request(512, 512)
    bad.host_a = None
    assert nbytes(bad) == (Status.INVALID_ARGUMENT, 0)
    assert L.stitch_server_request_bytes(None, None) == Status.INVALID_ARGUMENT


def test_static_match_reports_argument_errors_like_stitch_s4_match():
    """stitch_s4_match_static runs stitch_s4_match's host checks first, so an
    invalid request gets the same status from both (INVALID_ARGUMENT), and
    only a valid request too large for the 4 MiB scratch gets
    INSUFFICIENT_WORKSPACE; neither reaches the device."""
    from crossstage_stitch_b200._abi import Descriptors, Keypoints, Matches
    L = _abi.load()
    cfg = S4Config()
    cfg.ratio_threshold = 0.8
    cfg.cross_check = 1
    big = 200000
    fake = 1 << 20   # aligned host-side stand-ins; nothing is dereferenced
    kp = Keypoints(0, 0, 0, big, fake)
    out = Matches(fake, fake, fake, big, fake)
    bad_desc = Descriptors(0, 32, 0, fake)     # stride 0: invalid
    good_desc = Descriptors(0, 32, 32, fake)
    args = lambda d: (C.byref(kp), C.byref(d), C.byref(kp), C.byref(d), C.byref(cfg), C.byref(out))
    assert L.stitch_s4_match_static(*args(bad_desc), None) == Status.INVALID_ARGUMENT
    assert L.stitch_s4_match(*args(bad_desc), None, 0, None) == Status.INVALID_ARGUMENT
    assert L.stitch_s4_match_static(*args(good_desc), None) == Status.INSUFFICIENT_WORKSPACE
    assert L.stitch_s4_match(*args(good_desc), None, 0, None) == Status.INSUFFICIENT_WORKSPACE
    short = Matches(fake, fake, fake, big - 1, fake)   # output capacity below the query capacity
    assert L.stitch_s4_match_static(C.byref(kp), C.byref(good_desc), C.byref(kp), C.byref(good_desc),
                                    C.byref(cfg), C.byref(short), None) == Status.INVALID_ARGUMENT


def test_matcher_choice_is_per_thread():
    """The S4 matcher is a property of the calling host thread: another
    thread's choice does not change this one's."""
    import threading
    L = _abi.load()
    mine = L.stitch_s4_matcher()
    assert L.stitch_s4_set_matcher(7) == Status.INVALID_ARGUMENT
    seen = {}

    def other():
        seen["default"] = L.stitch_s4_matcher()
        seen["set"] = L.stitch_s4_set_matcher(1 - mine)
        seen["after"] = L.stitch_s4_matcher()

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen == {"default": 1, "set": 0, "after": 1 - mine}
    assert L.stitch_s4_matcher() == mine
    assert L.stitch_batch_set_matcher(None, 0) == Status.INVALID_ARGUMENT
