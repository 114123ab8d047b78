"""Resolution buckets and K classes of the autotuner (host logic only)."""
from crossstage_stitch_b200 import tune


def test_buckets_and_k_classes():
    assert tune.bucket_of(640, 480, 640, 480) == "vga"
    assert tune.bucket_of(1280, 720, 1200, 700) == "720p"
    assert tune.bucket_of(1920, 1080, 640, 480) == "1080p"   # the larger image decides
    assert tune.bucket_of(3840, 2160, 3840, 2160) == "4k"
    assert tune.bucket_of(512, 512, 512, 512) == "vga"
    assert [tune.k_class(k) for k in (1, 500, 1000, 2000, 4000, 8000, 20000)] == \
        ["k500", "k500", "k500", "k2000", "k2000", "k8000", "k8000"]
    # every tuning field has its default first and valid values only
    assert tune.SPACE["fast_ctas_per_sm"][0] == 7 and tune.SPACE["resize_tile_h"][0] == 64
    assert all(1 <= m <= 5 for m in tune.SPACE["matcher"])
