"""The ensemble's bucket-size rule (host logic only, no GPU call): cases
of one size share launches up to what keeps their finest multigrid level
within half the L2 and the stacked grid within the z limit; a cap set per
size overrides the rule and is clipped to the grid limit; the autotuner's
JSON cache re-installs it."""
import json

import pytest


def _cap(n, fp32=True):
    from warpflow import autotune
    return autotune.bucket_cap(n, fp32)


def _rule(n, fp32):
    lvl = 2 * (n + 2) ** 3 * (4 if fp32 else 8)
    return max(1, min(60000 // (n + 6), (64 << 20) // lvl))


@pytest.mark.parametrize("fp32", [True, False])
def test_default_rule(fp32):
    for n in (8, 16, 32, 48, 56, 64, 80, 96, 128, 256):
        assert _cap(n, fp32) == _rule(n, fp32), n
    assert _cap(256, fp32) == 1 and _cap(96, True) == 8 and _cap(80, True) == 15


def test_override_and_clip():
    from warpflow import _abi, autotune
    try:
        autotune.set_bucket_cap(80, 6)
        assert _cap(80) == 6 and _cap(80, fp32=False) == _rule(80, False)
        autotune.set_bucket_cap(32, 10 ** 6)
        assert _cap(32) == 60000 // (32 + 6)
        autotune.set_bucket_cap(32, 1)
        assert _cap(32) == 1
    finally:
        autotune.set_bucket_cap(80, 0)
        autotune.set_bucket_cap(32, 0)
    assert _cap(80) == _rule(80, True) and _cap(32) == _rule(32, True)
    with pytest.raises(RuntimeError):
        autotune.set_bucket_cap(2, 4)
    with pytest.raises(RuntimeError):
        autotune.set_bucket_cap(32, -1)


def test_cache_round_trip(tmp_path):
    from warpflow import autotune
    p = tmp_path / "tune.json"
    coarse = {20: {"best": 2, "us": {"2": 1.0}}}
    buckets = {48: {"cap": 1, "ms": {"bucket": 3.0, "branches": 2.0}},
               96: {"cap": 8, "ms": {"bucket": 9.0, "branches": 12.0}}}
    try:
        autotune.save(coarse, p, buckets=buckets)
        doc = json.loads(p.read_text())
        assert set(doc) == {"coarse", "buckets"}
        autotune.load_and_apply(p)
        assert _cap(48) == 1 and _cap(96) == 8
    finally:
        autotune.set_bucket_cap(48, 0)
        autotune.set_bucket_cap(96, 0)
        autotune.set_strategy(20, 2)
        autotune.set_strategy(20, 2, fp32=True)


def test_launch_shapes_set_validate_and_cache(tmp_path):
    """Launch-shape table (host only): defaults, accepted and rejected
    shapes, reset, and the JSON cache."""
    from warpflow import autotune
    # built-in shapes by size (the tuner's measurements on B200)
    assert autotune.shape("conv", 80) == (32, 4, 2)
    assert autotune.shape("conv", 48) == (32, 8, 1)
    assert autotune.shape("conv", 256) == (32, 4, 4)
    assert autotune.shape("split", 80) == (4, 8, 1)
    assert autotune.shape("split", 128) == (2, 8, 1)
    assert autotune.shape("split", 256) == (4, 2, 1)
    try:
        autotune.set_shape("conv", 80, 16, 16, 4)
        autotune.set_shape("split", 80, 4, 2)
        assert autotune.shape("conv", 80) == (16, 16, 4)
        assert autotune.shape("split", 80) == (4, 2, 1)
        assert autotune.shape("conv", 96) == (32, 4, 2)      # per size
        for kind, a, b, c in (("conv", 24, 8, 1), ("conv", 32, 16, 1), ("conv", 16, 1, 1),
                              ("conv", 32, 8, 0), ("conv", 32, 8, 17),
                              ("split", 3, 8, 1), ("split", 16, 8, 1), ("split", 2, 16, 1),
                              ("split", 2, 8, 2)):
            with pytest.raises(RuntimeError):
                autotune.set_shape(kind, 80, a, b, c)
        p = tmp_path / "tune.json"
        autotune.save({}, p, shapes={"conv": {80: {"best": [64, 4, 2], "us": {}}},
                                     "split": {80: {"best": [1, 4, 1], "us": {}}}})
        autotune.load_and_apply(p)
        assert autotune.shape("conv", 80) == (64, 4, 2)
        assert autotune.shape("split", 80) == (1, 4, 1)
    finally:
        autotune.set_shape("conv", 80, 0, 0, 0)
        autotune.set_shape("split", 80, 0, 0, 0)
    assert autotune.shape("conv", 80) == (32, 4, 2)
