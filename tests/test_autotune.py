"""The launch-shape cache behind the autotuner (host functions of
libtct_b200.so; no GPU): keys, size buckets, enumeration and the JSON round
trip that carries tuned shapes across processes."""
import json

import pytest

from tectosaur_b200 import _lib, autotune


@pytest.fixture(autouse=True)
def _empty_cache():
    autotune.clear()
    yield
    autotune.clear()


def test_bucket_is_rounded_log2():
    b = _lib.lib.tct_tune_bucket
    assert b(0) == 0 and b(1) == 1
    assert b(1000) == b(1400) != b(1500)   # 1448 = 2^10.5 splits the buckets
    assert b(59858) == b(55000)


def test_set_get_and_buckets():
    F = _lib.TCT_TUNE_FARFIELD
    assert autotune.lookup(F, 6, 0, 3, 1, 59858, 59858) is None
    assert _lib.lib.tct_tune_set(F, 6, 0, 3, 1, 59858, 59858, 6, 1) == 0
    assert autotune.lookup(F, 6, 0, 3, 1, 59858, 59858) == (6, 1)
    assert autotune.lookup(F, 6, 0, 3, 1, 60500, 57000) == (6, 1)   # same buckets
    assert autotune.lookup(F, 6, 1, 3, 1, 59858, 59858) is None     # other precision
    assert autotune.lookup(F, 6, 0, 4, 1, 59858, 59858) is None     # other rule
    assert _lib.lib.tct_tune_set(F, 6, 0, 3, 1, 1, 1, 0, 1) == _lib.TCT_ERR_ARG
    assert _lib.lib.tct_tune_set(9, 6, 0, 3, 1, 1, 1, 1, 1) == _lib.TCT_ERR_ARG


def test_save_load_round_trip(tmp_path):
    B = _lib.TCT_TUNE_BSR9
    _lib.lib.tct_tune_set(B, -1, 1, 0, 1, 400000, 1, 4, 16)
    _lib.lib.tct_tune_set(_lib.TCT_TUNE_FARFIELD, 0, 1, 4, 1, 722, 722, 24, 1)
    path = str(tmp_path / "tune.json")
    autotune.save(path)
    doc = json.load(open(path))
    assert len(doc["entries"]) == 2
    autotune.clear()
    assert autotune.entries() == []
    assert autotune.load(path) == 2
    assert autotune.lookup(B, -1, 1, 0, 1, 400000, 1) == (4, 16)
    # entries tuned on another GPU are not restored unless asked
    doc["gpu"] = "another GPU"
    json.dump(doc, open(path, "w"))
    autotune.clear()
    assert autotune.load(path) == 0
    assert autotune.load(path, any_gpu=True) == 2
