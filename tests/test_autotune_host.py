"""Autotuner bookkeeping that needs no GPU: the cache file and the shape
validation of the tile settings it applies."""

import json

import pytest

from qforte_b200 import autotune
from qforte_b200._lib import check, lib
from qforte_b200.device import gates_config


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("QFB_TUNE_CACHE", str(tmp_path / "t.json"))
    autotune._store(autotune.gate_key(28), [11, 4, 3])
    autotune._store("ucc:n=20:nparam=875:batch=64", [12, 11, 3])
    d = json.loads((tmp_path / "t.json").read_text())
    assert d["gates:n=28"] == [11, 4, 3] and d["ucc:n=20:nparam=875:batch=64"] == [12, 11, 3]
    try:
        assert autotune.apply_cached(nqubit=28) == {"gates": (11, 4, 3)}
    finally:
        gates_config(0, 3)
    assert autotune.apply_cached(nqubit=30) == {}


def test_window_tile_validation():
    assert lib().qfb_ucc_tiles(12, 11, 3) == 0
    for bad in ((14, 11, 3), (12, 13, 3), (4, 11, 3), (12, 11, 7)):
        with pytest.raises(ValueError):
            check(lib().qfb_ucc_tiles(*bad), "qfb_ucc_tiles")
    assert lib().qfb_ucc_tiles(12, 11, 3) == 0
