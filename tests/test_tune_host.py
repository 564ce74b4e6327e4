"""The autotuner's process-wide cache through the C ABI (host only: no GPU needed)."""
import pytest

import elsa_b200
from elsa_b200 import _capi


@pytest.fixture(autouse=True)
def _empty_cache():
    elsa_b200.tune_cache_clear()
    yield
    elsa_b200.tune_cache_clear()


def test_put_get_size_clear():
    assert elsa_b200.tune_cache_size() == 0
    assert elsa_b200.tune_cache_get("0:3:64,64,64:96,96,60") is None
    elsa_b200.tune_cache_put("0:3:64,64,64:96,96,60", [-1, 16, -1, 0, -1, -1])
    elsa_b200.tune_cache_put("1:2:128,128,1:182,1,180", [256, 32, -1, 1, -1, -1])
    assert elsa_b200.tune_cache_size() == 2
    assert elsa_b200.tune_cache_get("0:3:64,64,64:96,96,60") == [-1, 16, -1, 0, -1, -1]
    elsa_b200.tune_cache_put("0:3:64,64,64:96,96,60", [-1, 8, -1, 0, -1, -1])  # replaces
    assert elsa_b200.tune_cache_get("0:3:64,64,64:96,96,60") == [-1, 8, -1, 0, -1, -1]
    assert elsa_b200.tune_cache_size() == 2
    elsa_b200.tune_cache_clear()
    assert elsa_b200.tune_cache_size() == 0


def test_save_load_round_trip(tmp_path):
    entries = {"0:3:64,64,64:96,96,60": [-1, 16, -1, 0, -1, -1], "2:3:128,128,128:192,192,180": [-1, -1, 128, -1, 0, -1],
               "1:2:128,128,1:182,1,180": [512, 64, -1, 1, -1, -1]}
    for k, v in entries.items():
        elsa_b200.tune_cache_put(k, v)
    path = tmp_path / "tune.txt"
    elsa_b200.tune_cache_save(str(path))
    lines = path.read_text().splitlines()
    assert len(lines) == 3 and all(len(line.split()) == 1 + _capi.KNOB_COUNT for line in lines)
    elsa_b200.tune_cache_clear()
    elsa_b200.tune_cache_load(str(path))
    assert elsa_b200.tune_cache_size() == 3
    for k, v in entries.items():
        assert elsa_b200.tune_cache_get(k) == v


def test_malformed_file_changes_nothing(tmp_path):
    elsa_b200.tune_cache_put("0:3:32,32,32:48,48,24", [-1, 4, -1, 0, -1, -1])
    bad = tmp_path / "bad.txt"
    bad.write_text("0:3:64,64,64:96,96,60 -1 16 -1 0 -1 -1\n0:3:8,8,8:8,8,8 -1 x -1 0 -1 -1\n")
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.tune_cache_load(str(bad))
    assert elsa_b200.tune_cache_size() == 1
    assert elsa_b200.tune_cache_get("0:3:64,64,64:96,96,60") is None
    bad.write_text("0:3:64,64,64:96,96,60 -1 16 -1 0 -1 -1 7\n")  # one value too many
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.tune_cache_load(str(bad))
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.tune_cache_load(str(tmp_path / "missing.txt"))


def test_invalid_entries_rejected():
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.tune_cache_put("has space", [1, 1, 1, 0, 0, -1])
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.tune_cache_put("", [1, 1, 1, 0, 0, -1])
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.tune_cache_put("k", [1, -2, 1, 0, 0, -1])
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.tune_cache_put("k", [1, 1])
    assert elsa_b200.tune_cache_size() == 0
