"""Autotuner host logic (CPU only): the native settings table (keying,
wildcard n_rhs entries, validation), the on-disk cache (persistence, keying by
device model, replacement) and the mapping of the reference's block_dim /
block_size arguments onto launch settings."""
import json

import pytest
import torch

from socu_b200 import _lib, autotune
from socu_b200.block_tridiag_solver import _settings


@pytest.fixture(autouse=True)
def clean_table():
    lib = _lib.load()
    lib.socu_tuning_clear()
    yield
    lib.socu_tuning_clear()


def test_table_exact_and_wildcard_entries():
    autotune.install(torch.float32, 64, 0, {"node_threads": 128, "sweep_tensor_cores": 2})
    autotune.install(torch.float32, 64, 8, {"sweep_threads": 256})
    # exact entry on top of the wildcard one
    assert autotune.current_settings(torch.float32, 64, 8) == {
        "node_threads": 128, "update_threads": 0, "sweep_threads": 256, "sweep_tensor_cores": 2,
        "update_tile": 0, "ragged_units": 0, "update_tensor_cores": 0, "node_tensor_cores": 0}
    # other n_rhs: wildcard only
    assert autotune.current_settings(torch.float32, 64, 3)["node_threads"] == 128
    assert autotune.current_settings(torch.float32, 64, 3)["sweep_threads"] == 0
    # other dtype / n: nothing
    assert not any(autotune.current_settings(torch.float64, 64, 8).values())
    assert not any(autotune.current_settings(torch.float32, 32, 8).values())
    # replace, then remove
    autotune.install(torch.float32, 64, 8, {"sweep_threads": 64})
    assert autotune.current_settings(torch.float32, 64, 8)["sweep_threads"] == 64
    autotune.install(torch.float32, 64, 8, None)
    assert autotune.current_settings(torch.float32, 64, 8)["sweep_threads"] == 0


@pytest.mark.parametrize("bad", [{"node_threads": 96}, {"update_tile": 8}, {"sweep_tensor_cores": 3},
                                 {"ragged_units": 65}, {"sweep_threads": 512}, {"update_tensor_cores": 3},
                                 {"node_tensor_cores": 5}])
def test_table_rejects_invalid_settings(bad):
    with pytest.raises(RuntimeError):
        autotune.install(torch.float64, 16, 1, bad)


def test_cache_persists_and_is_keyed_by_device(tmp_path):
    path = tmp_path / "tune.json"
    autotune.save_entry("NVIDIA B200", torch.float64, 64, 8, {"node_threads": 256}, 0.7, (1, 1024), path=path)
    autotune.save_entry("NVIDIA B200", torch.float32, 64, 8, {"sweep_tensor_cores": 1}, 0.4, (1, 1024), path=path)
    autotune.save_entry("Other GPU", torch.float64, 64, 8, {"node_threads": 64}, 1.0, (1, 1024), path=path)
    # replacing an entry keeps one per key
    autotune.save_entry("NVIDIA B200", torch.float64, 64, 8, {"node_threads": 128}, 0.6, (1, 1024), path=path)
    data = json.loads(path.read_text())
    assert data["version"] == 1 and len(data["entries"]) == 3
    assert autotune.load_cache(path=path, device_name="NVIDIA B200") == 2
    assert autotune.current_settings(torch.float64, 64, 8)["node_threads"] == 128
    assert autotune.current_settings(torch.float32, 64, 8)["sweep_tensor_cores"] == 1
    # read once per (file, device)
    assert autotune.load_cache(path=path, device_name="NVIDIA B200") == 0


def test_corrupt_cache_is_ignored(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text("{not json")
    assert autotune.load_cache(path=path, device_name="NVIDIA B200") == 0
    autotune.save_entry("NVIDIA B200", torch.float64, 16, 1, {}, 0.1, (1, 64), path=path)
    assert len(json.loads(path.read_text())["entries"]) == 1


def test_candidates_cover_the_knobs_that_matter():
    c = autotune.candidates(64, 8, torch.float32)
    assert "sweep_tensor_cores" in c and "update_tile" not in c
    c = autotune.candidates(128, 32, torch.float64)
    assert "update_tile" in c and "sweep_tensor_cores" not in c
    for vals in c.values():
        assert vals[0] == 0    # the built-in heuristic is always a candidate


def test_block_dim_and_block_size_map_to_settings():
    assert _settings(None, None) is None
    assert _settings(64, None) == {"node_threads": 64, "update_threads": 64, "sweep_threads": 64}
    assert _settings(100, None)["node_threads"] == 128
    assert _settings(1024, None)["sweep_threads"] == 256
    assert _settings(None, 16) == {"update_tile": 16}
    assert _settings(None, 32) == {"update_tile": 32}
    with pytest.raises(AssertionError):
        _settings(0, None)
