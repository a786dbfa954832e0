"""The autotuner's choices persist per (device, data shape) in a JSON file
(the reference keeps its fitted switch in the package,
estimate_threshold.py:29-96 and random_forest.py:278-289).  Host only."""
import json

from cudatree_b200 import tune_cache


def test_round_trip_through_the_file(tmp_path, monkeypatch):
    f = tmp_path / "tune.json"
    monkeypatch.setenv(tune_cache.ENV, str(f))
    tune_cache.clear_memory()
    k = tune_cache.key("NVIDIA B200", ("batched", 581012, 54, 7, 7, 4, True, 1))
    opts = {"scan_piece": 2048, "subtree_cutoff": 32, "bfs_threshold": 0, "part_shape": 2, "huge_rows": 16384,
            "sample_trees": 16, "sample_ms": 12.5}
    assert tune_cache.get(k) is None
    tune_cache.put(k, opts)
    tune_cache.clear_memory()  # a new process
    assert tune_cache.get(k) == opts
    data = json.loads(f.read_text())
    assert data["format"] == tune_cache.FORMAT and k in data["entries"]
    other = tune_cache.key("NVIDIA B200", ("batched", 10000, 3000, 100, 55, 2, True, 1))
    tune_cache.put(other, dict(opts, part_shape=1))
    tune_cache.clear_memory()
    assert tune_cache.get(k)["part_shape"] == 2 and tune_cache.get(other)["part_shape"] == 1


def test_corrupt_file_reads_as_empty_and_is_replaced(tmp_path, monkeypatch):
    f = tmp_path / "tune.json"
    f.write_text("{not json")
    monkeypatch.setenv(tune_cache.ENV, str(f))
    tune_cache.clear_memory()
    k = tune_cache.key("dev", ("plain", 1, 2))
    assert tune_cache.get(k) is None
    tune_cache.put(k, {"bfs_threshold": 4000})
    tune_cache.clear_memory()
    assert tune_cache.get(k) == {"bfs_threshold": 4000}


def test_off_keeps_choices_in_the_process(tmp_path, monkeypatch):
    monkeypatch.setenv(tune_cache.ENV, "off")
    tune_cache.clear_memory()
    assert tune_cache.path() is None
    k = tune_cache.key("dev", ("batched", 5))
    tune_cache.put(k, {"scan_piece": 1024})
    assert tune_cache.get(k) == {"scan_piece": 1024}
    tune_cache.clear_memory()
    assert tune_cache.get(k) is None
    assert not any(tmp_path.iterdir())
