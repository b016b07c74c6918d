"""The autotuner's cache and key logic on the host (no GPU): the key names
the potential, the network shapes, the GPU model and the neighbour-capacity
class; stored choices round-trip; the last entry of a key wins; malformed
lines and invalid choices are rejected."""
import os

import pytest

from ace_b200 import NNPError, nnp, potential, synth

CHOICES = {"symm_minb": 3, "force_minb": 2, "force_unroll": 2, "force_chunk": 192, "tc_per_sm": 2}


@pytest.fixture
def cache(tmp_path, monkeypatch):
    d = tmp_path / "cache"
    monkeypatch.setenv("NNP_CACHE_DIR", str(d))
    return d


def pot_file(tmp_path, k, seed=1234, name="p"):
    path = str(tmp_path / ("%s%d_%d.nnp" % (name, k, seed)))
    potential.write(path, synth.potential_config(k, seed=seed))
    return path


def test_key_names_potential_gpu_and_capacity_class(tmp_path, cache):
    p2 = pot_file(tmp_path, 2)
    k = nnp.tune_cache_key(p2, "NVIDIA B200", 148, 96)
    assert k == nnp.tune_cache_key(p2, "NVIDIA B200", 148, 96)            # stable
    assert k == nnp.tune_cache_key(p2, "NVIDIA B200", 148, 128)           # same class (65..128 slots)
    assert k != nnp.tune_cache_key(p2, "NVIDIA B200", 148, 136)           # next class
    assert k != nnp.tune_cache_key(p2, "NVIDIA H100", 132, 96)            # another GPU
    assert k != nnp.tune_cache_key(pot_file(tmp_path, 5), "NVIDIA B200", 148, 96)   # another basis
    # the same basis with other network weights shares the key (the kernels are the same)
    assert k == nnp.tune_cache_key(pot_file(tmp_path, 2, seed=99), "NVIDIA B200", 148, 96)
    assert "NVIDIA_B200" in k and k.endswith(":cap128")


def test_store_load_roundtrip_and_last_entry_wins(tmp_path, cache):
    key = nnp.tune_cache_key(pot_file(tmp_path, 3), "NVIDIA B200", 148, 100)
    assert nnp.tune_cache_load(key) is None
    nnp.tune_cache_store(key, CHOICES)
    assert nnp.tune_cache_load(key) == CHOICES
    later = dict(CHOICES, force_chunk=288)
    nnp.tune_cache_store(key, later)
    assert nnp.tune_cache_load(key) == later
    assert nnp.tune_cache_load(key + "x") is None
    assert os.path.exists(cache / "tuning.txt")


def test_malformed_lines_and_invalid_choices(tmp_path, cache):
    key = nnp.tune_cache_key(pot_file(tmp_path, 3), "NVIDIA B200", 148, 100)
    nnp.tune_cache_store(key, CHOICES)
    with open(cache / "tuning.txt", "a") as f:
        f.write(key + " symm_minb=9 force_minb=1 force_unroll=1 force_chunk=288 tc_per_sm=0\n")   # out of range
        f.write(key + " garbage\n")
        f.write(key + "\n")
    assert nnp.tune_cache_load(key) == CHOICES
    with pytest.raises(NNPError):
        nnp.tune_cache_store(key, dict(CHOICES, force_chunk=4096))
