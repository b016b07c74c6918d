"""Autotuning on the GPU: the first energy+force call with autotuning on
times the candidate launch and tile choices on its own batch, keeps the
fastest, stores them in the cache, and returns the same results as the
default choices (to FP32 summation order); a second handle of the same
potential loads the choices from the cache instead of timing again."""
import numpy as np
import pytest

from ace_b200 import NNP, potential, synth

pytestmark = pytest.mark.gpu


def test_autotune_then_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("NNP_CACHE_DIR", str(tmp_path / "cache"))
    pot = synth.potential_config(2)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    b = synth.config2(seed=5, n_struct=64)
    nn = NNP.read(path)
    _, _, G = nn.compute_batch(b.atom_off[:9], b.pos[:b.atom_off[8]], b.type[:b.atom_off[8]], b.cell[:8], symm=True)
    nn.close()
    synth.condition(pot, G, b.type[:b.atom_off[8]])
    potential.write(path, pot)

    ref = NNP.read(path)
    E0, F0 = ref.compute_batch(b.atom_off, b.pos, b.type, b.cell)
    assert ref.tune_params()[1] == "default"
    ref.close()

    nn = NNP.read(path)
    nn.set_precision(2)
    nn.set_autotune(True)
    E1, F1 = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell)
    choices, source, log = nn.tune_params()
    print(source, choices, log)
    assert source == "tuned" and "ms" in log
    E2, F2 = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell)   # tuned kernels, no second tuning
    assert nn.tune_params()[1] == "tuned"
    nn.close()
    nat = np.diff(b.atom_off)
    for E, F in ((E1, F1), (E2, F2)):
        assert (np.abs(E - E0) / nat).max() < 2e-5       # BF16x3 networks against FP32 ones
        assert np.abs(F - F0).max() < 2e-4

    again = NNP.read(path)
    again.set_precision(2)
    again.set_autotune(True)
    E3, F3 = again.compute_batch(b.atom_off, b.pos, b.type, b.cell)
    c3, s3, _ = again.tune_params()
    again.close()
    assert s3 == "cache" and c3 == choices
    assert np.abs(F3 - F2).max() < 1e-6
