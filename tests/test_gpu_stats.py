"""Input statistics and preconditioning (nnp_input_stats, nnp_precondition)
against nnptefr's formulas (nnptefr.cpp:689-880) evaluated in FP64 on the
reference's own symmetry functions (the golden fixtures' rows).

Tolerances: with the symmetry functions evaluated in FP64 (NNP_SYMM_FP64,
rows stored as FP32) every statistic agrees to 1e-6 relative to the
largest magnitude of that input over the batch (the FP32 storage of the
rows); with FP32 terms to 1e-5.  The harmonic mean N / sum(1/G) is held
relative to itself: it is set by the smallest values of G, whose FP32
relative error is the largest, so 1e-5 with FP64 terms and 1e-4 with FP32
terms (measured 1.5e-5)."""
import os

import numpy as np
import pytest

from ace_b200 import NNP, NNPError, potential
from ace_b200.nnp import STATS

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def reference_stats(G, types, pot):
    """nnptefr.cpp:689-781 on FP64 rows: per element count, max, min,
    harmonic mean, mean, sample standard deviation, rms."""
    out = {}
    for t in range(pot.ntypes):
        g = G[types == t, :pot.n_input(t)]
        n = len(g)
        avg = g.sum(0) / n
        with np.errstate(divide="ignore"):
            har = n / (1.0 / g).sum(0)
        out[t] = {"count": n, "max": g.max(0), "min": g.min(0), "harmonic": har, "mean": avg,
                  "dev": np.sqrt(((avg - g) ** 2).sum(0) / (n - 1.0)), "rms": np.sqrt((g * g).sum(0) / n)}
    return out


def load(name, tmp_path):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    path = str(tmp_path / "pot.nnp")
    with open(path, "wb") as f:
        f.write(z["potential"].tobytes())
    return z, path


@pytest.mark.parametrize("acc,tol", [(2, 1e-6), (0, 1e-5)], ids=["fp64-terms", "fp32-terms"])
@pytest.mark.parametrize("name", ["config2", "config5", "forms_sech_gauss2"])
def test_input_stats_match_reference_formulas(tmp_path, name, acc, tol):
    z, path = load(name, tmp_path)
    pot = potential.read(path)
    ref = reference_stats(z["symm"], z["type"], pot)
    nn = NNP.read(path)
    nn.set_accumulation(acc)
    cnt, st = nn.input_stats(z["atom_off"], z["pos"], z["type"], z["cell"])
    nn.close()
    for t in range(pot.ntypes):
        assert cnt[t] == ref[t]["count"]
        nin = pot.n_input(t)
        scale = np.maximum(np.abs(ref[t]["max"]), np.abs(ref[t]["min"]))
        for s in STATS:
            got, want = st[s][t, :nin], ref[t][s]
            if s == "harmonic":
                err = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
                assert err.max() < (1e-5 if acc == 2 else 1e-4), (t, s, err.max())
            else:
                err = np.abs(got - want) / np.maximum(scale, 1e-300)
                assert err.max() < tol, (t, s, err.max())


@pytest.mark.parametrize("prebias,prescale", [("MEAN", "DEV"), ("MID", "MINMAX"), ("HAR", "MAX"),
                                              ("RMS", "IDENTITY"), ("MIN", "DEV"), ("IDENTITY", "MINMAX")])
def test_precondition_sets_input_bias_and_scale(tmp_path, prebias, prescale):
    z, path = load("config3", tmp_path)
    pot = potential.read(path)
    ref = reference_stats(z["symm"], z["type"], pot)
    nn = NNP.read(path)
    nn.set_accumulation(2)
    nn.precondition(z["atom_off"], z["pos"], z["type"], z["cell"], prebias, prescale, inbias=0.25, inscale=2.0)
    out = str(tmp_path / "cond.nnp")
    nn.write(out)
    nn.close()
    got = potential.read(out)
    for t in range(pot.ntypes):
        r = ref[t]
        b = {"MEAN": -r["mean"], "HAR": -r["harmonic"], "RMS": -r["rms"], "MID": -0.5 * (r["max"] + r["min"]),
             "MIN": -r["min"], "IDENTITY": np.zeros_like(r["mean"])}[prebias] + 0.25
        if prescale == "DEV":
            w = np.where(r["dev"] == 0, 1.0, 1.0 / np.where(r["dev"] == 0, 1.0, r["dev"]))
        elif prescale == "MINMAX":
            d = r["max"] - r["min"]
            w = np.where(d > 0, 1.0 / np.where(d > 0, d, 1.0), 1.0)
        elif prescale == "MAX":
            w = np.where(r["max"] > 0, 1.0 / np.where(r["max"] > 0, r["max"], 1.0), 1.0)
        else:
            w = np.ones_like(r["mean"])
        w = 2.0 * w
        net = got.nets[t]
        scale = np.maximum(np.abs(r["max"]), np.abs(r["min"]))
        assert np.all(np.abs(net.inpb - b) <= 1e-6 * np.maximum(scale, 1.0) + 1e-12)
        assert np.all(np.abs(net.inpw - w) <= 1e-5 * np.abs(w))
        assert np.all(net.outb == 0) and np.all(net.outw == 1)


def test_precondition_rejects_none(tmp_path):
    z, path = load("config3", tmp_path)
    nn = NNP.read(path)
    with pytest.raises(NNPError, match="Invalid input bias"):
        nn.precondition(z["atom_off"], z["pos"], z["type"], z["cell"], 6, "DEV")
    with pytest.raises(NNPError, match="Invalid input scaling"):
        nn.precondition(z["atom_off"], z["pos"], z["type"], z["cell"], "MEAN", 4)
    nn.close()
