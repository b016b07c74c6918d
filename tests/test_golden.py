"""Golden fixtures written by the reference itself (tests/golden/make_golden.py,
from the reference's own NNP code compiled in oracle/_ref): the FP64 oracle
must reproduce them to rounding, and the potential files must round-trip
byte for byte through the writer.  When oracle/_ref is built, the oracle is
also compared with the live reference on fresh random structures."""
import glob
import os

import numpy as np
import pytest

from ace_b200 import potential, synth
from oracle import oracle as orc
from oracle import ref

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("train_", "large_")))
TOL = 1e-10     # FP64 against FP64: summation order only


def load(path, tmp_path):
    z = np.load(path)
    pot_path = str(tmp_path / "pot.nnp")
    with open(pot_path, "wb") as f:
        f.write(z["potential"].tobytes())
    return z, pot_path


def test_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in GOLDEN}
    assert {"config1", "config2", "config3", "config4", "config5", "small_cells", "free_cluster"} <= names
    assert set(synth.FORM_POTENTIALS) <= names


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_fixture(path, tmp_path):
    z, pot_path = load(path, tmp_path)
    op = orc.OraclePot.from_file(pot_path)
    off = z["atom_off"]
    pbc = bool(z["pbc"])
    for s in range(len(off) - 1):
        a, b = int(off[s]), int(off[s + 1])
        pos, typ, cell = z["pos"][a:b], z["type"][a:b], z["cell"][s]
        e, f, _ = orc.compute(op, pos, typ, cell, pbc=pbc)
        G = orc.compute_symm(op, pos, typ, cell, pbc=pbc)
        ev = orc.compute_energy(op, typ, G)
        n = b - a
        assert abs(e - z["energy"][s]) / n < TOL
        assert abs(ev - z["energy_vacuum"][s]) / n < TOL
        assert np.abs(f - z["forces"][a:b]).max() < TOL
        gs = G.shape[1]
        assert np.abs(G - z["symm"][a:b, :gs]).max() < TOL * max(1.0, np.abs(G).max())


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_potential_file_roundtrip(path, tmp_path):
    """The reference wrote nothing here, but the fixture's file is what
    NNP::write produces for this potential; reading it and writing it again
    must give the same bytes."""
    z, pot_path = load(path, tmp_path)
    pot = potential.read(pot_path)
    out = str(tmp_path / "again.nnp")
    potential.write(out, pot)
    assert open(out, "rb").read() == z["potential"].tobytes()


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref (compiled reference) not built")
@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_oracle_matches_live_reference(k, tmp_path):
    nt = {1: 1, 2: 3, 3: 2, 4: 2, 5: 4}[k]
    rng = np.random.default_rng(900 + k)
    b = synth.config1() if k == 1 else synth.batch_random(900 + k, rng.integers(8, 64, size=3), nt)
    pot = synth.potential_config(k, seed=77 + k)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    op = orc.OraclePot.from_file(path)
    rp = ref.RefNNP(path)
    for s in range(b.n_struct):
        p, t, c = b.structure(s)
        e, f, ev, g = rp.compute(p, t, c, want_symm=True)
        eo, fo, _ = orc.compute(op, p, t, c)
        Go = orc.compute_symm(op, p, t, c)
        assert abs(e - eo) / len(t) < TOL
        assert np.abs(f - fo).max() < TOL
        assert np.abs(g[:, :Go.shape[1]] - Go).max() < TOL * max(1.0, np.abs(Go).max())
    rp.close()
