"""Training gradients against the reference's own analytic gradient
(tests/golden/train_config3.npz, written by tests/golden/make_golden.py from
the reference code compiled in oracle/_ref).

Energy term: the reference's ANN::fpbp + NN::Cost::grad per atom
(ml/nn.cpp:1402-1420, 1747-1805) on its own NNP::compute_symm, accumulated
with NNPTEFR::error_cost_o1's loss factor (nnptefr.cpp:1292-1380) for every
norm mode and loss kind, averaged over the batch (nnptefr.cpp:996-1000).
Force term: the reference's NN::D2ODZDI (ml/nn.cpp:2047-2137) contracted
with the change of its compute_symm along the force adjoint (central
differences).  The FP64 oracle must reproduce both; the CUDA path is held to
the same fixture in tests/test_gpu_train.py."""
import os

import numpy as np
import pytest

from ace_b200 import synth
from oracle import oracle as orc
from oracle import ref

FIX = os.path.join(os.path.dirname(__file__), "golden", "train_config3.npz")
E_TOL = 1e-10   # FP64 against FP64, same algorithm: summation order only
F_TOL = 1e-8    # force term: the fixture's tangent is a central difference (error ~1e-10 relative)


def load(tmp_path):
    z = np.load(FIX)
    paths = {}
    for k in ("potential_e", "potential_f"):
        p = str(tmp_path / (k + ".nnp"))
        with open(p, "wb") as f:
            f.write(z[k].tobytes())
        paths[k] = p
    b = synth.Batch(z["atom_off"], z["pos"], z["type"], z["cell"].reshape(-1, 3, 3), True)
    return z, paths, b


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_energy_loss_grad_matches_reference(tmp_path):
    z, paths, b = load(tmp_path)
    op = orc.OraclePot.from_file(paths["potential_e"])
    G = np.concatenate([orc.compute_symm(op, *b.structure(s)) for s in range(b.n_struct)])
    for c, (nm, kind, delta) in enumerate(z["cases"]):
        L, g = orc.energy_loss_grad(op, b.atom_off, b.type, G, z["e_ref"], int(nm), int(kind), float(delta))
        assert abs(L - z["loss_e"][c]) <= E_TOL * abs(z["loss_e"][c]), (nm, kind)
        assert np.abs(g - z["grad_e"][c]).max() <= E_TOL * np.abs(z["grad_e"][c]).max(), (nm, kind)


def test_energy_force_loss_grad_matches_reference(tmp_path):
    z, paths, b = load(tmp_path)
    op = orc.OraclePot.from_file(paths["potential_f"])
    L, g, _, _ = orc.ef_loss_grad(op, b, z["e_ref"], z["f_ref"], float(z["w_f"]), norm_mode=1)
    assert abs(L - z["loss_ef"]) <= E_TOL * abs(z["loss_ef"])
    assert rel(g, z["grad_ef"]) < F_TOL
    # the force term is a sizeable part of the gradient (the check is not the energy term alone)
    Le, ge = orc.energy_loss_grad(op, b.atom_off, b.type,
                                  np.concatenate([orc.compute_symm(op, *b.structure(s)) for s in range(b.n_struct)]),
                                  z["e_ref"], 1)
    assert rel(ge, z["grad_ef"]) > 1e-2


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref (compiled reference) not built")
def test_live_reference_reproduces_fixture(tmp_path):
    """The compiled reference still gives the stored energy-loss gradients."""
    z, paths, b = load(tmp_path)
    rp = ref.RefNNP(paths["potential_e"])
    for c, (nm, kind, delta) in enumerate(z["cases"]):
        L, g, _, _ = rp.energy_loss_grad(b, z["e_ref"], int(nm), int(kind), float(delta))
        assert abs(L - z["loss_e"][c]) <= 1e-14 * abs(z["loss_e"][c])
        assert np.abs(g - z["grad_e"][c]).max() <= 1e-14 * np.abs(z["grad_e"][c]).max()
    rp.close()
