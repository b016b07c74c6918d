"""Tensor-core network layers (NNP_PREC_BF16, NNP_PREC_BF16X3) against the
reference's own outputs (tests/golden/*.npz).

Tolerances: BF16X3 (hi*hi + hi*lo + lo*hi, ~16 significant bits, FP32
accumulation) -- 2e-5 eV/atom and 2e-4 eV/A, well inside the north-star
bound of 1 meV/atom and 10 meV/A (measured <= 7e-6 eV/atom, 3.6e-5 eV/A).
BF16 (one BF16 product per MMA) does NOT meet that bound on these inputs
(measured up to 5.4 meV/atom and 20 meV/A: the conditioned network inputs
and the weights each lose ~3 significant digits), so it is tested against
1e-2 eV/atom and 4e-2 eV/A only.  Symmetry functions and the basis
derivatives of the forces stay FP32 in both modes."""
import glob
import os

import numpy as np
import pytest

from ace_b200 import NNP

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
PREC = {"bf16": (1, 1e-2, 4e-2), "bf16x3": (2, 2e-5, 2e-4)}


def run(path, tmp_path, prec):
    z = np.load(path)
    pot_path = str(tmp_path / "pot.nnp")
    with open(pot_path, "wb") as f:
        f.write(z["potential"].tobytes())
    nn = NNP.read(pot_path)
    nn.set_precision(prec)
    off, pbc = z["atom_off"], bool(z["pbc"])
    E, F = nn.compute_batch(off, z["pos"], z["type"], z["cell"], pbc=pbc)
    EV, _ = nn.compute_batch(off, z["pos"], z["type"], z["cell"], pbc=pbc, vacuum=True)
    nn.close()
    nat = np.maximum(np.diff(off), 1)
    e_err = max((np.abs(E - z["energy"]) / nat).max(), (np.abs(EV - z["energy_vacuum"]) / nat).max())
    f_err = np.abs(F - z["forces"]).max()
    return e_err, f_err


@pytest.mark.parametrize("prec", sorted(PREC))
@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_tensor_core_networks_match_reference(path, prec, tmp_path):
    code, e_tol, f_tol = PREC[prec]
    e_err, f_err = run(path, tmp_path, code)
    print("%s %s: E/atom %.2e eV  F %.2e eV/A" % (os.path.basename(path), prec, e_err, f_err))
    assert e_err < e_tol
    assert f_err < f_tol


def test_precision_switch_back_to_fp32(tmp_path):
    """Switching back to FP32 gives the FP32 results again (same handle)."""
    path = [p for p in GOLDEN if p.endswith("config2.npz")][0]
    z = np.load(path)
    pot_path = str(tmp_path / "pot.nnp")
    with open(pot_path, "wb") as f:
        f.write(z["potential"].tobytes())
    nn = NNP.read(pot_path)
    E0, F0 = nn.compute_batch(z["atom_off"], z["pos"], z["type"], z["cell"])
    nn.set_precision(1)
    nn.compute_batch(z["atom_off"], z["pos"], z["type"], z["cell"])
    nn.set_precision(0)
    E1, F1 = nn.compute_batch(z["atom_off"], z["pos"], z["type"], z["cell"])
    nn.close()
    assert np.abs(E1 - E0).max() < 1e-9 and np.abs(F1 - F0).max() < 1e-7
