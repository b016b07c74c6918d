"""Tensor-core network layers (NNP_PREC_BF16, NNP_PREC_BF16X3) against the
reference's own outputs (tests/golden/*.npz).

Tolerances: BF16X3 (hi*hi + hi*lo + lo*hi, ~16 significant bits, FP32
accumulation) -- 2e-5 eV/atom and 2e-4 eV/A, well inside the bound of
1 meV/atom and 10 meV/A that the tensor-core networks are held to (measured
<= 7e-6 eV/atom, 3.6e-5 eV/A).
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

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("train_", "large_")))
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


def test_bf16x3_many_tiles_four_elements(tmp_path):
    """Config-5 potential (4 elements, 64-48-48-1) on 400 structures of its
    stream (~150 k atoms): the tensor-core kernel's CTAs run several tiles and
    restage weights and per-element vectors when the element changes.  BF16X3
    against the FP32 networks on the same handle, every call of three: the
    BF16X3 rounding is ~5e-5 eV/A on these forces (measured), bounded here by
    5e-4 eV/A and 5e-5 eV/atom."""
    from ace_b200 import potential, synth
    pot = synth.potential_config(5, seed=1234)
    path = str(tmp_path / "pot5.nnp")
    potential.write(path, pot)
    full = synth.config5(n_struct=400)
    nn = NNP.read(path)
    _, _, G = nn.compute_batch(full.atom_off[:33] - 0, full.pos[:full.atom_off[32]], full.type[:full.atom_off[32]],
                               full.cell[:32], symm=True)
    nn.close()
    synth.condition(pot, G, full.type[:full.atom_off[32]])
    potential.write(path, pot)
    nn = NNP.read(path)
    E0, F0 = nn.compute_batch(full.atom_off, full.pos, full.type, full.cell)
    nn.set_precision(2)
    nat = np.maximum(np.diff(full.atom_off), 1)
    for _ in range(3):
        E1, F1 = nn.compute_batch(full.atom_off, full.pos, full.type, full.cell)
        assert (np.abs(E1 - E0) / nat).max() < 5e-5
        assert np.abs(F1 - F0).max() < 5e-4
    nn.close()


def test_mma_wait_timeout_returns_error_and_handle_recovers(tmp_path):
    """A tensor-core wait that runs out ends the call with NNP_ERR_CUDA, not a
    hang: with a bound of one barrier test per MMA chain every wait gives up
    (a chain takes far longer than one test), the block leaves its tile loop
    as one, drains the chain in flight and frees its tensor memory.  The same
    handle then gives the reference's results with the default bound."""
    from ace_b200 import NNPError
    from ace_b200.nnp import ERRORS
    path = [p for p in GOLDEN if p.endswith("config2.npz")][0]
    z = np.load(path)
    pot_path = str(tmp_path / "pot.nnp")
    with open(pot_path, "wb") as f:
        f.write(z["potential"].tobytes())
    nn = NNP.read(pot_path)
    nn.set_precision(2)
    nn.set_mma_wait(1)
    for _ in range(2):
        with pytest.raises(NNPError) as ei:
            nn.compute_batch(z["atom_off"], z["pos"], z["type"], z["cell"])
        assert ERRORS[ei.value.code] == "CUDA" and "timed out" in str(ei.value)
    nn.set_mma_wait(0)
    E, F = nn.compute_batch(z["atom_off"], z["pos"], z["type"], z["cell"])
    nn.close()
    nat = np.maximum(np.diff(z["atom_off"]), 1)
    assert (np.abs(E - z["energy"]) / nat).max() < PREC["bf16x3"][1]
    assert np.abs(F - z["forces"]).max() < PREC["bf16x3"][2]
