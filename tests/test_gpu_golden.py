"""The CUDA path against the reference's own outputs (tests/golden/*.npz,
written by the compiled reference): same potential file, same structures.

Tolerances of the FP32 path, as in test_gpu_parity.py: symmetry functions
2e-5 relative to the atom's largest |G|, energies 2e-6 eV/atom and 1e-6
relative to the total energy with vacuum energies, forces 1e-5 eV/A.
Configuration 1, whose input scaling amplifies the rounding of the
symmetry-function terms (see test_gpu_parity.py), runs with its terms in
FP64 (NNP_SYMM_FP64)."""
import glob
import os

import numpy as np
import pytest

from ace_b200 import NNP

pytestmark = pytest.mark.gpu

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("train_", "large_")))
G_RTOL = 2e-5
E_ATOL = 2e-6
E_RTOL = 1e-6
F_ATOL = 1e-5


@pytest.mark.parametrize("jit", [True, False], ids=["specialised", "generic"])
@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_cuda_matches_reference_fixture(path, jit, tmp_path):
    z = np.load(path)
    pot_path = str(tmp_path / "pot.nnp")
    with open(pot_path, "wb") as f:
        f.write(z["potential"].tobytes())
    nn = NNP.read(pot_path)
    nn.set_specialization(jit)
    if int(z["config"]) == 1:
        nn.set_accumulation(2)          # NNP_SYMM_FP64
    off, pbc = z["atom_off"], bool(z["pbc"])
    E, F, G = nn.compute_batch(off, z["pos"], z["type"], z["cell"], pbc=pbc, symm=True)
    EV, _ = nn.compute_batch(off, z["pos"], z["type"], z["cell"], pbc=pbc, vacuum=True)
    nn.close()
    nat = np.maximum(np.diff(off), 1)
    Gr = z["symm"]
    gs = Gr.shape[1]
    scale = np.maximum(np.abs(Gr).max(axis=1, keepdims=True), 1e-30)
    g_err = (np.abs(G[:, :gs] - Gr) / scale).max()
    e_err = (np.abs(E - z["energy"]) / nat).max()
    ev_err = (np.abs(EV - z["energy_vacuum"]) / nat).max()
    f_err = np.abs(F - z["forces"]).max()
    e_rel = (np.abs(EV - z["energy_vacuum"]) / np.abs(z["energy_vacuum"])).max()
    print("%s: G rel %.2e  E/atom %.2e  E+vac/atom %.2e  E rel %.2e  F %.2e" %
          (os.path.basename(path), g_err, e_err, ev_err, e_rel, f_err))
    assert g_err < G_RTOL
    assert e_err < E_ATOL and ev_err < E_ATOL
    assert e_rel < E_RTOL
    assert f_err < F_ATOL
