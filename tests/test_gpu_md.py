"""The molecular-dynamics force call (nnp_compute_md): per-atom energies and
per-structure virials.

Per-atom energies against the FP64 oracle's network energy of every atom
(ANN::fpbp on the oracle's symmetry functions): 2e-6 eV, as the energies of
test_gpu_parity.py.  The virial has no reference counterpart; it is checked
against central finite differences of the oracle's energy under a
homogeneous strain of positions and cell, W_ab = -dE/de_ab (step 1e-5, FP64),
to 2e-4 relative to the largest |W| of the structure (FP32 pair terms summed
over all pairs)."""
import numpy as np
import pytest

from ace_b200 import NNP, potential, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

E_ATOL = 2e-6
W_RTOL = 2e-4


def setup(tmp_path, k, n=4, seed=61):
    nt = {1: 1, 2: 3, 3: 2, 4: 2, 5: 4}[k]
    rng = np.random.default_rng(seed + k)
    b = synth.config1() if k == 1 else synth.batch_random(seed + k, rng.integers(12, 60, size=n), nt)
    pot = synth.potential_config(k)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    op = orc.OraclePot.from_file(path)
    G = np.concatenate([orc.compute_symm(op, *b.structure(s)) for s in range(b.n_struct)])
    synth.condition(pot, G, b.type)
    potential.write(path, pot)
    return b, path


def strained_energy(op, pos, typ, cell, eps):
    M = np.eye(3) + eps
    cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)        # rows = lattice vectors
    e, _, _ = orc.compute(op, pos @ M.T, typ, cell @ M.T)
    return e


@pytest.mark.parametrize("k", [2, 3, 5])
def test_atom_energies_and_virial(tmp_path, k):
    b, path = setup(tmp_path, k)
    op = orc.OraclePot.from_file(path)
    nn = NNP.read(path)
    E, F, A, W = nn.compute_md(b.atom_off, b.pos, b.type, b.cell)
    E0, F0 = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell)
    EV, _, AV, _ = nn.compute_md(b.atom_off, b.pos, b.type, b.cell, vacuum=True)
    nn.close()
    # the MD call gives the same energies and forces as nnp_compute
    assert np.abs(E - E0).max() < 1e-9 and np.abs(F - F0).max() < 1e-9
    pot = potential.read(path)
    vac = {t: pot.types[t].energy for t in range(pot.ntypes)}
    for s in range(b.n_struct):
        p, t, c = b.structure(s)
        a0, a1 = int(b.atom_off[s]), int(b.atom_off[s + 1])
        # per-atom energies against the oracle's network energy of each atom
        G = orc.compute_symm(op, p, t, c)
        ref = np.array([orc.ann_fpbp(op, int(t[i]), G[i])[0] for i in range(len(t))])
        assert np.abs(A[a0:a1] - ref).max() < E_ATOL
        assert np.abs(AV[a0:a1] - (ref + np.array([vac[int(x)] for x in t]))).max() < E_ATOL
        assert abs(A[a0:a1].sum() - E[s]) < 1e-9 * max(1, a1 - a0)
        # virial against finite differences of the strained energy
        h = 1e-5
        Wfd = np.zeros((3, 3))
        for a in range(3):
            for c2 in range(3):
                eps = np.zeros((3, 3))
                eps[a, c2] = h
                Wfd[a, c2] = -(strained_energy(op, p, t, c, eps) - strained_energy(op, p, t, c, -eps)) / (2 * h)
        scale = max(1.0, np.abs(Wfd).max())
        print("config %d structure %d: |W| %.3e, max |W - W_fd| %.2e" % (k, s, np.abs(Wfd).max(), np.abs(W[s] - Wfd).max()))
        assert np.abs(W[s] - Wfd).max() < W_RTOL * scale
        assert np.abs(W[s] - W[s].T).max() < W_RTOL * scale


def test_md_call_errors(tmp_path):
    b, path = setup(tmp_path, 2, n=1)
    nn = NNP.read(path)
    from ace_b200 import nnp as _n
    rc = _n.lib().nnp_compute_md(nn._h, None, None, None, None, None, 0)
    assert rc == -1
    nn.close()
