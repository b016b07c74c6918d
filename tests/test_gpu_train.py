"""Weight gradient of the energy(+force) loss on the GPU (nnp_train_grad)
against the FP64 oracle (orc_ef_loss_grad, whose energy term follows
NNPTEFR::error_cost_o1 and is checked against finite differences in
test_oracle.py).

Training configuration 3: two elements, 48-32-32-1 tanh networks; labels from
a teacher potential of the same architecture (different seed) plus Gaussian
noise (1 meV/atom on energies, 20 meV/A on forces).

Tolerances (FP32 device arithmetic, FP64 sums across blocks): loss 1e-5
relative; gradient 1e-3 relative in the L2 norm and 1e-3 of the largest
component elementwise."""
import numpy as np
import pytest

from ace_b200 import NNP, NNPError, potential, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

L_RTOL = 1e-5
G_RTOL = 1e-3


def setup(tmp_path, n=6, seed=31):
    rng = np.random.default_rng(seed)
    b = synth.batch_random(seed, rng.integers(16, 64, size=n), 2)
    pot = synth.potential_config(3, seed=5)
    teacher = synth.potential_config(3, seed=6)
    paths = {}
    for name, p in (("model", pot), ("teacher", teacher)):
        path = str(tmp_path / (name + ".nnp"))
        potential.write(path, p)
        op = orc.OraclePot.from_file(path)
        G = np.concatenate([orc.compute_symm(op, *b.structure(s)) for s in range(b.n_struct)])
        synth.condition(p, G, b.type)
        potential.write(path, p)
        paths[name] = path
    tp = orc.OraclePot.from_file(paths["teacher"])
    E_t, F_t = orc.compute_batch(tp, b)
    nat = np.diff(b.atom_off)
    e_ref = E_t + rng.normal(0, 1e-3, size=b.n_struct) * nat
    f_ref = F_t + rng.normal(0, 0.02, size=F_t.shape)
    return b, paths["model"], e_ref, f_ref


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("w_f", [0.0, 0.5])
@pytest.mark.parametrize("jit", [True, False], ids=["specialised", "generic"])
def test_train_grad_matches_oracle(tmp_path, w_f, jit):
    b, path, e_ref, f_ref = setup(tmp_path)
    op = orc.OraclePot.from_file(path)
    nn = NNP.read(path)
    nn.set_specialization(jit)
    L, g, eo, fo = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, w_f, norm_mode=1)
    Lo, go, eoo, foo = orc.ef_loss_grad(op, b, e_ref, f_ref, w_f, norm_mode=1)
    nn.close()
    print("w_f %.1f: loss %.6e vs %.6e, grad rel L2 %.2e, max %.2e" %
          (w_f, L, Lo, rel(g, go), np.abs(g - go).max() / np.abs(go).max()))
    assert abs(L - Lo) <= L_RTOL * abs(Lo)
    assert rel(g, go) < G_RTOL
    assert np.abs(g - go).max() < G_RTOL * np.abs(go).max()
    assert np.abs(fo - foo).max() < 1e-5


@pytest.mark.parametrize("norm_mode", [0, 1, 2, 3, 4])
def test_energy_loss_norm_modes(tmp_path, norm_mode):
    """Energy-only loss for every nnptefr norm (IDENTITY, LINEAR, SQRT, CBRT,
    LOG) against orc_energy_loss_grad on the oracle's symmetry functions."""
    b, path, e_ref, f_ref = setup(tmp_path, n=4, seed=41)
    op = orc.OraclePot.from_file(path)
    G = np.concatenate([orc.compute_symm(op, *b.structure(s)) for s in range(b.n_struct)])
    Lo, go = orc.energy_loss_grad(op, b.atom_off, b.type, G, e_ref, norm_mode)
    nn = NNP.read(path)
    L, g, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, 0.0, norm_mode=norm_mode)
    nn.close()
    assert abs(L - Lo) <= L_RTOL * abs(Lo)
    assert rel(g, go) < G_RTOL


def test_train_grad_errors(tmp_path):
    b, path, e_ref, f_ref = setup(tmp_path, n=2, seed=51)
    nn = NNP.read(path)
    with pytest.raises(NNPError):
        nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, 0.5, norm_mode=9)
    with pytest.raises(NNPError):
        nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, -1.0)
    nn.close()
