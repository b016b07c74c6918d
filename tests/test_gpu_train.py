"""Weight gradient of the energy(+force) loss on the GPU (nnp_train_grad)
against the reference's own analytic gradient (tests/golden/train_config3.npz:
ANN::fpbp + Cost::grad with error_cost_o1's loss factors for the energy term,
D2ODZDI contracted with dG/dr for the force term) and against the FP64
oracle (orc_ef_loss_grad, which reproduces that fixture, tests/
test_train_golden.py, and finite differences, test_oracle.py).

Training configuration 3: two elements, 48-32-32-1 tanh networks; labels from
a teacher potential of the same architecture (different seed) plus Gaussian
noise (1 meV/atom on energies, 20 meV/A on forces).

Tolerances (FP32 device arithmetic, FP64 sums across blocks): loss 1e-5
relative; gradient 1e-3 relative in the L2 norm and 1e-3 of the largest
component elementwise."""
import os

import numpy as np
import pytest

from ace_b200 import NNP, NNPError, potential, synth
from ace_b200.nnp import LOSS_MSE
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


def load_fixture(tmp_path):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "train_config3.npz"))
    paths = {}
    for k in ("potential_e", "potential_f"):
        p = str(tmp_path / (k + ".nnp"))
        with open(p, "wb") as f:
            f.write(z[k].tobytes())
        paths[k] = p
    b = synth.Batch(z["atom_off"], z["pos"], z["type"], z["cell"].reshape(-1, 3, 3), True)
    return z, paths, b


@pytest.mark.parametrize("jit", [True, False], ids=["specialised", "generic"])
def test_energy_loss_grad_matches_reference_gradient(tmp_path, jit):
    """Every norm mode and loss kind (MSE, MAE, HUBER, ASINH) against the
    reference's Cost::grad / error_cost_o1 gradient of the fixture."""
    z, paths, b = load_fixture(tmp_path)
    nn = NNP.read(paths["potential_e"])
    nn.set_specialization(jit)
    f0 = np.zeros((b.n_atoms, 3))
    for c, (nm, kind, delta) in enumerate(z["cases"]):
        nn.set_loss(int(kind), float(delta))
        L, g, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, z["e_ref"], f0, 0.0, norm_mode=int(nm))
        gr = z["grad_e"][c]
        print("norm %d loss %d: loss %.6e vs %.6e, grad rel L2 %.2e" % (nm, kind, L, z["loss_e"][c], rel(g, gr)))
        assert abs(L - z["loss_e"][c]) <= L_RTOL * abs(z["loss_e"][c])
        assert rel(g, gr) < G_RTOL
        assert np.abs(g - gr).max() < G_RTOL * np.abs(gr).max()
    nn.set_loss(LOSS_MSE)
    nn.close()


@pytest.mark.parametrize("jit", [True, False], ids=["specialised", "generic"])
def test_energy_force_loss_grad_matches_reference_gradient(tmp_path, jit):
    """Energy + force loss (w_f = 0.5) against the reference's gradient: its
    Cost::grad energy term plus its D2ODZDI force term."""
    z, paths, b = load_fixture(tmp_path)
    nn = NNP.read(paths["potential_f"])
    nn.set_specialization(jit)
    L, g, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, z["e_ref"], z["f_ref"], float(z["w_f"]),
                               norm_mode=1)
    nn.close()
    gr = z["grad_ef"]
    print("loss %.6e vs %.6e, grad rel L2 %.2e, max %.2e" %
          (L, float(z["loss_ef"]), rel(g, gr), np.abs(g - gr).max() / np.abs(gr).max()))
    assert abs(L - float(z["loss_ef"])) <= L_RTOL * abs(float(z["loss_ef"]))
    assert rel(g, gr) < G_RTOL
    assert np.abs(g - gr).max() < G_RTOL * np.abs(gr).max()


def test_set_loss_errors(tmp_path):
    z, paths, b = load_fixture(tmp_path)
    nn = NNP.read(paths["potential_e"])
    with pytest.raises(NNPError):
        nn.set_loss(0)
    with pytest.raises(NNPError):
        nn.set_loss(3, 0.0)
    nn.close()


def adam_reference(p, g, m, v, t, gamma, eps=1e-16):
    """opt::algo::ADAM::step (opt/algo.cpp:280-296), step t = 1, 2, ..."""
    b1, b2 = 0.9, 0.999
    m = m * b1 + (1.0 - b1) * g
    v = v * b2 + (1.0 - b2) * g * g
    b1ii, b2ii = 1.0 / (1.0 - b1 ** t), 1.0 / (1.0 - b2 ** t)
    return p - gamma * b1ii * m / (np.sqrt(b2ii * v) + eps), m, v


def test_adam_on_device_matches_reference_step(tmp_path):
    """Three device ADAM steps equal the reference's step formula applied to
    the same gradients, and the host model follows the device parameters."""
    b, path, e_ref, f_ref = setup(tmp_path, n=4, seed=61)
    nn = NNP.read(path)
    p = nn.get_params()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for t in range(1, 4):
        _, g, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, 0.5, norm_mode=1)
        nn.opt_adam(1e-3)
        p, m, v = adam_reference(p, g, m, v, t, 1e-3)
        assert np.abs(nn.get_params() - p).max() <= 1e-12 * np.abs(p).max()
    with pytest.raises(NNPError):
        nn.opt_adam(1e-3)                       # the gradient was used
    nn.close()


def test_device_training_loop_reduces_loss(tmp_path):
    """train_grad + opt_adam on the device for 30 steps: the energy+force
    loss of configuration 3's batch falls."""
    b, path, e_ref, f_ref = setup(tmp_path, n=6, seed=71)
    nn = NNP.read(path)
    losses = []
    for _ in range(30):
        L, _, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, 0.5, norm_mode=1)
        losses.append(L)
        nn.opt_adam(2e-3)
    nn.close()
    print("loss %.4e -> %.4e" % (losses[0], losses[-1]))
    assert losses[-1] < 0.5 * losses[0]


@pytest.mark.parametrize("reg", ["NONE", "LASSO", "RIDGE", "HUBER", "ASINH"])
def test_opt_step_matches_nnptefr_sequence(tmp_path, reg):
    """nnp_opt_step = nnptefr's decay, ADAM step and weight decay of the
    weights (nnptefr.cpp:1032-1057), three steps, against a restatement."""
    from ace_b200.nnp import decay_step
    b, path, e_ref, f_ref = setup(tmp_path, n=3, seed=81)
    nn = NNP.read(path)
    p = nn.get_params()
    counts = [nn.nparams(t) for t in range(nn.ntypes)]
    # weight mask: per type, biases then weights (nnptefr.cpp:916-929)
    pot = potential.read(path)
    wm = np.concatenate([np.concatenate([np.zeros(sum(net.nodes[1:])),
                                         np.ones(sum(a * c for a, c in zip(net.nodes[:-1], net.nodes[1:])))])
                         for net in pot.nets])
    assert len(wm) == sum(counts)
    rfun = {"NONE": lambda x: 0 * x, "LASSO": np.sign, "RIDGE": lambda x: x,
            "HUBER": lambda x: x / np.sqrt(1 + x * x), "ASINH": np.arcsinh}[reg]
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    g_rate = g_ref = 2e-3
    for t in range(1, 4):
        _, g, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, 0.5, norm_mode=1)
        g_rate = nn.opt_step(g_rate, t, "INV", 0.1, 0, reg, 1e-2)
        g_ref = decay_step("INV", 0.1, 0, g_ref, t)
        assert g_rate == g_ref
        pold = p.copy()
        p, m, v = adam_reference(p, g, m, v, t, g_ref)
        p = p - g_ref * 1e-2 * wm * rfun(pold)
        assert np.abs(nn.get_params() - p).max() <= 1e-12 * np.abs(p).max()
    nn.close()


def test_device_pointer_training_matches_host(tmp_path):
    """nnp_train_grad with every array on the device gives the host-pointer
    call's loss and gradient (the same device arithmetic), and a device
    loop of train_grad + opt_step lowers the loss without host copies."""
    import torch
    b, path, e_ref, f_ref = setup(tmp_path, n=5, seed=91)
    nn = NNP.read(path)
    L, g, eo, fo = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, 0.5, norm_mode=2)
    dev = torch.device("cuda", 0)
    off = torch.tensor(b.atom_off, device=dev)
    pos = torch.tensor(b.pos, device=dev)
    typ = torch.tensor(b.type, device=dev)
    cell = torch.tensor(b.cell.reshape(-1, 9), device=dev)
    er = torch.tensor(e_ref, device=dev)
    fr = torch.tensor(f_ref, device=dev)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    grad = torch.zeros(len(g), dtype=torch.float64, device=dev)
    nn.train_grad_device(off.data_ptr(), pos.data_ptr(), typ.data_ptr(), cell.data_ptr(), b.n_struct, er.data_ptr(),
                         fr.data_ptr(), 0.5, loss.data_ptr(), grad.data_ptr(), norm_mode=2)
    torch.cuda.synchronize()
    assert abs(loss.item() - L) <= 1e-12 * abs(L)
    # the parameter gradient is summed per block in FP32 shared-memory
    # atomics, whose order changes from launch to launch: float rounding
    assert np.abs(grad.cpu().numpy() - g).max() <= 1e-5 * np.abs(g).max()
    losses = []
    gamma = 2e-3
    for t in range(1, 16):
        nn.train_grad_device(off.data_ptr(), pos.data_ptr(), typ.data_ptr(), cell.data_ptr(), b.n_struct,
                             er.data_ptr(), fr.data_ptr(), 0.5, loss.data_ptr(), 0, norm_mode=2)
        losses.append(loss.item())
        gamma = nn.opt_step(gamma, t, "EXP", 1e-3, 0, "NONE", 0.0)
    nn.close()
    assert losses[-1] < 0.7 * losses[0]


@pytest.mark.parametrize("w_f", [0.0, 0.5])
def test_tiled_gradient_matches_warp_kernel(tmp_path, monkeypatch, w_f):
    """The tiled network-gradient kernel (tiles of 32 atoms of one element,
    the default when its arrays fit in shared memory) gives the warp-per-atom
    kernel's gradient (NNP_TRAIN_TILE=0) to FP32 summation order, on a batch
    of 600+ atoms whose tiles of two elements are shared out over the CTAs."""
    b, path, e_ref, f_ref = setup(tmp_path, n=14, seed=57)
    assert b.n_atoms > 500
    nn = NNP.read(path)
    L1, g1, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, w_f, norm_mode=1)
    nn.close()
    monkeypatch.setenv("NNP_TRAIN_TILE", "0")
    nn = NNP.read(path)
    L0, g0, _, _ = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, w_f, norm_mode=1)
    nn.close()
    assert abs(L1 - L0) <= 1e-12 * abs(L0)
    assert np.abs(g1 - g0).max() <= 1e-5 * np.abs(g0).max()
