"""Writes the golden fixtures of tests/golden/ from the reference itself.

train_config3.npz holds the reference's own training gradients (see
make_train).

Each fixture holds a potential file (text, as NNP::write writes it), a small
CSR batch of structures, and the reference's outputs for every structure:
NNP::compute_force energy (no vacuum terms) and forces, NNP::compute_energy
(with vacuum terms), and the symmetry functions of NNP::compute_symm.  The
reference is the compiled reference code in oracle/_ref (built by
oracle/ref/Makefile from the reference sources), so this script needs the
reference checkout; the fixtures it writes do not.

    make -C oracle/ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ace_b200 import potential, synth  # noqa: E402
from oracle import ref  # noqa: E402


def cases():
    """(name, config number, batch, pbc) of every fixture."""
    out = [("config1", 1, synth.config1(), True)]
    for k, nt in [(2, 3), (3, 2), (4, 2), (5, 4)]:
        rng = np.random.default_rng(500 + k)
        out.append(("config%d" % k, k, synth.batch_random(500 + k, rng.integers(8, 72, size=4), nt), True))
    # cells smaller than the cutoff: an atom sees its own periodic images
    rng = np.random.default_rng(77)
    small = synth.Batch(atom_off=np.array([0, 2, 5], dtype=np.int64),
                        pos=rng.uniform(0, 3.2, size=(5, 3)),
                        type=np.array([0, 1, 2, 0, 1], dtype=np.int32),
                        cell=np.stack([np.diag([3.2, 3.4, 3.6]),
                                       np.diag([3.5, 3.5, 3.5]) + np.array([[0, 0.4, 0], [0, 0, 0], [0.3, 0, 0]])]),
                        pbc=True)
    out.append(("small_cells", 2, small, True))
    # free boundaries (zero cell): a cluster
    rng = np.random.default_rng(78)
    cl = synth.grid_positions(rng, 40, np.eye(3) * 12.0)
    free = synth.Batch(atom_off=np.array([0, 40], dtype=np.int64), pos=cl,
                       type=rng.integers(0, 3, size=40).astype(np.int32), cell=np.zeros((1, 3, 3)), pbc=False)
    out.append(("free_cluster", 2, free, False))
    return out


def make_large(name, k, b):
    """A full-size fixture: the reference's energies and forces (no symmetry
    functions, to keep the file small) of one large structure of
    configuration k, potential conditioned as for the small fixtures."""
    import tempfile
    pot = synth.potential_config(k)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "pot.nnp")
        potential.write(path, pot)
        rp = ref.RefNNP(path)
        cb = conditioning_batch(k)
        G = np.concatenate([rp.compute(*cb.structure(s), want_symm=True)[3] for s in range(cb.n_struct)])
        rp.close()
        synth.condition(pot, G[:, :max(pot.n_input(t) for t in range(pot.ntypes))], cb.type)
        potential.write(path, pot)
        text = open(path).read()
        rp = ref.RefNNP(path)
        E, EV, F = [], [], []
        for s in range(b.n_struct):
            e, f, ev, _ = rp.compute(*b.structure(s))
            E.append(e)
            EV.append(ev)
            F.append(f)
        rp.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), potential=np.frombuffer(text.encode(), dtype=np.uint8),
                        atom_off=b.atom_off, pos=b.pos, type=b.type, cell=np.asarray(b.cell).reshape(-1, 9),
                        pbc=np.array(True), energy=np.array(E), energy_vacuum=np.array(EV),
                        forces=np.concatenate(F), config=np.array(k))


def large_cases():
    """Configuration 4's jittered FCC lattice at 10^3 cells (4000 atoms,
    rc 6.5 A) and one 2048-atom structure of configuration 5's generator."""
    rng = np.random.default_rng(705)
    return [("large_config4", 4, synth.config4(seed=704, ncell=10)),
            ("large_config5", 5, synth.batch_random(705, [2048], 4))]


def form_cases():
    """(name, batch) of the fixtures of the other basis forms, cutoffs and
    activations (synth.FORM_POTENTIALS): 4 periodic structures of 8-48 atoms."""
    out = []
    for n, name in enumerate(sorted(synth.FORM_POTENTIALS)):
        nt = len(synth.FORM_POTENTIALS[name][3])
        rng = np.random.default_rng(600 + n)
        out.append((name, synth.batch_random(600 + n, rng.integers(8, 48, size=4), nt)))
    return out


def make_forms(name, b):
    """A fixture of one FORM_POTENTIALS potential, conditioned on its own
    batch's symmetry functions (the reference's), with the reference's
    energies, forces and symmetry functions."""
    import tempfile
    pot = synth.potential_forms(name)
    nt = pot.ntypes
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "pot.nnp")
        potential.write(path, pot)
        rp = ref.RefNNP(path)
        G = np.concatenate([rp.compute(*b.structure(s), want_symm=True)[3] for s in range(b.n_struct)])
        rp.close()
        synth.condition(pot, G[:, :max(pot.n_input(t) for t in range(nt))], b.type)
        potential.write(path, pot)
        text = open(path).read()
        rp = ref.RefNNP(path)
        E, EV, F, Gs = [], [], [], []
        for s in range(b.n_struct):
            e, f, ev, g = rp.compute(*b.structure(s), want_symm=True)
            E.append(e)
            EV.append(ev)
            F.append(f)
            Gs.append(g)
        rp.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), potential=np.frombuffer(text.encode(), dtype=np.uint8),
                        atom_off=b.atom_off, pos=b.pos, type=b.type, cell=np.asarray(b.cell).reshape(-1, 9),
                        pbc=np.array(True), energy=np.array(E), energy_vacuum=np.array(EV),
                        forces=np.concatenate(F), symm=np.concatenate(Gs), config=np.array(0))


def conditioning_batch(k):
    """Periodic structures of configuration k whose symmetry-function mean
    and spread set the network's input bias and scale (nnptefr's PREBIAS MEAN
    / PRESCALE DEV); a tiny fixture alone would give near-zero spreads."""
    if k == 1:
        return synth.config1()
    nt = {2: 3, 3: 2, 4: 2, 5: 4}[k]
    rng = np.random.default_rng(400 + k)
    return synth.batch_random(400 + k, rng.integers(32, 96, size=6), nt)


def make(name, k, b, pbc, seed=1234):
    import tempfile
    pot = synth.potential_config(k, seed=seed)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "pot.nnp")
        potential.write(path, pot)
        rp = ref.RefNNP(path)
        cb = conditioning_batch(k)
        G = np.concatenate([rp.compute(*cb.structure(s), want_symm=True)[3] for s in range(cb.n_struct)])
        rp.close()
        synth.condition(pot, G[:, :max(pot.n_input(t) for t in range(pot.ntypes))], cb.type)
        potential.write(path, pot)
        text = open(path).read()
        rp = ref.RefNNP(path)
        E, EV, F, Gs = [], [], [], []
        for s in range(b.n_struct):
            e, f, ev, g = rp.compute(*b.structure(s), pbc=pbc, want_symm=True)
            E.append(e)
            EV.append(ev)
            F.append(f)
            Gs.append(g)
        rp.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), potential=np.frombuffer(text.encode(), dtype=np.uint8),
                        atom_off=b.atom_off, pos=b.pos, type=b.type, cell=np.asarray(b.cell).reshape(-1, 9),
                        pbc=np.array(pbc), energy=np.array(E), energy_vacuum=np.array(EV),
                        forces=np.concatenate(F), symm=np.concatenate(Gs), config=np.array(k))


# (norm mode, loss kind, delta) of the energy-loss gradients in train_config3.npz:
# every nnptefr norm with MSE, then MAE / HUBER / ASINH with the LINEAR norm
TRAIN_CASES = [(0, 1, 1.0), (1, 1, 1.0), (2, 1, 1.0), (3, 1, 1.0), (4, 1, 1.0),
               (1, 2, 1.0), (1, 3, 0.05), (1, 4, 0.05)]
TRAIN_W_F = 0.5


def fold_input_scaling(pot):
    """The same networks with inpw = 1, inpb = 0: the input scale and bias
    moved into the first layer (W0' = W0 diag(inpw), b0' = b0 + W0 (inpw * inpb))."""
    for net in pot.nets:
        w0 = net.w[0]
        net.b[0] = net.b[0] + w0 @ (net.inpw * net.inpb)
        net.w[0] = w0 * net.inpw[None, :]
        net.inpw = np.ones_like(net.inpw)
        net.inpb = np.zeros_like(net.inpb)
    return pot


def make_train():
    """Training configuration 3 (two elements, 48-32-32-1 tanh) on 4 small
    structures, labels from a teacher potential (other seed) evaluated by the
    reference plus Gaussian noise (1 meV/atom, 20 meV/A).

    potential_e: conditioned potential (inpw != 1).  For each case of
    TRAIN_CASES, grad_e[c] / loss_e[c] are the reference's energy-loss gradient
    and loss: NNP::compute_symm, then ANN::fpbp + Cost::grad per atom and
    NNPTEFR::error_cost_o1's loss factor and batch average (ref_energy_loss_grad).

    potential_f: the same networks with the input scaling folded into the
    first layer (inpw = 1, for which the reference's D2ODZDI is exact).
    grad_ef / loss_ef: the energy(MSE, LINEAR)+force loss with w_f = TRAIN_W_F,
    the energy term as above and the force term -sum_i d/dtheta(dE_i/dG_i . C_i)
    from the reference's D2ODZDI contracted with C_i, the change of the
    reference's compute_symm along the force adjoint (central differences,
    largest displacement 1e-5 A)."""
    import tempfile
    rng = np.random.default_rng(31)
    b = synth.batch_random(31, rng.integers(16, 40, size=4), 2)
    cb = conditioning_batch(3)
    pots = {}
    with tempfile.TemporaryDirectory() as d:
        for name, seed in (("model", 5), ("teacher", 6)):
            pot = synth.potential_config(3, seed=seed)
            path = os.path.join(d, name + ".nnp")
            potential.write(path, pot)
            rp = ref.RefNNP(path)
            G = np.concatenate([rp.compute(*cb.structure(s), want_symm=True)[3] for s in range(cb.n_struct)])
            rp.close()
            synth.condition(pot, G, cb.type)
            potential.write(path, pot)
            pots[name] = path
        rt = ref.RefNNP(pots["teacher"])
        Et, Ft = [], []
        for s in range(b.n_struct):
            e, f, _, _ = rt.compute(*b.structure(s))
            Et.append(e)
            Ft.append(f)
        rt.close()
        nat = np.diff(b.atom_off)
        e_ref = np.array(Et) + rng.normal(0, 1e-3, size=b.n_struct) * nat
        f_ref = np.concatenate(Ft) + rng.normal(0, 0.02, size=(b.n_atoms, 3))
        text_e = open(pots["model"]).read()
        rp = ref.RefNNP(pots["model"])
        grad_e, loss_e = [], []
        for nm, kind, delta in TRAIN_CASES:
            L, g, _, _ = rp.energy_loss_grad(b, e_ref, norm_mode=nm, loss_kind=kind, delta=delta)
            grad_e.append(g)
            loss_e.append(L)
        rp.close()
        pot = fold_input_scaling(potential.read(pots["model"]))
        path_f = os.path.join(d, "folded.nnp")
        potential.write(path_f, pot)
        text_f = open(path_f).read()
        rp = ref.RefNNP(path_f)
        L_e, g, _, _ = rp.energy_loss_grad(b, e_ref, norm_mode=1, loss_kind=1)
        B = b.n_struct
        lf = 0.0
        for s in range(B):
            p, t, c = b.structure(s)
            a0, a1 = int(b.atom_off[s]), int(b.atom_off[s + 1])
            _, f, _, _ = rp.compute(p, t, c)
            df = f - f_ref[a0:a1]
            fs = TRAIN_W_F / (3.0 * (a1 - a0))
            lf += 0.5 * fs * float((df * df).sum()) / B
            v = fs * df / B
            g -= rp.force_term_grad(p, t, c, v, 1e-5 / np.abs(v).max())
        rp.close()
    np.savez_compressed(os.path.join(HERE, "train_config3.npz"),
                        potential_e=np.frombuffer(text_e.encode(), dtype=np.uint8),
                        potential_f=np.frombuffer(text_f.encode(), dtype=np.uint8),
                        atom_off=b.atom_off, pos=b.pos, type=b.type, cell=np.asarray(b.cell).reshape(-1, 9),
                        e_ref=e_ref, f_ref=f_ref, cases=np.array(TRAIN_CASES), grad_e=np.array(grad_e),
                        loss_e=np.array(loss_e), w_f=np.array(TRAIN_W_F), grad_ef=g, loss_ef=np.array(L_e + lf))


if __name__ == "__main__":
    which = sys.argv[1:]
    for name, k, b, pbc in cases():
        if which and name not in which:
            continue
        make(name, k, b, pbc)
        print("wrote", name, os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")
    for name, b in form_cases():
        if which and name not in which:
            continue
        make_forms(name, b)
        print("wrote", name, os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")
    for name, k, b in large_cases():
        if which and name not in which:
            continue
        make_large(name, k, b)
        print("wrote", name, os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")
    if not which or "train_config3" in which:
        make_train()
        print("wrote train_config3", os.path.getsize(os.path.join(HERE, "train_config3.npz")), "bytes")
