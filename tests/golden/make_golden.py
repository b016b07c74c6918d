"""Writes the golden fixtures of tests/golden/ from the reference itself.

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


if __name__ == "__main__":
    for name, k, b, pbc in cases():
        make(name, k, b, pbc)
        print("wrote", name, os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")
