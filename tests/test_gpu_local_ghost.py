"""The pair-style force call (nnp_compute_local_ghost) against the periodic
call on the same atoms: a domain given its ghost atoms explicitly -- the
periodic images within rc of the domain, as a LAMMPS-style communication
builds them -- has the periodic energy, per-atom energies and virial, and
its forces, with each ghost's force added back onto the atom it images
(the reverse communication), are the periodic forces.

Two decompositions: the whole cell as one domain (a few thousand atoms with
ghosts, so the free-boundary search runs on a cell grid over the bounding
box), and the cell split into two domains whose energies and folded forces
add up to the periodic ones.  Tolerances: the same FP32 path on both sides,
only the order in which an atom's neighbours are summed differs: total
energies 1e-6 eV/atom, per-atom energies (FP32 network outputs, a few ulp
of their ~1-10 eV) 1e-5 eV, forces 1e-5 eV/A, virial 1e-5 relative to its
largest component."""
import numpy as np
import pytest

from ace_b200 import NNP, potential, synth

pytestmark = pytest.mark.gpu


def fcc_cell(n, seed=3):
    b = synth.config4(seed=seed, ncell=n)
    return b.pos.copy(), b.type.copy(), float(b.cell[0][0][0])


def make(tmp_path):
    pot = synth.potential_config(4)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    s = synth.config4(seed=997, ncell=4)
    nn = NNP.read(path)
    _, _, G = nn.compute_batch(s.atom_off, s.pos, s.type, s.cell, symm=True)
    nn.close()
    synth.condition(pot, G, s.type)
    potential.write(path, pot)
    return path, pot.rc


def ghosts_of(pos, typ, L, lo, hi, rc):
    """Periodic images (and, for a sub-domain, other atoms) within rc of the
    box [lo, hi) (per direction): positions, types and the owning atom."""
    gp, gt, go = [], [], []
    inside = np.all((pos >= lo) & (pos < hi), axis=1)
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sz in (-1, 0, 1):
                sh = np.array([sx, sy, sz]) * L
                q = pos + sh
                near = np.all((q >= lo - rc) & (q < hi + rc), axis=1)
                if sx == sy == sz == 0:
                    near &= ~inside
                gp.append(q[near])
                gt.append(typ[near])
                go.append(np.nonzero(near)[0])
    return np.concatenate(gp), np.concatenate(gt), np.concatenate(go), inside


@pytest.mark.parametrize("ncell", [4, 6])
def test_one_domain_with_ghosts_equals_periodic(tmp_path, ncell):
    path, rc = make(tmp_path)
    pos, typ, L = fcc_cell(ncell)
    pos = pos - L * np.floor(pos / L)
    nn = NNP.read(path)
    E, F, A, W = nn.compute_md(np.array([0, len(pos)]), pos, typ, np.eye(3)[None] * L)
    gp, gt, go, inside = ghosts_of(pos, typ, L, np.zeros(3), np.full(3, L), rc)
    assert inside.all()
    e, f, a, w = nn.compute_local_ghost(pos, typ, gp, gt)
    nn.close()
    n = len(pos)
    folded = f[:n].copy()
    np.add.at(folded, go, f[n:])
    print("ncell %d: %d local + %d ghosts: dE/atom %.2e  dF %.2e  dW %.2e" %
          (ncell, n, len(gp), abs(e - E[0]) / n, np.abs(folded - F).max(), np.abs(w - W[0]).max()))
    assert abs(e - E[0]) / n < 1e-6
    assert np.abs(a - A).max() < 1e-5
    assert np.abs(folded - F).max() < 1e-5
    assert np.abs(w - W[0]).max() < 1e-5 * np.abs(W[0]).max()


def test_two_domains_add_up_to_periodic(tmp_path):
    path, rc = make(tmp_path)
    pos, typ, L = fcc_cell(5)
    pos = pos - L * np.floor(pos / L)
    nn = NNP.read(path)
    E, F, A, W = nn.compute_md(np.array([0, len(pos)]), pos, typ, np.eye(3)[None] * L)
    n = len(pos)
    Fsum = np.zeros_like(F)
    Esum = 0.0
    Wsum = np.zeros((3, 3))
    for lo_x, hi_x in ((0.0, 0.5 * L), (0.5 * L, L)):
        lo, hi = np.array([lo_x, 0.0, 0.0]), np.array([hi_x, L, L])
        gp, gt, go, inside = ghosts_of(pos, typ, L, lo, hi, rc)
        own = np.nonzero(inside)[0]
        e, f, a, w = nn.compute_local_ghost(pos[own], typ[own], gp, gt)
        assert np.abs(a - A[own]).max() < 1e-5
        Esum += e
        Wsum += w
        np.add.at(Fsum, own, f[:len(own)])
        np.add.at(Fsum, go, f[len(own):])
    nn.close()
    assert abs(Esum - E[0]) / n < 1e-6
    assert np.abs(Fsum - F).max() < 1e-5
    assert np.abs(Wsum - W[0]).max() < 1e-5 * np.abs(W[0]).max()


def test_errors_and_empty(tmp_path):
    path, rc = make(tmp_path)
    nn = NNP.read(path)
    e, f, a, w = nn.compute_local_ghost(np.zeros((0, 3)), np.zeros(0, dtype=np.int32), np.zeros((0, 3)),
                                        np.zeros(0, dtype=np.int32))
    assert e == 0.0 and np.all(w == 0)
    from ace_b200 import NNPError
    with pytest.raises(NNPError):
        nn.compute_local_ghost(np.zeros((2, 3)) + [[0, 0, 0], [2, 0, 0]], np.array([0, 5], dtype=np.int32),
                               np.zeros((0, 3)), np.zeros(0, dtype=np.int32))
    nn.close()
