"""The neighbour-search prologue of a small periodic batch runs in one
thread block (k_prologue_small: at most 2048 atoms and 32 structures); larger
batches use the launch sequence (k_type_count ... k_cell_pos).  Both build
the same cell lists, work items and neighbour lists: the structures of a
small batch get the same energies and forces alone (one-block prologue) and
inside a batch that is too large for it (launch sequence), up to the order
of the FP64 force atomics."""
import numpy as np
import pytest

from ace_b200 import NNP, potential, synth

pytestmark = pytest.mark.gpu


def conditioned(tmp_path, b):
    pot = synth.potential_config(2)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    nn = NNP.read(path)
    _, _, G = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell, symm=True)
    nn.close()
    synth.condition(pot, G, b.type)
    potential.write(path, pot)
    return path


@pytest.mark.parametrize("jit", [True, False], ids=["specialised", "generic"])
@pytest.mark.parametrize("grow", ["atoms", "structures"])
def test_one_block_prologue_matches_launch_sequence(tmp_path, jit, grow):
    big = synth.config2(seed=23, n_struct=64, nmin=16, nmax=512)
    counts = np.diff(big.atom_off)
    # a small batch: the first structures up to ~1500 atoms (includes
    # single-cell structures of fewer than ~86 atoms when the draw has them)
    k = int(np.searchsorted(np.cumsum(counts), 1500))
    k = max(2, min(k, 20))
    small = big.subset(range(k))
    assert small.n_atoms <= 2048 and small.n_struct <= 32
    if grow == "atoms":
        extra = [i for i in range(k, big.n_struct)]
        order = list(range(k)) + extra[:8]
        large = big.subset(order)
        assert large.n_atoms > 2048
    else:
        # more than 32 structures, few atoms: the same small structures
        # followed by copies of the smallest one
        smallest = int(np.argmin(counts[:k]))
        large = big.subset(list(range(k)) + [smallest] * (33 - k + 1))
        assert large.n_struct > 32
    path = conditioned(tmp_path, small)
    nn = NNP.read(path)
    nn.set_specialization(jit)
    E1, F1 = nn.compute_batch(small.atom_off, small.pos, small.type, small.cell)
    E2, F2 = nn.compute_batch(large.atom_off, large.pos, large.type, large.cell)
    nn.close()
    F2 = F2.reshape(-1, 3)[: small.n_atoms].reshape(F1.shape)
    assert np.abs(E2[:k] - E1).max() < 1e-9
    assert np.abs(F2 - F1).max() < 1e-9
