"""Neighbour lists against the oracle, count for count: per atom and
element, the neighbours found by the cell-list search (nnp_neighbor_counts
after a compute call) equal the oracle's list (orc_nlist: every atom and
every image within rc, the displacement test of neighbor.cpp:46-88) exactly.
The cases go through both prologue forms (one thread block for a periodic
batch of at most 2048 atoms and 32 structures, the launch sequence above),
the work items that split a big cell over several blocks (periodic
structures small enough to be one cell, seen through 27 images; a free
cluster that is one cell), triclinic shear and several elements."""
import numpy as np
import pytest

from ace_b200 import NNP, potential, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def oracle_counts(rc, b, ntypes):
    out = []
    for s in range(b.n_struct):
        pos, typ, cell = b.structure(s)
        nl = orc.nlist(rc, pos, cell, pbc=b.pbc, cap=4096)
        c = np.zeros((len(pos), ntypes), np.int32)
        for i, (idx, _) in enumerate(nl):
            np.add.at(c[i], typ[idx], 1)
        out.append(c)
    return np.concatenate(out)


def batches():
    big = synth.config2(seed=31, n_struct=40, nmin=16, nmax=512)
    counts = np.diff(big.atom_off)
    k = int(max(2, min(20, np.searchsorted(np.cumsum(counts), 1800))))
    free = synth.batch_random(62, [700, 40, 1900], 3)
    return {
        "config1_cell": (1, synth.config1()),
        "mixed_one_block": (2, big.subset(range(k))),
        "mixed_launch_sequence": (2, big),
        "free_clusters": (2, synth.Batch(free.atom_off, free.pos, free.type, free.cell, pbc=False)),
    }


@pytest.mark.parametrize("name", ["config1_cell", "mixed_one_block", "mixed_launch_sequence", "free_clusters"])
def test_neighbour_counts_match_oracle(tmp_path, name):
    k, b = batches()[name]
    pot = synth.potential_config(k)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    nn = NNP.read(path)
    if b.pbc:
        nn.compute_batch(b.atom_off, b.pos, b.type, b.cell)
    else:
        nn.compute_batch(b.atom_off, b.pos, b.type, None, pbc=False)
    got = nn.neighbor_counts(b.n_atoms)
    nn.close()
    want = oracle_counts(pot.rc, b, len(pot.types))
    assert got.shape == want.shape
    bad = np.argwhere(got != want)
    assert bad.size == 0, "first mismatches (atom, element): %s" % bad[:5].tolist()
