"""CUDA-graph replay of the device-side step (nnp_set_graphs): an MD-like
loop of calls with the same shape and moving atoms gives exactly the results
of eager launches, including the call that captures, the calls that replay,
a change of shape, and a neighbour-capacity overflow in the middle of
replays (which must drop the graph and retry eagerly)."""
import numpy as np
import pytest
import torch

from ace_b200 import NNP, potential, synth

pytestmark = pytest.mark.gpu


def make(tmp_path):
    rng = np.random.default_rng(8)
    b = synth.batch_random(8, rng.integers(20, 60, size=5), 3)
    pot = synth.potential_config(2)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    nn = NNP.read(path)
    _, _, G = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell, symm=True)
    nn.close()
    synth.condition(pot, G, b.type)
    potential.write(path, pot)
    return b, path


def run_loop(path, b, graphs, steps=6, squeeze_at=None):
    nn = NNP.read(path)
    s = torch.cuda.Stream()
    nn.set_stream(s.cuda_stream)          # graphs need a capturable (non-default) stream
    nn.set_graphs(graphs)
    rng = np.random.default_rng(3)
    out = []
    pos = b.pos.copy()
    cell = b.cell.copy()
    for k in range(steps):
        pos = pos + rng.normal(0, 0.01, size=pos.shape)      # atoms move, shape stays
        if squeeze_at is not None and k == squeeze_at:
            pos = pos * 0.8                                    # denser: more neighbours than the capacity
            cell = cell * 0.8
        E, F = nn.compute_batch(b.atom_off, pos, b.type, cell)
        out.append((E.copy(), F.copy()))
    launches = nn.launch_count()
    nn.close()
    return out, launches


@pytest.mark.parametrize("squeeze_at", [None, 4])
def test_graph_replay_matches_eager(tmp_path, squeeze_at):
    b, path = make(tmp_path)
    eager, _ = run_loop(path, b, False, squeeze_at=squeeze_at)
    replay, _ = run_loop(path, b, True, squeeze_at=squeeze_at)
    for (E0, F0), (E1, F1) in zip(eager, replay):
        # same kernels on the same inputs; only FP64 atomics may reorder
        assert np.abs(E1 - E0).max() < 1e-9
        assert np.abs(F1 - F0).max() < 1e-9


def test_graph_follows_shape_change(tmp_path):
    b, path = make(tmp_path)
    small = b.subset([0, 1])
    nn = NNP.read(path)
    s = torch.cuda.Stream()
    nn.set_stream(s.cuda_stream)
    ref = NNP.read(path)
    ref.set_graphs(False)
    for batch in [b, b, b, small, small, small, b, b]:
        E, F = nn.compute_batch(batch.atom_off, batch.pos, batch.type, batch.cell)
        E0, F0 = ref.compute_batch(batch.atom_off, batch.pos, batch.type, batch.cell)
        assert np.abs(E - E0).max() < 1e-9 and np.abs(F - F0).max() < 1e-9
    nn.close()
    ref.close()
