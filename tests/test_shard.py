"""Multi-rank path on CPU: structure splitting, and the training step's one
exchange (batch-average loss and gradient via all-reduce), with world size 2
over gloo.  The per-rank work is the FP64 oracle, so nothing needs a GPU."""
import os
import socket

import numpy as np
import pytest

from ace_b200 import potential, shard, synth


def test_split_by_atoms_covers_everything():
    rng = np.random.default_rng(3)
    for S in [1, 2, 5, 37]:
        counts = rng.integers(1, 500, size=S)
        off = np.concatenate([[0], np.cumsum(counts)])
        for world in [1, 2, 3, 8]:
            parts = shard.split_by_atoms(off, world)
            assert len(parts) == world
            assert parts[0][0] == 0 and parts[-1][1] == S
            for (a, b), (c, d) in zip(parts, parts[1:]):
                assert b == c and a <= b
            if S >= world:
                assert all(b > a for a, b in parts)
    # balanced by atoms: equal-size structures split evenly
    off = np.arange(0, 101) * 10
    assert shard.split_by_atoms(off, 4) == [(0, 25), (25, 50), (50, 75), (75, 100)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, path, out_dir):
    import torch.distributed as dist
    from oracle import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b, e_ref, f_ref = _data()
        local, (s0, s1) = shard.local_batch(b, rank, world)
        a0, a1 = int(b.atom_off[s0]), int(b.atom_off[s1])
        op = orc.OraclePot.from_file(path)
        L, g, _, _ = orc.ef_loss_grad(op, local, e_ref[s0:s1], f_ref[a0:a1], 0.3, norm_mode=1)
        Lc, gc = shard.combine_loss_grad(L, g, s1 - s0)
        np.save(os.path.join(out_dir, "rank%d.npy" % rank), np.concatenate([[Lc], gc]))
    finally:
        dist.destroy_process_group()


def _data():
    rng = np.random.default_rng(11)
    b = synth.batch_random(11, rng.integers(8, 40, size=5), 2)
    e_ref = rng.normal(0, 1, size=b.n_struct)
    f_ref = rng.normal(0, 0.5, size=(b.n_atoms, 3))
    return b, e_ref, f_ref


def test_two_rank_training_gradient_equals_full_batch(tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle as orc
    pot = synth.potential_config(3, seed=8)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, path, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = np.load(str(tmp_path / "rank0.npy"))
    r1 = np.load(str(tmp_path / "rank1.npy"))
    np.testing.assert_array_equal(r0, r1)          # every rank holds the same result
    b, e_ref, f_ref = _data()
    op = orc.OraclePot.from_file(path)
    L, g, _, _ = orc.ef_loss_grad(op, b, e_ref, f_ref, 0.3, norm_mode=1)
    assert abs(r0[0] - L) < 1e-12 * max(1.0, abs(L))
    assert np.abs(r0[1:] - g).max() < 1e-12 * max(1.0, np.abs(g).max())
