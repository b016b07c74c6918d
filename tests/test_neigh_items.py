"""CPU checks of the neighbour search's work items (ace_b200/csrc/nnp_kernels.cu:
neigh_parts, sort_cell's item ranges, the neigh_items reservation in
run_prepare), restated here with the device code's integer steps: every
cell's parts are non-empty, cover its atoms [0, n) exactly once in order,
give each warp of a block at least one atom at the finest split, and the
parts of a whole batch fit the reserved N + ceil(N / 4) + 1 items."""
import numpy as np
import pytest

NEIGH_WARPS = 4


def neigh_parts(n, O, budget):
    if n <= 0:
        return 0
    p = (O * n * n + budget - 1) // budget
    pmax = (n + NEIGH_WARPS - 1) // NEIGH_WARPS
    return int(min(max(p, 1), pmax))


def item_ranges(n, parts):
    return [(p * n // parts, (p + 1) * n // parts) for p in range(parts)]


def budget_for(N, nblocks=148 * 7):
    return int(min(1 << 16, max(2048, N * 216 // nblocks)))


@pytest.mark.parametrize("O", [1, 27, 125, 343])
def test_parts_cover_each_cell(O):
    for budget in (2048, 9000, 1 << 16):
        for n in range(0, 700):
            parts = neigh_parts(n, O, budget)
            if n == 0:
                assert parts == 0
                continue
            assert 1 <= parts <= (n + NEIGH_WARPS - 1) // NEIGH_WARPS
            r = item_ranges(n, parts)
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(a < b for a, b in r)                               # non-empty
            assert all(r[i][1] == r[i + 1][0] for i in range(len(r) - 1))  # contiguous, in order
            assert max(b - a for a, b in r) <= max(NEIGH_WARPS, (n + parts - 1) // parts)


def test_small_periodic_cell_splits_to_warps():
    """The 64-atom cell (one cell, its 27 images) splits into one part per
    four atoms: 16 blocks search it instead of one."""
    assert neigh_parts(64, 27, budget_for(64)) == 16


def test_items_fit_the_reservation():
    rng = np.random.default_rng(5)
    for _ in range(200):
        ncell = int(rng.integers(1, 400))
        counts = rng.integers(0, 90, size=ncell)
        counts[rng.random(ncell) < 0.3] = 0
        N = int(counts.sum())
        if N == 0:
            continue
        O = int(rng.choice([1, 27, 125]))
        b = budget_for(N)
        total = sum(neigh_parts(int(n), O, b) for n in counts)
        assert total <= N + (N + NEIGH_WARPS - 1) // NEIGH_WARPS + 1
