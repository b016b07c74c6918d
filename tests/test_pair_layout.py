"""CPU checks of the index arithmetic that the force kernel's slot pass uses
(ace_b200/csrc/nnp_device.cuh: Blk, PairIt, tri_half, force_slots, small_div),
restated here in Python: for every chunking of a block's pairs, each pair is
summed exactly once by the owner of its first slot and once by the owner of
its second slot, at the coefficient index the pair pass wrote it to.  The GPU
tests run the kernels themselves (forced small chunks, dense neighbour lists);
these pin the enumeration for many block shapes in a second."""
import numpy as np
import pytest


def tri_pairs(n):
    """Pair numbering of a J == K block of n slots: p = g n + f couples slot f
    with slot (f + g + 1) mod n for g < (n-1)/2, plus the half row g = n/2-1,
    f < n/2, for even n."""
    out = []
    h = (n - 1) // 2
    for g in range(h):
        out += [(f, (f + g + 1) % n) for f in range(n)]
    if n % 2 == 0 and n >= 2:
        g = n // 2 - 1
        out += [(f, (f + g + 1) % n) for f in range(n // 2)]
    return out


def tri_half(n, x, second, g, c0, c1):
    """Pair index (or None) of row g in which slot x is the first or second member."""
    h = (n - 1) >> 1
    on = g != h or (x >= (n >> 1) if second else x < (n >> 1))
    o = x - g - 1 if second else x + g + 1
    o = o + n if o < 0 else (o - n if o >= n else o)
    p = g * n + (o if second else x)
    return p if (on and c0 <= p < c1) else None


@pytest.mark.parametrize("chunk", [7, 32, 256])
def test_tri_slots_cover_every_pair_twice(chunk):
    for n in range(2, 70):
        pairs = tri_pairs(n)
        assert len(pairs) == n * (n - 1) // 2
        assert len({tuple(sorted(q)) for q in pairs}) == len(pairs)      # every unordered pair once
        got = {x: [] for x in range(n)}
        for c0 in range(0, len(pairs), chunk):
            c1 = min(len(pairs), c0 + chunk)
            gmin, gmax = c0 // n, min((c1 - 1) // n, (n >> 1) - 1)
            for x in range(n):
                for g in range(gmin, gmax + 1):
                    for second in (False, True):
                        p = tri_half(n, x, second, g, c0, c1)
                        if p is not None:
                            a, b = pairs[p]
                            assert (b if second else a) == x
                            got[x].append(p)
        for x in range(n):
            assert sorted(got[x]) == [p for p, q in enumerate(pairs) if x in q]


@pytest.mark.parametrize("chunk", [7, 32, 256])
def test_rect_slots_cover_every_pair_twice(chunk):
    """J != K: pair p = g nb + f; a row owner reads its row's run inside the
    chunk, a column owner one entry per row (rows may be split by chunks)."""
    for na in list(range(1, 18)) + [40]:
        for nb in list(range(1, 18)) + [33, 200, 255]:
            npairs = na * nb
            rows, cols = {}, {}
            for c0 in range(0, npairs, chunk):
                c1 = min(npairs, c0 + chunk)
                for sl in range(na + nb):
                    is_row = sl < na
                    pb = sl * nb
                    lo, hi = max(c0, pb), min(c1, pb + nb)
                    f = sl - na
                    glo = -(-(c0 - f) // nb) if c0 > f else 0
                    ghi = (c1 - 1 - f) // nb + 1 if c1 > f else 0
                    cnt = hi - lo if is_row else ghi - glo
                    q0 = lo - c0 if is_row else glo * nb + f - c0
                    qs = 1 if is_row else nb
                    for j in range(max(cnt, 0)):
                        q = q0 + j * qs
                        assert 0 <= q < c1 - c0
                        g, ff = divmod(c0 + q, nb)
                        if is_row:
                            assert g == sl
                            rows.setdefault(sl, []).append(c0 + q)
                        else:
                            assert ff == f
                            cols.setdefault(f, []).append(c0 + q)
            for g in range(na):
                assert sorted(rows[g]) == [g * nb + f for f in range(nb)]
            for f in range(nb):
                assert sorted(cols[f]) == [g * nb + f for g in range(na)]


def test_small_div_correction():
    """small_div: a float quotient within a few ulps of p/m, corrected by two
    comparisons, is the exact integer quotient for p < 2^22, m <= 1024."""
    rng = np.random.default_rng(0)
    for m in range(1, 1025):
        ps = np.concatenate([np.arange(300), rng.integers(0, 1 << 22, 64),
                             m * rng.integers(0, (1 << 22) // m, 64), m * rng.integers(1, (1 << 22) // m, 64) - 1])
        for p in ps.tolist():
            qf = np.float32(p) / np.float32(m)
            for d in (-2, 0, 2):
                a = qf
                for _ in range(abs(d)):
                    a = np.nextafter(a, np.float32(np.inf if d > 0 else -np.inf))
                q = int(a)
                q += 1 if (q + 1) * m <= p else 0
                q -= 1 if q * m > p else 0
                assert q == p // m
