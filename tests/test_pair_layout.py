"""CPU checks of the index arithmetic that the force kernel's pair and slot
passes use (ace_b200/csrc/nnp_device.cuh: make_blk, chunk_rows, PairIt,
force_pairs_generic's coefficient index, tri_visits, tri_visits2, force_slots, small_div),
restated here in Python with the device code's integer steps: for every
block shape up to the staging capacity and the chunk sizes the tuner may
pick, the pair pass writes each pair of a chunk to a distinct coefficient
inside the chunk's area, and the slot pass sums each pair exactly once for
its first and once for its second slot, reading the coefficient the pair
pass wrote it to.  Coefficient indices stay below the per-array length
coef_len(chunk, cap) = max(chunk, cap), checked at the smallest capacity a
block can have (its own slots).  The GPU tests run the kernels themselves;
these pin the enumeration for all block shapes in seconds."""
import numpy as np
import pytest

NNP_PCH = 288
CAPACITY = 256


def coef_len(chunk, cap):
    return max(chunk, cap)


def small_div(p, m):
    assert 0 <= p < (1 << 22) and 1 <= m <= 1024
    return p // m


def make_blk(n0, n1, tri):
    """Blk of a block whose J segment starts at slot 0 and K segment at n0"""
    if tri:
        k = dict(sa=0, na=n0, sb=0, nb=n0, tri=True, npairs=n0 * (n0 - 1) // 2, rows=n0 >> 1, s=n0)
    else:
        s0, s1 = 0, n0
        if n1 > n0:
            k = dict(sa=s1, na=n1, sb=s0, nb=n0)
        else:
            k = dict(sa=s0, na=n0, sb=s1, nb=n1)
        k.update(tri=False, npairs=k["na"] * k["nb"], rows=k["na"], s=k["nb"] | 1)
    if k["npairs"] == 0:
        return None
    k["m"] = k["nb"]
    k["q32"] = small_div(32, k["m"])
    k["r32"] = 32 - k["q32"] * k["m"]
    return k


def chunk_rows(k, chunk):
    R = small_div(chunk, k["s"])
    if not k["tri"] and k["nb"] < 32:
        R = min(R, 32 - k["nb"])
    return max(R, 1)


def pair_pass(k, c0, c1, q0):
    """(coefficient index, first slot, second slot) of the pairs [c0, c1), as
    the lanes' PairIt walks them (p = lane + 32 t)"""
    out = []
    for lane in range(32):
        p = c0 + lane
        g = small_div(p, k["m"])
        f = p - g * k["m"]
        while p < c1:
            if k["tri"]:
                bb = f + g + 1
                a, b = k["sa"] + f, k["sa"] + (bb - k["m"] if bb >= k["m"] else bb)
            else:
                a, b = k["sa"] + g, k["sb"] + f
            out.append((g * k["s"] + f - q0, a, b))
            p += 32
            f += k["r32"]
            g += k["q32"]
            if f >= k["m"]:
                f -= k["m"]
                g += 1
    return out


def tri_visits(k, x, second, g0, g1):
    """(coefficient index, partner) of slot x's pairs in rows [g0, g1)"""
    n = k["m"]
    hn, hr = n >> 1, (-1 if n & 1 else (n >> 1) - 1)
    o = x - g0 - 1 if second else x + g0 + 1
    o += n if o < 0 else 0
    o -= n if o >= n else 0
    base, out = 0, []
    for g in range(g0, g1):
        first = o if second else x
        if g != hr or first < hn:
            out.append((base + first, k["sa"] + o))
        base += n
        o = (n - 1 if o == 0 else o - 1) if second else (0 if o == n - 1 else o + 1)
    return out


def tri_visits2(k, x, g0, g1):
    """tri_visits of both halves in one walk (J == K blocks of more than 16
    slots): (coefficient index, side, partner) in walk order"""
    n = k["m"]
    hn, hr = n >> 1, (-1 if n & 1 else (n >> 1) - 1)
    of, os = x + g0 + 1, x - g0 - 1
    of -= n if of >= n else 0
    os += n if os < 0 else 0
    base, out = 0, []
    for g in range(g0, g1):
        half = g == hr
        if not half or x < hn:
            out.append((base + x, "A", k["sa"] + of))
        if not half or os < hn:
            out.append((base + os, "C", k["sa"] + os))
        base += n
        of = 0 if of == n - 1 else of + 1
        os = n - 1 if os == 0 else os - 1
    return out


def slot_pass(k, g0, g1):
    """slot -> list of (coefficient index, side, partner): side 'A' = the
    slot is the pair's first member (cA), 'C' = second member (cC)"""
    got = {}
    if k["tri"]:
        for x in range(k["m"]):
            if k["m"] > 16:                                   # one walk over both halves
                got[k["sa"] + x] = tri_visits2(k, x, g0, g1)
                continue
            for second in (False, True):
                for q, o in tri_visits(k, x, second, g0, g1):
                    got.setdefault(k["sa"] + x, []).append((q, "C" if second else "A", o))
        return got
    nr = g1 - g0
    for sl in range(nr + k["nb"]):
        is_row = sl < nr
        slot = k["sa"] + g0 + sl if is_row else k["sb"] + (sl - nr)
        cnt = k["nb"] if is_row else nr
        q0 = sl * k["s"] if is_row else sl - nr
        qs = 1 if is_row else k["s"]
        up = k["sb"] if is_row else k["sa"] + g0
        for j in range(cnt):
            got.setdefault(slot, []).append((q0 + j * qs, "A" if is_row else "C", up + j))
    return got


def check(n0, n1, tri, chunk):
    k = make_blk(n0, n1, tri)
    if tri:
        want = {frozenset((a, b)) for a in range(n0) for b in range(a + 1, n0)}
    else:
        want = {frozenset((a, b)) for a in range(n0) for b in range(n0, n0 + n1)}
    if k is None:
        assert not want
        return
    if not tri:
        assert k["na"] >= k["nb"] and k["s"] % 2 == 1                # larger segment as rows, odd stride
    R = chunk_rows(k, chunk)
    area = coef_len(chunk, n0 if tri else n0 + n1)                  # smallest capacity holding the block
    seen = []
    for g0 in range(0, k["rows"], R):
        g1 = min(k["rows"], g0 + R)
        c0, c1, q0 = g0 * k["m"], min(k["npairs"], g1 * k["m"]), g0 * k["s"]
        written = {}
        for q, a, b in pair_pass(k, c0, c1, q0):
            assert 0 <= q < area and q not in written             # inside the coefficient arrays, once
            written[q] = (a, b)
            seen.append(frozenset((a, b)))
        if not tri and k["nb"] < 32:
            assert (g1 - g0) + k["nb"] <= 32                       # one lane per row and column
        visits = {}
        for slot, lst in slot_pass(k, g0, g1).items():
            for q, side, partner in lst:
                assert q in written                                 # reads what the pair pass wrote
                a, b = written[q]
                assert (a, b) == ((slot, partner) if side == "A" else (partner, slot))
                visits[(q, side)] = visits.get((q, side), 0) + 1
        assert all(c == 1 for c in visits.values())
        assert len(visits) == 2 * len(written)                     # every pair once per member
    assert len(seen) == len(want) and set(seen) == want


@pytest.mark.parametrize("chunk", [NNP_PCH, 192, 144, 40, 7])
def test_tri_blocks(chunk):
    for n in range(0, CAPACITY + 1, 1 if chunk == NNP_PCH else 5):
        check(n, n, True, chunk)


@pytest.mark.parametrize("chunk", [NNP_PCH, 192, 144, 40, 7])
def test_rect_blocks(chunk):
    sizes = list(range(0, 34)) + [47, 64, 65, 100, 128, 200, 255]
    for n0 in sizes[:: (1 if chunk == NNP_PCH else 3)]:
        for n1 in sizes:
            if n0 + n1 <= CAPACITY:
                check(n0, n1, False, chunk)


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
