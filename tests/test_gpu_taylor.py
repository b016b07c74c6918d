"""Taylor expansion of a training set on the GPU (nnp_taylor_expand) against
nnptefr's force perturbation (nnptefr.cpp:2733-2830) restated here in FP64:
the same copies (structures with a mean force norm above 1e-12, nadd each,
originals first), the same counter-based random numbers, displacements and
first-order energies to rounding (1e-12 A, 1e-9 eV).  A second check is the
physics: with small displacements the first-order energies agree with the
model's energies at the displaced positions to second order."""
import math

import numpy as np
import pytest

from ace_b200 import NNP, NNPError, potential, synth
from ace_b200.nnp import DISTRIBUTIONS, taylor_expand

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def mix64(z):
    z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & M64
    z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & M64
    return z ^ (z >> 31)


def uniform(seed, o, j, k):
    h = mix64(mix64(mix64((seed + 0x9e3779b97f4a7c15) & M64) ^ o) ^ ((j * 4 + k) & M64))
    return ((h >> 11) + 0.5) / 9007199254740992.0


def radius(dist, w, u1, u2):
    if dist == 1:
        return u1 * w
    if dist == 2:
        p = u1 - 0.5
        return -w * np.sign(p) * math.log(1.0 - 2.0 * abs(p))
    if dist == 3:
        return w * math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)
    if dist == 5:
        return w * 2.0 / math.pi * math.log(math.tan(0.5 * math.pi * u1))
    if dist == 6:
        return w * math.log(u1 / (1.0 - u1))
    t = math.sqrt(-2.0 * math.log(u1 if u1 < 0.5 else 1.0 - u1))
    v = w * (0.820251 - 0.806770 * t + 0.093247 * t * t)
    return v if u1 < 0.5 else -v


def expand_reference(off, pos, energy, forces, nadd, dist, w, seed):
    oo, op, oe, src = [0], [], [], []
    o = 0
    for s in range(len(off) - 1):
        a0, a1 = off[s], off[s + 1]
        f = forces[a0:a1]
        favg = np.linalg.norm(f, axis=1).mean() if a1 > a0 else 0.0
        for m in range(1 + (nadd if favg > 1e-12 else 0)):
            x = pos[a0:a1].copy()
            de = 0.0
            if m > 0:
                for j in range(a1 - a0):
                    vr = radius(dist, w, uniform(seed, o, j, 0), uniform(seed, o, j, 3))
                    ct = 2.0 * uniform(seed, o, j, 1) - 1.0
                    st = math.sqrt(1.0 - ct * ct)
                    ph = (2.0 * uniform(seed, o, j, 2) - 1.0) * math.pi
                    d = np.array([vr * st * math.cos(ph), vr * st * math.sin(ph), vr * ct])
                    x[j] += d
                    de += d @ f[j]
            op.append(x)
            oe.append(energy[s] - de)
            src.append(s)
            oo.append(oo[-1] + a1 - a0)
            o += 1
    return np.array(oo), np.concatenate(op), np.array(oe), np.array(src)


@pytest.mark.parametrize("dist", sorted(DISTRIBUTIONS))
def test_expansion_matches_restatement(dist):
    rng = np.random.default_rng(4)
    b = synth.batch_random(8, rng.integers(5, 30, size=5), 2)
    E = rng.normal(size=b.n_struct)
    F = rng.normal(size=(b.n_atoms, 3))
    F[b.atom_off[2]:b.atom_off[3]] = 0.0                # a structure without forces is kept, not expanded
    oo, op, ot, oe, src = taylor_expand(b.atom_off, b.pos, b.type, E, F, 3, dist, 0.05, seed=1234)
    roo, rop, roe, rsrc = expand_reference(b.atom_off, b.pos, E, F, 3, DISTRIBUTIONS[dist], 0.05, 1234)
    np.testing.assert_array_equal(oo, roo)
    np.testing.assert_array_equal(src, rsrc)
    assert len(src) == b.n_struct * 4 - 3
    assert np.abs(op - rop).max() < 1e-12
    assert np.abs(oe - roe).max() < 1e-9
    np.testing.assert_array_equal(ot, np.concatenate([b.type[b.atom_off[s]:b.atom_off[s + 1]] for s in src]))


def test_first_order_energies_against_model(tmp_path):
    """Copies of model-labelled structures: the first-order energy differs
    from the model's energy at the displaced positions by O(|dr|^2)."""
    pot = synth.potential_config(3)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    b = synth.batch_random(9, [40, 60, 50], 2)
    nn = NNP.read(path)
    E, F = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell)
    errs = {}
    for w in (0.01, 0.02):       # wide enough that the second-order term dwarfs the FP32 energy noise (~3e-6 eV)
        oo, op, ot, oe, src = taylor_expand(b.atom_off, b.pos, b.type, E, F, 2, "UNIFORM", w, seed=7)
        Em, _ = nn.compute_batch(oo, op, ot, b.cell[src])
        errs[w] = np.abs(Em - oe).max()
    nn.close()
    print("first-order error: %.3e (w 0.01), %.3e (w 0.02)" % (errs[0.01], errs[0.02]))
    assert errs[0.01] < 0.05
    assert 2.5 < errs[0.02] / max(errs[0.01], 1e-15) < 6.0       # second order: x4 for twice the width


def test_errors():
    with pytest.raises(NNPError, match="distribution"):
        taylor_expand(np.array([0, 1]), np.zeros((1, 3)), np.zeros(1, dtype=np.int32), np.zeros(1),
                      np.ones((1, 3)), 1, 4, 0.1)
