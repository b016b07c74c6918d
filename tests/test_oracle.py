"""CPU checks of the FP64 oracle: the reference's own property tests, as
assertions (the reference's tests only print, src/nnp/test_*.cpp,
src/ml/test_nn_*.cpp)."""
import numpy as np
import pytest

from ace_b200 import potential, synth
from oracle import oracle as orc


def _pot(tmp_path, k, cond=True, seed=1234):
    pot = synth.potential_config(k, seed=seed)
    path = str(tmp_path / ("p%d.nnp" % k))
    potential.write(path, pot)
    if cond:
        b = synth.config1() if k == 1 else _small_batch(k)
        op = orc.OraclePot.from_file(path)
        G = np.concatenate([orc.compute_symm(op, *b.structure(s)) for s in range(b.n_struct)])
        synth.condition(pot, G, b.type)
        potential.write(path, pot)
    return pot, path, orc.OraclePot.from_file(path)


def _small_batch(k, n=3, seed=5):
    ntypes = {1: 1, 2: 3, 3: 2, 4: 2, 5: 4}[k]
    rng = np.random.default_rng(seed)
    return synth.batch_random(seed, rng.integers(12, 40, size=n), ntypes)


def test_special_functions():
    xs = np.linspace(-30, 5, 101)
    for x in xs:
        assert orc.lib().orc_fmexp(x) == pytest.approx(np.exp(x), rel=1e-13)
    for x in np.linspace(0, np.pi, 33):
        assert orc.lib().orc_coscut(x) == pytest.approx(np.cos(x), abs=1e-10)
        assert orc.lib().orc_sincut(x) == pytest.approx(np.sin(x), abs=1e-10)


@pytest.mark.parametrize("cut", [1, 2, 3, 4])
def test_cutoff_gradient(cut):
    """test_nnp_cutoff.cpp:18-76: cutoff slope against central differences."""
    rc = 6.0
    for r in np.linspace(0.1, 5.9, 37):
        fd = (orc.lib().orc_cutf(cut, rc, r + 1e-6) - orc.lib().orc_cutf(cut, rc, r - 1e-6)) / 2e-6
        assert orc.lib().orc_cutg(cut, rc, r) == pytest.approx(fd, abs=1e-6)
    assert orc.lib().orc_cutf(cut, rc, 6.5) == 0.0


def test_potential_roundtrip(tmp_path):
    for k in (1, 2, 5):
        pot = synth.potential_config(k)
        p1 = str(tmp_path / "a.nnp")
        p2 = str(tmp_path / "b.nnp")
        potential.write(p1, pot)
        q = potential.read(p1)
        potential.write(p2, q)
        assert open(p1).read() == open(p2).read()
        assert q.nparams() == pot.nparams()
        v = q.get_params()
        q.set_params(v)
        assert np.array_equal(q.get_params(), v)


def test_nlist_counts_small_cell():
    """Small periodic cell (side < 2 rc): multiple images and self-images."""
    b = synth.config1()
    p, t, c = b.structure(0)
    nl = orc.nlist(6.0, p, c)
    counts = np.array([len(x[0]) for x in nl])
    assert counts.mean() == pytest.approx(4.0 / 3.0 * np.pi * 216 * 64 / 8.5 ** 3, rel=0.1)
    # several images of the same atom appear (side 8.5 < 2 rc)
    assert any(len(np.unique(x[0])) < len(x[0]) for x in nl)
    # a cell smaller than rc: every atom sees its own images
    small = synth.batch_random(4, [6], 1, density=0.05 * (6 / 5.0) ** 0)
    ps, ts, cs = small.structure(0)
    nls = orc.nlist(6.0, ps, cs)
    assert all((x[0] == i).any() for i, x in enumerate(nls))
    # the list is symmetric: i sees j with shift n  <=>  j sees i with shift -n
    pairs = set()
    for i, (idx, img) in enumerate(nl):
        for j, s in zip(idx, img):
            pairs.add((i, int(j), tuple(np.round(s).astype(int))))
    for (i, j, s) in pairs:
        assert (j, i, tuple(-x for x in s)) in pairs


def test_force_vs_finite_difference(tmp_path):
    """test_nnp_force.cpp:40-167: analytic forces against central differences."""
    pot, path, op = _pot(tmp_path, 2)
    b = _small_batch(2, n=1, seed=9)
    p, t, c = b.structure(0)
    e, f, g = orc.compute(op, p, t, c)
    eps = 1e-5
    rng = np.random.default_rng(0)
    for a in rng.choice(len(p), size=6, replace=False):
        for d in range(3):
            pp = p.copy(); pp[a, d] += eps
            pm = p.copy(); pm[a, d] -= eps
            fd = -(orc.compute(op, pp, t, c)[0] - orc.compute(op, pm, t, c)[0]) / (2 * eps)
            assert f[a, d] == pytest.approx(fd, abs=2e-6, rel=1e-6)
    assert np.abs(f.sum(axis=0)).max() < 1e-10


def test_supercell_invariance(tmp_path):
    """test_nnp_symm.cpp:383-490: G of a cell equals G of the same atoms in its 2x2x2 supercell."""
    pot, path, op = _pot(tmp_path, 3, cond=False)
    b = synth.batch_random(3, [20], 2)
    p, t, c = b.structure(0)
    G = orc.compute_symm(op, p, t, c)
    shifts = np.array([[i, j, k] for i in range(2) for j in range(2) for k in range(2)])
    P2 = np.concatenate([p + s @ c for s in shifts])
    T2 = np.tile(t, 8)
    G2 = orc.compute_symm(op, P2, T2, 2 * c)
    for s in range(8):
        np.testing.assert_allclose(G2[s * 20:(s + 1) * 20], G, rtol=1e-10, atol=1e-10)


def test_energy_consistency(tmp_path):
    """compute_energy (with vacuum energies) = compute_force energy + sum of vacuum energies."""
    pot, path, op = _pot(tmp_path, 5)
    b = _small_batch(5, n=1)
    p, t, c = b.structure(0)
    e, f, g = orc.compute(op, p, t, c)
    ev = orc.compute_energy(op, t, g)
    vac = np.array([x.energy for x in pot.types])
    assert ev == pytest.approx(e + vac[t].sum(), rel=1e-12)


def test_nn_input_gradient(tmp_path):
    """test_nn_grad.cpp:15-120 (DODZ): dE/dG against central differences."""
    pot, path, op = _pot(tmp_path, 2)
    rng = np.random.default_rng(1)
    x = rng.normal(size=op.a["n_input"][1]) * 3 + 10
    out, dodi = orc.ann_fpbp(op, 1, x)
    for k in range(0, len(x), 5):
        xp = x.copy(); xp[k] += 1e-6
        xm = x.copy(); xm[k] -= 1e-6
        fd = (orc.ann_fpbp(op, 1, xp)[0] - orc.ann_fpbp(op, 1, xm)[0]) / 2e-6
        assert dodi[k] == pytest.approx(fd, abs=1e-7, rel=1e-6)


def test_cost_grad(tmp_path):
    """test_nn_cost.cpp:12-229: Cost::grad against central differences in the parameters."""
    pot, path, op = _pot(tmp_path, 3)
    rng = np.random.default_rng(2)
    x = rng.normal(size=op.a["n_input"][0])
    out, g = orc.cost_grad(op, 0, x)
    o, m = op.param_slice(0)
    par = op.a["nn_par"]
    for k in rng.choice(m, size=25, replace=False):
        v = par[o + k]
        par[o + k] = v + 1e-6
        up = orc.cost_grad(op, 0, x)[0]
        par[o + k] = v - 1e-6
        dn = orc.cost_grad(op, 0, x)[0]
        par[o + k] = v
        assert g[k] == pytest.approx((up - dn) / 2e-6, abs=1e-7, rel=1e-6)


def test_loss_gradient_fd(tmp_path):
    """Energy+force loss gradient against central differences of the oracle loss."""
    pot, path, op = _pot(tmp_path, 3)
    b = synth.batch_random(21, [10, 14], 2)
    rng = np.random.default_rng(3)
    e_ref = rng.normal(size=2)
    f_ref = rng.normal(size=(b.n_atoms, 3))
    loss, g, _, _ = orc.ef_loss_grad(op, b, e_ref, f_ref, w_f=0.7)
    p0 = op.get_params()
    for k in rng.choice(len(p0), size=20, replace=False):
        p = p0.copy(); p[k] += 1e-6
        op.set_params(p)
        up = orc.ef_loss_grad(op, b, e_ref, f_ref, 0.7, want_grad=False)[0]
        p[k] -= 2e-6
        op.set_params(p)
        dn = orc.ef_loss_grad(op, b, e_ref, f_ref, 0.7, want_grad=False)[0]
        op.set_params(p0)
        assert g[k] == pytest.approx((up - dn) / 2e-6, abs=1e-7, rel=1e-5)


def test_energy_loss_matches_ef_with_zero_force_weight(tmp_path):
    pot, path, op = _pot(tmp_path, 3)
    b = synth.batch_random(22, [10, 14, 9], 2)
    G = np.concatenate([orc.compute_symm(op, *b.structure(s)) for s in range(b.n_struct)])
    e_ref = np.array([1.0, -2.0, 0.5])
    l1, g1 = orc.energy_loss_grad(op, b.atom_off, b.type, G, e_ref)
    l2, g2, _, _ = orc.ef_loss_grad(op, b, e_ref, np.zeros((b.n_atoms, 3)), 0.0)
    assert l1 == pytest.approx(l2, rel=1e-12)
    np.testing.assert_allclose(g1, g2, rtol=1e-10, atol=1e-14)
