"""Structure files into a CSR batch (nnp_read_structures; host only) against
the reference's own readers (XYZ::read, VASP::POSCAR::read, compiled in
oracle/_ref): element types, positions (periodic frames wrapped into the
cell, as the reference does), forces, energies and cells, to 1e-12."""
import os

import numpy as np
import pytest

from ace_b200 import NNPError, nnp
from oracle import ref

NAMES = ["Si", "O", "H"]


def frame_text(rng, n, lattice=True, forces=True, energy=True):
    cell = np.diag(rng.uniform(6, 9, size=3)) + rng.uniform(-0.5, 0.5, size=(3, 3)) * (1 - np.eye(3))
    names = [NAMES[k] for k in rng.integers(0, 3, size=n)]
    pos = rng.uniform(-3, 12, size=(n, 3))
    frc = rng.normal(size=(n, 3))
    props = "Properties=species:S:1:pos:R:3" + (":forces:R:3" if forces else "")
    head = [props]
    if energy:
        head.append("potential_energy=%.12f" % rng.normal(-50, 5))
    if lattice:
        head.append('Lattice="%s"' % " ".join("%.12f" % x for x in cell.reshape(-1)))
    lines = ["%d" % n, " ".join(head)]
    for i in range(n):
        row = [names[i]] + ["%.12f" % x for x in pos[i]] + (["%.12f" % x for x in frc[i]] if forces else [])
        lines.append(" ".join(row))
    return "\n".join(lines) + "\n"


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref (compiled reference) not built")
def test_xyz_frames_match_reference_reader(tmp_path):
    rng = np.random.default_rng(5)
    frames = [frame_text(rng, 12), frame_text(rng, 7, forces=False), frame_text(rng, 9, lattice=False),
              frame_text(rng, 5, energy=False)]
    allpath = str(tmp_path / "all.xyz")
    with open(allpath, "w") as f:
        f.write("".join(frames))
    off, pos, typ, cells, pbc, en, frc = nnp.read_structures(allpath, NAMES, "xyz")
    assert len(off) == 5
    for s, text in enumerate(frames):
        one = str(tmp_path / ("f%d.xyz" % s))
        with open(one, "w") as f:
            f.write(text)
        names, rp, rf, pe, rcell = ref.read_structure(one, "xyz")
        a0, a1 = off[s], off[s + 1]
        assert [NAMES[t] for t in typ[a0:a1]] == names
        assert np.abs(pos[a0:a1] - rp).max() < 1e-12
        assert np.abs(frc[a0:a1] - rf).max() < 1e-12
        assert abs(en[s] - pe) < 1e-12
        assert np.abs(cells[s] - rcell).max() < 1e-12
        assert pbc[s] == (np.abs(rcell).max() > 0)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref (compiled reference) not built")
@pytest.mark.parametrize("direct", [True, False])
def test_poscar_matches_reference_reader(tmp_path, direct):
    rng = np.random.default_rng(6)
    R = np.diag([5.1, 6.2, 7.3]) + rng.uniform(-0.4, 0.4, size=(3, 3)) * (1 - np.eye(3))
    counts = [3, 2, 4]
    x = rng.uniform(0, 1, size=(9, 3)) if direct else rng.uniform(0, 6, size=(9, 3))
    lines = ["comment", "1.05"] + [" ".join("%.12f" % v for v in R[n]) for n in range(3)]
    lines += [" ".join(NAMES), " ".join(str(c) for c in counts), "Direct" if direct else "Cartesian"]
    lines += [" ".join("%.12f" % v for v in row) for row in x]
    path = str(tmp_path / "POSCAR")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    off, pos, typ, cells, pbc, en, frc = nnp.read_structures(path, NAMES, "vasp")
    names, rp, _, _, rcell = ref.read_structure(path, "vasp")
    assert list(off) == [0, 9] and pbc[0]
    assert [NAMES[t] for t in typ] == names
    assert np.abs(pos - rp).max() < 1e-12
    assert np.abs(cells[0] - rcell).max() < 1e-12


def test_reader_errors(tmp_path):
    path = str(tmp_path / "x.xyz")
    with open(path, "w") as f:
        f.write("2\nProperties=species:S:1:pos:R:3\nSi 0 0 0\nXe 1 1 1\n")
    with pytest.raises(NNPError, match="Xe"):
        nnp.read_structures(path, NAMES, "xyz")
    with open(path, "w") as f:
        f.write("3\n\nSi 0 0 0\n")
    with pytest.raises(NNPError):
        nnp.read_structures(path, NAMES, "xyz")
    with pytest.raises(NNPError):
        nnp.read_structures(str(tmp_path / "missing.xyz"), NAMES, "xyz")
    # plain XYZ without a Properties field: "name x y z"
    with open(path, "w") as f:
        f.write("2\nplain\nSi 0 0 0\nO 1.5 0 0\n")
    off, pos, typ, cells, pbc, en, frc = nnp.read_structures(path, NAMES, "xyz")
    assert list(typ) == [0, 1] and not pbc[0] and pos[1, 0] == 1.5
