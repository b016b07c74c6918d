"""Seeded synthetic workloads: potentials and structure batches.

The reference publishes no dataset for its NNP path, so every workload is
generated here from a seed with the shapes the benchmark configurations
name.  Choices the configurations leave open are fixed as follows:

* radial functions are GAUSSIAN with centres evenly spaced on [0.5, rc_r]
  and width eta = 1.0 A^-1 (the reference's eta multiplies (r-rs), so
  "eta = 1 A^-2" in the eta*r^2 convention is eta = 1 here);
* angular functions are GAUSS with eta in {1/sqrt(0.005), 1/sqrt(0.02)} A
  (the reference's eta is a length: exp(-(rij^2+rik^2)/eta^2)), eta
  outermost so equal-eta runs share one damping factor, then
  zeta in {1,2,4,8} and lambda = +-1;
* an angular block of m functions takes m evenly spaced members of the
  16-function set eta x zeta x lambda (eta outermost), so every block
  spans zeta up to 8;
* networks are tanh with a linear output, Xavier-normal weights
  (sigma_w = 1), biases N(0, 0.001 * Xavier scale) (ml/nn.cpp:1193-1209);
* batched structures place atoms on a randomly chosen subset of a jittered
  grid in the (sheared) cell, which fixes the density exactly and keeps
  every pair at least ~0.7 A apart.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

from .potential import BasisA, BasisR, ElementType, Network, Potential, tt_index

ETA_A = (1.0 / math.sqrt(0.005), 1.0 / math.sqrt(0.02))
NAMES = ["A", "B", "C", "D", "E", "F", "G", "H"]


@dataclasses.dataclass
class Batch:
    """CSR batch of structures: atoms of structure s are atom_off[s]:atom_off[s+1].

    cell[s] holds the lattice vectors as rows (cell[s, n, :] = a_n), which is
    Cell::R (lattice vectors as columns) read column by column."""
    atom_off: np.ndarray   # int64 [n_struct+1]
    pos: np.ndarray        # float64 [N,3]
    type: np.ndarray       # int32 [N]
    cell: np.ndarray       # float64 [n_struct,3,3]
    pbc: bool = True

    @property
    def n_struct(self) -> int:
        return len(self.atom_off) - 1

    @property
    def n_atoms(self) -> int:
        return int(self.atom_off[-1])

    def structure(self, s: int):
        a, b = int(self.atom_off[s]), int(self.atom_off[s + 1])
        return self.pos[a:b], self.type[a:b], self.cell[s]

    def subset(self, idx: Sequence[int]) -> "Batch":
        pos, typ, cells, off = [], [], [], [0]
        for s in idx:
            p, t, c = self.structure(int(s))
            pos.append(p)
            typ.append(t)
            cells.append(c)
            off.append(off[-1] + len(p))
        return Batch(np.array(off, dtype=np.int64), np.concatenate(pos).reshape(-1, 3),
                     np.concatenate(typ).astype(np.int32), np.array(cells), self.pbc)


def angular_params(m: int):
    """m functions picked evenly from the 16-function set ordered eta-outermost:
    eta in ETA_A x (zeta, lambda) in (1,+1),(1,-1),(2,+1),(2,-1),...,(8,-1)."""
    full = [(e, z, l) for e in ETA_A for z in (1.0, 2.0, 4.0, 8.0) for l in (1, -1)]
    idx = np.round(np.linspace(0, len(full) - 1, m)).astype(int) if m > 1 else np.array([0])
    pick = [full[k] for k in idx]
    return (np.array([p[0] for p in pick]), np.array([p[1] for p in pick]),
            np.array([p[2] for p in pick], dtype=np.int32))


def xavier_net(rng: np.random.Generator, nodes: Sequence[int], neuron: str = "TANH") -> Network:
    b, w = [], []
    for l in range(len(nodes) - 1):
        ni, no = nodes[l], nodes[l + 1]
        s = math.sqrt(2.0 / (no + ni))
        b.append(rng.normal(0.0, 0.001 * s, size=no))
        w.append(rng.normal(0.0, 1.0 * s, size=(no, ni)))
    nin, nout = nodes[0], nodes[-1]
    return Network(list(nodes), neuron, 1.0, np.ones(nin), np.zeros(nin), np.ones(nout), np.zeros(nout), b, w)


def make_potential(ntypes: int, rc: float, n_rad: int, ang_sizes: Sequence[int], hidden: Sequence[int],
                   seed: int, neuron="TANH", cut: str = "COS",
                   energies: Optional[Sequence[float]] = None, rform: str = "GAUSSIAN",
                   aform: str = "GAUSS") -> Potential:
    """ntypes elements, n_rad radial functions per neighbour element, angular
    block sizes in TensorTri order (len = ntypes*(ntypes+1)/2).  neuron is one
    activation name for every element's network or a list of one per element;
    rform / aform name the radial / angular form (basis_radial.hpp:27-35,
    basis_angular.hpp:27-35), cut the cutoff (cutoff.hpp:23-29)."""
    TT = ntypes * (ntypes + 1) // 2
    if len(ang_sizes) != TT:
        raise ValueError("need %d angular block sizes" % TT)
    neurons = [neuron] * ntypes if isinstance(neuron, str) else list(neuron)
    if len(neurons) != ntypes:
        raise ValueError("need one activation per element")
    rng = np.random.default_rng(seed)
    types = [ElementType(name=NAMES[i], energy=(energies[i] if energies else -1.0 - 0.5 * i),
                         mass=1.0 + i) for i in range(ntypes)]
    rs = np.linspace(0.5, min(6.0, rc), n_rad) if n_rad > 1 else np.array([0.5])
    basis_r = [[BasisR(cut, rc, rform, rs.copy(), np.ones(n_rad)) for _ in range(ntypes)]
               for _ in range(ntypes)]
    basis_a = []
    for _ in range(ntypes):
        row = []
        for t in range(TT):
            e, z, l = angular_params(ang_sizes[t])
            row.append(BasisA(cut, rc, aform, e, z, l))
        basis_a.append(row)
    nin = ntypes * n_rad + sum(ang_sizes)
    nets = [xavier_net(rng, [nin] + list(hidden) + [1], neurons[i]) for i in range(ntypes)]
    return Potential(types, rc, basis_r, basis_a, nets)


# Potentials of the other basis forms, cutoffs and activations the reference
# supports, two or three elements each (6 radial functions per neighbour
# element, 4 angular per block, 24-16-16-1 or 30-16-16-1 networks):
# name -> (cutoff, radial form, angular form, activation of each element)
FORM_POTENTIALS = {
    "forms_sech_gauss2": ("TANH", "SECH", "GAUSS2", ["SIGMOID", "SWISH"]),
    "forms_logistic_sech": ("POLY3", "LOGISTIC", "SECH", ["GELU", "SOFTPLUS"]),
    "forms_tanh_student3": ("COS", "TANH", "STUDENT3", ["ISRU", "ARCTAN"]),
    "forms_logcosh_student4": ("TANH", "LOGCOSH", "STUDENT4", ["ELU", "MISH"]),
    "forms_logcosh2_student5": ("POLY3", "LOGCOSH2", "STUDENT5", ["PFLU", "LOGISH"]),
    "forms_step_gauss": ("STEP", "GAUSSIAN", "GAUSS", ["SQPLUS", "ATISH"]),
    "forms_activations": ("COS", "GAUSSIAN", "GAUSS", ["IERF", "TANHRE", "SQRE"]),
    "forms_relu_linear": ("COS", "SECH", "GAUSS2", ["RELU", "LINEAR"]),
}


def potential_forms(name: str, seed: int = 4321) -> Potential:
    cut, rform, aform, neurons = FORM_POTENTIALS[name]
    nt = len(neurons)
    return make_potential(nt, 6.0, 6, [4] * (nt * (nt + 1) // 2), [16, 16], seed, neuron=neurons, cut=cut,
                          rform=rform, aform=aform)


# --------------------------------------------------------------------------
# the benchmark configurations' potentials
# --------------------------------------------------------------------------

def potential_config(k: int, seed: int = 1234) -> Potential:
    if k == 1:   # 1 element, 16 radial + 16 angular, 32-20-20-1
        return make_potential(1, 6.0, 16, [16], [20, 20], seed)
    if k == 2:   # 3 elements, 3x8 radial + 32 angular, 56-32-32-1
        return make_potential(3, 6.0, 8, [6, 5, 5, 6, 5, 5], [32, 32], seed)
    if k == 3:   # 2 elements, 2x12 radial + 3x8 angular, 48-32-32-1
        return make_potential(2, 6.0, 12, [8, 8, 8], [32, 32], seed)
    if k == 4:   # 2 elements, 2x16 radial + 3x16 angular, 80-64-64-1, rc 6.5
        return make_potential(2, 6.5, 16, [16, 16, 16], [64, 64], seed)
    if k == 5:   # 4 elements, 4x6 radial + 10x4 angular, 64-48-48-1
        return make_potential(4, 6.0, 6, [4] * 10, [48, 48], seed)
    raise ValueError(k)


# --------------------------------------------------------------------------
# structures
# --------------------------------------------------------------------------

def _min_image_ok(p: np.ndarray, q: np.ndarray, L: float, dmin: float) -> bool:
    d = p[None, :] - q
    d -= L * np.round(d / L)
    return bool(np.all(np.einsum("ij,ij->i", d, d) >= dmin * dmin))


def config1(seed: int = 7, natoms: int = 64, side: float = 8.5, dmin: float = 1.8) -> Batch:
    """64 atoms, seeded uniform with rejection at dmin, cubic periodic cell."""
    rng = np.random.default_rng(seed)
    pos = np.zeros((0, 3))
    while len(pos) < natoms:
        p = rng.uniform(0.0, side, size=3)
        if len(pos) == 0 or _min_image_ok(p, pos, side, dmin):
            pos = np.vstack([pos, p])
    return Batch(np.array([0, natoms], dtype=np.int64), pos, np.zeros(natoms, dtype=np.int32),
                 np.eye(3)[None] * side, True)


def random_cell(rng: np.random.Generator, natoms: int, density: float, shear: float) -> np.ndarray:
    """Cube of volume N/density times (I+S), S off-diagonal U(-shear, shear).
    Returned with lattice vectors as rows."""
    L = (natoms / density) ** (1.0 / 3.0)
    S = rng.uniform(-shear, shear, size=(3, 3))
    np.fill_diagonal(S, 0.0)
    R = L * (np.eye(3) + S)          # columns are lattice vectors
    return R.T.copy()


def grid_positions(rng: np.random.Generator, natoms: int, cell_rows: np.ndarray,
                   sites_per_atom: float = 4.0, jitter: float = 0.3) -> np.ndarray:
    """Random subset of a jittered fractional grid mapped through the cell."""
    n = max(1, int(math.ceil((sites_per_atom * natoms) ** (1.0 / 3.0))))
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    pick = rng.choice(len(g), size=natoms, replace=False)
    frac = (g[pick] + 0.5 + rng.uniform(-jitter, jitter, size=(natoms, 3))) / n
    return frac @ cell_rows


def batch_random(seed: int, counts: Sequence[int], ntypes: int, density: float = 0.05,
                 shear: float = 0.1, dirichlet: bool = True) -> Batch:
    rng = np.random.default_rng(seed)
    off = np.zeros(len(counts) + 1, dtype=np.int64)
    off[1:] = np.cumsum(counts)
    pos = np.zeros((int(off[-1]), 3))
    typ = np.zeros(int(off[-1]), dtype=np.int32)
    cells = np.zeros((len(counts), 3, 3))
    for s, n in enumerate(counts):
        cells[s] = random_cell(rng, int(n), density, shear)
        pos[off[s]:off[s + 1]] = grid_positions(rng, int(n), cells[s])
        if ntypes > 1:
            p = rng.dirichlet(np.ones(ntypes)) if dirichlet else np.full(ntypes, 1.0 / ntypes)
            typ[off[s]:off[s + 1]] = rng.choice(ntypes, size=int(n), p=p)
    return Batch(off, pos, typ, cells, True)


def config2(seed: int = 11, n_struct: int = 4096, nmin: int = 16, nmax: int = 512) -> Batch:
    rng = np.random.default_rng(seed)
    counts = rng.integers(nmin, nmax + 1, size=n_struct)
    return batch_random(seed + 1, counts, 3)


def config3(seed: int = 13, n_struct: int = 256, nmin: int = 64, nmax: int = 256) -> Batch:
    rng = np.random.default_rng(seed)
    counts = rng.integers(nmin, nmax + 1, size=n_struct)
    return batch_random(seed + 1, counts, 2)


def config4(seed: int = 17, ncell: int = 32, a: float = 4.05, sigma: float = 0.1) -> Batch:
    """Jittered FCC, ncell^3 conventional cells, 50/50 two elements."""
    rng = np.random.default_rng(seed)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell), indexing="ij"), -1).reshape(-1, 3)
    pos = ((g[:, None, :] + basis[None]) * a).reshape(-1, 3)
    pos = pos + rng.normal(0.0, sigma, size=pos.shape)
    n = len(pos)
    typ = np.zeros(n, dtype=np.int32)
    typ[: n // 2] = 1
    rng.shuffle(typ)
    return Batch(np.array([0, n], dtype=np.int64), pos, typ, np.eye(3)[None] * (a * ncell), True)


def config5(seed: int = 19, n_struct: int = 20000, nmin: int = 8, nmax: int = 2048) -> Batch:
    rng = np.random.default_rng(seed)
    counts = np.floor(np.exp(rng.uniform(math.log(nmin), math.log(nmax + 1), size=n_struct))).astype(np.int64)
    counts = np.clip(counts, nmin, nmax)
    return batch_random(seed + 1, counts, 4)


def condition(pot: Potential, symm: np.ndarray, types: np.ndarray) -> Potential:
    """Set every network's input bias/scale from input statistics the way
    nnptefr's PREBIAS MEAN / PRESCALE DEV do (nnptefr.cpp:786-880):
    inpb = -mean(G), inpw = 1/dev(G) (1 where dev == 0), outb = 0, outw = 1.
    symm holds one row per atom (at least n_input(type) columns)."""
    for II in range(pot.ntypes):
        n = pot.n_input(II)
        g = symm[types == II, :n]
        net = pot.nets[II]
        if len(g) == 0:
            continue
        avg = g.mean(axis=0)
        dev = np.sqrt(((g - avg) ** 2).mean(axis=0))
        net.inpb = -avg
        net.inpw = np.where(dev == 0, 1.0, 1.0 / np.where(dev == 0, 1.0, dev))
        net.outb = np.zeros(1)
        net.outw = np.ones(1)
    return pot
