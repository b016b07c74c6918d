"""Potential model and the reference's potential text format.

A potential is a set of per-element Hamiltonians (NNH): for each centre
element II a radial basis per neighbour element J, an angular basis per
unordered neighbour pair (J,K) stored in TensorTri order, and an atomic
network.  ``write`` produces exactly the text ``NNP::write`` emits
(src/nnp/nnp.cpp:197-236, nnh.cpp:95-108, basis_radial.cpp:108-116,
basis_angular.cpp:101-109, ml/nn.cpp:1471-1511) and ``read`` parses it the
way ``NNP::read`` does (nnp.cpp:243-307), so files round-trip with the
reference.  Basis parameters are printed with ``%f`` and network
parameters with ``%.15f`` as in the reference, so a value that goes through
a file is rounded the same way on both sides.
"""
from __future__ import annotations

import dataclasses
from typing import List

import numpy as np

CUTOFFS = ["NONE", "STEP", "COS", "TANH", "POLY3"]                      # cutoff.hpp:23-29
RADIAL = ["NONE", "GAUSSIAN", "SECH", "LOGISTIC", "TANH", "LOGCOSH", "LOGCOSH2"]  # basis_radial.hpp:27-35
ANGULAR = ["NONE", "GAUSS", "GAUSS2", "SECH", "STUDENT3", "STUDENT4", "STUDENT5"]  # basis_angular.hpp:27-35
NEURONS = ["NONE", "LINEAR", "SIGMOID", "TANH", "ISRU", "ARCTAN", "RELU", "ELU", "TANHRE", "SQRE",
           "SWISH", "GELU", "MISH", "PFLU", "LOGISH", "SOFTPLUS", "SQPLUS", "ATISH", "IERF", "TEST"]  # nn.hpp:84-112
TYPE_FIELDS = ["energy", "mass", "charge", "radius", "z", "alpha", "ie", "rcov", "rvdw", "amp"]  # nnh.cpp:95-108


def tt_index(i: int, j: int) -> int:
    """TensorTri rank-2 linear index (src/nnp/tensortri.hpp:196-200)."""
    return i * (i + 1) // 2 + j if i > j else j * (j + 1) // 2 + i


@dataclasses.dataclass
class BasisR:
    cut: str
    rc: float
    form: str
    rs: np.ndarray
    eta: np.ndarray

    @property
    def size(self) -> int:
        return len(self.rs)


@dataclasses.dataclass
class BasisA:
    cut: str
    rc: float
    form: str
    eta: np.ndarray
    zeta: np.ndarray
    lam: np.ndarray

    @property
    def size(self) -> int:
        return len(self.eta)

    def rflag(self) -> np.ndarray:
        """Radial-damping groups: adjacent equal eta (BasisA::init, basis_angular.cpp:178-205)."""
        out = np.zeros(self.size, dtype=np.int32)
        flag = 0
        for n in range(1, self.size):
            if abs(self.eta[n] - self.eta[n - 1]) >= 1.0e-6:
                flag += 1
            out[n] = flag
        return out


@dataclasses.dataclass
class Network:
    """ANN: nodes = [n_in, h1, ..., n_out]; w[l] has shape (nodes[l+1], nodes[l])."""
    nodes: List[int]
    neuron: str
    c: float
    inpw: np.ndarray
    inpb: np.ndarray
    outw: np.ndarray
    outb: np.ndarray
    b: List[np.ndarray]
    w: List[np.ndarray]

    @property
    def nlayer(self) -> int:
        return len(self.nodes) - 1

    def nparams(self) -> int:
        return sum(self.nodes[l + 1] * (self.nodes[l] + 1) for l in range(self.nlayer))

    def pack(self) -> np.ndarray:
        """Parameter vector in the reference packing (ml/nn.cpp:881-894): all
        biases by layer, then each weight matrix column-major."""
        parts = [bb for bb in self.b] + [ww.reshape(-1, order="F") for ww in self.w]
        return np.concatenate(parts).astype(np.float64)

    def unpack(self, v: np.ndarray) -> None:
        """Inverse of ``pack`` (ml/nn.cpp:902-915)."""
        v = np.asarray(v, dtype=np.float64)
        if v.size != self.nparams():
            raise ValueError("Invalid size: vector and network mismatch.")
        k = 0
        for l in range(self.nlayer):
            n = self.nodes[l + 1]
            self.b[l] = v[k:k + n].copy()
            k += n
        for l in range(self.nlayer):
            no, ni = self.nodes[l + 1], self.nodes[l]
            self.w[l] = v[k:k + no * ni].reshape((no, ni), order="F").copy()
            k += no * ni


@dataclasses.dataclass
class ElementType:
    name: str
    energy: float = 0.0
    mass: float = 0.0
    charge: float = 0.0
    radius: float = 0.0
    z: float = 0.0
    alpha: float = 0.0
    ie: float = 0.0
    rcov: float = 0.0
    rvdw: float = 0.0
    amp: float = 0.0


@dataclasses.dataclass
class Potential:
    types: List[ElementType]
    rc: float
    basis_r: List[List[BasisR]]      # [II][J]
    basis_a: List[List[BasisA]]      # [II][tt]
    nets: List[Network]              # [II]

    @property
    def ntypes(self) -> int:
        return len(self.types)

    def index(self, name: str) -> int:
        for i, t in enumerate(self.types):
            if t.name == name:
                return i
        raise KeyError(name)

    def n_input_r(self, II: int) -> int:
        return sum(b.size for b in self.basis_r[II])

    def n_input(self, II: int) -> int:
        return self.n_input_r(II) + sum(b.size for b in self.basis_a[II])

    def offset_r(self, II: int) -> List[int]:
        """NNH::init_input radial offsets (nnh.cpp:186-191)."""
        out, s = [], 0
        for b in self.basis_r[II]:
            out.append(s)
            s += b.size
        return out

    def offset_a(self, II: int) -> List[int]:
        """NNH::init_input angular offsets, TensorTri linear order (nnh.cpp:193-198)."""
        out, s = [], 0
        for b in self.basis_a[II]:
            out.append(s)
            s += b.size
        return out

    def nparams(self) -> int:
        return sum(n.nparams() for n in self.nets)

    def get_params(self) -> np.ndarray:
        """All networks' packed parameters, types in index order (nnptefr.cpp:1171-1175)."""
        return np.concatenate([n.pack() for n in self.nets])

    def set_params(self, v: np.ndarray) -> None:
        k = 0
        for n in self.nets:
            m = n.nparams()
            n.unpack(v[k:k + m])
            k += m


# --------------------------------------------------------------------------
# text format
# --------------------------------------------------------------------------

def _f(x: float) -> str:
    return "%f" % x


def _f15(x: float) -> str:
    return "%.15f" % x


def write(path_or_file, pot: Potential) -> None:
    """NNP::write (nnp.cpp:197-236)."""
    lines = ["ann\n", "ntypes %i\n" % pot.ntypes]
    for t in pot.types:
        s = "name %s " % t.name
        for f in TYPE_FIELDS:
            s += "%s %s " % (f, _f(getattr(t, f)))
        lines.append(s + "\n")
    lines.append("rc %s\n" % _f(pot.rc))
    T = pot.ntypes
    for i in range(T):
        lines.append("basis %s\n" % pot.types[i].name)
        for j in range(T):
            lines.append("basis_radial %s\n" % pot.types[j].name)
            b = pot.basis_r[i][j]
            lines.append("BasisR %s %s %s %i\n" % (b.cut, _f(b.rc), b.form, b.size))
            for n in range(b.size):
                lines.append("\t%s %s\n" % (_f(b.rs[n]), _f(b.eta[n])))
        for j in range(T):
            for k in range(j, T):
                lines.append("basis_angular %s %s\n" % (pot.types[j].name, pot.types[k].name))
                b = pot.basis_a[i][tt_index(j, k)]
                lines.append("BasisA %s %s %s %i\n" % (b.cut, _f(b.rc), b.form, b.size))
                rf = b.rflag()
                for n in range(b.size):
                    lines.append("\t%s %s %i %i\n" % (_f(b.eta[n]), _f(b.zeta[n]), int(b.lam[n]), int(rf[n])))
    for i in range(T):
        lines.append("nn %s\n" % pot.types[i].name)
        nn = pot.nets[i]
        lines.append("nn " + "".join("%i " % n for n in nn.nodes) + "\n")
        lines.append("neuron %s %s\n" % (nn.neuron, _f(nn.c)))
        for tag, arr in (("inpw", nn.inpw), ("outw", nn.outw), ("inpb", nn.inpb), ("outb", nn.outb)):
            lines.append(tag + " " + "".join(_f15(x) + " " for x in arr) + "\n")
        for l in range(nn.nlayer):
            lines.append("bias[%i] " % (l + 1) + "".join(_f15(x) + " " for x in nn.b[l]) + "\n")
        for l in range(nn.nlayer):
            lines.append("weight[%i,%i] " % (l, l + 1) + "".join(_f15(x) + " " for x in nn.w[l].reshape(-1)) + "\n")
    text = "".join(lines)
    if hasattr(path_or_file, "write"):
        path_or_file.write(text)
    else:
        with open(path_or_file, "w") as fh:
            fh.write(text)


class _Lines:
    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.k = 0

    def next(self) -> List[str]:
        if self.k >= len(self.lines):
            raise ValueError("unexpected end of potential file")
        tok = self.lines[self.k].split()
        self.k += 1
        return tok


def _read_basis_r(L: _Lines) -> BasisR:
    h = L.next()       # BasisR <cut> <rc> <form> <n>   (basis_radial.cpp:123-143)
    n = int(h[4])
    rs, eta = np.zeros(n), np.zeros(n)
    for i in range(n):
        t = L.next()
        rs[i], eta[i] = float(t[0]), float(t[1])
    if h[1] not in CUTOFFS[1:] or h[3] not in RADIAL[1:]:
        raise ValueError("invalid radial basis header: %s" % " ".join(h))
    return BasisR(h[1], float(h[2]), h[3], rs, eta)


def _read_basis_a(L: _Lines) -> BasisA:
    h = L.next()       # BasisA <cut> <rc> <form> <n>   (basis_angular.cpp:116-138)
    n = int(h[4])
    eta, zeta, lam = np.zeros(n), np.zeros(n), np.zeros(n, dtype=np.int32)
    for i in range(n):
        t = L.next()
        eta[i], zeta[i], lam[i] = float(t[0]), float(t[1]), int(t[2])
    if h[1] not in CUTOFFS[1:] or h[3] not in ANGULAR[1:]:
        raise ValueError("invalid angular basis header: %s" % " ".join(h))
    return BasisA(h[1], float(h[2]), h[3], eta, zeta, lam)


def _read_net(L: _Lines) -> Network:
    nodes = [int(x) for x in L.next()[1:]]           # ml/nn.cpp:1558-1559
    t = L.next()
    neuron, c = t[1], float(t[2])
    if neuron not in NEURONS[1:]:
        raise ValueError("ANN::read(FILE*,ANN&): Invalid neuron.")
    nin, nout = nodes[0], nodes[-1]
    inpw = np.array([float(x) for x in L.next()[1:1 + nin]])
    outw = np.array([float(x) for x in L.next()[1:1 + nout]])
    inpb = np.array([float(x) for x in L.next()[1:1 + nin]])
    outb = np.array([float(x) for x in L.next()[1:1 + nout]])
    nl = len(nodes) - 1
    b = [np.array([float(x) for x in L.next()[1:1 + nodes[l + 1]]]) for l in range(nl)]
    w = []
    for l in range(nl):
        vals = np.array([float(x) for x in L.next()[1:1 + nodes[l + 1] * nodes[l]]])
        w.append(vals.reshape(nodes[l + 1], nodes[l]))
    return Network(nodes, neuron, c, inpw, inpb, outw, outb, b, w)


def read(path_or_text) -> Potential:
    """NNP::read (nnp.cpp:243-307)."""
    if "\n" in str(path_or_text):
        text = str(path_or_text)
    else:
        with open(path_or_text) as fh:
            text = fh.read()
    L = _Lines(text)
    L.next()                                  # header "ann"
    ntypes = int(L.next()[1])
    if ntypes <= 0:
        raise ValueError("NNP::read(FILE*,NNP&): invalid number of types.")
    types = []
    for _ in range(ntypes):
        tok = L.next()
        et = ElementType(name="NONE")
        k = 0
        while k < len(tok):                   # NNH::Type::read (nnh.cpp:65-93)
            tag = tok[k].upper()
            k += 1
            if tag == "NAME":
                et.name = tok[k]
                k += 1
            elif tag.lower() in TYPE_FIELDS:
                setattr(et, tag.lower(), float(tok[k]))
                k += 1
        types.append(et)
    names = [t.name for t in types]
    rc = float(L.next()[1])
    if rc <= 0:
        raise ValueError("NNP::read(FILE*,NNP&): invalid cutoff.")
    T = ntypes
    TT = T * (T + 1) // 2
    basis_r = [[None] * T for _ in range(T)]
    basis_a = [[None] * TT for _ in range(T)]
    for _ in range(T):
        II = names.index(L.next()[1])
        for _ in range(T):
            JJ = names.index(L.next()[1])
            basis_r[II][JJ] = _read_basis_r(L)
        for _ in range(TT):
            t = L.next()
            JJ, KK = names.index(t[1]), names.index(t[2])
            basis_a[II][tt_index(JJ, KK)] = _read_basis_a(L)
    nets = [None] * T
    for _ in range(T):
        II = names.index(L.next()[1])
        nets[II] = _read_net(L)
    pot = Potential(types, rc, basis_r, basis_a, nets)
    for II in range(T):
        if nets[II].nodes[0] != pot.n_input(II):
            raise ValueError("network input size %d != basis size %d for %s"
                             % (nets[II].nodes[0], pot.n_input(II), names[II]))
    return pot
