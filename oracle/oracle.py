"""ctypes front end of the FP64 oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product.  It has its own parser of
the reference's potential text format (NNP::read, src/nnp/nnp.cpp:243-307)
so that the product's C++ parser is checked against an independent reading
of the same file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
MAXL = 8

CUT = {"STEP": 1, "COS": 2, "TANH": 3, "POLY3": 4}
RAD = {"GAUSSIAN": 1, "SECH": 2, "LOGISTIC": 3, "TANH": 4, "LOGCOSH": 5, "LOGCOSH2": 6}
ANG = {"GAUSS": 1, "GAUSS2": 2, "SECH": 3, "STUDENT3": 4, "STUDENT4": 5, "STUDENT5": 6}
NEU = {n: i for i, n in enumerate(["NONE", "LINEAR", "SIGMOID", "TANH", "ISRU", "ARCTAN", "RELU", "ELU",
                                   "TANHRE", "SQRE", "SWISH", "GELU", "MISH", "PFLU", "LOGISH",
                                   "SOFTPLUS", "SQPLUS", "ATISH", "IERF", "TEST"])}


def build(force: bool = False) -> str:
    """Compile liboracle.so from oracle.c (no FMA contraction, as the reference
    is built without -march=native here)."""
    src = os.path.join(HERE, "oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        d, i, p = C.c_double, C.c_int, C.c_void_p
        _lib.orc_fmexp.restype = d
        _lib.orc_fmexp.argtypes = [d]
        _lib.orc_coscut.restype = d
        _lib.orc_coscut.argtypes = [d]
        _lib.orc_sincut.restype = d
        _lib.orc_sincut.argtypes = [d]
        _lib.orc_cutf.restype = d
        _lib.orc_cutf.argtypes = [i, d, d]
        _lib.orc_cutg.restype = d
        _lib.orc_cutg.argtypes = [i, d, d]
        _lib.orc_nlist.restype = i
        _lib.orc_nlist.argtypes = [d, i, p, p, i, i, p, p, p]
        _lib.orc_compute_symm.restype = i
        _lib.orc_compute_symm.argtypes = [p, i, p, p, p, i, i, p]
        _lib.orc_compute_energy.restype = d
        _lib.orc_compute_energy.argtypes = [p, i, p, i, p]
        _lib.orc_compute_force.restype = d
        _lib.orc_compute_force.argtypes = [p, i, p, p, p, i, i, p, p, p]
        _lib.orc_compute.restype = d
        _lib.orc_compute.argtypes = [p, i, p, p, p, i, i, p, p]
        _lib.orc_ann_fpbp.restype = d
        _lib.orc_ann_fpbp.argtypes = [p, i, p, p]
        _lib.orc_cost_grad.restype = d
        _lib.orc_cost_grad.argtypes = [p, i, p, p]
        _lib.orc_nparams.restype = i
        _lib.orc_nparams.argtypes = [p, i]
        _lib.orc_energy_loss_grad.restype = d
        _lib.orc_energy_loss_grad.argtypes = [p, i, p, p, i, p, p, i, i, d, p]
        _lib.orc_ef_loss_grad.restype = d
        _lib.orc_ef_loss_grad.argtypes = [p, i, p, p, p, p, i, p, p, d, i, i, d, p, p, p]
    return _lib


class _Pot(C.Structure):
    _fields_ = [("ntypes", C.c_int32), ("rc", C.c_double)] + [
        (n, C.c_void_p) for n in (
            "r_cut", "r_rc", "r_form", "r_n", "r_off", "r_rs", "r_eta",
            "a_cut", "a_rc", "a_form", "a_n", "a_off", "a_eta", "a_zeta", "a_lambda",
            "n_input", "n_input_r", "offset_r", "offset_a",
            "nn_nlayer", "nn_nodes", "nn_neuron", "nn_c", "nn_off", "nn_par", "energy")]


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _tt(i, j):
    return i * (i + 1) // 2 + j if i > j else j * (j + 1) // 2 + i


class OraclePot:
    """A potential flattened into the arrays of orc_pot (oracle.h)."""

    def __init__(self, text: str):
        self._parse(text)
        self._flatten()

    @classmethod
    def from_file(cls, path: str) -> "OraclePot":
        with open(path) as fh:
            return cls(fh.read())

    # -- parsing (NNP::read, nnp.cpp:243-307) --
    def _parse(self, text: str):
        lines = [ln.split() for ln in text.splitlines()]
        k = 1
        T = int(lines[k][1]); k += 1
        self.names, self.energy = [], []
        for _ in range(T):
            tok = lines[k]; k += 1
            name, e = "NONE", 0.0
            for q in range(0, len(tok) - 1):
                if tok[q].upper() == "NAME":
                    name = tok[q + 1]
                elif tok[q].upper() == "ENERGY":
                    e = float(tok[q + 1])
            self.names.append(name)
            self.energy.append(e)
        self.rc = float(lines[k][1]); k += 1
        TT = T * (T + 1) // 2
        self.T, self.TT = T, TT
        self.br = [None] * (T * T)
        self.ba = [None] * (T * TT)
        for _ in range(T):
            II = self.names.index(lines[k][1]); k += 1
            for _ in range(T):
                JJ = self.names.index(lines[k][1]); k += 1
                h = lines[k]; k += 1
                n = int(h[4])
                vals = np.array([[float(x) for x in lines[k + q][:2]] for q in range(n)]).reshape(n, 2)
                k += n
                self.br[II * T + JJ] = (CUT[h[1]], float(h[2]), RAD[h[3]], vals[:, 0].copy(), vals[:, 1].copy())
            for _ in range(TT):
                t = lines[k]; k += 1
                jk = _tt(self.names.index(t[1]), self.names.index(t[2]))
                h = lines[k]; k += 1
                n = int(h[4])
                vals = [lines[k + q] for q in range(n)]
                k += n
                self.ba[II * TT + jk] = (CUT[h[1]], float(h[2]), ANG[h[3]],
                                         np.array([float(v[0]) for v in vals]),
                                         np.array([float(v[1]) for v in vals]),
                                         np.array([int(v[2]) for v in vals], dtype=np.int32))
        self.nets = [None] * T
        for _ in range(T):
            II = self.names.index(lines[k][1]); k += 1
            nodes = [int(x) for x in lines[k][1:]]; k += 1
            neuron, c = lines[k][1], float(lines[k][2]); k += 1
            nin, nout, nl = nodes[0], nodes[-1], len(nodes) - 1
            inpw = [float(x) for x in lines[k][1:1 + nin]]; k += 1
            outw = [float(x) for x in lines[k][1:1 + nout]]; k += 1
            inpb = [float(x) for x in lines[k][1:1 + nin]]; k += 1
            outb = [float(x) for x in lines[k][1:1 + nout]]; k += 1
            b = []
            for l in range(nl):
                b.append(np.array([float(x) for x in lines[k][1:1 + nodes[l + 1]]])); k += 1
            w = []
            for l in range(nl):
                m = np.array([float(x) for x in lines[k][1:1 + nodes[l + 1] * nodes[l]]]); k += 1
                w.append(m.reshape(nodes[l + 1], nodes[l]))       # file order is row-major
            self.nets[II] = dict(nodes=nodes, neuron=NEU[neuron], c=c, inpw=inpw, inpb=inpb,
                                 outw=outw, outb=outb, b=b, w=w)

    def _flatten(self):
        T, TT = self.T, self.TT
        i32, f64 = np.int32, np.float64
        self.a = {}
        A = self.a
        A["r_cut"] = np.array([b[0] for b in self.br], i32)
        A["r_rc"] = np.array([b[1] for b in self.br], f64)
        A["r_form"] = np.array([b[2] for b in self.br], i32)
        A["r_n"] = np.array([len(b[3]) for b in self.br], i32)
        A["r_off"] = np.concatenate([[0], np.cumsum(A["r_n"])[:-1]]).astype(i32)
        A["r_rs"] = np.concatenate([b[3] for b in self.br] + [np.zeros(1)]).astype(f64)
        A["r_eta"] = np.concatenate([b[4] for b in self.br] + [np.zeros(1)]).astype(f64)
        A["a_cut"] = np.array([b[0] for b in self.ba], i32)
        A["a_rc"] = np.array([b[1] for b in self.ba], f64)
        A["a_form"] = np.array([b[2] for b in self.ba], i32)
        A["a_n"] = np.array([len(b[3]) for b in self.ba], i32)
        A["a_off"] = np.concatenate([[0], np.cumsum(A["a_n"])[:-1]]).astype(i32)
        A["a_eta"] = np.concatenate([b[3] for b in self.ba] + [np.zeros(1)]).astype(f64)
        A["a_zeta"] = np.concatenate([b[4] for b in self.ba] + [np.zeros(1)]).astype(f64)
        A["a_lambda"] = np.concatenate([b[5] for b in self.ba] + [np.zeros(1, i32)]).astype(i32)
        # NNH::init_input offsets (nnh.cpp:183-201)
        nir, ni = np.zeros(T, i32), np.zeros(T, i32)
        offr, offa = np.zeros(T * T, i32), np.zeros(T * TT, i32)
        for II in range(T):
            s = 0
            for J in range(T):
                offr[II * T + J] = s
                s += A["r_n"][II * T + J]
            nir[II] = s
            s2 = 0
            for t in range(TT):
                offa[II * TT + t] = s2
                s2 += A["a_n"][II * TT + t]
            ni[II] = s + s2
        A["n_input"], A["n_input_r"], A["offset_r"], A["offset_a"] = ni, nir, offr, offa
        A["nn_nlayer"] = np.array([len(n["nodes"]) - 1 for n in self.nets], i32)
        nodes = np.zeros(T * MAXL, i32)
        par, off = [], []
        pos = 0
        for II, n in enumerate(self.nets):
            nodes[II * MAXL: II * MAXL + len(n["nodes"])] = n["nodes"]
            v = list(n["inpw"]) + list(n["inpb"]) + list(n["outw"]) + list(n["outb"])
            for bb in n["b"]:
                v += list(bb)
            for ww in n["w"]:
                v += list(ww.reshape(-1, order="F"))
            off.append(pos)
            pos += len(v)
            par += v
        A["nn_nodes"] = nodes
        A["nn_neuron"] = np.array([n["neuron"] for n in self.nets], i32)
        A["nn_c"] = np.array([n["c"] for n in self.nets], f64)
        A["nn_off"] = np.array(off, np.int64)
        A["nn_par"] = np.array(par, f64)
        A["energy"] = np.array(self.energy, f64)
        self.s = _Pot()
        self.s.ntypes = T
        self.s.rc = self.rc
        for name in A:
            setattr(self.s, name, A[name].ctypes.data)
        self.ref = C.pointer(self.s)

    # -- helpers --
    @property
    def gstride(self) -> int:
        return int(self.a["n_input"].max())

    def nparams(self, II: int) -> int:
        return int(lib().orc_nparams(self.ref, II))

    def nparams_total(self) -> int:
        return sum(self.nparams(t) for t in range(self.T))

    def param_slice(self, II: int):
        """(offset, size) of type II's packed parameters inside nn_par."""
        n = self.nets[II]
        o = int(self.a["nn_off"][II]) + 2 * n["nodes"][0] + 2 * n["nodes"][-1]
        return o, self.nparams(II)

    def set_params(self, v: np.ndarray):
        k = 0
        for II in range(self.T):
            o, m = self.param_slice(II)
            self.a["nn_par"][o:o + m] = v[k:k + m]
            k += m

    def get_params(self) -> np.ndarray:
        return np.concatenate([self.a["nn_par"][o:o + m] for o, m in (self.param_slice(t) for t in range(self.T))])


def _struct_args(pos, cell):
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    cell = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
    return pos, cell


def nlist(rc, pos, cell, pbc=True, cap=512):
    pos, cell = _struct_args(pos, cell)
    n = len(pos)
    cnt = np.zeros(max(n, 1), np.int32)
    idx = np.zeros(max(n, 1) * cap, np.int32)
    img = np.zeros(max(n, 1) * cap * 3, np.float64)
    rcode = lib().orc_nlist(rc, n, _ptr(pos), _ptr(cell), int(pbc), cap, _ptr(cnt), _ptr(idx), _ptr(img))
    if rcode != 0:
        raise RuntimeError("oracle neighbour list overflow")
    out = []
    for i in range(n):
        c = int(cnt[i])
        out.append((idx[i * cap:i * cap + c].copy(), img[i * cap * 3:(i * cap + c) * 3].reshape(c, 3).copy()))
    return out


def compute(pot: OraclePot, pos, typ, cell, pbc=True):
    """NNP::compute: returns (E without vacuum, forces [N,3], symm [N,gstride])."""
    pos, cell = _struct_args(pos, cell)
    typ = np.ascontiguousarray(typ, dtype=np.int32)
    n = len(pos)
    gs = pot.gstride
    symm = np.zeros((max(n, 1), gs))
    force = np.zeros((max(n, 1), 3))
    e = lib().orc_compute(pot.ref, n, _ptr(pos), _ptr(typ), _ptr(cell), int(pbc), gs, _ptr(symm), _ptr(force))
    return e, force[:n], symm[:n]


def compute_symm(pot: OraclePot, pos, typ, cell, pbc=True):
    pos, cell = _struct_args(pos, cell)
    typ = np.ascontiguousarray(typ, dtype=np.int32)
    n = len(pos)
    symm = np.zeros((max(n, 1), pot.gstride))
    lib().orc_compute_symm(pot.ref, n, _ptr(pos), _ptr(typ), _ptr(cell), int(pbc), pot.gstride, _ptr(symm))
    return symm[:n]


def compute_energy(pot: OraclePot, typ, symm):
    typ = np.ascontiguousarray(typ, dtype=np.int32)
    symm = np.ascontiguousarray(symm, dtype=np.float64)
    return lib().orc_compute_energy(pot.ref, len(typ), _ptr(typ), symm.shape[1], _ptr(symm))


def compute_force(pot: OraclePot, pos, typ, cell, symm, pbc=True, want_dedg=False):
    pos, cell = _struct_args(pos, cell)
    typ = np.ascontiguousarray(typ, dtype=np.int32)
    symm = np.ascontiguousarray(symm, dtype=np.float64)
    n = len(pos)
    force = np.zeros((max(n, 1), 3))
    dedg = np.zeros((max(n, 1), symm.shape[1])) if want_dedg else None
    e = lib().orc_compute_force(pot.ref, n, _ptr(pos), _ptr(typ), _ptr(cell), int(pbc), symm.shape[1],
                                _ptr(symm), _ptr(force), _ptr(dedg) if want_dedg else None)
    return (e, force[:n], dedg[:n]) if want_dedg else (e, force[:n])


def compute_batch(pot: OraclePot, batch, want_symm=False):
    """Per-structure NNP::compute over a CSR batch: (E[n_struct] excl. vacuum, F[N,3])."""
    E = np.zeros(batch.n_struct)
    F = np.zeros((batch.n_atoms, 3))
    G = np.zeros((batch.n_atoms, pot.gstride)) if want_symm else None
    for s in range(batch.n_struct):
        p, t, c = batch.structure(s)
        a = int(batch.atom_off[s])
        E[s], f, g = compute(pot, p, t, c, batch.pbc)
        F[a:a + len(p)] = f
        if want_symm:
            G[a:a + len(p)] = g
    return (E, F, G) if want_symm else (E, F)


def ann_fpbp(pot: OraclePot, II, inp):
    inp = np.ascontiguousarray(inp, dtype=np.float64)
    dodi = np.zeros(len(inp))
    out = lib().orc_ann_fpbp(pot.ref, II, _ptr(inp), _ptr(dodi))
    return out, dodi


def cost_grad(pot: OraclePot, II, inp):
    inp = np.ascontiguousarray(inp, dtype=np.float64)
    g = np.zeros(pot.nparams(II))
    out = lib().orc_cost_grad(pot.ref, II, _ptr(inp), _ptr(g))
    return out, g


def energy_loss_grad(pot: OraclePot, atom_off, typ, symm, e_ref, norm_mode=1, loss_kind=1, delta=1.0):
    atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
    typ = np.ascontiguousarray(typ, dtype=np.int32)
    symm = np.ascontiguousarray(symm, dtype=np.float64)
    e_ref = np.ascontiguousarray(e_ref, dtype=np.float64)
    g = np.zeros(pot.nparams_total())
    loss = lib().orc_energy_loss_grad(pot.ref, len(atom_off) - 1, _ptr(atom_off), _ptr(typ), symm.shape[1],
                                      _ptr(symm), _ptr(e_ref), norm_mode, loss_kind, float(delta), _ptr(g))
    return loss, g


def ef_loss_grad(pot: OraclePot, batch, e_ref, f_ref, w_f, norm_mode=1, want_grad=True, loss_kind=1, delta=1.0):
    off = np.ascontiguousarray(batch.atom_off, dtype=np.int64)
    pos = np.ascontiguousarray(batch.pos, dtype=np.float64)
    typ = np.ascontiguousarray(batch.type, dtype=np.int32)
    cell = np.ascontiguousarray(batch.cell, dtype=np.float64)
    e_ref = np.ascontiguousarray(e_ref, dtype=np.float64)
    f_ref = np.ascontiguousarray(f_ref, dtype=np.float64)
    g = np.zeros(pot.nparams_total()) if want_grad else None
    eo = np.zeros(batch.n_struct)
    fo = np.zeros((batch.n_atoms, 3))
    loss = lib().orc_ef_loss_grad(pot.ref, batch.n_struct, _ptr(off), _ptr(pos), _ptr(typ), _ptr(cell),
                                  int(batch.pbc), _ptr(e_ref), _ptr(f_ref), float(w_f), norm_mode, loss_kind,
                                  float(delta), _ptr(g) if want_grad else None, _ptr(eo), _ptr(fo))
    return loss, g, eo, fo
