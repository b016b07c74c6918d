"""Python front end of libnnp_b200.so (the C ABI in include/nnp_b200.h).

``NNP`` keeps the method names of the reference's ``NNP`` class
(src/nnp/nnp.hpp:64-121): ``read``, ``write``, ``compute_symm``,
``compute_energy``, ``compute_force``, ``compute``, ``index``, ``ntypes``,
``rc``.  Errors raise ``NNPError`` (the reference throws
``std::invalid_argument`` / ``std::runtime_error``).  The library is loaded
from this package directory; there is no fallback when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libnnp_b200.so")

NNP_OK = 0
ERRORS = {-1: "ARG", -2: "IO", -3: "PARSE", -4: "CUDA", -5: "CAPACITY", -6: "UNSUPPORTED", -7: "TYPE",
          -8: "NOT_FINITE"}
PREC_FP32, PREC_BF16, PREC_BF16X3 = 0, 1, 2
ACC_FP32, ACC_FP64, SYMM_FP64 = 0, 1, 2
LOSS_MSE, LOSS_MAE, LOSS_HUBER, LOSS_ASINH = 1, 2, 3, 4   # opt::Loss (opt/loss.hpp:18-24)
DECAY = {"CONST": 1, "EXP": 2, "GAUSS": 3, "SQRT": 4, "INV": 5, "STEP": 6}   # opt::Decay::Name
REG = {"LASSO": 0, "RIDGE": 1, "HUBER": 2, "ASINH": 3, "NONE": 4}              # Regularization
STATS = ("max", "min", "harmonic", "mean", "dev", "rms")   # nnp_input_stats, NNP_STAT_* order
PREBIAS = {"IDENTITY": 0, "MEAN": 1, "HAR": 2, "RMS": 3, "MID": 4, "MIN": 5}      # nnptefr.hpp:97-107
PRESCALE = {"IDENTITY": 0, "DEV": 1, "MINMAX": 2, "MAX": 3}                     # nnptefr.hpp:69-77
ENERGY, FORCES, VACUUM, DEVICE_PTRS, SYMM = 1, 2, 4, 8, 16


class NNPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%s)" % (msg, ERRORS.get(code, code)))
        self.code = code


class _Batch(C.Structure):
    _fields_ = [("n_struct", C.c_int32), ("atom_off", C.c_void_p), ("pos", C.c_void_p), ("type", C.c_void_p),
                ("cell", C.c_void_p), ("pbc", C.c_int32)]


_lib = None


def lib():
    """Load the CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise ImportError("libnnp_b200.so is not built (run make -C ace_b200 or __graft_entry__.build())")
        L = C.CDLL(LIBPATH)
        p, i, d, u = C.c_void_p, C.c_int32, C.c_double, C.c_uint32
        sig = {
            "nnp_create_from_file": ([C.c_char_p, C.POINTER(p)], i),
            "nnp_create_from_basis": ([i, p, d, p, p, C.POINTER(p)], i),
            "nnp_destroy": ([p], i),
            "nnp_write": ([p, C.c_char_p], i),
            "nnp_set_precision": ([p, i], i),
            "nnp_set_stream": ([p, p], i),
            "nnp_ntypes": ([p, C.POINTER(i)], i),
            "nnp_type_index": ([p, C.c_char_p, C.POINTER(i)], i),
            "nnp_rc": ([p, C.POINTER(d)], i),
            "nnp_n_input": ([p, i, C.POINTER(i)], i),
            "nnp_compute": ([p, C.POINTER(_Batch), p, p, p, u], i),
            "nnp_compute_md": ([p, C.POINTER(_Batch), p, p, p, p, u], i),
            "nnp_compute_local_ghost": ([p, C.c_int64, C.c_int64, p, p, p, p, p, p, u], i),
            "nnp_input_stats": ([p, C.POINTER(_Batch), p, p], i),
            "nnp_read_structures": ([i, p, C.c_char_p, i, C.POINTER(i), C.POINTER(C.c_int64), p, p, p, p, p, p, p], i),
            "nnp_type_name": ([p, i, C.POINTER(C.c_char_p)], i),
            "nnp_taylor_expand": ([i, p, p, p, p, p, i, i, d, C.c_uint64, p, p, p, p, p, C.POINTER(i)], i),
            "nnp_precondition": ([p, C.POINTER(_Batch), i, i, d, d], i),
            "nnp_set_graphs": ([p, i], i),
            "nnp_compute_energy_symm": ([p, i, p, p, p, i, p], i),
            "nnp_nparams": ([p, i, C.POINTER(i)], i),
            "nnp_get_params": ([p, p], i),
            "nnp_set_params": ([p, p], i),
            "nnp_train_grad": ([p, C.POINTER(_Batch), p, p, d, i, p, p, p, p, u], i),
            "nnp_set_loss": ([p, i, d], i),
            "nnp_opt_adam": ([p, d, d], i),
            "nnp_opt_reset": ([p], i),
            "nnp_opt_step": ([p, C.POINTER(d), i, i, d, i, i, d, d], i),
            "nnp_decay_step": ([i, d, i, d, i, C.POINTER(d)], i),
            "nnp_set_mma_wait": ([p, C.c_int64], i),
            "nnp_set_autotune": ([p, i], i),
            "nnp_tune_params": ([p, p, i, C.POINTER(i), C.POINTER(C.c_char_p)], i),
            "nnp_tune_cache_key": ([C.c_char_p, C.c_char_p, i, i, C.c_char_p, i], i),
            "nnp_tune_cache_store": ([C.c_char_p, p, i], i),
            "nnp_tune_cache_load": ([C.c_char_p, p, i], i),
            "nnp_set_accumulation": ([p, i], i),
            "nnp_set_specialization": ([p, i], i),
            "nnp_specialization": ([p, C.POINTER(i), C.POINTER(C.c_char_p)], i),
            "nnp_set_timing": ([p, i], i),
            "nnp_stage_times": ([p, p, i], i),
            "nnp_neighbor_counts": ([p, p], i),
            "nnp_launch_count": ([p, C.POINTER(C.c_int64)], i),
            "nnp_last_error": ([p], C.c_char_p),
            "nnp_version": ([], C.c_char_p),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class NNP:
    """A potential resident on the GPU (one C-ABI handle)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self.precision = PREC_FP32

    # ---- construction: NNP::read (nnp.cpp:181-190)
    @classmethod
    def read(cls, path: str) -> "NNP":
        h = C.c_void_p()
        rc = lib().nnp_create_from_file(os.fsencode(path), C.byref(h))
        if rc != NNP_OK:
            raise NNPError(rc, lib().nnp_last_error(None).decode())
        return cls(h)

    @classmethod
    def from_basis(cls, type_lines: Sequence[str], rc: float, basis_paths: Sequence[str],
                   network_texts: Sequence[str]) -> "NNP":
        """NNP::read_basis per element + a network per element (nnptefr.cpp:2023-2031)."""
        n = len(type_lines)
        tl = (C.c_char_p * n)(*[s.encode() for s in type_lines])
        bp = (C.c_char_p * n)(*[os.fsencode(s) for s in basis_paths])
        nt = (C.c_char_p * n)(*[s.encode() for s in network_texts])
        h = C.c_void_p()
        r = lib().nnp_create_from_basis(n, C.cast(tl, C.c_void_p), float(rc), C.cast(bp, C.c_void_p),
                                        C.cast(nt, C.c_void_p), C.byref(h))
        if r != NNP_OK:
            raise NNPError(r, lib().nnp_last_error(None).decode())
        return cls(h)

    def close(self):
        if self._h:
            lib().nnp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != NNP_OK:
            raise NNPError(rc, lib().nnp_last_error(self._h).decode())

    # ---- NNP::write (nnp.cpp:165-174)
    def write(self, path: str):
        self._check(lib().nnp_write(self._h, os.fsencode(path)))

    # ---- access (nnp.hpp:78-87)
    @property
    def ntypes(self) -> int:
        v = C.c_int32()
        self._check(lib().nnp_ntypes(self._h, C.byref(v)))
        return v.value

    @property
    def rc(self) -> float:
        v = C.c_double()
        self._check(lib().nnp_rc(self._h, C.byref(v)))
        return v.value

    def index(self, name: str) -> int:
        v = C.c_int32()
        self._check(lib().nnp_type_index(self._h, name.encode(), C.byref(v)))
        return v.value

    def n_input(self, t: int) -> int:
        v = C.c_int32()
        self._check(lib().nnp_n_input(self._h, t, C.byref(v)))
        return v.value

    @property
    def gstride(self) -> int:
        g = max(self.n_input(t) for t in range(self.ntypes))
        return (g + 3) & ~3

    def set_precision(self, prec: int):
        self._check(lib().nnp_set_precision(self._h, prec))
        self.precision = prec

    def set_loss(self, kind: int, delta: float = 1.0):
        """Energy-loss kind of train_grad (LOSS_MSE, LOSS_MAE, LOSS_HUBER,
        LOSS_ASINH) and its width, as nnptefr's loss / delta settings."""
        self._check(lib().nnp_set_loss(self._h, kind, float(delta)))

    def opt_adam(self, gamma: float, eps: float = 1e-16):
        """One ADAM step on the device with the last train_grad gradient."""
        self._check(lib().nnp_opt_adam(self._h, float(gamma), float(eps)))

    def opt_step(self, gamma: float, step: int, decay="CONST", alpha=0.0, period=0, reg="NONE", eta=0.0,
                 eps: float = 1e-16) -> float:
        """nnptefr's optimiser step on the device: decayed rate, ADAM, weight
        decay; returns the rate used."""
        g = C.c_double(gamma)
        dk = DECAY[decay] if isinstance(decay, str) else decay
        rk = REG[reg] if isinstance(reg, str) else reg
        self._check(lib().nnp_opt_step(self._h, C.byref(g), int(step), int(dk), float(alpha), int(period), int(rk),
                                       float(eta), float(eps)))
        return g.value

    def opt_reset(self):
        self._check(lib().nnp_opt_reset(self._h))

    def set_mma_wait(self, polls: int):
        """Bound of each tensor-core MMA-chain wait (0: the default)."""
        self._check(lib().nnp_set_mma_wait(self._h, int(polls)))

    def type_names(self):
        out = []
        for t in range(self.ntypes):
            v = C.c_char_p()
            self._check(lib().nnp_type_name(self._h, t, C.byref(v)))
            out.append(v.value.decode())
        return out

    def read_structures(self, path: str, fmt: str = "xyz"):
        """read_structures with this potential's element names."""
        return read_structures(path, self.type_names(), fmt)

    def _batch(self, atom_off, pos, types, cells, pbc):
        atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        types = np.ascontiguousarray(types, dtype=np.int32)
        S = len(atom_off) - 1
        cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(S, 9) if pbc else None
        keep = (atom_off, pos, types, cells)
        return _Batch(S, atom_off.ctypes.data, pos.ctypes.data, types.ctypes.data,
                      cells.ctypes.data if cells is not None else None, 1 if pbc else 0), keep

    def input_stats(self, atom_off, pos, types, cells, pbc=True):
        """Per-element statistics of the network inputs over a batch
        (nnptefr.cpp:689-781): (count [ntypes], {name: array [ntypes, gstride]})."""
        b, keep = self._batch(atom_off, pos, types, cells, pbc)
        T = self.ntypes
        gs = max(self.n_input(t) for t in range(T))
        gs = (gs + 3) & ~3
        cnt = np.zeros(T, dtype=np.int64)
        st = np.zeros((T, len(STATS), gs))
        self._check(lib().nnp_input_stats(self._h, C.byref(b), _ptr(cnt), _ptr(st)))
        return cnt, {name: st[:, k, :] for k, name in enumerate(STATS)}

    def precondition(self, atom_off, pos, types, cells, prebias="MEAN", prescale="DEV", inbias=0.0, inscale=1.0,
                     pbc=True):
        """nnptefr's input preconditioning (nnptefr.cpp:783-880) from the batch's statistics."""
        b, keep = self._batch(atom_off, pos, types, cells, pbc)
        pb = PREBIAS.get(prebias, prebias) if isinstance(prebias, str) else prebias
        ps = PRESCALE.get(prescale, prescale) if isinstance(prescale, str) else prescale
        self._check(lib().nnp_precondition(self._h, C.byref(b), int(pb) if not isinstance(pb, str) else 99,
                                           int(ps) if not isinstance(ps, str) else 99, float(inbias),
                                           float(inscale)))

    def compute_local_ghost(self, pos_local, type_local, pos_ghost, type_ghost, vacuum=False):
        """One domain of a pair style: local atoms then ghost atoms, no cell.
        Returns (energy of the local atoms, forces [n_local + n_ghost, 3],
        per-atom energies [n_local], virial [3, 3])."""
        pos = np.ascontiguousarray(np.concatenate([np.reshape(pos_local, (-1, 3)), np.reshape(pos_ghost, (-1, 3))]),
                                   dtype=np.float64)
        typ = np.ascontiguousarray(np.concatenate([np.asarray(type_local), np.asarray(type_ghost)]), dtype=np.int32)
        nl, ng = len(pos_local), len(pos_ghost)
        e = np.zeros(1)
        f = np.zeros((max(nl + ng, 1), 3))
        ea = np.zeros(max(nl, 1))
        w = np.zeros(9)
        self._check(lib().nnp_compute_local_ghost(self._h, nl, ng, _ptr(pos), _ptr(typ), _ptr(e), _ptr(f), _ptr(ea),
                                                  _ptr(w), VACUUM if vacuum else 0))
        return float(e[0]), f[:nl + ng], ea[:nl], w.reshape(3, 3)

    def set_autotune(self, on: bool = True):
        """Tune the kernels' launch and tile choices on the first energy+force
        call of each neighbour-capacity class (cached on disk)."""
        self._check(lib().nnp_set_autotune(self._h, 1 if on else 0))

    TUNE_NAMES = ("symm_minb", "force_minb", "force_unroll", "force_chunk", "tc_per_sm")

    def tune_params(self):
        """(choices as a dict, source: "default" | "cache" | "tuned", log)."""
        v = np.zeros(5, dtype=np.int32)
        src = C.c_int32()
        log = C.c_char_p()
        self._check(lib().nnp_tune_params(self._h, _ptr(v), 5, C.byref(src), C.byref(log)))
        return (dict(zip(self.TUNE_NAMES, (int(x) for x in v))), ("default", "cache", "tuned")[src.value],
                (log.value or b"").decode())

    def set_graphs(self, on: bool = True):
        """Replay the device-side step as a CUDA graph while calls repeat their shape."""
        self._check(lib().nnp_set_graphs(self._h, 1 if on else 0))

    def set_accumulation(self, mode=1):
        """Precision of the symmetry functions: ACC_FP32 (0, or False), ACC_FP64
        (1, or True: FP64 running sums of FP32 terms) or SYMM_FP64 (2: FP64
        terms and sums)."""
        self._check(lib().nnp_set_accumulation(self._h, int(mode)))

    def set_specialization(self, on: bool = True):
        """Use the kernels compiled for this basis at creation (True) or the prebuilt ones."""
        self._check(lib().nnp_set_specialization(self._h, 1 if on else 0))

    def specialization(self):
        """(active, CUDA source of the specialised kernels)."""
        a = C.c_int32()
        s = C.c_char_p()
        self._check(lib().nnp_specialization(self._h, C.byref(a), C.byref(s)))
        return bool(a.value), (s.value or b"").decode()

    def set_stream(self, stream_ptr: int):
        self._check(lib().nnp_set_stream(self._h, C.c_void_p(stream_ptr)))

    # ---- stage timers (the reference's phase clocks) and counters
    STAGES = ("neighbors", "symm", "networks", "forces", "energies")

    def set_timing(self, on: bool = True):
        self._check(lib().nnp_set_timing(self._h, 1 if on else 0))

    def stage_times(self) -> dict:
        ms = np.zeros(5, dtype=np.float32)
        self._check(lib().nnp_stage_times(self._h, _ptr(ms), 5))
        return dict(zip(self.STAGES, (float(x) for x in ms)))

    def launch_count(self) -> int:
        v = C.c_int64()
        self._check(lib().nnp_launch_count(self._h, C.byref(v)))
        return v.value

    def neighbor_counts(self, n_atoms: int) -> np.ndarray:
        """[N, ntypes] neighbour counts by type of the last compute call."""
        c = np.zeros((max(n_atoms, 1), self.ntypes), dtype=np.int32)
        self._check(lib().nnp_neighbor_counts(self._h, _ptr(c)))
        return c[:n_atoms]

    def nparams(self, t: int = -1) -> int:
        v = C.c_int32()
        self._check(lib().nnp_nparams(self._h, t, C.byref(v)))
        return v.value

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.nparams())
        self._check(lib().nnp_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float64)
        if p.size != self.nparams():
            raise NNPError(-1, "Invalid size: vector and network mismatch.")
        self._check(lib().nnp_set_params(self._h, _ptr(p)))

    # ---- batched compute
    def compute_batch(self, atom_off, pos, types, cells, pbc=True, energy=True, forces=True,
                      symm=False, vacuum=False, out_e=None, out_f=None):
        """Energies [n_struct], forces [N,3] (and symmetry functions [N,gstride]) of a CSR batch.
        out_e / out_f may be caller-owned (e.g. pinned) float64 arrays to write into."""
        atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        types = np.ascontiguousarray(types, dtype=np.int32)
        S = len(atom_off) - 1
        cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(S, 9) if pbc else None
        N = int(atom_off[-1]) if S else 0
        b = _Batch(S, atom_off.ctypes.data, pos.ctypes.data, types.ctypes.data,
                   cells.ctypes.data if cells is not None else None, 1 if pbc else 0)
        E = out_e if out_e is not None else np.zeros(max(S, 1))
        F = out_f if out_f is not None else np.zeros((max(N, 1), 3))
        if E.dtype != np.float64 or not E.flags.c_contiguous or F.dtype != np.float64 or not F.flags.c_contiguous:
            raise NNPError(-1, "output arrays must be contiguous float64")
        gs = self.gstride
        G = np.zeros((max(N, 1), gs)) if symm else None
        flags = (ENERGY if energy else 0) | (FORCES if forces else 0) | (SYMM if symm else 0) | (VACUUM if vacuum else 0)
        self._check(lib().nnp_compute(self._h, C.byref(b), _ptr(E), _ptr(F), _ptr(G), flags))
        out = [E[:S], F[:N]]
        if symm:
            out.append(G[:N])
        return tuple(out)

    def compute_md(self, atom_off, pos, types, cells, pbc=True, vacuum=False):
        """nnp_compute_md: energies [n_struct], forces [N,3], per-atom energies
        [N] and virials [n_struct,3,3] (W = -dE/d strain, eV)."""
        atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        types = np.ascontiguousarray(types, dtype=np.int32)
        S = len(atom_off) - 1
        cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(S, 9) if pbc else None
        N = int(atom_off[-1]) if S else 0
        b = _Batch(S, atom_off.ctypes.data, pos.ctypes.data, types.ctypes.data,
                   cells.ctypes.data if cells is not None else None, 1 if pbc else 0)
        E = np.zeros(max(S, 1))
        F = np.zeros((max(N, 1), 3))
        A = np.zeros(max(N, 1))
        W = np.zeros((max(S, 1), 3, 3))
        self._check(lib().nnp_compute_md(self._h, C.byref(b), _ptr(E), _ptr(F), _ptr(A), _ptr(W),
                                         VACUUM if vacuum else 0))
        return E[:S], F[:N], A[:N], W[:S]

    def compute_device(self, atom_off_ptr: int, pos_ptr: int, type_ptr: int, cell_ptr: int, n_struct: int,
                       energy_ptr: int, force_ptr: int, pbc: bool = True, vacuum: bool = False):
        """Same as compute_batch on device-resident arrays (raw CUDA pointers)."""
        b = _Batch(n_struct, atom_off_ptr, pos_ptr, type_ptr, cell_ptr, 1 if pbc else 0)
        flags = ENERGY | FORCES | DEVICE_PTRS | (VACUUM if vacuum else 0)
        self._check(lib().nnp_compute(self._h, C.byref(b), C.c_void_p(energy_ptr), C.c_void_p(force_ptr), None,
                                      flags))

    # ---- per-structure calls with the reference's names and semantics
    def compute_symm(self, pos, types, cell, pbc=True) -> np.ndarray:
        """NNP::compute_symm (nnp.cpp:350-398): symmetry functions, one row per atom."""
        n = len(types)
        _, _, G = self.compute_batch([0, n], pos, types, cell, pbc, energy=False, forces=False, symm=True)
        return G

    def compute_energy(self, types, symm) -> float:
        """NNP::compute_energy (nnp.cpp:329-338): sum of network(G) + vacuum energies."""
        types = np.ascontiguousarray(types, dtype=np.int32)
        symm = np.ascontiguousarray(symm, dtype=np.float64)
        off = np.array([0, len(types)], dtype=np.int64)
        E = np.zeros(1)
        self._check(lib().nnp_compute_energy_symm(self._h, 1, _ptr(off), _ptr(types), _ptr(symm), symm.shape[1],
                                                  _ptr(E)))
        return float(E[0])

    def compute_force(self, pos, types, cell, pbc=True):
        """NNP::compute_force (nnp.cpp:412-482): (energy without vacuum terms, forces)."""
        n = len(types)
        E, F = self.compute_batch([0, n], pos, types, cell, pbc)
        return float(E[0]), F

    compute = compute_force   # NNP::compute (nnp.cpp:489-494) = build + symm + force

    def train_grad_device(self, atom_off_ptr: int, pos_ptr: int, type_ptr: int, cell_ptr: int, n_struct: int,
                          e_ref_ptr: int, f_ref_ptr: int, w_f: float, loss_ptr: int, grad_ptr: int = 0,
                          norm_mode: int = 1, pbc: bool = True):
        """train_grad on device-resident arrays (raw CUDA pointers); loss and
        grad (optional) are device pointers too."""
        b = _Batch(n_struct, atom_off_ptr, pos_ptr, type_ptr, cell_ptr, 1 if pbc else 0)
        self._check(lib().nnp_train_grad(self._h, C.byref(b), C.c_void_p(e_ref_ptr), C.c_void_p(f_ref_ptr or None),
                                         float(w_f), norm_mode, C.c_void_p(loss_ptr), C.c_void_p(grad_ptr or None),
                                         None, None, DEVICE_PTRS))

    def train_grad(self, atom_off, pos, types, cells, e_ref, f_ref, w_f, norm_mode=1, pbc=True):
        """Energy+force loss, its weight gradient, and the model's E and F."""
        atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        types = np.ascontiguousarray(types, dtype=np.int32)
        S = len(atom_off) - 1
        N = int(atom_off[-1])
        cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(S, 9)
        e_ref = np.ascontiguousarray(e_ref, dtype=np.float64)
        f_ref = np.ascontiguousarray(f_ref, dtype=np.float64).reshape(-1, 3)
        b = _Batch(S, atom_off.ctypes.data, pos.ctypes.data, types.ctypes.data, cells.ctypes.data, 1 if pbc else 0)
        loss = np.zeros(1)
        g = np.zeros(self.nparams())
        eo = np.zeros(S)
        fo = np.zeros((N, 3))
        self._check(lib().nnp_train_grad(self._h, C.byref(b), _ptr(e_ref), _ptr(f_ref), float(w_f), norm_mode,
                                         _ptr(loss), _ptr(g), _ptr(eo), _ptr(fo), 0))
        return float(loss[0]), g, eo, fo


def tune_cache_key(potential_path: str, device_name: str, n_sm: int, cap: int) -> str:
    """Key of the tuning cache for a potential on a GPU model and capacity (no GPU needed)."""
    buf = C.create_string_buffer(256)
    rc = lib().nnp_tune_cache_key(os.fsencode(potential_path), device_name.encode(), n_sm, cap, buf, len(buf))
    if rc != NNP_OK:
        raise NNPError(rc, "tune_cache_key failed")
    return buf.value.decode()


def tune_cache_store(key: str, params: dict) -> None:
    v = np.array([params[k] for k in NNP.TUNE_NAMES], dtype=np.int32)
    rc = lib().nnp_tune_cache_store(key.encode(), _ptr(v), 5)
    if rc != NNP_OK:
        raise NNPError(rc, "tune_cache_store failed")


def tune_cache_load(key: str):
    """The stored choices of key as a dict, or None."""
    v = np.zeros(5, dtype=np.int32)
    rc = lib().nnp_tune_cache_load(key.encode(), _ptr(v), 5)
    return None if rc != NNP_OK else dict(zip(NNP.TUNE_NAMES, (int(x) for x in v)))


DISTRIBUTIONS = {"UNIFORM": 1, "LAPLACE": 2, "NORMAL": 3, "SECH": 5, "LOGISTIC": 6, "COSINE": 7}   # rng::dist::Name


def taylor_expand(atom_off, pos, types, energy, forces, nadd, dist="NORMAL", rdelta=0.01, seed=0):
    """nnptefr's force perturbation on the GPU (nnptefr.cpp:2733-2830):
    returns (atom_off, pos [N',3], types [N'], energy [S'], source structure [S'])."""
    atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    types = np.ascontiguousarray(types, dtype=np.int32)
    energy = np.ascontiguousarray(energy, dtype=np.float64)
    forces = np.ascontiguousarray(forces, dtype=np.float64).reshape(-1, 3)
    S = len(atom_off) - 1
    N = int(atom_off[-1]) if S else 0
    So, No = S * (1 + nadd), N * (1 + nadd)
    oo = np.zeros(So + 1, dtype=np.int64)
    op = np.zeros((max(No, 1), 3))
    ot = np.zeros(max(No, 1), dtype=np.int32)
    oe = np.zeros(max(So, 1))
    osrc = np.zeros(max(So, 1), dtype=np.int32)
    n = C.c_int32()
    d = DISTRIBUTIONS.get(dist, dist) if isinstance(dist, str) else dist
    rc = lib().nnp_taylor_expand(S, _ptr(atom_off), _ptr(pos), _ptr(types), _ptr(energy), _ptr(forces), int(nadd),
                                 int(d) if not isinstance(d, str) else 0, float(rdelta), int(seed) & (2**64 - 1),
                                 _ptr(oo), _ptr(op), _ptr(ot), _ptr(oe), _ptr(osrc), C.byref(n))
    if rc != NNP_OK:
        raise NNPError(rc, lib().nnp_last_error(None).decode())
    k = n.value
    na = int(oo[k])
    return oo[:k + 1], op[:na], ot[:na], oe[:k], osrc[:k]


def read_structures(path: str, type_names, fmt: str = "xyz"):
    """Structures of an extended-XYZ or VASP file as a CSR batch (host only):
    (atom_off, pos [N,3], types [N], cells [S,3,3] (vectors as rows),
    pbc [S], energies [S], forces [N,3])."""
    code = {"xyz": 1, "vasp": 2}[fmt.lower()]
    T = len(type_names)
    names = (C.c_char_p * max(T, 1))(*[n.encode() for n in type_names])
    ns, na = C.c_int32(), C.c_int64()
    rc = lib().nnp_read_structures(T, C.cast(names, C.c_void_p), os.fsencode(path), code, C.byref(ns), C.byref(na),
                                   None, None, None, None, None, None, None)
    if rc != NNP_OK:
        raise NNPError(rc, lib().nnp_last_error(None).decode())
    S, N = ns.value, na.value
    off = np.zeros(S + 1, dtype=np.int64)
    pos = np.zeros((max(N, 1), 3))
    typ = np.zeros(max(N, 1), dtype=np.int32)
    cell = np.zeros((max(S, 1), 3, 3))
    pbc = np.zeros(max(S, 1), dtype=np.int32)
    en = np.zeros(max(S, 1))
    frc = np.zeros((max(N, 1), 3))
    rc = lib().nnp_read_structures(T, C.cast(names, C.c_void_p), os.fsencode(path), code, C.byref(ns), C.byref(na),
                                   _ptr(off), _ptr(pos), _ptr(typ), _ptr(cell), _ptr(pbc), _ptr(en), _ptr(frc))
    if rc != NNP_OK:
        raise NNPError(rc, lib().nnp_last_error(None).decode())
    return off, pos[:N], typ[:N], cell[:S], pbc[:S].astype(bool), en[:S], frc[:N]


def decay_step(kind, alpha, period, gamma, step):
    """opt::Decay::step: the next learning rate (host only)."""
    out = C.c_double()
    rc = lib().nnp_decay_step(DECAY[kind] if isinstance(kind, str) else kind, float(alpha), int(period), float(gamma),
                              int(step), C.byref(out))
    if rc != NNP_OK:
        raise NNPError(rc, lib().nnp_last_error(None).decode())
    return out.value
