"""ctypes wrapper of the reference's own NNP code compiled into
oracle/_ref/libref.so by oracle/ref/Makefile (from the reference sources,
with the project's small Eigen header).

TEST INFRASTRUCTURE ONLY: used by the tests (to pin the oracle and the CUDA
path to the reference), by tests/golden/make_golden.py, and by bench.py's
CPU baseline / reference arm.  Never used by the library."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_ref", "libref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise ImportError("oracle/_ref/libref.so is not built (make -C oracle/ref)")
        L = C.CDLL(LIBPATH)
        p = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.ref_nnp_read.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.ref_nnp_read.restype = p
        L.ref_nnp_free.argtypes = [p]
        L.ref_nnp_ntypes.argtypes = [p]
        L.ref_nnp_rc.argtypes = [p]
        L.ref_nnp_rc.restype = C.c_double
        L.ref_nnp_ninput.argtypes = [p, C.c_int]
        L.ref_nnp_compute.argtypes = [p, C.c_int, dp, C.POINTER(C.c_int), dp, C.c_int, C.c_int, dp, dp, dp, dp,
                                      C.c_char_p, C.c_int]
        L.ref_nnp_nparams.argtypes = [p, C.c_int]
        L.ref_decay_step.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, C.c_int]
        L.ref_decay_step.restype = C.c_double
        L.ref_read_structure.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int), dp, dp, dp, dp,
                                         C.c_char_p, C.c_int, C.c_char_p, C.c_int]
        L.ref_energy_loss_grad.argtypes = [p, C.c_int, C.POINTER(C.c_int64), dp, C.POINTER(C.c_int), dp, C.c_int,
                                           dp, C.c_int, C.c_int, C.c_double, dp, dp, dp, dp, C.c_char_p, C.c_int]
        L.ref_force_term_grad.argtypes = [p, C.c_int, dp, C.POINTER(C.c_int), dp, C.c_int, dp, C.c_double, dp,
                                          dp, C.c_char_p, C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class RefNNP:
    """The reference's NNP read from a potential file."""

    def __init__(self, path: str):
        err = C.create_string_buffer(512)
        self.h = lib().ref_nnp_read(os.fsencode(path), err, len(err))
        if not self.h:
            raise RuntimeError("reference NNP::read failed: " + err.value.decode())
        self.ntypes = lib().ref_nnp_ntypes(self.h)
        self.rc = lib().ref_nnp_rc(self.h)
        self.gstride = max(lib().ref_nnp_ninput(self.h, t) for t in range(self.ntypes))

    def close(self):
        if self.h:
            lib().ref_nnp_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compute(self, pos, types, cell, pbc=True, want_symm=False):
        """One structure through NNP::compute_symm + compute_force (+
        compute_energy): returns (energy without vacuum terms, forces [n,3],
        energy with vacuum terms, symm [n, gstride] or None)."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        types = np.ascontiguousarray(types, dtype=np.int32)
        cell = np.ascontiguousarray(cell if cell is not None else np.zeros(9), dtype=np.float64).reshape(9)
        e = np.zeros(1)
        ev = np.zeros(1)
        f = np.zeros((max(n, 1), 3))
        g = np.zeros((max(n, 1), self.gstride)) if want_symm else None
        err = C.create_string_buffer(512)
        rc = lib().ref_nnp_compute(self.h, n, _dp(pos), types.ctypes.data_as(C.POINTER(C.c_int)), _dp(cell),
                                   1 if pbc else 0, self.gstride, _dp(e), _dp(f), _dp(g), _dp(ev), err, len(err))
        if rc != 0:
            raise RuntimeError("reference compute failed: " + err.value.decode())
        return float(e[0]), f[:n], float(ev[0]), (g[:n] if want_symm else None)


    def nparams(self, t: int) -> int:
        """ANN::size of type t's network."""
        return int(lib().ref_nnp_nparams(self.h, t))

    def nparams_total(self) -> int:
        return sum(self.nparams(t) for t in range(self.ntypes))

    def energy_loss_grad(self, batch, e_ref, norm_mode=1, loss_kind=1, delta=1.0):
        """Energy-loss gradient of a batch through the reference's fpbp +
        Cost::grad per atom and NNPTEFR::error_cost_o1's loss factors:
        returns (loss, grad in the per-element packing, rmse, energies)."""
        off = np.ascontiguousarray(batch.atom_off, dtype=np.int64)
        pos = np.ascontiguousarray(batch.pos, dtype=np.float64)
        typ = np.ascontiguousarray(batch.type, dtype=np.int32)
        cell = np.ascontiguousarray(np.asarray(batch.cell).reshape(-1, 9), dtype=np.float64)
        e_ref = np.ascontiguousarray(e_ref, dtype=np.float64)
        g = np.zeros(self.nparams_total())
        loss, rmse = np.zeros(1), np.zeros(1)
        en = np.zeros(batch.n_struct)
        err = C.create_string_buffer(512)
        rc = lib().ref_energy_loss_grad(self.h, batch.n_struct, off.ctypes.data_as(C.POINTER(C.c_int64)), _dp(pos),
                                        typ.ctypes.data_as(C.POINTER(C.c_int)), _dp(cell), int(batch.pbc),
                                        _dp(e_ref), norm_mode, loss_kind, float(delta), _dp(g), _dp(loss),
                                        _dp(rmse), _dp(en), err, len(err))
        if rc != 0:
            raise RuntimeError("reference energy-loss gradient failed: " + err.value.decode())
        return float(loss[0]), g, float(rmse[0]), en

    def force_term_grad(self, pos, types, cell, v, fd_h, pbc=True, want_tangent=False):
        """sum_i d/dtheta (dE_i/dG_i . C_i) for one structure, C_i the change of
        G_i along the displacement field v, from the reference's D2ODZDI and
        central differences of its compute_symm (potential with inpw = 1)."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        types = np.ascontiguousarray(types, dtype=np.int32)
        cell = np.ascontiguousarray(cell if cell is not None else np.zeros(9), dtype=np.float64).reshape(9)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        g = np.zeros(self.nparams_total())
        ct = np.zeros((n, self.gstride)) if want_tangent else None
        err = C.create_string_buffer(512)
        rc = lib().ref_force_term_grad(self.h, n, _dp(pos), types.ctypes.data_as(C.POINTER(C.c_int)), _dp(cell),
                                       1 if pbc else 0, _dp(v), float(fd_h), _dp(g), _dp(ct), err, len(err))
        if rc != 0:
            raise RuntimeError("reference force-term gradient failed: " + err.value.decode())
        return (g, ct) if want_tangent else g


def read_structure(path: str, fmt: str = "xyz", cap: int = 100000):
    """One structure through the reference's XYZ::read / VASP::POSCAR::read:
    (names, positions [n,3], forces [n,3], pe, cell [3,3] with the lattice
    vectors as rows)."""
    n = C.c_int()
    pos = np.zeros((cap, 3))
    frc = np.zeros((cap, 3))
    pe = np.zeros(1)
    cell = np.zeros(9)
    names = C.create_string_buffer(16 * cap + 16)
    err = C.create_string_buffer(512)
    rc = lib().ref_read_structure(os.fsencode(path), 1 if fmt == "xyz" else 2, cap, C.byref(n), _dp(pos), _dp(frc),
                                  _dp(pe), _dp(cell), names, len(names), err, len(err))
    if rc != 0:
        raise RuntimeError("reference read failed: " + err.value.decode())
    k = n.value
    return names.value.decode().split(), pos[:k], frc[:k], float(pe[0]), cell.reshape(3, 3)
