"""nnp_energy_symm_noalloc (allocation-free energies from device-resident
symmetry functions) against nnp_compute on the same batch, through the C ABI.

The energies must agree to 1e-7 eV per atom (both paths run the same FP32
network arithmetic on the same FP32 symmetry functions and sum in FP64)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from ace_b200 import NNP, nnp, potential, synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
E_TOL = 1e-7    # eV per atom


def max_atoms():
    text = open(os.path.join(ROOT, "include", "nnp_b200.h")).read()
    m = re.search(r"#define NNP_NOALLOC_MAX_ATOMS \(1 << (\d+)\)", text)
    return 1 << int(m.group(1))


def entry():
    f = nnp.lib().nnp_energy_symm_noalloc
    f.argtypes = [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_uint32,
                  C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_energies_match_compute(tmp_path):
    import torch
    rng = np.random.default_rng(21)
    b = synth.batch_random(21, rng.integers(8, 120, size=12), 3)
    pot = synth.potential_config(2)
    path = str(tmp_path / "pot.nnp")
    potential.write(path, pot)
    nn = NNP.read(path)
    _, _, G = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell, symm=True)
    synth.condition(pot, G, b.type)
    potential.write(path, pot)
    nn.close()

    nn = NNP.read(path)
    E_ref, _, G = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell, symm=True)
    E_vac, _ = nn.compute_batch(b.atom_off, b.pos, b.type, b.cell, vacuum=True)
    nat = np.diff(b.atom_off)
    S, N, gstride = b.n_struct, b.n_atoms, G.shape[1]

    dev = torch.device("cuda", 0)
    off = torch.tensor(b.atom_off, dtype=torch.int64, device=dev)
    typ = torch.tensor(b.type, dtype=torch.int32, device=dev)
    Gd = torch.tensor(G, dtype=torch.float32, device=dev)      # FP32 rows, exactly as computed
    out = torch.empty(S, dtype=torch.float64, device=dev)
    f = entry()

    def call(flags):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = f(nn._h, S, N, off.data_ptr(), typ.data_ptr(), Gd.data_ptr(), gstride, flags, out.data_ptr())
        assert rc == 0, nnp.lib().nnp_last_error(nn._h)
        torch.cuda.synchronize()
        return out.cpu().numpy().copy()

    # two calls in a row, then one with vacuum energies
    for _ in range(2):
        E = call(0)
        assert np.isfinite(E).all()
        assert (np.abs(E - E_ref) / nat).max() < E_TOL
    E = call(4)      # NNP_VACUUM
    assert (np.abs(E - E_vac) / nat).max() < E_TOL

    # larger than the scratch array: rejected before any launch
    rc = f(nn._h, 1, max_atoms() + 1, off.data_ptr(), typ.data_ptr(), Gd.data_ptr(), gstride, 0, out.data_ptr())
    assert rc == -5     # NNP_ERR_CAPACITY
    assert b"at most" in nnp.lib().nnp_last_error(nn._h)
    # rows shorter than the networks' input: rejected
    rc = f(nn._h, S, N, off.data_ptr(), typ.data_ptr(), Gd.data_ptr(), 4, 0, out.data_ptr())
    assert rc == -1     # NNP_ERR_ARG
    nn.close()
