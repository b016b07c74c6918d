"""The C ABI library loads without a GPU and exports every function that
include/nnp_b200.h declares; host-only entry points behave as documented."""
import ctypes
import os
import re

import pytest

from ace_b200 import nnp, potential, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nnp_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nnp_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_path():
    names = declared_functions()
    for must in ["nnp_create_from_file", "nnp_destroy", "nnp_compute", "nnp_train_grad", "nnp_get_params",
                 "nnp_set_params", "nnp_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    raw = ctypes.CDLL(nnp.LIBPATH)
    missing = [n for n in declared_functions() if not hasattr(raw, n)]
    assert not missing, missing


def test_version_and_errors_without_gpu():
    L = nnp.lib()
    assert L.nnp_version().decode().startswith("nnp_b200")
    h = ctypes.c_void_p()
    rc = L.nnp_create_from_file(b"/nonexistent/potential.nnp", ctypes.byref(h))
    assert rc == -2            # NNP_ERR_IO
    assert b"open" in L.nnp_last_error(None)


@pytest.mark.parametrize("k", [1, 2, 5])
def test_specialised_kernels_compile_without_gpu(tmp_path, monkeypatch, k):
    """The run-time specialised kernels are generated and compiled by NVRTC
    for sm_100a on the host alone."""
    path = str(tmp_path / "pot.nnp")
    potential.write(path, synth.potential_config(k))
    buf = ctypes.create_string_buffer(1 << 20)
    monkeypatch.setenv("NNP_CACHE_DIR", str(tmp_path / "cache"))
    rc = nnp.lib().nnp_specialization_check(path.encode(), buf, len(buf))
    assert rc == 0, buf.value.decode()[:2000]
    assert b"k_symm_jit" in buf.value and b"k_force_jit" in buf.value
