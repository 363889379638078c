"""The C-ABI library loads without a GPU and exports every function include/ibpm_b200.h declares."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ibpm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ibpm_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("ibpm_create", "ibpm_destroy", "ibpm_set_state", "ibpm_get_state", "ibpm_advance", "ibpm_get_forces",
              "ibpm_last_error"):
        assert n in names


def test_library_exports_all_declared(ib):
    from importlib import import_module

    abi = import_module(ib.__name__ + "._abi")
    lib = ctypes.CDLL(abi.LIB_PATH)
    for n in declared_functions():
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(ibpm_\w+)", out))
    assert set(declared_functions()) <= exported


def test_header_constants_match_the_python_mirror(ib):
    """Every integer #define of the header that the ctypes mirror also names has
    the same value there (modes, precisions, fields, error codes)."""
    from importlib import import_module

    abi = import_module(ib.__name__ + "._abi")
    defines = dict((k, int(v)) for k, v in re.findall(r"#define\s+(IBPM_\w+)\s+\(?(-?\d+)\)?", open(HEADER).read()))
    shared = [k for k in defines if hasattr(abi, k)]
    assert {"IBPM_WS_PREVIOUS", "IBPM_WS_DIRECT", "IBPM_WS_PRECONDITIONED", "IBPM_FP64"} <= set(shared), shared
    for k in shared:
        assert getattr(abi, k) == defines[k], k


def test_create_without_gpu_fails_loudly(ib):
    """With no CUDA device the library refuses to create a solver (no CPU fallback)."""
    import torch

    if torch.cuda.is_available():
        return
    prob = ib.configs.small_cylinder(32, 2)
    try:
        ib.create_solver(ib.State(prob))
    except RuntimeError as e:
        assert "CUDA" in str(e) or "device" in str(e)
    else:
        raise AssertionError("create_solver succeeded without a GPU")
