"""ibpm_lap_inv_noalloc: the Laplacian-inverse solve for callers that cannot
allocate device memory (code inside another framework's memory pool or a fixed
arena, or a host loop that must not allocate between steps).  The caller passes
device buffers for b and x; the entry point's scratch fields and transform
tables live in a static device array of the library, limited to 262144 cells.

Checked through the C ABI against the allocating path (ibpm_diag_solve with
op 0, the same Δinv operator) on two calls in a row, at the tolerance of the
operator-level solve tests, plus a size change and the size limit; and against
the CPU oracle's Δinv (src/fluid.jl:145-166) on non-square grids up to the
largest transform length the limit allows (1024 x 256), where the x and y
tables differ, and with x given the same buffer as b."""
import ctypes as C

import numpy as np
import pytest

from fixtures import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-13  # the operator-level solve tolerance (tests/test_gpu_operators.py)


def _noalloc(lib, nx, ny, b, alias=False):
    import torch

    bd = torch.from_numpy(np.asfortranarray(b).ravel(order="F")).cuda()
    xd = bd if alias else torch.empty_like(bd)
    rc = lib.ibpm_lap_inv_noalloc(nx, ny, C.c_void_p(bd.data_ptr()), C.c_void_p(xd.data_ptr()),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0, lib.ibpm_noalloc_last_error().decode()
    return xd.cpu().numpy().reshape(b.shape, order="F")


def test_noalloc_matches_allocating_solve(ib):
    import importlib

    abi = importlib.import_module(ib.__name__ + "._abi")
    lib = abi.load()
    for n, calls in ((256, 2), (200, 1), (256, 1)):
        prob = ib.configs.small_cylinder(n, 2)
        solver = ib.create_solver(ib.State(prob))
        rng = np.random.default_rng(n)
        for _ in range(calls):  # consecutive calls share the static scratch
            b = rng.standard_normal((n - 1, n - 1))
            ref = solver.diag_solve(0, 1, b)
            x = _noalloc(lib, n, n, b)
            assert rel_l2(x, ref) <= TOL


def test_noalloc_matches_oracle_on_non_square_grids(ib, orc):
    import importlib

    abi = importlib.import_module(ib.__name__ + "._abi")
    lib = abi.load()
    for nx, ny, alias in ((512, 256, False), (256, 512, False), (1024, 256, False), (1024, 256, True),
                          (384, 256, False)):
        rng = np.random.default_rng(nx + 7 * ny)
        b = rng.standard_normal((nx - 1, ny - 1))
        ref = orc.lap_inv(nx, ny, orc.lap_eigs(nx, ny), b)
        for _ in range(2):  # two calls in a row on the shared scratch
            x = _noalloc(lib, nx, ny, b, alias=alias)
            assert rel_l2(x, ref) <= TOL, (nx, ny, alias, rel_l2(x, ref))


def test_noalloc_rejects_sizes_beyond_its_limit(ib):
    import importlib

    import torch

    abi = importlib.import_module(ib.__name__ + "._abi")
    lib = abi.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.ibpm_lap_inv_noalloc(1024, 1024, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), None)
    assert rc == abi.IBPM_ERR_INVALID
    assert "no-alloc limit" in lib.ibpm_noalloc_last_error().decode()
