"""ibpm_create rejects malformed problem descriptions before touching a device
(so these run without a GPU): the caller gets IBPM_ERR_INVALID and a message."""
import ctypes as C

import numpy as np
import pytest


def _problem(abi, xb, ds, starts, kinds, h=0.04):
    p = abi.ibpm_problem(nx=64, ny=64, nlevel=2, h=h, x0=-1.28, y0=-1.28, Re=100.0, dt=0.004,
                         npanel=int(ds.size), nbody=int(kinds.size), body_kind=kinds.ctypes.data_as(abi._ip),
                         body_start=starts.ctypes.data_as(abi._ip), body_xb=abi.dptr(xb), body_ds=abi.dptr(ds),
                         grid_moving=0)
    return p


def _create(ib, p, opt=None):
    abi = ib._abi
    lib = abi.load()
    h = C.c_void_p()
    if opt is None:
        opt = abi.ibpm_options()
        lib.ibpm_default_options(C.byref(opt))
    rc = lib.ibpm_create(C.byref(p), C.byref(opt), C.byref(h))
    return rc, lib.ibpm_last_error(None).decode()


def _circle(n=40, r=0.3):
    t = np.linspace(0, 2 * np.pi, n, endpoint=False)
    xb = np.asfortranarray(np.stack([r * np.cos(t), r * np.sin(t)], axis=1))
    return xb, np.full(n, 2 * np.pi * r / n)


def test_decreasing_body_start_is_rejected(ib):
    xb, ds = _circle()
    kinds = np.array([0, 0], dtype=np.int32)
    starts = np.array([0, 30, 40], dtype=np.int32)
    starts[1] = 50  # 0, 50, 40: the second body would run backwards
    rc, msg = _create(ib, _problem(ib._abi, xb, ds, starts, kinds))
    assert rc == ib._abi.IBPM_ERR_INVALID and "must not decrease" in msg


def test_non_finite_body_point_is_rejected(ib):
    xb, ds = _circle()
    xb[3, 1] = np.nan
    rc, msg = _create(ib, _problem(ib._abi, xb, ds, np.array([0, 40], np.int32), np.array([0], np.int32)))
    assert rc == ib._abi.IBPM_ERR_INVALID and "non-finite" in msg


def test_negative_cg_option_is_rejected(ib):
    abi = ib._abi
    xb, ds = _circle()
    opt = abi.ibpm_options()
    abi.load().ibpm_default_options(C.byref(opt))
    opt.cg_reltol = -1.0
    rc, msg = _create(ib, _problem(abi, xb, ds, np.array([0, 40], np.int32), np.array([0], np.int32)), opt)
    assert rc == abi.IBPM_ERR_INVALID and "CG options" in msg


@pytest.mark.parametrize("bad", ["h", "nlevel"])
def test_bad_grid_is_rejected(ib, bad):
    abi = ib._abi
    xb, ds = _circle()
    p = _problem(abi, xb, ds, np.array([0, 40], np.int32), np.array([0], np.int32))
    if bad == "h":
        p.h = float("inf")
    else:
        p.nlevel = 0
    rc, msg = _create(ib, p)
    assert rc == abi.IBPM_ERR_INVALID
