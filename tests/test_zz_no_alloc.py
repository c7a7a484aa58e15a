"""Allocation-free reduction (mt_case_reduce_noalloc) through the C ABI: the
same mass / momentum / kinetic-energy sums as mt_case_reduce on two calls in
a row, its size limit, and a context that stays usable after the rejection.

Kept in its own file, named to be collected last, so that it runs both in a
fresh process (first call on the device does the set-up) and after every
other GPU test of a session."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the static scratch holds one partial per 256-cell block for 16384 blocks
MAX_CELLS = 256 * 16384


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def _dense_tgv(ctx, n, q, collision, storage):
    from mortontrie_amr_b200.case import taylor_green_fields, uniform_box_case
    from mortontrie_amr_b200.lbm import DenseCase, morton_order_fields
    case = uniform_box_case(q=q, n=(n, n, n), nu=1.0 / 30.0, collision=collision, storage=storage)
    d = DenseCase(ctx, case, storage)
    d.init_fields(*morton_order_fields(n, *taylor_green_fields((n, n, n), 0.03)))
    return d


def _reduce_noalloc(ctx, d):
    from mortontrie_amr_b200.lbm import lib
    out = np.full(5, np.nan)
    ctx.check(lib().mt_case_reduce_noalloc(ctx.h, d.id, out.ctypes.data_as(C.POINTER(C.c_double))),
              "mt_case_reduce_noalloc")
    return out


def _reduce(ctx, d):
    r = d.reduce()
    return np.array([r["mass"], *r["momentum"], r["kinetic_energy"]])


class _PoolWatch:
    """High-water mark of the device's default memory pool, which every
    stream-ordered allocation of the library draws from: reset before a
    stretch of calls, read after it."""

    def __init__(self, device=0):
        from cuda.bindings import runtime as rt
        self.rt = rt
        err, self.pool = rt.cudaDeviceGetDefaultMemPool(device)
        assert err == rt.cudaError_t.cudaSuccess, err

    def _get(self, attr):
        err, v = self.rt.cudaMemPoolGetAttribute(self.pool, attr)
        assert err == self.rt.cudaError_t.cudaSuccess, err
        return int(v)

    def reset(self):
        A = self.rt.cudaMemPoolAttr
        from cuda.bindings import driver
        err, = self.rt.cudaMemPoolSetAttribute(self.pool, A.cudaMemPoolAttrUsedMemHigh, driver.cuuint64_t(0))
        assert err == self.rt.cudaError_t.cudaSuccess, err
        return self._get(A.cudaMemPoolAttrUsedMemCurrent)

    def high(self):
        return self._get(self.rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh)


@pytest.mark.parametrize("n,q,collision,storage", [
    (32, 19, "LBGK", "f64"),
    (64, 19, "LBGK", "f16"),
    (32, 27, "Cumulant", "f32"),
    (128, 19, "LBGK", "bf16"),
])
def test_noalloc_matches_reduce_twice(ctx, n, q, collision, storage):
    """Two calls in a row after some steps equal the allocating entry point
    bit for bit (same kernels, same grid, same summation order), and the
    pair of calls takes nothing from the device's memory pool."""
    d = _dense_tgv(ctx, n, q, collision, storage)
    d.step(7)
    ref = _reduce(ctx, d)
    ctx.synchronize()
    pool = _PoolWatch(0)
    used = pool.reset()
    launches0 = ctx.launch_count()
    a = _reduce_noalloc(ctx, d)
    b = _reduce_noalloc(ctx, d)
    assert ctx.launch_count() - launches0 == 4
    assert pool.high() == used, "the allocation-free reduction drew memory from the pool"
    for got in (a, b):
        assert np.all(np.isfinite(got))
        np.testing.assert_array_equal(got, ref)
    # the state moves on; the next pair of calls follows it
    d.step(3)
    ref2 = _reduce(ctx, d)
    assert not np.array_equal(ref2[4], ref[4])
    np.testing.assert_array_equal(_reduce_noalloc(ctx, d), ref2)
    np.testing.assert_array_equal(_reduce_noalloc(ctx, d), ref2)
    d.close()


def test_noalloc_rejects_cases_beyond_scratch(ctx):
    """256^3 cells (4x the scratch limit) is refused with MT_ERR_ARG and a
    message naming the limit; the context keeps working."""
    from mortontrie_amr_b200.lbm import MTError
    big = _dense_tgv(ctx, 256, 19, "LBGK", "f16")
    assert big.n > MAX_CELLS
    with pytest.raises(MTError, match="MT_ERR_ARG") as info:
        _reduce_noalloc(ctx, big)
    assert str(MAX_CELLS) in str(info.value)
    ref = _reduce(ctx, big)
    assert np.isfinite(ref).all()
    big.close()
    small = _dense_tgv(ctx, 128, 19, "LBGK", "f16")
    assert small.n == 2 * 1024 * 1024
    np.testing.assert_array_equal(_reduce_noalloc(ctx, small), _reduce(ctx, small))
    small.close()
