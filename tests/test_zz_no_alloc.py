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


@pytest.mark.parametrize("n,q,collision,storage", [
    (32, 19, "LBGK", "f64"),
    (64, 19, "LBGK", "f16"),
    (32, 27, "Cumulant", "f32"),
    (128, 19, "LBGK", "bf16"),
])
def test_noalloc_matches_reduce_twice(ctx, n, q, collision, storage):
    """Two calls in a row after some steps equal the allocating entry point
    (same kernels, same summation order: identical up to rounding, tested at
    1e-12 relative on the mass and 1e-12 of the mass on the other sums)."""
    d = _dense_tgv(ctx, n, q, collision, storage)
    d.step(7)
    ref = _reduce(ctx, d)
    launches0 = ctx.launch_count()
    a = _reduce_noalloc(ctx, d)
    b = _reduce_noalloc(ctx, d)
    assert ctx.launch_count() - launches0 == 4
    scale = abs(ref[0])
    for got in (a, b):
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * scale)
    # the state moves on; the next pair of calls follows it
    d.step(3)
    ref2 = _reduce(ctx, d)
    assert not np.array_equal(ref2[4], ref[4])
    np.testing.assert_allclose(_reduce_noalloc(ctx, d), ref2, rtol=1e-12, atol=1e-12 * scale)
    np.testing.assert_allclose(_reduce_noalloc(ctx, d), ref2, rtol=1e-12, atol=1e-12 * scale)
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
    np.testing.assert_allclose(_reduce_noalloc(ctx, small), _reduce(ctx, small), rtol=1e-12,
                               atol=1e-12 * small.n)
    small.close()
