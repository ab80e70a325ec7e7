"""GPU parity tests for the Fr vector operations (*_arr_mont_*, lib/cbits/curves/array/mont/bn128_arr_mont.c)
through the drop-in C ABI and the native zkg_fr_* calls.

Every drop-in function is compared byte for byte with golden vectors of the reference C, and at
larger sizes (many threads, many elements per thread) with the oracle restatement, including the
reference's edge behaviour: a zero anywhere in a batch inversion zeroes every output, and
mul_by_powers leaves tgt[0] unwritten.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

import zkutil as Z

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import ARR_FUNCS, call_arr  # noqa: E402

pytestmark = pytest.mark.gpu


def golden(curve):
    return np.load(os.path.join(Z.GOLDEN, "arr_%s.npz" % Z.NAMES[curve]))


@pytest.mark.parametrize("curve", Z.CURVES)
def test_fr_ops_golden_reference_vectors(zk, curve):
    L = zk.lib()
    d = golden(curve)
    A, B = d["A"], d["B"]
    cases = sorted({k.split("__")[0] for k in d.files if "__" in k and not k.startswith("sparse")})
    checked = 0
    for cname in cases:
        a, b, c = d[cname + "__a"], d[cname + "__b"], d[cname + "__c"]
        n = a.shape[0]
        tgt0 = np.full((n, 4), 0xABABABABABABABAB, np.uint64)
        for fn, pat in ARR_FUNCS:
            key = "%s__%s" % (cname, fn)
            if key not in d.files:
                continue
            got = call_arr(L, curve, fn, pat, n, a, b, c, A, B, tgt0)
            assert L.zkg_last_status() == 0, (key, L.zkg_last_error())
            assert np.array_equal(got, d[key]), key
            checked += 1
    assert checked >= 150
    name = Z.NAMES[curve]
    for key in sorted({k.rsplit("__", 1)[0] for k in d.files if k.startswith("sparse")}):
        rows, cols, co, src = d[key + "__rows"], d[key + "__cols"], d[key + "__coeffs"], d[key + "__src"]
        N = d[key + "__tgt"].shape[0]
        out = np.full((N, 4), 7, np.uint64)
        L["%s_arr_mont_sparse_matrix_mul" % name](ctypes.c_int(N), ctypes.c_int(rows.shape[0]), Z.ptr(rows),
                                                   Z.ptr(cols), Z.ptr(co), Z.ptr(src), Z.ptr(out))
        assert L.zkg_last_status() == 0
        assert np.array_equal(out, d[key + "__tgt"]), key


@pytest.mark.parametrize("curve", Z.CURVES)
def test_fr_data_movement_entries(zk, curve):
    L = zk.lib()
    name = Z.NAMES[curve]
    a = Z.rand_fr(curve, 10, 1)
    b = Z.rand_fr(curve, 5, 2)
    out = np.zeros((15, 4), np.uint64)
    L["%s_arr_mont_append" % name](10, 5, Z.ptr(a), Z.ptr(b), Z.ptr(out))
    assert np.array_equal(out, np.concatenate([a, b]))
    out[:] = 0
    ns = (ctypes.c_int * 3)(5, 0, 10)
    srcs = (ctypes.c_void_p * 3)(b.ctypes.data, a.ctypes.data, a.ctypes.data)
    L["%s_arr_mont_concat" % name](3, ns, srcs, Z.ptr(out))
    assert np.array_equal(out, np.concatenate([b, a]))
    L["%s_arr_mont_copy" % name](10, Z.ptr(a), Z.ptr(out))
    assert np.array_equal(out[:10], a)
    L["%s_arr_mont_set_zero" % name](15, Z.ptr(out))
    assert not np.any(out)
    L["%s_arr_mont_set_one" % name](15, Z.ptr(out))
    assert np.all(out == Z.to_limbs((1 << 256) % Z.R[curve], 4))
    L["%s_arr_mont_set_const" % name](15, Z.ptr(b[2]), Z.ptr(out))
    assert np.all(out == b[2])


@pytest.mark.parametrize("curve", Z.CURVES)
def test_fr_ops_large_vs_oracle(zk, curve):
    """(1 << 18) + 5 elements: more elements than threads in every kernel"""
    n = (1 << 18) + 5
    a, b, c = (Z.rand_fr(curve, n, 9800 + k) for k in range(3))
    A, B = Z.rand_fr(curve, 1, 9810)[0], Z.rand_fr(curve, 1, 9811)[0]
    L = zk.lib()
    for fn, (op, order) in Z.FR_OPS.items():
        if fn.endswith("inplace") or fn == "sub_inplace_reverse":
            continue
        ins = {"a": a, "b": b, "c": c}
        args = [ins[ch] for ch in order] + [None] * (3 - len(order))
        init = np.full((n, 4), 0x5A5A5A5A5A5A5A5A, np.uint64)
        want = Z.oracle_fr_op(curve, op, *args, ka=A, kb=B, n=n, out=init)
        got = init.copy()
        ps = [None if x is None else Z.ptr(np.ascontiguousarray(x)) for x in args]
        assert L.zkg_fr_map(curve, op, n, *ps, Z.ptr(A), Z.ptr(B), Z.ptr(got)) == 0, (fn, L.zkg_last_error())
        assert np.array_equal(got, want), fn
    # batch inversion with one zero at the far end
    a2 = a.copy()
    a2[n - 2] = 0
    got = np.ones((n, 4), np.uint64)
    assert L.zkg_fr_map(curve, 7, n, Z.ptr(a2), None, None, None, None, Z.ptr(got)) == 0
    assert not np.any(got)
    # dot product and predicates
    out = np.zeros(4, np.uint64)
    assert L.zkg_fr_dot(curve, n, Z.ptr(a), Z.ptr(b), Z.ptr(out)) == 0
    want = np.zeros(4, np.uint64)
    Z.oracle().oracle_fr_dot(curve, n, Z.ptr(a), Z.ptr(b), Z.ptr(want))
    assert np.array_equal(out, want)
    res = ctypes.c_int(-1)
    for which, arr, arr2, expect in ((0, a, None, 1), (1, a, None, 0), (3, a, a.copy(), 1), (3, a, b, 0)):
        assert L.zkg_fr_predicate(curve, which, n, Z.ptr(arr), None if arr2 is None else Z.ptr(arr2),
                                  ctypes.byref(res)) == 0
        assert res.value == expect, which
    bad = a.copy()
    bad[n - 1] = Z.to_limbs(Z.R[curve], 4)   # r itself is not a valid element
    assert L.zkg_fr_predicate(curve, 0, n, Z.ptr(bad), None, ctypes.byref(res)) == 0 and res.value == 0


@pytest.mark.parametrize("curve", Z.CURVES)
def test_fr_device_api_in_place(zk, curve):
    import torch
    n = 100003
    a, b = Z.rand_fr(curve, n, 9900), Z.rand_fr(curve, n, 9901)
    A = Z.rand_fr(curve, 1, 9902)[0]
    L = zk.lib()
    d_a = torch.from_numpy(a.view(np.int64).copy()).cuda()
    d_b = torch.from_numpy(b.view(np.int64).copy()).cuda()
    # a <- A*a + b in place, then a <- 1/a in place
    assert L.zkg_fr_map_device(curve, 12, n, ctypes.c_void_p(d_a.data_ptr()), ctypes.c_void_p(d_b.data_ptr()), None,
                               Z.ptr(A), None, ctypes.c_void_p(d_a.data_ptr())) == 0
    assert L.zkg_fr_map_device(curve, 7, n, ctypes.c_void_p(d_a.data_ptr()), None, None, None, None,
                               ctypes.c_void_p(d_a.data_ptr())) == 0
    torch.cuda.synchronize()
    want = Z.oracle_fr_op(curve, 7, Z.oracle_fr_op(curve, 12, a, b, ka=A))
    assert np.array_equal(d_a.cpu().numpy().view(np.uint64), want)
    out = np.zeros(4, np.uint64)
    assert L.zkg_fr_dot_device(curve, n, ctypes.c_void_p(d_a.data_ptr()), ctypes.c_void_p(d_b.data_ptr()),
                               Z.ptr(out)) == 0
    w = np.zeros(4, np.uint64)
    Z.oracle().oracle_fr_dot(curve, n, Z.ptr(want), Z.ptr(b), Z.ptr(w))
    assert np.array_equal(out, w)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_fr_sparse_matrix_mul_large(zk, curve):
    N, M, K = 3000, 5000, 200000
    rows = (Z.splitmix64(1, K) % np.uint64(N)).astype(np.uint64)
    rows[:1000] = 7                     # one heavy row
    cols = (Z.splitmix64(2, K) % np.uint64(M)).astype(np.uint64)
    co = Z.rand_fr(curve, K, 3)
    src = Z.rand_fr(curve, M, 4)
    L = zk.lib()
    out = np.zeros((N, 4), np.uint64)
    assert L.zkg_fr_sparse_matrix_mul(curve, N, K, Z.ptr(rows), Z.ptr(cols), Z.ptr(co), Z.ptr(src), Z.ptr(out)) == 0
    want = np.zeros((N, 4), np.uint64)
    Z.oracle().oracle_fr_sparse(curve, N, K, Z.ptr(rows), Z.ptr(cols), Z.ptr(co), Z.ptr(src), Z.ptr(want))
    assert np.array_equal(out, want)
    bad = rows.copy()
    bad[5] = N
    assert L.zkg_fr_sparse_matrix_mul(curve, N, K, Z.ptr(bad), Z.ptr(cols), Z.ptr(co), Z.ptr(src), Z.ptr(out)) != 0


def test_fr_rejects_bad_arguments(zk):
    L = zk.lib()
    x = np.zeros((4, 4), np.uint64)
    assert L.zkg_fr_map(0, 99, 4, Z.ptr(x), Z.ptr(x), None, None, None, Z.ptr(x)) != 0
    assert L.zkg_fr_map(0, 3, -1, Z.ptr(x), Z.ptr(x), None, None, None, Z.ptr(x)) != 0
    assert L.zkg_fr_map(0, 3, 4, Z.ptr(x), None, None, None, None, Z.ptr(x)) != 0   # add needs b
    assert L.zkg_fr_map(2, 3, 4, Z.ptr(x), Z.ptr(x), None, None, None, Z.ptr(x)) != 0
    assert L.zkg_fr_map(0, 3, 0, None, None, None, None, None, None) == 0
