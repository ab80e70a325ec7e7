"""Host-buffer entry points from pageable and from page-locked arrays.

Pageable caller arrays (numpy, or the Haskell FFI's pinned-but-not-page-locked arrays) are staged
through the library's 32 MB page-locked slots; page-locked ones go straight to the copy engine.
Sizes here span several slots with a ragged last chunk, and every result must equal the device
path's (and, for the Fr product, the oracle's).
"""
import numpy as np
import pytest
import torch

import zkutil as Z

pytestmark = pytest.mark.gpu


def page_locked(a):
    """a copy of `a` in page-locked host memory (the tensor keeps the memory alive)"""
    t = torch.empty(a.size, dtype=torch.int64, pin_memory=True)
    v = t.numpy().view(np.uint64).reshape(a.shape)
    v[...] = a
    return t, v


def test_fr_mul_pageable_and_page_locked(zk):
    n = (1 << 21) + 3   # 64 MB + 96 B per operand: three staging chunks, the last one 96 bytes
    a = Z.rand_fr(Z.BN254, n, 41000)
    b = Z.rand_fr(Z.BN254, n, 41001)
    want = Z.oracle_fr_op(Z.BN254, Z.FR_OPS["mul"][0], a, b)
    assert np.array_equal(zk.fr_map(Z.BN254, "mul", a, b), want)
    ta, pa = page_locked(a)
    tb, pb = page_locked(b)
    to, po = page_locked(np.zeros_like(a))
    zk.fr_map(Z.BN254, "mul", pa, pb, out=po)
    assert np.array_equal(po, want)


def test_ntt_pageable_and_page_locked(zk):
    m = 21
    x = Z.rand_fr(Z.BN254, 1 << m, 41100)
    d_x = torch.from_numpy(x.view(np.int64)).cuda()
    d_y = torch.empty_like(d_x)
    zk.ntt_device(Z.BN254, m, d_x, d_y)
    want = d_y.cpu().numpy().view(np.uint64).reshape(-1, 4)
    assert np.array_equal(zk.forward_ntt(Z.BN254, m, x), want)
    tx, px = page_locked(x)
    assert np.array_equal(zk.forward_ntt(Z.BN254, m, px), want)
    assert np.array_equal(zk.inverse_ntt(Z.BN254, m, want), x)


@pytest.mark.parametrize("n", [(1 << 19) + 7, (1 << 21) + 5])
@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_pageable_and_page_locked(zk, curve, n):
    # 2^19 + 7: two point-range parts, bases of 34-50 MB span two staging chunks; 2^21 + 5: four
    # parts whose bucket arrays are merged in one pass, bases of 134-201 MB over many chunks
    nl = Z.NLP[curve]
    d_k = torch.from_numpy(Z.rand_fr(curve, n, 41200 + curve).view(np.int64)).cuda()
    d_b = torch.empty((n, 2 * nl), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(curve, n, d_k, d_b)
    ks = Z.rand_fr(curve, n, 41300 + curve)
    want = zk.msm_device(curve, n, torch.from_numpy(ks.view(np.int64)).cuda(), d_b)
    bases = d_b.cpu().numpy().view(np.uint64)
    assert np.array_equal(zk.msm_affine(curve, ks, bases), want)
    tk, pk = page_locked(ks)
    tb, pb = page_locked(bases)
    assert np.array_equal(zk.msm_affine(curve, pk, pb), want)
