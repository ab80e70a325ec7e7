"""Direct GPU tests of the field arithmetic (BN254 / BLS12-381 Fp and Fr) on both product paths.

Every MSM, NTT and group-FFT result rests on these operations. Each is compared, bit for bit,
with the oracle's Montgomery arithmetic (which the golden vectors pin to the reference C,
bn128_Fp_mont.c:189, bls12_381_Fp_mont.c:203 and the Fr twins) on every pair of edge values
(0, 1, 2, R mod p, p - 1, p - 2, (p - 1) / 2, (p + 1) / 2, 2^k - 1 below p, R^2 mod p) and on
2^16 random pairs: the 32-bit-limb CIOS product, the FP64-pipe product through the radix
conversions the kernels use, the raw FP64 product a b 2^-(52 L), the paired-product calls,
additions, subtractions and negations, and the same operations on the MSM bucket pipeline's
redundant range [0, 2p) with operands given as x and as x + p, and the FP64 product in the
reference's own radix (no conversions) that the Fr vector operations use.
"""
import ctypes

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu

MUL, SQR, ADD, SUB, NEG, RAW, PAIR_A, PAIR_B, SQR_PAIR = range(9)
FIELDS = [(c, f) for c in Z.CURVES for f in (0, 1)]


def modulus(curve, field):
    return Z.R[curve] if field else Z.P[curve]


def nlimbs(curve, field):
    return 4 if field else Z.NLP[curve]


def operands(curve, field, nrand, seed):
    p = modulus(curve, field)
    nl = nlimbs(curve, field)
    Rm = 1 << (64 * nl)
    edges = [0, 1, 2, Rm % p, p - 1, p - 2, (p - 1) // 2, (p + 1) // 2, Rm * Rm % p,
             (1 << (p.bit_length() - 1)) - 1, (1 << 64) - 1, p - (1 << 64)]
    a = [x for x in edges for _ in edges]
    b = [y for _ in edges for y in edges]
    rng = np.random.default_rng(seed)
    for _ in range(nrand):
        a.append(int.from_bytes(rng.bytes(8 * nl), "little") % p)
        b.append(int.from_bytes(rng.bytes(8 * nl), "little") % p)
    return Z.ints_to_array(a, nl), Z.ints_to_array(b, nl)


def device_op(zk, curve, field, path, op, a, b):
    import torch
    L = zk.lib()
    f = L.zkg_field_test_device
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]
    d_a = torch.from_numpy(a.view(np.int64)).cuda()
    d_b = torch.from_numpy(b.view(np.int64)).cuda()
    d_o = torch.full_like(d_a, -1)
    st = f(curve, field, path, op, a.shape[0], vp(d_a.data_ptr()), vp(d_b.data_ptr()), vp(d_o.data_ptr()))
    assert st == 0, L.zkg_last_error()
    return d_o.cpu().numpy().view(np.uint64)


def oracle_op(curve, field, op, a, b=None):
    """oracle_field_op codes: 2 mul, 3 add, 4 sub, 5 neg"""
    a = np.ascontiguousarray(a)
    out = np.zeros_like(a)
    Z.oracle().oracle_field_op(curve, field, op, a.shape[0], Z.ptr(a),
                               None if b is None else Z.ptr(np.ascontiguousarray(b)), Z.ptr(out))
    return out


@pytest.mark.parametrize("curve,field,path",
                         [(c, f, p) for c, f in FIELDS for p in (0, 1, 2, 3) if p != 2 or f == 0])
def test_field_ops_edge_values_and_random_pairs(zk, curve, field, path):
    """path 0: 32-bit limbs, 1: FP64 products, 2: the MSM pipeline's redundant range [0, 2p)
    (operands in both representatives x and x + p), 3: FP64 products in the reference's radix"""
    a, b = operands(curve, field, 1 << 16, 50000 + 10 * curve + field)
    want_mul = oracle_op(curve, field, 2, a, b)
    assert np.array_equal(device_op(zk, curve, field, path, MUL, a, b), want_mul)
    assert np.array_equal(device_op(zk, curve, field, path, PAIR_A, a, b), want_mul)
    assert np.array_equal(device_op(zk, curve, field, path, PAIR_B, a, b), want_mul)
    want_sqr = oracle_op(curve, field, 2, a, a)
    assert np.array_equal(device_op(zk, curve, field, path, SQR, a, b), want_sqr)
    assert np.array_equal(device_op(zk, curve, field, path, SQR_PAIR, a, b), want_sqr)
    assert np.array_equal(device_op(zk, curve, field, path, ADD, a, b), oracle_op(curve, field, 3, a, b))
    assert np.array_equal(device_op(zk, curve, field, path, SUB, a, b), oracle_op(curve, field, 4, a, b))
    assert np.array_equal(device_op(zk, curve, field, path, NEG, a, b), oracle_op(curve, field, 5, a))


@pytest.mark.parametrize("curve,field", FIELDS)
def test_raw_fp64_product_is_a_b_over_2_to_52L(zk, curve, field):
    """the FP64 product itself, without radix conversions: a b 2^-(52 L) mod p, with
    L = 5 limbs for 254/255-bit moduli and 8 for the 381-bit one"""
    a, b = operands(curve, field, 1 << 14, 51000 + 10 * curve + field)
    p = modulus(curve, field)
    nl = nlimbs(curve, field)
    Lb = 52 * (8 if p.bit_length() > 300 else 5)
    # a b 2^-Lb = mont(mont(a, b), c) with c = R^2 2^-Lb (standard integer), R = 2^(64 nl)
    c = (1 << (128 * nl)) * pow(1 << Lb, -1, p) % p
    cc = np.repeat(Z.to_limbs(c, nl)[None, :], a.shape[0], axis=0)
    want = oracle_op(curve, field, 2, oracle_op(curve, field, 2, a, b), cc)
    assert np.array_equal(device_op(zk, curve, field, 0, RAW, a, b), want)
    # spot check with Python integers
    for i in (0, 17, 143, a.shape[0] - 1):
        x, y = Z.from_limbs(a[i]), Z.from_limbs(b[i])
        assert Z.from_limbs(want[i]) == x * y * pow(1 << Lb, -1, p) % p
