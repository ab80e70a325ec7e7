"""GPU parity tests for the NTT (forward / inverse, BN254 and BLS12-381 Fr) through the C ABI.

Bit-exact against: the reference's own outputs (golden vectors), the oracle restatement on the
same seeded inputs, the reference C's whole output vectors at 2^20 and 2^24 for both curves
(SHA-256 digests of its bytes), and at full size (2^24) size-independent properties: round trip
and evaluation identities y_k = f(g^k).
"""
import ctypes
import os

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu


def golden(curve):
    return np.load(os.path.join(Z.GOLDEN, "ntt_%s.npz" % Z.NAMES[curve]))


def dropin(zk, curve, inverse, m, gen, x):
    L = zk.lib()
    fn = getattr(L, "%s_poly_mont_ntt_%s" % (Z.NAMES[curve], "inverse" if inverse else "forward"))
    x = np.ascontiguousarray(x, dtype=np.uint64)
    gen = np.ascontiguousarray(gen, dtype=np.uint64)
    out = np.zeros_like(x)
    fn(ctypes.c_int(m), Z.ptr(gen), Z.ptr(x), Z.ptr(out))
    assert L.zkg_last_status() == 0, L.zkg_last_error()
    return out


@pytest.mark.parametrize("curve", Z.CURVES)
def test_ntt_golden_reference_vectors(zk, curve):
    d = golden(curve)
    names = sorted({k.split("__")[0] for k in d.files})
    for name in names:
        m, gen, x = int(d[name + "__m"][0]), d[name + "__gen"], d[name + "__x"]
        assert np.array_equal(dropin(zk, curve, False, m, gen, x), d[name + "__fwd"]), name
        assert np.array_equal(dropin(zk, curve, True, m, gen, x), d[name + "__inv"]), name


@pytest.mark.parametrize("curve", Z.CURVES)
def test_ntt_vs_oracle_all_small_sizes(zk, curve):
    for m in range(0, 17):
        x = Z.rand_fr(curve, 1 << m, 11000 + m)
        gen = Z.fft_gen(curve, m)
        for inv in (False, True):
            got = dropin(zk, curve, inv, m, gen, x)
            assert np.array_equal(got, Z.oracle_ntt(curve, m, gen, x, inv)), (m, inv)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_ntt_pass_splits_agree(zk, curve):
    """every pass schedule (largest pass 2^1 .. 2^11) computes the same network"""
    m = 13
    x = Z.rand_fr(curve, 1 << m, 12000)
    gen = Z.fft_gen(curve, m)
    want_f = Z.oracle_ntt(curve, m, gen, x, False)
    want_i = Z.oracle_ntt(curve, m, gen, x, True)
    L = zk.lib()
    prev = L.zkg_set_ntt_kmax(8)
    try:
        for k in (1, 2, 3, 4, 5, 6, 7, 9, 10, 11):
            L.zkg_set_ntt_kmax(k)
            assert np.array_equal(dropin(zk, curve, False, m, gen, x), want_f), k
            assert np.array_equal(dropin(zk, curve, True, m, gen, x), want_i), k
    finally:
        L.zkg_set_ntt_kmax(prev)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_ntt_arbitrary_generator_exact_network(zk, curve):
    """for a generator that is not a primitive root the reference's butterfly network is not a
    DFT; the GPU factorisation must still reproduce it exactly"""
    for m, seed in ((12, 13001), (15, 13002)):
        x = Z.rand_fr(curve, 1 << m, seed)
        gen = Z.rand_fr(curve, 1, seed + 7)[0]
        for inv in (False, True):
            assert np.array_equal(dropin(zk, curve, inv, m, gen, x), Z.oracle_ntt(curve, m, gen, x, inv)), (m, inv)


def test_ntt_bn254_2pow20_vs_oracle(zk):
    m = 20
    x = Z.rand_fr(Z.BN254, 1 << m, 14000)
    gen = Z.fft_gen(Z.BN254, m)
    for inv in (False, True):
        assert np.array_equal(dropin(zk, Z.BN254, inv, m, gen, x), Z.oracle_ntt(Z.BN254, m, gen, x, inv))


@pytest.mark.parametrize("curve", Z.CURVES)
def test_ntt_2pow24_round_trip_and_evaluations(zk, curve):
    m = 24
    x = Z.rand_fr(curve, 1 << m, 15000 + curve)
    gen = Z.fft_gen(curve, m)
    y = dropin(zk, curve, False, m, gen, x)
    assert np.array_equal(dropin(zk, curve, True, m, gen, y), x)
    # y_k = f(g^k) at a few k, f evaluated by the oracle's Horner rule
    r = Z.R[curve]
    g = Z.from_limbs(gen) * pow(1 << 256, -1, r) % r
    for k in (0, 1, 12345, (1 << m) - 1):
        pt = Z.to_limbs(pow(g, k, r) * (1 << 256) % r, 4)
        out = np.zeros(4, np.uint64)
        Z.oracle().oracle_eval_at(curve, 1 << m, Z.ptr(x), Z.ptr(pt), Z.ptr(out))
        assert np.array_equal(out, y[k]), k


def test_ntt_device_api_matches_host_api(zk):
    import torch
    m = 14
    x = Z.rand_fr(Z.BN254, 1 << m, 16000)
    gen = Z.fft_gen(Z.BN254, m)
    d_x = torch.from_numpy(x.view(np.int64)).cuda()
    d_y = torch.empty_like(d_x)
    zk.ntt_device(Z.BN254, m, d_x, d_y, inverse=False, gen=gen)
    torch.cuda.synchronize()
    assert np.array_equal(d_y.cpu().numpy().view(np.uint64), dropin(zk, Z.BN254, False, m, gen, x))


def test_ntt_rejects_bad_arguments(zk):
    L = zk.lib()
    x = np.zeros((4, 4), np.uint64)
    gen = Z.fft_gen(Z.BN254, 2)
    assert L.zkg_ntt(0, 31, Z.ptr(gen), Z.ptr(x), Z.ptr(x.copy()), 0) != 0   # beyond the reference's int N
    assert L.zkg_ntt(0, 2, Z.ptr(gen), Z.ptr(x), Z.ptr(x), 0) != 0   # aliasing
    assert L.zkg_ntt(7, 2, Z.ptr(gen), Z.ptr(x), Z.ptr(x.copy()), 0) != 0


def _shifted(zk, curve, name, eta, m, gen, x):
    L = zk.lib()
    fn = getattr(L, "%s_poly_mont_ntt_%s" % (Z.NAMES[curve], name))
    x = np.ascontiguousarray(x, dtype=np.uint64)
    out = np.zeros_like(x)
    fn(Z.ptr(np.ascontiguousarray(eta, dtype=np.uint64)), ctypes.c_int(m), Z.ptr(np.ascontiguousarray(gen)),
       Z.ptr(x), Z.ptr(out))
    assert L.zkg_last_status() == 0, L.zkg_last_error()
    return out


def _asym(zk, curve, ms, mt, gs, gt, x):
    L = zk.lib()
    fn = getattr(L, "%s_poly_mont_ntt_forward_asymmetric" % Z.NAMES[curve])
    x = np.ascontiguousarray(x, dtype=np.uint64)
    out = np.zeros((1 << mt, 4), np.uint64)
    fn(ctypes.c_int(ms), ctypes.c_int(mt), Z.ptr(np.ascontiguousarray(gs)), Z.ptr(np.ascontiguousarray(gt)),
       Z.ptr(x), Z.ptr(out))
    assert L.zkg_last_status() == 0, L.zkg_last_error()
    return out


@pytest.mark.parametrize("curve", Z.CURVES)
def test_shifted_and_asymmetric_ntt_golden_reference_vectors(zk, curve):
    d = np.load(os.path.join(Z.GOLDEN, "ntt_shifted_%s.npz" % Z.NAMES[curve]))
    for name in sorted({k.split("__")[0] for k in d.files}):
        if name.startswith("asymmetric"):
            got = _asym(zk, curve, int(d[name + "__ms"][0]), int(d[name + "__mt"][0]), d[name + "__gs"],
                        d[name + "__gt"], d[name + "__x"])
        else:
            fn = "inverse_shifted" if name.startswith("inverse") else "forward_shifted"
            got = _shifted(zk, curve, fn, d[name + "__eta"], int(d[name + "__m"][0]), d[name + "__gen"], d[name + "__x"])
        assert np.array_equal(got, d[name + "__out"]), name


@pytest.mark.parametrize("curve", Z.CURVES)
def test_shifted_and_asymmetric_ntt_vs_oracle(zk, curve):
    for m in (0, 1, 11, 16):
        x = Z.rand_fr(curve, 1 << m, 17000 + m)
        eta = Z.rand_fr(curve, 1, 17100 + m)[0]
        gen = Z.fft_gen(curve, m)
        for inv, name in ((False, "forward_shifted"), (True, "inverse_shifted")):
            assert np.array_equal(_shifted(zk, curve, name, eta, m, gen, x),
                                  Z.oracle_ntt_shifted(curve, m, eta, gen, x, inv)), (m, name)
    for ms, mt in ((0, 3), (3, 3), (10, 13), (14, 16)):
        x = Z.rand_fr(curve, 1 << ms, 17200 + ms)
        gs, gt = Z.fft_gen(curve, ms), Z.fft_gen(curve, mt)
        assert np.array_equal(_asym(zk, curve, ms, mt, gs, gt, x), Z.oracle_ntt_asymmetric(curve, ms, mt, gs, gt, x)), (ms, mt)


@pytest.mark.parametrize("key", ["bn128_20", "bls12_381_20", "bn128_24", "bls12_381_24"])
def test_ntt_whole_vector_matches_reference_digest(zk, key):
    """forward and inverse NTT of the seeded 2^20 / 2^24 vector, through the drop-in entry points
    and the device entry point, byte-equal to the reference C's output
    (bn128_poly_mont.c:452-473, 601-622 and the BLS12-381 twins)"""
    import torch
    case = Z.ntt_large_cases()[key]
    curve, m = case["curve"], case["m"]
    x = Z.rand_fr(curve, 1 << m, case["seed"])
    assert Z.sha256(x) == case["input_sha256"]
    gen = Z.fft_gen(curve, m)
    assert Z.sha256(dropin(zk, curve, False, m, gen, x)) == case["forward_sha256"]
    assert Z.sha256(dropin(zk, curve, True, m, gen, x)) == case["inverse_sha256"]
    d_x = torch.from_numpy(x.view(np.int64)).cuda()
    d_y = torch.empty_like(d_x)
    for inv, k in ((False, "forward_sha256"), (True, "inverse_sha256")):
        zk.ntt_device(curve, m, d_x, d_y, inverse=inv, gen=gen)
        torch.cuda.synchronize()
        assert Z.sha256(d_y.cpu().numpy().view(np.uint64)) == case[k], (key, inv)


def _free_device_memory(zk):
    import torch
    zk.lib().zkg_release_cache()
    torch.cuda.empty_cache()
    return torch.cuda.mem_get_info()[0]


def test_ntt_maximum_sizes(zk):
    """The library's largest transforms: m up to 30, the bound of the reference's `int N = 1 << m`
    (bn128_poly_mont.c:453; the reference itself aborts from m = 27, where its int buffer size
    overflows), with any generator. BLS12-381 at 2^30 (a generator of order 2^30 exists): a sparse
    input's transform y_k = sum_j v_j g^(jk) at sampled k. BN254 at 2^29 (beyond its two-adicity:
    an arbitrary generator, so no closed form): a dense round trip, which holds for any generator
    because every butterfly is inverted exactly. Device buffers only (4 GB-34 GB vectors)."""
    import torch
    need = 150 << 30
    if _free_device_memory(zk) < need:
        pytest.skip("needs 150 GB of free device memory")
    try:
        # BLS12-381, m = 30, sparse input
        curve, m = Z.BLS12_381, 30
        N = 1 << m
        r = Z.R[curve]
        rng = np.random.default_rng(18000)
        terms = {int(j): int(rng.integers(1, 1 << 62)) for j in rng.integers(0, N, 5)}
        terms[0] = 7
        terms[N - 1] = 11
        x = torch.zeros((N, 4), dtype=torch.int64, device="cuda")
        for j, v in terms.items():
            x[j] = torch.from_numpy(Z.to_limbs(v, 4).view(np.int64))
        y = torch.empty_like(x)
        gen = Z.fft_gen(curve, m)
        zk.ntt_device(curve, m, x, y, inverse=False, gen=gen)
        torch.cuda.synchronize()
        g = Z.from_limbs(gen) * pow(1 << 256, -1, r) % r
        for k in [0, 1, 2, N // 2, N - 1] + [int(t) for t in rng.integers(0, N, 8)]:
            want = sum(v * pow(g, j * k, r) for j, v in terms.items()) % r
            got = Z.from_limbs(y[k].cpu().numpy().view(np.uint64))
            assert got == want, k
        del x, y
        _free_device_memory(zk)
        # BN254, m = 29, dense round trip with an arbitrary generator
        curve, m = Z.BN254, 29
        N = 1 << m
        x = torch.randint(0, 256, (N * 32,), dtype=torch.uint8, device="cuda").view(torch.int64).view(N, 4)
        x[:, 3] &= (1 << 61) - 1   # below r (r > 2^253)
        gen = Z.to_limbs(123456789123456789 * (1 << 256) % Z.R[curve], 4)
        y = torch.empty_like(x)
        zk.ntt_device(curve, m, x, y, inverse=False, gen=gen)
        z = torch.empty_like(x)
        zk.ntt_device(curve, m, y, z, inverse=True, gen=gen)
        torch.cuda.synchronize()
        assert not torch.equal(y, x)
        assert torch.equal(z, x)
        del x, y, z
    finally:
        _free_device_memory(zk)
