"""GPU parity tests for the G1 group FFT and the binary MSMs through the drop-in C ABI.

Group FFT (*_G1_{proj,jac}_fft_{forward,inverse}, lib/cbits/curves/g1/proj/bn128_G1_proj.c:791-902):
the reference normalises its outputs, so outputs are compared byte for byte with the golden
vectors of the reference C and with the oracle restatement; at larger sizes the FFT of k_i G must
be [NTT(k)_j] G and the inverse must undo the forward.

Binary MSMs (*_MSM_binary_coeff_*, *_multi_MSM_binary_coeff_*, bn128_G1_proj.c:684-782): affine
outputs byte for byte, projective / Jacobian after normalisation; at larger sizes against the
oracle on sampled rows and through row + complement = sum of all bases.
"""
import ctypes
import os

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu


def golden(kind, curve):
    return np.load(os.path.join(Z.GOLDEN, "%s_%s.npz" % (kind, Z.NAMES[curve])))


def case_names(d):
    return sorted({k.split("__")[0] for k in d.files})


def fft_call(zk, curve, fam, fn, m, gen, src):
    L = zk.lib()
    src = np.ascontiguousarray(src, dtype=np.uint64)
    gen = np.ascontiguousarray(gen, dtype=np.uint64)
    out = np.zeros_like(src)
    getattr(L, "%s_G1_%s_fft_%s" % (Z.NAMES[curve], fam, fn))(ctypes.c_int(m), Z.ptr(gen), Z.ptr(src), Z.ptr(out))
    assert L.zkg_last_status() == 0, L.zkg_last_error()
    return out


def affine_rows(curve, fam, pts):
    conv = Z.proj_to_affine if fam == "proj" else Z.jac_to_affine
    return np.stack([conv(curve, p) for p in pts])


def rand_points(curve, n, seed, jac):
    aff = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, seed))
    lam = [Z.from_limbs(v) for v in Z.rand_fr(curve, n, seed + 1)]
    return Z.scaled_points(curve, aff, lam, jac)


# ------------------------------------------------------------------------------ group FFT

@pytest.mark.parametrize("curve", Z.CURVES)
def test_g1_fft_golden_reference_vectors(zk, curve):
    d = golden("g1fft", curve)
    names = case_names(d)
    assert len(names) >= 10
    for name in names:
        m, gen = int(d[name + "__m"][0]), d[name + "__gen"]
        for fam in ("proj", "jac"):
            src = d[name + "__src_" + fam]
            for fn in ("forward", "inverse"):
                got = fft_call(zk, curve, fam, fn, m, gen, src)
                assert np.array_equal(got, d["%s__%s_%s" % (name, fam, fn)]), (name, fam, fn)


@pytest.mark.parametrize("curve", Z.CURVES)
@pytest.mark.parametrize("m", [1, 2, 7, 8])
def test_g1_fft_random_vs_oracle(zk, curve, m):
    for fam in ("proj", "jac"):
        src = rand_points(curve, 1 << m, 9100 + m, fam == "jac")
        src[3 % (1 << m)] = src[0]          # a repeated point (doubling inside the butterflies)
        for gen, tag in ((Z.fft_gen(curve, m), "std"), (Z.rand_fr(curve, 1, 9200 + m)[0], "odd")):
            for inv, fn in ((0, "forward"), (1, "inverse")):
                got = fft_call(zk, curve, fam, fn, m, gen, src)
                want = Z.oracle_g1_fft(curve, fam == "jac", m, gen, src, inv)
                assert np.array_equal(got, want), (fam, tag, fn)


def _discrete_log_check(zk, curve, m, seed):
    """x_i = k_i G: forward FFT must give [NTT(k)_j] G, and the inverse must return x"""
    import torch
    n = 1 << m
    nl = Z.NLP[curve]
    ks = Z.rand_fr(curve, n, seed)
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((n, 2 * nl), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(curve, n, d_k, d_b)
    torch.cuda.synchronize()
    aff = d_b.cpu().numpy().view(np.uint64)
    lam = [Z.from_limbs(v) for v in Z.rand_fr(curve, n, seed + 1)]
    src = Z.scaled_points(curve, aff, lam, False)
    gen = Z.fft_gen(curve, m)
    y = zk.forward_fft(curve, m, src)
    # NTT of the exponents on the CPU oracle, then [.]G on the device
    e = Z.fr_from_mont_array(curve, Z.oracle_ntt(curve, m, gen, Z.fr_to_mont_array(curve, ks), 0))
    d_e = torch.from_numpy(np.ascontiguousarray(e).view(np.int64)).cuda()
    zk.g1_gen_mul_device(curve, n, d_e, d_b)
    torch.cuda.synchronize()
    want_aff = d_b.cpu().numpy().view(np.uint64)
    one = Z.to_limbs((1 << (64 * nl)) % Z.P[curve], nl)
    want = np.zeros((n, 3 * nl), np.uint64)
    want[:, :2 * nl] = want_aff
    want[:, 2 * nl:] = one
    inf = np.all(want_aff == 0, axis=1)
    want[inf] = 0
    want[inf, nl:2 * nl] = one
    assert np.array_equal(y, want)
    back = zk.inverse_fft(curve, m, y)
    norm = np.zeros_like(src)
    norm[:, :2 * nl] = aff
    norm[:, 2 * nl:] = one
    ainf = np.all(aff == 0, axis=1)
    norm[ainf] = 0
    norm[ainf, nl:2 * nl] = one
    assert np.array_equal(back, norm)


def test_g1_fft_bn254_2pow14_discrete_logs(zk):
    _discrete_log_check(zk, Z.BN254, 14, 9300)


def test_g1_fft_bls12_381_2pow12_discrete_logs(zk):
    _discrete_log_check(zk, Z.BLS12_381, 12, 9400)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_g1_fft_device_api_matches_host(zk, curve):
    import torch
    m = 6
    for jac in (False, True):
        src = rand_points(curve, 1 << m, 9500, jac)
        d_src = torch.from_numpy(src.view(np.int64)).cuda()
        d_out = torch.empty_like(d_src)
        for inv in (False, True):
            zk.g1_fft_device(curve, m, d_src, d_out, inverse=inv, jac=jac)
            host = (zk.inverse_fft if inv else zk.forward_fft)(curve, m, src, jac=jac)
            assert np.array_equal(d_out.cpu().numpy().view(np.uint64), host)
        # in place
        zk.g1_fft_device(curve, m, d_src, d_src, inverse=False, jac=jac)
        assert np.array_equal(d_src.cpu().numpy().view(np.uint64), zk.forward_fft(curve, m, src, jac=jac))


def test_g1_fft_rejects_bad_arguments(zk):
    L = zk.lib()
    g = np.zeros(4, np.uint64)
    buf = np.zeros(24, np.uint64)
    assert L.zkg_g1_fft(0, 0, -1, Z.ptr(g), Z.ptr(buf), Z.ptr(buf), 0) != 0
    assert L.zkg_g1_fft(0, 0, 27, Z.ptr(g), Z.ptr(buf), Z.ptr(buf), 0) != 0
    assert L.zkg_g1_fft(7, 0, 1, Z.ptr(g), Z.ptr(buf), Z.ptr(buf), 0) != 0
    assert L.zkg_g1_fft(0, 0, 1, None, Z.ptr(buf), Z.ptr(buf), 0) != 0


# ------------------------------------------------------------------------------ binary MSMs

BIN_KINDS = [("proj", "proj"), ("proj", "affine"), ("jac", "jac"), ("jac", "affine")]


def bin_call(zk, curve, fam, kind, coeffs, bases, multi):
    L = zk.lib()
    nl = Z.NLP[curve]
    co = np.ascontiguousarray(coeffs, dtype=np.uint8)
    b = np.ascontiguousarray(bases, dtype=np.uint64)
    nrows, npts = co.shape
    out = np.zeros((nrows, (2 if kind == "affine" else 3) * nl), np.uint64)
    name = Z.NAMES[curve]
    if multi:
        fn = getattr(L, "%s_G1_%s_multi_MSM_binary_coeff_%s_out" % (name, fam, kind))
        fn(ctypes.c_int(nrows), ctypes.c_int(npts), Z.row_pointers(co), Z.ptr(b), Z.ptr(out))
    else:
        assert nrows == 1
        fn = getattr(L, "%s_G1_%s_MSM_binary_coeff_%s_out" % (name, fam, kind))
        fn(ctypes.c_int(npts), Z.ptr(co), Z.ptr(b), Z.ptr(out))
    assert L.zkg_last_status() == 0, L.zkg_last_error()
    return out


def bin_affine(curve, fam, kind, out):
    if kind == "affine":
        return out
    return affine_rows(curve, fam, out) if out.shape[0] else out[:, :2 * Z.NLP[curve]]


@pytest.mark.parametrize("curve", Z.CURVES)
def test_binary_msm_golden_reference_vectors(zk, curve):
    d = golden("msm_binary", curve)
    names = case_names(d)
    assert len(names) >= 20
    nl = Z.NLP[curve]
    one = Z.to_limbs((1 << (64 * nl)) % Z.P[curve], nl)
    for name in names:
        co, bases = d[name + "__coeffs"], d[name + "__bases"]
        multi = name.startswith("multi")
        want = d[name + "__proj_affine"]
        for fam, kind in BIN_KINDS:
            got = bin_call(zk, curve, fam, kind, co, bases, multi)
            assert np.array_equal(bin_affine(curve, fam, kind, got), want), (name, fam, kind)
            if kind != "affine":
                # normalised outputs: (x, y, 1); identity (0,1,0) projective, (1,1,0) Jacobian
                for r in range(co.shape[0]):
                    if np.all(want[r] == np.uint64(Z.U64)):
                        x0 = one if fam == "jac" else np.zeros(nl, np.uint64)
                        assert np.array_equal(got[r], np.concatenate([x0, one, np.zeros(nl, np.uint64)])), name
                    else:
                        assert np.array_equal(got[r], np.concatenate([want[r], one])), name


@pytest.mark.parametrize("curve", Z.CURVES)
@pytest.mark.parametrize("nrows,npts", [(1, 3000), (3, 500), (17, 700), (64, 1000), (300, 200), (1000, 64)])
def test_binary_msm_random_vs_oracle(zk, curve, nrows, npts):
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, npts, 9600 + npts))
    co = (Z.splitmix64(9700 + nrows, nrows * npts) & np.uint64(1)).astype(np.uint8).reshape(nrows, npts)
    got = bin_call(zk, curve, "proj", "affine", co, bases, True)
    want = affine_rows(curve, "proj", Z.oracle_msm_binary(curve, co, bases))
    assert np.array_equal(got, want)
    if nrows == 1:
        assert np.array_equal(bin_call(zk, curve, "proj", "affine", co, bases, False), want)


def _binary_large(zk, curve, nrows, npts, seed, sample_rows):
    """large binary MSMs (several column chunks): sampled rows against the oracle, and
    row + complement = sum of all bases for every row"""
    import torch
    nl = Z.NLP[curve]
    ks = Z.rand_fr(curve, npts, seed)
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((npts, 2 * nl), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(curve, npts, d_k, d_b)
    torch.cuda.synchronize()
    bases = d_b.cpu().numpy().view(np.uint64)
    co = (Z.splitmix64(seed + 1, nrows * npts) & np.uint64(1)).astype(np.uint8).reshape(nrows, npts)
    got = zk.binary_multi_msm(curve, co, bases, affine=True)
    comp = zk.binary_multi_msm(curve, 1 - co, bases, affine=True)
    total = zk.binary_multi_msm(curve, np.ones((1, npts), np.uint8), bases, affine=True)[0]
    tot_std = Z.py_affine_std(curve, total)
    for r in range(nrows):
        s = Z.py_add(curve, Z.py_affine_std(curve, got[r]), Z.py_affine_std(curve, comp[r]))
        assert s == tot_std, r
    for r in sample_rows:
        want = affine_rows(curve, "proj", Z.oracle_msm_binary(curve, co[r:r + 1], bases))[0]
        assert np.array_equal(got[r], want), r
    # device API on the same data
    d_co = torch.from_numpy(co).cuda()
    d_out = torch.empty((nrows, 2 * nl), dtype=torch.int64, device="cuda")
    zk.msm_binary_device(curve, nrows, npts, d_co, npts, d_b, d_out, kind=zk.OUT_AFFINE)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy().view(np.uint64), got)


def test_binary_msm_bn254_many_rows_chunked(zk):
    _binary_large(zk, Z.BN254, 64, 1 << 20, 9800, [0, 63])


def test_binary_msm_bls12_381_single_row_chunked(zk):
    _binary_large(zk, Z.BLS12_381, 1, (1 << 19) + 12345, 9900, [0])


def test_binary_msm_rejects_bad_arguments(zk):
    L = zk.lib()
    b = np.zeros(16, np.uint64)
    out = np.zeros(12, np.uint64)
    co = np.ones(2, np.uint8)
    rows = Z.row_pointers(co.reshape(1, 2))
    assert L.zkg_msm_binary(0, 2, -1, 2, rows, Z.ptr(b), Z.ptr(out)) != 0
    assert L.zkg_msm_binary(0, 2, 1, -2, rows, Z.ptr(b), Z.ptr(out)) != 0
    assert L.zkg_msm_binary(0, 9, 1, 2, rows, Z.ptr(b), Z.ptr(out)) != 0
    assert L.zkg_msm_binary(3, 2, 1, 2, rows, Z.ptr(b), Z.ptr(out)) != 0
    assert L.zkg_msm_binary(0, 2, 1, 2, None, Z.ptr(b), Z.ptr(out)) != 0
