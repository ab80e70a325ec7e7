"""CPU tests: the oracle restatement (oracle/zkoracle.c) is pinned to the reference.

1. against golden vectors produced by the reference C itself (tests/golden/make_golden.py);
2. against the reference C compiled here (oracle/_ref), when it was built;
3. against an independent pure-Python group law / DFT for tiny sizes.
"""
import os

import numpy as np
import pytest

import zkutil as Z


def golden(kind, curve):
    return np.load(os.path.join(Z.GOLDEN, "%s_%s.npz" % (kind, Z.NAMES[curve])))


def case_names(d):
    return sorted({k.split("__")[0] for k in d.files})


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_msm_matches_reference_golden(curve):
    d = golden("msm", curve)
    names = case_names(d)
    assert len(names) >= 20
    for name in names:
        scal, bases, nl = d[name + "__scalars"], d[name + "__bases"], int(d[name + "__nlimbs"][0])
        n = bases.shape[0]
        for mont in (0, 1):
            if mont and nl != 4:
                continue
            coeff = "mont" if mont else "std"
            proj = np.zeros(3 * Z.NLP[curve], np.uint64)
            s = np.ascontiguousarray(scal.reshape(-1))
            b = np.ascontiguousarray(bases.reshape(-1))
            assert Z.oracle().oracle_msm_proj(curve, n, Z.ptr(s), nl, mont, Z.ptr(b), Z.ptr(proj), 0) == 0
            # same algorithm and formulas as the reference: even the projective bytes agree
            assert np.array_equal(proj, d[name + "__proj_%s_proj" % coeff]), (name, coeff)
            assert np.array_equal(Z.proj_to_affine(curve, proj), d[name + "__proj_%s_affine" % coeff]), name
            assert np.array_equal(d[name + "__jac_%s_affine" % coeff], d[name + "__proj_%s_affine" % coeff])
            assert np.array_equal(Z.jac_to_affine(curve, d[name + "__jac_%s_jac" % coeff]),
                                  d[name + "__proj_%s_affine" % coeff]), name


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_ntt_matches_reference_golden(curve):
    d = golden("ntt", curve)
    for name in case_names(d):
        m, gen, x = int(d[name + "__m"][0]), d[name + "__gen"], d[name + "__x"]
        assert np.array_equal(Z.oracle_ntt(curve, m, gen, x, False), d[name + "__fwd"]), name
        assert np.array_equal(Z.oracle_ntt(curve, m, gen, x, True), d[name + "__inv"]), name


@pytest.mark.parametrize("curve", Z.CURVES)
def test_golden_bases_are_k_times_g(curve):
    """the golden bases came from the reference's scalar multiplication; the oracle's base
    generator must reproduce them (it builds the GPU-test inputs)"""
    d = golden("msm", curve)
    b = d["rand_n17__bases"]
    # regenerate with the same seed the generator used
    ks = Z.rand_fr(curve, 17, 2000 + 17)
    assert np.array_equal(Z.gen_bases_cpu(curve, ks), b)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_msm_vs_python_group_law(curve):
    ks = Z.rand_fr(curve, 5, 77)
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, 5, 78))
    aff = Z.oracle_msm_affine(curve, ks, 4, False, bases)
    pts = [Z.py_affine_std(curve, b) for b in bases]
    exp = Z.py_msm(curve, [Z.from_limbs(k) for k in ks], pts)
    assert Z.py_affine_std(curve, aff) == exp
    # Montgomery coefficients: value k*R^-1
    rinv = pow(1 << 256, -1, Z.R[curve])
    aff_m = Z.oracle_msm_affine(curve, ks, 4, True, bases)
    exp_m = Z.py_msm(curve, [Z.from_limbs(k) * rinv % Z.R[curve] for k in ks], pts)
    assert Z.py_affine_std(curve, aff_m) == exp_m


@pytest.mark.parametrize("curve", Z.CURVES)
@pytest.mark.parametrize("m", [0, 1, 2, 3, 5])
def test_oracle_ntt_vs_dft_definition(curve, m):
    """y_k = sum_i x_i g^(ik); inverse = N^-1 sum_k y_k g^(-ik)  (also covers m <= 1, where the
    reference's own NTT overruns its twiddle buffer and cannot be run)"""
    r = Z.R[curve]
    N = 1 << m
    x = Z.rand_fr(curve, N, 90 + m)
    gen = Z.fft_gen(curve, m)
    rinv = pow(1 << 256, -1, r)
    g = Z.from_limbs(gen) * rinv % r
    xs = [Z.from_limbs(v) * rinv % r for v in x]
    y = Z.oracle_ntt(curve, m, gen, x, False)
    ys = [Z.from_limbs(v) * rinv % r for v in y]
    assert ys == [sum(xs[i] * pow(g, i * k, r) for i in range(N)) % r for k in range(N)]
    z = Z.oracle_ntt(curve, m, gen, x, True)
    zs = [Z.from_limbs(v) * rinv % r for v in z]
    ninv = pow(N, -1, r)
    assert zs == [ninv * sum(xs[k] * pow(g, -i * k, r) for k in range(N)) % r for i in range(N)]


@pytest.mark.skipif(Z.reference() is None, reason="reference C not built (make -C oracle ref)")
@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_vs_reference_c_random(curve):
    import ctypes
    L = Z.reference()
    name = Z.NAMES[curve]
    for n in (7, 300):
        ks = Z.rand_fr(curve, n, 500 + n)
        bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 600 + n))
        proj = np.zeros(3 * Z.NLP[curve], np.uint64)
        getattr(L, "%s_G1_proj_MSM_mont_coeff_proj_out" % name)(ctypes.c_int(n), Z.ptr(ks), Z.ptr(bases),
                                                                Z.ptr(proj), ctypes.c_int(4))
        mine = np.zeros_like(proj)
        Z.oracle().oracle_msm_proj(curve, n, Z.ptr(ks), 4, 1, Z.ptr(bases), Z.ptr(mine), 0)
        assert np.array_equal(proj, mine)
    for m in (11, 12):
        x = Z.rand_fr(curve, 1 << m, 700 + m)
        gen = Z.fft_gen(curve, m)
        for inv, fn in ((False, "forward"), (True, "inverse")):
            out = np.zeros_like(x)
            getattr(L, "%s_poly_mont_ntt_%s" % (name, fn))(ctypes.c_int(m), Z.ptr(gen), Z.ptr(x), Z.ptr(out))
            assert np.array_equal(out, Z.oracle_ntt(curve, m, gen, x, inv))


def test_reference_window_rule():
    """c = round(log2 n - 3.5) clamped to [1, 64] (bn128_G1_proj.c:597-605)"""
    w = Z.oracle().oracle_msm_window
    assert [w(n) for n in (0, 1, 2, 1 << 10, 1 << 16, 1 << 20, 1 << 22, 1 << 24)] == [1, 1, 1, 7, 13, 17, 19, 21]


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_shifted_and_asymmetric_ntt_match_reference_golden(curve):
    d = golden("ntt_shifted", curve)
    for name in case_names(d):
        if name.startswith("asymmetric"):
            got = Z.oracle_ntt_asymmetric(curve, int(d[name + "__ms"][0]), int(d[name + "__mt"][0]),
                                          d[name + "__gs"], d[name + "__gt"], d[name + "__x"])
        else:
            got = Z.oracle_ntt_shifted(curve, int(d[name + "__m"][0]), d[name + "__eta"], d[name + "__gen"],
                                       d[name + "__x"], name.startswith("inverse"))
        assert np.array_equal(got, d[name + "__out"]), name


def normalized_affine(curve, fam, pts):
    """rows of projective (fam 'proj') or Jacobian ('jac') points -> affine rows (0xff infinity)"""
    conv = Z.proj_to_affine if fam == "proj" else Z.jac_to_affine
    return np.stack([conv(curve, p) for p in np.atleast_2d(pts)]) if len(pts) else np.zeros((0, 2 * Z.NLP[curve]),
                                                                                             np.uint64)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_g1_fft_matches_reference_golden(curve):
    d = golden("g1fft", curve)
    names = case_names(d)
    assert len(names) >= 10
    for name in names:
        m, gen = int(d[name + "__m"][0]), d[name + "__gen"]
        for fam in ("proj", "jac"):
            src = d[name + "__src_" + fam]
            for inv, fn in ((0, "forward"), (1, "inverse")):
                out = Z.oracle_g1_fft(curve, fam == "jac", m, gen, src, inv)
                # the reference normalises its outputs, so the bytes agree
                assert np.array_equal(out, d["%s__%s_%s" % (name, fam, fn)]), (name, fam, fn)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_g1_fft_is_the_ntt_on_discrete_logs(curve):
    """[NTT(k)_j] G == FFT([k_i] G)_j: the group FFT agrees with the field NTT on exponents"""
    m = 3
    ks = Z.rand_fr(curve, 1 << m, 8901)
    gen = Z.fft_gen(curve, m)
    nl = Z.NLP[curve]
    pts = Z.gen_bases_cpu(curve, ks)
    src = np.zeros((1 << m, 3 * nl), np.uint64)
    one = Z.to_limbs((1 << (64 * nl)) % Z.P[curve], nl)
    for i in range(1 << m):
        src[i, :2 * nl] = pts[i]
        src[i, 2 * nl:] = one
    for inv in (0, 1):
        out = Z.oracle_g1_fft(curve, 0, m, gen, src, inv)
        ks_m = Z.fr_to_mont_array(curve, ks)
        y = Z.fr_from_mont_array(curve, Z.oracle_ntt(curve, m, gen, ks_m, inv))
        want = Z.gen_bases_cpu(curve, y)
        got = normalized_affine(curve, "proj", out)
        want = np.where(np.all(want == 0, axis=1, keepdims=True), np.uint64(Z.U64), want)
        assert np.array_equal(got, want), inv


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_binary_msm_matches_reference_golden(curve):
    d = golden("msm_binary", curve)
    names = case_names(d)
    assert len(names) >= 20
    for name in names:
        co, bases = d[name + "__coeffs"], d[name + "__bases"]
        out = Z.oracle_msm_binary(curve, co, bases)
        aff = normalized_affine(curve, "proj", out)
        assert np.array_equal(aff, d[name + "__proj_affine"]), name
        assert np.array_equal(aff, d[name + "__jac_affine"]), name
        assert np.array_equal(aff, normalized_affine(curve, "proj", d[name + "__proj_proj"])), name
        assert np.array_equal(aff, normalized_affine(curve, "jac", d[name + "__jac_jac"])), name


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_fr_vector_ops_match_reference_golden(curve):
    d = golden("arr", curve)
    A, B = d["A"], d["B"]
    cases = sorted({k.split("__")[0] for k in d.files if "__" in k and not k.startswith("sparse")})
    assert len(cases) >= 6
    checked = 0
    for cname in cases:
        a, b, c = d[cname + "__a"], d[cname + "__b"], d[cname + "__c"]
        n = a.shape[0]
        ins = {"a": a, "b": b, "c": c}
        for fn, (op, order) in Z.FR_OPS.items():
            key = "%s__%s" % (cname, fn)
            if key not in d.files:
                continue
            args = [ins[ch] for ch in order] + [None] * (3 - len(order))
            init = np.full((n, 4), 0xABABABABABABABAB, np.uint64)
            got = Z.oracle_fr_op(curve, op, *args, ka=A, kb=B, n=n, out=init)
            assert np.array_equal(got, d[key]), key
            checked += 1
        if cname + "__dot_prod" in d.files:
            out = np.zeros(4, np.uint64)
            Z.oracle().oracle_fr_dot(curve, n, Z.ptr(np.ascontiguousarray(a)), Z.ptr(np.ascontiguousarray(b)), Z.ptr(out))
            assert np.array_equal(out, d[cname + "__dot_prod"]), cname
    assert checked >= 100
    for key in sorted({k.rsplit("__", 1)[0] for k in d.files if k.startswith("sparse")}):
        rows, cols, co, src = d[key + "__rows"], d[key + "__cols"], d[key + "__coeffs"], d[key + "__src"]
        N = d[key + "__tgt"].shape[0]
        out = np.zeros((N, 4), np.uint64)
        Z.oracle().oracle_fr_sparse(curve, N, rows.shape[0], Z.ptr(rows), Z.ptr(cols), Z.ptr(co), Z.ptr(src), Z.ptr(out))
        assert np.array_equal(out, d[key + "__tgt"]), key


@pytest.mark.parametrize("curve", Z.CURVES)
def test_reference_batch_inverse_zero_semantics(curve):
    """the reference's batch inversion inverts one product: a single zero zeroes every output"""
    d = golden("arr", curve)
    assert not np.any(d["zeros_n50__inv"])
    assert not np.any(d["zeros_n50__div"])
    assert np.any(d["rand_n100__inv"])


@pytest.mark.parametrize("curve", Z.CURVES)
def test_oracle_ntt_2pow20_matches_reference_digests(curve):
    """whole 2^20 vectors, forward and inverse: the restatement reproduces the reference C's
    output bytes (SHA-256 digests from tests/golden/make_golden.py ntt_large)"""
    case = Z.ntt_large_cases()["%s_20" % Z.NAMES[curve]]
    m = case["m"]
    x = Z.rand_fr(curve, 1 << m, case["seed"])
    assert Z.sha256(x) == case["input_sha256"]
    gen = Z.fft_gen(curve, m)
    assert Z.sha256(Z.oracle_ntt(curve, m, gen, x, False)) == case["forward_sha256"]
    assert Z.sha256(Z.oracle_ntt(curve, m, gen, x, True)) == case["inverse_sha256"]


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_identity_helper_matches_oracle(curve):
    """the pure-numpy (sum s_i k_i) G check used for full-size MSMs equals the oracle's MSM"""
    n = 3000
    ks = Z.rand_fr(curve, n, 52000 + curve)
    ss = Z.rand_fr(curve, n, 52100 + curve)
    bases = Z.gen_bases_cpu(curve, ks)
    assert np.array_equal(Z.msm_identity_affine(curve, ks, ss), Z.oracle_msm_affine(curve, ss, 4, True, bases))
    zero = np.zeros_like(ss)
    assert np.array_equal(Z.msm_identity_affine(curve, ks, zero), np.full(2 * Z.NLP[curve], Z.U64, np.uint64))


def test_closed_form_signed_digit_carry():
    """the MSM's window-major digits use carry_w = [(s mod 2^(wc)) > H_w], H_w = sum_{j<w}
    2^(jc + c - 1), in place of the sequential recoding carry (raw > 2^(c-1) -> carry 1); the
    two agree for every window of random, all-ones and boundary scalars"""
    rng = np.random.default_rng(53000)
    for c in (2, 3, 5, 13, 16, 17, 19):
        nwin = (256 + 1 + c - 1) // c
        H = [sum(1 << (j * c + c - 1) for j in range(w)) for w in range(nwin)]
        scalars = [int.from_bytes(rng.bytes(32), "little") for _ in range(200)] + [(1 << 256) - 1, 0, 1]
        scalars += [H[w] for w in range(nwin)] + [H[w] + 1 for w in range(nwin)]
        for s in scalars:
            carry = 0
            for w in range(nwin):
                assert carry == int((s % (1 << (w * c))) > H[w]), (c, w, s)
                raw = ((s >> (w * c)) & ((1 << c) - 1)) + carry
                carry = 1 if raw > (1 << (c - 1)) else 0
