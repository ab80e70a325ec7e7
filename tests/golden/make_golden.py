"""Generates tests/golden/*.npz from the reference C itself.

The reference's generated C (lib/cbits) is compiled from its own sources by `make -C oracle ref`
into oracle/_ref/libzkref.so (with corrected carry primitives; see oracle/refpatch/platform.h).
This script calls the reference's own entry points on seeded inputs and stores inputs and
outputs, so the GPU library and the oracle restatement are both pinned to the reference:

  msm_<curve>.npz  per case: bases (from the reference's *_G1_affine_scl_Fr_std of seeded k),
                   scalars, limb count, and the outputs of all eight MSM entry points
                   (*_G1_proj_MSM_{std,mont}_coeff_{proj,affine}_out, *_G1_jac_MSM_..._{jac,affine}_out)
  ntt_<curve>.npz  per case: m, generator, input, *_poly_mont_ntt_forward and _inverse outputs
  ntt_shifted_<curve>.npz  *_poly_mont_ntt_{forward,inverse}_shifted and _forward_asymmetric
  g1fft_<curve>.npz  per case: projective and Jacobian input points (random Z, some at infinity),
                   generator, *_G1_{proj,jac}_fft_forward and _inverse outputs
  msm_binary_<curve>.npz  per case: byte coefficient rows, bases, and the outputs of
                   *_G1_{proj,jac}_MSM_binary_coeff_* (one row) or *_multi_MSM_binary_coeff_*
  arr_<curve>.npz  per case: Fr input arrays a, b, c and constants A, B, and the outputs of every
                   *_arr_mont_* function (bn128_arr_mont.c) on them
  ntt_large_digests.json  SHA-256 digests of the reference's *_poly_mont_ntt_forward and _inverse
                   outputs on seeded 2^20 and 2^24 inputs (both curves; too large to store), with
                   the digest of the input so a test can check that it regenerated the same vector

m <= 1 is not generated: the reference's ntt_forward/ntt_inverse write gpows[1] into a buffer of
N/2 elements (bn128_poly_mont.c:459-460, 606-615) and corrupt the heap there; those sizes are
pinned in the tests against the DFT definition instead.

Usage: make -C oracle ref && python tests/golden/make_golden.py [msm ntt ... ntt_large]
"""
import ctypes
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import zkutil as Z  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def ref_lib():
    L = Z.reference()
    if L is None:
        raise SystemExit("oracle/_ref/libzkref.so missing: run `make -C oracle ref` first")
    return L


def ref_bases(L, curve, ks):
    name = Z.NAMES[curve]
    nl = Z.NLP[curve]
    gen = (ctypes.c_uint64 * (2 * nl)).in_dll(L, "%s_G1_affine_gen_G1" % name)
    out = np.zeros((ks.shape[0], 2 * nl), dtype=np.uint64)
    fn = getattr(L, "%s_G1_affine_scl_Fr_std" % name)
    for i in range(ks.shape[0]):
        k = np.ascontiguousarray(ks[i])
        fn(Z.ptr(k), gen, Z.ptr(out[i]))
    # the reference writes all-0xff for the identity; MSM inputs use (0,0)
    inf = np.all(out == np.uint64(Z.U64), axis=1)
    out[inf] = 0
    return out


def msm_outputs(L, curve, scalars, nlimbs, bases):
    name = Z.NAMES[curve]
    nl = Z.NLP[curve]
    n = bases.shape[0]
    res = {}
    s = np.ascontiguousarray(scalars.reshape(-1))
    b = np.ascontiguousarray(bases.reshape(-1))
    for coeff in ("std", "mont"):
        if coeff == "mont" and nlimbs != 4:
            continue
        for fam, kinds in (("proj", ("proj", "affine")), ("jac", ("jac", "affine"))):
            for kind in kinds:
                out = np.zeros((2 if kind == "affine" else 3) * nl, dtype=np.uint64)
                fn = getattr(L, "%s_G1_%s_MSM_%s_coeff_%s_out" % (name, fam, coeff, kind))
                fn(ctypes.c_int(n), Z.ptr(s), Z.ptr(b), Z.ptr(out), ctypes.c_int(nlimbs))
                res["%s_%s_%s" % (fam, coeff, kind)] = out
    return res


def msm_cases(curve, L):
    r = Z.R[curve]
    cases = {}

    def bases_for(n, seed):
        return ref_bases(L, curve, Z.rand_fr(curve, n, seed))

    for n in (0, 1, 2, 3, 5, 17, 64, 100, 257, 1000):
        cases["rand_n%d" % n] = (Z.rand_fr(curve, n, 1000 + n), 4, bases_for(n, 2000 + n))
    cases["zeros_n50"] = (np.zeros((50, 4), np.uint64), 4, bases_for(50, 3001))
    rep = np.repeat(bases_for(1, 3002), 64, axis=0)
    cases["repeat_base_n64"] = (Z.rand_fr(curve, 64, 3003), 4, rep)
    eq = np.repeat(Z.rand_fr(curve, 1, 3004), 64, axis=0)
    cases["repeat_base_same_scalar_n64"] = (eq, 4, rep.copy())
    # P, -P pairs with equal scalars (bucket sums that cancel) plus a tail of random terms
    pb = bases_for(16, 3005)
    neg = pb.copy()
    nl = Z.NLP[curve]
    for i in range(16):
        y = Z.from_limbs(pb[i, nl:])
        neg[i, nl:] = Z.to_limbs((Z.P[curve] - y) % Z.P[curve], nl)
    pairs = np.empty((32, 2 * nl), np.uint64)
    pairs[0::2], pairs[1::2] = pb, neg
    ps = np.repeat(Z.rand_fr(curve, 16, 3006), 2, axis=0)
    cases["neg_pairs_n32"] = (ps, 4, pairs)
    cases["neg_pairs_only_cancel_n32"] = (ps.copy(), 4, pairs.copy())
    cases["neg_pairs_plus_rand_n40"] = (np.concatenate([ps, Z.rand_fr(curve, 8, 3007)]), 4,
                                        np.concatenate([pairs, bases_for(8, 3008)]))
    ib = bases_for(40, 3009)
    ib[::3] = 0
    cases["inf_bases_n40"] = (Z.rand_fr(curve, 40, 3010), 4, ib)
    cases["equal_scalars_n200"] = (np.repeat(Z.rand_fr(curve, 1, 3011), 200, axis=0), 4, bases_for(200, 3012))
    cases["small_scalars_n100"] = (Z.ints_to_array(list(range(100)), 4), 4, bases_for(100, 3013))
    cases["max_scalar_n20"] = (Z.ints_to_array([r - 1] * 20, 4), 4, bases_for(20, 3014))
    full = Z.splitmix64(3015, 64 * 4).reshape(64, 4)
    cases["std_full_256bit_n64"] = (full, 4, bases_for(64, 3016))
    cases["std_all_ones_n16"] = (np.full((16, 4), Z.U64, np.uint64), 4, bases_for(16, 3017))
    for nlimbs, n in ((1, 50), (2, 50), (3, 30), (5, 30), (8, 10)):
        cases["std_nlimbs%d_n%d" % (nlimbs, n)] = (Z.splitmix64(4000 + nlimbs, n * nlimbs).reshape(n, nlimbs),
                                                   nlimbs, bases_for(n, 4100 + nlimbs))
    return cases


def make_msm(curve):
    L = ref_lib()
    data = {}
    for name, (scal, nlimbs, bases) in msm_cases(curve, L).items():
        data[name + "__scalars"] = np.ascontiguousarray(scal, dtype=np.uint64)
        data[name + "__bases"] = np.ascontiguousarray(bases, dtype=np.uint64)
        data[name + "__nlimbs"] = np.array([nlimbs])
        for k, v in msm_outputs(L, curve, scal, nlimbs, bases).items():
            data[name + "__" + k] = v
    path = os.path.join(OUT, "msm_%s.npz" % Z.NAMES[curve])
    np.savez_compressed(path, **data)
    return path


def make_ntt(curve):
    L = ref_lib()
    name = Z.NAMES[curve]
    data = {}
    cases = [("std_m%d" % m, m, Z.fft_gen(curve, m)) for m in range(2, 11)]
    # arbitrary (non-primitive) generators pin the exact butterfly network, not only the DFT
    for m, seed in ((4, 5001), (7, 5002), (9, 5003)):
        cases.append(("oddgen_m%d" % m, m, Z.rand_fr(curve, 1, seed)[0]))
    cases.append(("gen_one_m5", 5, Z.to_limbs((1 << 256) % Z.R[curve], 4)))
    for cname, m, gen in cases:
        x = Z.rand_fr(curve, 1 << m, 6000 + m)
        gen = np.ascontiguousarray(gen, dtype=np.uint64)
        fwd = np.zeros_like(x)
        inv = np.zeros_like(x)
        getattr(L, "%s_poly_mont_ntt_forward" % name)(ctypes.c_int(m), Z.ptr(gen), Z.ptr(x), Z.ptr(fwd))
        getattr(L, "%s_poly_mont_ntt_inverse" % name)(ctypes.c_int(m), Z.ptr(gen), Z.ptr(x), Z.ptr(inv))
        data[cname + "__m"] = np.array([m])
        data[cname + "__gen"] = gen
        data[cname + "__x"] = x
        data[cname + "__fwd"] = fwd
        data[cname + "__inv"] = inv
    path = os.path.join(OUT, "ntt_%s.npz" % name)
    np.savez_compressed(path, **data)
    return path


def make_ntt_shifted(curve):
    """*_poly_mont_ntt_forward_shifted / _inverse_shifted / _forward_asymmetric
    (bn128_poly_mont.c:477-555, 626-641)"""
    L = ref_lib()
    name = Z.NAMES[curve]
    data = {}
    for m in (2, 5, 9):
        x = Z.rand_fr(curve, 1 << m, 7000 + m)
        eta = np.ascontiguousarray(Z.rand_fr(curve, 1, 7100 + m)[0])
        gen = np.ascontiguousarray(Z.fft_gen(curve, m))
        for fn in ("forward_shifted", "inverse_shifted"):
            out = np.zeros_like(x)
            getattr(L, "%s_poly_mont_ntt_%s" % (name, fn))(Z.ptr(eta), ctypes.c_int(m), Z.ptr(gen), Z.ptr(x), Z.ptr(out))
            key = "%s_m%d" % (fn, m)
            data[key + "__m"] = np.array([m])
            data[key + "__eta"] = eta
            data[key + "__gen"] = gen
            data[key + "__x"] = x
            data[key + "__out"] = out
    for ms, mt in ((2, 4), (4, 4), (5, 8), (7, 9)):
        x = Z.rand_fr(curve, 1 << ms, 7200 + 16 * ms + mt)
        gs = np.ascontiguousarray(Z.fft_gen(curve, ms))
        gt = np.ascontiguousarray(Z.fft_gen(curve, mt))
        out = np.zeros((1 << mt, 4), np.uint64)
        L_fn = getattr(L, "%s_poly_mont_ntt_forward_asymmetric" % name)
        L_fn(ctypes.c_int(ms), ctypes.c_int(mt), Z.ptr(gs), Z.ptr(gt), Z.ptr(x), Z.ptr(out))
        key = "asymmetric_%d_%d" % (ms, mt)
        data[key + "__ms"] = np.array([ms])
        data[key + "__mt"] = np.array([mt])
        data[key + "__gs"] = gs
        data[key + "__gt"] = gt
        data[key + "__x"] = x
        data[key + "__out"] = out
    path = os.path.join(OUT, "ntt_shifted_%s.npz" % name)
    np.savez_compressed(path, **data)
    return path


def make_g1fft(curve):
    """*_G1_{proj,jac}_fft_forward / _inverse (bn128_G1_proj.c:831,893; bn128_G1_jac.c:880,942)"""
    L = ref_lib()
    name = Z.NAMES[curve]
    data = {}
    cases = [("std_m%d" % m, m, Z.fft_gen(curve, m), None) for m in range(0, 7)]
    cases.append(("oddgen_m3", 3, Z.rand_fr(curve, 1, 8101)[0], None))
    cases.append(("oddgen_m5", 5, Z.rand_fr(curve, 1, 8102)[0], None))
    cases.append(("gen_one_m3", 3, Z.to_limbs((1 << 256) % Z.R[curve], 4), None))
    cases.append(("inf_points_m4", 4, Z.fft_gen(curve, 4), "inf"))
    cases.append(("repeated_points_m4", 4, Z.fft_gen(curve, 4), "rep"))
    for cname, m, gen, special in cases:
        n = 1 << m
        aff = ref_bases(L, curve, Z.rand_fr(curve, n, 8200 + m))
        if special == "inf":
            aff[::3] = 0
        if special == "rep":
            aff[:] = aff[0]
        lam = [Z.from_limbs(v) for v in Z.rand_fr(curve, n, 8300 + m)]
        gen = np.ascontiguousarray(gen, dtype=np.uint64)
        data[cname + "__m"] = np.array([m])
        data[cname + "__gen"] = gen
        for fam in ("proj", "jac"):
            src = Z.scaled_points(curve, aff, lam, fam == "jac")
            data[cname + "__src_" + fam] = src
            for fn in ("forward", "inverse"):
                out = np.zeros_like(src)
                getattr(L, "%s_G1_%s_fft_%s" % (name, fam, fn))(ctypes.c_int(m), Z.ptr(gen), Z.ptr(src), Z.ptr(out))
                data["%s__%s_%s" % (cname, fam, fn)] = out
    path = os.path.join(OUT, "g1fft_%s.npz" % name)
    np.savez_compressed(path, **data)
    return path


def make_msm_binary(curve):
    """*_G1_{proj,jac}_MSM_binary_coeff_* (bn128_G1_proj.c:684-698, bn128_G1_jac.c:733-748) and
    *_multi_MSM_binary_coeff_* (bn128_G1_proj.c:718-782, bn128_G1_jac.c:767-835)"""
    L = ref_lib()
    name = Z.NAMES[curve]
    nl = Z.NLP[curve]
    data = {}
    cases = []
    for n in (0, 1, 5, 100, 1000):
        cases.append(("single_n%d" % n, 1, n, None))
    cases += [("single_zeros_n64", 1, 64, "zeros"), ("single_ones_n64", 1, 64, "ones"),
              ("single_inf_bases_n60", 1, 60, "inf"), ("single_repeat_n32", 1, 32, "rep"),
              ("single_negpairs_n32", 1, 32, "neg")]
    for nrows, npts in ((2, 64), (7, 100), (40, 300), (130, 64), (300, 40), (16, 1), (5, 0)):
        cases.append(("multi_r%d_n%d" % (nrows, npts), nrows, npts, None))
    cases += [("multi_repeat_r20_n48", 20, 48, "rep"), ("multi_negpairs_r20_n48", 20, 48, "neg"),
              ("multi_inf_bases_r20_n48", 20, 48, "inf")]
    for cname, nrows, npts, special in cases:
        seed = 8500 + 131 * nrows + npts
        bases = ref_bases(L, curve, Z.rand_fr(curve, npts, seed))
        if special == "inf":
            bases[::4] = 0
        if special == "rep":
            bases[:] = bases[0] if npts else bases
        if special == "neg":
            for i in range(1, npts, 2):
                bases[i, :nl] = bases[i - 1, :nl]
                y = Z.from_limbs(bases[i - 1, nl:])
                bases[i, nl:] = Z.to_limbs((Z.P[curve] - y) % Z.P[curve], nl)
        co = (Z.splitmix64(seed, nrows * npts) % np.uint64(4)).astype(np.uint8).reshape(nrows, npts)
        co[co == 3] = 200   # any non-zero byte selects the point
        co[co == 2] = 0
        if special == "zeros":
            co[:] = 0
        if special in ("ones", "neg") and nrows == 1:
            co[:] = 1
        co = np.ascontiguousarray(co)
        bases = np.ascontiguousarray(bases)
        data[cname + "__coeffs"] = co
        data[cname + "__bases"] = bases
        for fam, kinds in (("proj", ("proj", "affine")), ("jac", ("jac", "affine"))):
            for kind in kinds:
                w = (2 if kind == "affine" else 3) * nl
                out = np.zeros((nrows, w), np.uint64)
                if cname.startswith("single"):
                    fn = getattr(L, "%s_G1_%s_MSM_binary_coeff_%s_out" % (name, fam, kind))
                    fn(ctypes.c_int(npts), Z.ptr(co), Z.ptr(bases), Z.ptr(out))
                else:
                    fn = getattr(L, "%s_G1_%s_multi_MSM_binary_coeff_%s_out" % (name, fam, kind))
                    fn(ctypes.c_int(nrows), ctypes.c_int(npts), Z.row_pointers(co), Z.ptr(bases), Z.ptr(out))
                data["%s__%s_%s" % (cname, fam, kind)] = out
    path = os.path.join(OUT, "msm_binary_%s.npz" % name)
    np.savez_compressed(path, **data)
    return path


# (name, argument pattern) of the *_arr_mont_* functions (lib/cbits/curves/array/mont/bn128_arr_mont.h)
ARR_FUNCS = [
    ("from_std", "u"), ("to_std", "u"), ("neg", "u"), ("sqr", "u"), ("inv", "u"),
    ("add", "b"), ("sub", "b"), ("mul", "b"), ("div", "b"),
    ("mul_add", "t"), ("mul_sub", "t"),
    ("neg_inplace", "iu"), ("sqr_inplace", "iu"), ("inv_inplace", "iu"),
    ("add_inplace", "ib"), ("sub_inplace", "ib"), ("mul_inplace", "ib"), ("div_inplace", "ib"),
    ("sub_inplace_reverse", "ib"),
    ("dot_prod", "dot"), ("powers", "pow"), ("mul_by_powers", "mbp"),
    ("scale", "scale"), ("scale_inplace", "iscale"),
    ("Ax_plus_y", "axpy"), ("Ax_plus_y_inplace", "iaxpy"), ("Ax_plus_By", "axpby"), ("Ax_plus_By_inplace", "iaxpby"),
    ("is_valid", "pu"), ("is_zero", "pu"), ("is_one", "pu"), ("is_equal", "pb"),
]


def call_arr(L, curve, fn, pat, n, a, b, c, A, B, tgt0):
    """run one *_arr_mont_* function; returns its output array (or the predicate's byte)"""
    f = getattr(L, "%s_arr_mont_%s" % (Z.NAMES[curve], fn))
    ci = ctypes.c_int(n)
    tgt = np.array(tgt0, copy=True)
    if pat == "u":
        f(ci, Z.ptr(a), Z.ptr(tgt))
    elif pat == "b":
        f(ci, Z.ptr(a), Z.ptr(b), Z.ptr(tgt))
    elif pat == "t":
        f(ci, Z.ptr(a), Z.ptr(b), Z.ptr(c), Z.ptr(tgt))
    elif pat == "iu":
        tgt = np.array(a, copy=True)
        f(ci, Z.ptr(tgt))
    elif pat == "ib":
        tgt = np.array(a, copy=True)
        f(ci, Z.ptr(tgt), Z.ptr(b))
    elif pat == "dot":
        tgt = np.zeros(4, np.uint64)
        f(ci, Z.ptr(a), Z.ptr(b), Z.ptr(tgt))
    elif pat == "pow":
        f(ci, Z.ptr(A), Z.ptr(B), Z.ptr(tgt))
    elif pat == "mbp":
        f(ci, Z.ptr(A), Z.ptr(B), Z.ptr(a), Z.ptr(tgt))
    elif pat == "scale":
        f(ci, Z.ptr(A), Z.ptr(a), Z.ptr(tgt))
    elif pat == "iscale":
        tgt = np.array(a, copy=True)
        f(ci, Z.ptr(A), Z.ptr(tgt))
    elif pat == "axpy":
        f(ci, Z.ptr(A), Z.ptr(a), Z.ptr(b), Z.ptr(tgt))
    elif pat == "iaxpy":
        tgt = np.array(a, copy=True)
        f(ci, Z.ptr(A), Z.ptr(tgt), Z.ptr(b))
    elif pat == "axpby":
        f(ci, Z.ptr(A), Z.ptr(B), Z.ptr(a), Z.ptr(b), Z.ptr(tgt))
    elif pat == "iaxpby":
        tgt = np.array(a, copy=True)
        f(ci, Z.ptr(A), Z.ptr(B), Z.ptr(tgt), Z.ptr(b))
    elif pat in ("pu", "pb"):
        f.restype = ctypes.c_uint8
        r = f(ci, Z.ptr(a), Z.ptr(b)) if pat == "pb" else f(ci, Z.ptr(a))
        return np.array([r], np.uint8)
    return tgt


def arr_cases(curve):
    r = Z.R[curve]
    cases = {}
    for n in (1, 7, 100, 1000):
        a, b, c = (Z.rand_fr(curve, n, 9000 + 10 * n + k) for k in range(3))
        cases["rand_n%d" % n] = (a, b, c)
    a, b, c = (Z.rand_fr(curve, 50, 9100 + k) for k in range(3))
    a[17] = 0
    b[3] = 0
    cases["zeros_n50"] = (a, b, c)                      # inv / div: one zero empties the batch
    one = Z.to_limbs((1 << 256) % r, 4)
    cases["ones_n20"] = (np.tile(one, (20, 1)), np.tile(one, (20, 1)), np.zeros((20, 4), np.uint64))
    big = Z.splitmix64(9200, 64 * 4).reshape(64, 4)    # any 256-bit words: from_std reduces, is_valid fails
    cases["wide_n64"] = (big, big.copy(), Z.rand_fr(curve, 64, 9201))
    return cases


def make_arr(curve):
    """*_arr_mont_* (lib/cbits/curves/array/mont/bn128_arr_mont.c:26-278)"""
    L = ref_lib()
    name = Z.NAMES[curve]
    data = {}
    A = np.ascontiguousarray(Z.rand_fr(curve, 1, 9300)[0])
    B = np.ascontiguousarray(Z.rand_fr(curve, 1, 9301)[0])
    data["A"], data["B"] = A, B
    for cname, (a, b, c) in arr_cases(curve).items():
        a, b, c = (np.ascontiguousarray(x, dtype=np.uint64) for x in (a, b, c))
        n = a.shape[0]
        data[cname + "__a"], data[cname + "__b"], data[cname + "__c"] = a, b, c
        tgt0 = np.full((n, 4), 0xABABABABABABABAB, np.uint64)   # mul_by_powers leaves tgt[0] as it was
        for fn, pat in ARR_FUNCS:
            if cname == "wide_n64" and fn not in ("from_std", "is_valid", "is_zero", "is_equal", "to_std"):
                continue
            data["%s__%s" % (cname, fn)] = call_arr(L, curve, fn, pat, n, a, b, c, A, B, tgt0)
    # sparse matrix times vector (bn128_arr_mont.c:226-237)
    for N, M, K, seed in ((5, 7, 0, 1), (10, 20, 60, 2), (100, 64, 1000, 3)):
        rows = (Z.splitmix64(9400 + seed, K) % np.uint64(N)).astype(np.uint64)
        cols = (Z.splitmix64(9500 + seed, K) % np.uint64(M)).astype(np.uint64)
        co = Z.rand_fr(curve, K, 9600 + seed)
        src = Z.rand_fr(curve, M, 9700 + seed)
        tgt = np.zeros((N, 4), np.uint64)
        L["%s_arr_mont_sparse_matrix_mul" % name](ctypes.c_int(N), ctypes.c_int(K), Z.ptr(rows), Z.ptr(cols),
                                                   Z.ptr(co), Z.ptr(src), Z.ptr(tgt))
        key = "sparse_N%d_K%d" % (N, K)
        data[key + "__rows"], data[key + "__cols"], data[key + "__coeffs"] = rows, cols, co
        data[key + "__src"], data[key + "__tgt"] = src, tgt
    path = os.path.join(OUT, "arr_%s.npz" % name)
    np.savez_compressed(path, **data)
    return path


NTT_LARGE_SIZES = (20, 24)


def ntt_large_seed(curve, m):
    return 41000 + 100 * curve + m


def make_ntt_large():
    """Whole-vector parity at the sizes of the NTT configuration: the reference C's forward and
    inverse NTT (bn128_poly_mont.c:452-473, 601-622 and the BLS12-381 twins) of seeded inputs,
    stored as SHA-256 digests of the output bytes."""
    import hashlib
    import json
    import threading
    L = ref_lib()
    jobs, res = [], {}
    for curve in Z.CURVES:
        for m in NTT_LARGE_SIZES:
            x = Z.rand_fr(curve, 1 << m, ntt_large_seed(curve, m))
            g = np.ascontiguousarray(Z.fft_gen(curve, m))
            key = "%s_%d" % (Z.NAMES[curve], m)
            res[key] = {"curve": curve, "m": m, "seed": ntt_large_seed(curve, m),
                        "input_sha256": hashlib.sha256(x.tobytes()).hexdigest()}
            for inv in (False, True):
                jobs.append((key, curve, m, g, x, inv))

    def run(key, curve, m, g, x, inv):
        f = getattr(L, "%s_poly_mont_ntt_%s" % (Z.NAMES[curve], "inverse" if inv else "forward"))
        out = np.zeros_like(x)
        f(ctypes.c_int(m), Z.ptr(g), Z.ptr(x), Z.ptr(out))
        res[key]["inverse_sha256" if inv else "forward_sha256"] = hashlib.sha256(out.tobytes()).hexdigest()
        res[key]["inverse_first" if inv else "forward_first"] = [hex(int(v)) for v in out[0]]

    for lo in range(0, len(jobs), 4):   # four reference calls at a time (each holds ~1.4 GB)
        ths = [threading.Thread(target=run, args=j) for j in jobs[lo:lo + 4]]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
    with open(os.path.join(OUT, "ntt_large_digests.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if sys.argv[1:] == ["ntt_large"]:
        make_ntt_large()
        raise SystemExit(0)
    which = sys.argv[1:] or ["msm", "ntt", "ntt_shifted", "g1fft", "msm_binary", "arr"]
    for c in Z.CURVES:
        if "msm" in which:
            print(make_msm(c))
        if "ntt" in which:
            print(make_ntt(c))
        if "ntt_shifted" in which:
            print(make_ntt_shifted(c))
        if "g1fft" in which:
            print(make_g1fft(c))
        if "msm_binary" in which:
            print(make_msm_binary(c))
        if "arr" in which:
            print(make_arr(c))
