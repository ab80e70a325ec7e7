"""GPU parity tests for the MSM (BN254 and BLS12-381 G1) through the drop-in C ABI.

Affine outputs are compared byte for byte; projective / Jacobian outputs (returned normalised)
are compared after the reference's own normalisation. Sources of truth: golden vectors from the
reference C, the oracle restatement on the same seeded inputs, an independent scalar-sum identity
at full size, and degenerate cases mirroring the reference's special cases
(lib/cbits/curves/g1/proj/bn128_G1_proj.c:334-358).
"""
import ctypes
import os

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu

ENTRY = [("proj", "proj"), ("proj", "affine"), ("jac", "jac"), ("jac", "affine")]


def call(zk, curve, fam, coeff, kind, scalars, nlimbs, bases):
    L = zk.lib()
    nl = Z.NLP[curve]
    s = np.ascontiguousarray(np.asarray(scalars, dtype=np.uint64).reshape(-1))
    b = np.ascontiguousarray(np.asarray(bases, dtype=np.uint64).reshape(-1))
    n = b.size // (2 * nl)
    out = np.zeros((2 if kind == "affine" else 3) * nl, np.uint64)
    fn = getattr(L, "%s_G1_%s_MSM_%s_coeff_%s_out" % (Z.NAMES[curve], fam, coeff, kind))
    fn(ctypes.c_int(n), Z.ptr(s), Z.ptr(b), Z.ptr(out), ctypes.c_int(nlimbs))
    assert L.zkg_last_status() == 0, L.zkg_last_error()
    return out


def to_affine(curve, fam, kind, out):
    if kind == "affine":
        return out
    return Z.proj_to_affine(curve, out) if fam == "proj" else Z.jac_to_affine(curve, out)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_golden_reference_vectors(zk, curve):
    d = np.load(os.path.join(Z.GOLDEN, "msm_%s.npz" % Z.NAMES[curve]))
    names = sorted({k.split("__")[0] for k in d.files})
    nl = Z.NLP[curve]
    for name in names:
        scal, bases, nlimbs = d[name + "__scalars"], d[name + "__bases"], int(d[name + "__nlimbs"][0])
        for coeff in ("std", "mont"):
            if coeff == "mont" and nlimbs != 4:
                continue
            want = d[name + "__proj_%s_affine" % coeff]
            for fam, kind in ENTRY:
                got = call(zk, curve, fam, coeff, kind, scal, nlimbs, bases)
                assert np.array_equal(to_affine(curve, fam, kind, got), want), (name, coeff, fam, kind)
                if kind != "affine":
                    one = Z.to_limbs((1 << (64 * nl)) % Z.P[curve], nl)
                    zero = np.zeros(nl, np.uint64)
                    if np.all(want == np.uint64(Z.U64)):
                        # infinity in the reference's normalised encoding: proj (0,1,0)
                        # (bn128_G1_proj.c:96-100), jac (1,1,0) (bn128_G1_jac.c:182-187); the
                        # reference itself may return any (0,Y,0), which its is_equal normalises
                        ref = d[name + "__%s_%s_%s" % (fam, coeff, kind)]
                        assert np.all(ref[2 * nl:] == 0), name
                        exp = np.concatenate([zero if fam == "proj" else one, one, zero])
                        assert np.array_equal(got, exp), (name, fam)
                    else:
                        assert np.array_equal(got[2 * nl:], one)


@pytest.mark.parametrize("curve", Z.CURVES)
@pytest.mark.parametrize("n", [1, 2, 3, 31, 64, 1000, 4097, 1 << 14])
def test_msm_random_vs_oracle(zk, curve, n):
    ks = Z.rand_fr(curve, n, 20000 + n)
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 21000 + n))
    for mont in (True, False):
        want = Z.oracle_msm_affine(curve, ks, 4, mont, bases)
        got = call(zk, curve, "proj", "mont" if mont else "std", "affine", ks, 4, bases)
        assert np.array_equal(got, want), mont


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_every_window_width(zk, curve):
    """window widths 2..20 (bucket counts 2 .. 2^19) all give the same point"""
    n = 3000
    ks = Z.rand_fr(curve, n, 22000)
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 22001))
    want = Z.oracle_msm_affine(curve, ks, 4, True, bases)
    L = zk.lib()
    prev = L.zkg_set_msm_window(0)
    try:
        for c in range(2, 21):
            L.zkg_set_msm_window(c)
            assert np.array_equal(call(zk, curve, "proj", "mont", "affine", ks, 4, bases), want), c
    finally:
        L.zkg_set_msm_window(prev)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_pipelined_parts_agree(zk, curve):
    """host-buffer MSMs split into 1..4 point-range parts (copy/compute overlap) give the same point,
    including ragged last parts and parts smaller than a window's bucket count"""
    L = zk.lib()
    prev = L.zkg_set_msm_parts(0)
    try:
        for n in (5, 1000, 4099):
            ks = Z.rand_fr(curve, n, 28000 + n)
            bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 28100 + n))
            want = Z.oracle_msm_affine(curve, ks, 4, True, bases)
            for parts in (1, 2, 3, 4):
                L.zkg_set_msm_parts(parts)
                assert np.array_equal(call(zk, curve, "proj", "mont", "affine", ks, 4, bases), want), (n, parts)
    finally:
        L.zkg_set_msm_parts(prev)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_degenerate_cases(zk, curve):
    _degenerate_checks(zk, curve)


@pytest.mark.parametrize("curve", Z.CURVES)
@pytest.mark.parametrize("levels,slots", [(1, 4), (3, 5), (8, 32)])
def test_msm_degenerate_cases_affine_tree(zk, curve, levels, slots):
    """the same special cases with the affine tree levels forced on small MSMs: doublings,
    cancellations P + (-P) and (0, 0) bases inside the tree's pairs, thread batches that start and
    end inside segments, and more levels than a segment needs"""
    L = zk.lib()
    prev = L.zkg_set_msm_tree(levels, slots)
    try:
        _degenerate_checks(zk, curve)
    finally:
        L.zkg_set_msm_tree(prev, -1)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_affine_tree_levels_match_oracle(zk, curve):
    """random MSMs with 0..8 affine tree levels and several thread batch sizes equal the oracle"""
    L = zk.lib()
    prev = L.zkg_set_msm_tree(-1, 0)
    try:
        for n in (1000, 4099, 1 << 14):
            ks = Z.rand_fr(curve, n, 29000 + n)
            bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 29100 + n))
            want = Z.oracle_msm_affine(curve, ks, 4, True, bases)
            for levels, slots in ((0, 32), (1, 32), (2, 7), (4, 4), (6, 64), (8, 33)):
                L.zkg_set_msm_tree(levels, slots)
                assert np.array_equal(call(zk, curve, "proj", "mont", "affine", ks, 4, bases), want), (n, levels, slots)
    finally:
        L.zkg_set_msm_tree(prev, -1)


def _degenerate_checks(zk, curve):
    nl = Z.NLP[curve]
    n = 300
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 23000))
    ks = Z.rand_fr(curve, n, 23001)
    inf_aff = np.full(2 * nl, Z.U64, np.uint64)
    # all-zero scalars -> infinity (0xff affine, (0,1,0) proj, (1,1,0) jac)
    z = np.zeros((n, 4), np.uint64)
    assert np.array_equal(call(zk, curve, "proj", "std", "affine", z, 4, bases), inf_aff)
    one = Z.to_limbs((1 << (64 * nl)) % Z.P[curve], nl)
    pz = call(zk, curve, "proj", "mont", "proj", z, 4, bases)
    assert np.array_equal(pz, np.concatenate([np.zeros(nl, np.uint64), one, np.zeros(nl, np.uint64)]))
    jz = call(zk, curve, "jac", "std", "jac", z, 4, bases)
    assert np.array_equal(jz, np.concatenate([one, one, np.zeros(nl, np.uint64)]))
    # n = 0
    assert np.array_equal(call(zk, curve, "proj", "mont", "affine", z[:0], 4, bases[:0]), inf_aff)
    # every scalar equal: one bucket per window holds every point (load-balancing levels)
    eq = np.repeat(ks[:1], 5000, axis=0)
    b5 = Z.gen_bases_cpu(curve, Z.rand_fr(curve, 5000, 23002))
    assert np.array_equal(call(zk, curve, "proj", "mont", "affine", eq, 4, b5),
                          Z.oracle_msm_affine(curve, eq, 4, True, b5))
    # one base repeated with equal scalars: bucket additions hit the doubling case
    rep = np.repeat(bases[:1], 257, axis=0)
    eq2 = np.repeat(ks[:1], 257, axis=0)
    assert np.array_equal(call(zk, curve, "proj", "std", "affine", eq2, 4, rep),
                          Z.oracle_msm_affine(curve, eq2, 4, False, rep))
    # P and -P with equal scalars cancel inside buckets
    negb = bases.copy()
    for i in range(n):
        negb[i, nl:] = Z.to_limbs((Z.P[curve] - Z.from_limbs(bases[i, nl:])) % Z.P[curve], nl)
    pb = np.concatenate([bases, negb])
    pk = np.concatenate([ks, ks])
    assert np.array_equal(call(zk, curve, "proj", "mont", "affine", pk, 4, pb), inf_aff)
    pk2 = np.concatenate([ks, ks[::-1]])
    assert np.array_equal(call(zk, curve, "proj", "mont", "affine", pk2, 4, pb),
                          Z.oracle_msm_affine(curve, pk2, 4, True, pb))
    # affine (0,0) bases are the identity
    ib = bases.copy()
    ib[::2] = 0
    assert np.array_equal(call(zk, curve, "proj", "mont", "affine", ks, 4, ib),
                          Z.oracle_msm_affine(curve, ks, 4, True, ib))
    # standard scalars >= r, full 64*nlimbs bits, other limb counts
    for nlimbs in (1, 2, 3, 4, 5, 8):
        raw = Z.splitmix64(23100 + nlimbs, n * nlimbs).reshape(n, nlimbs)
        assert np.array_equal(call(zk, curve, "proj", "std", "affine", raw, nlimbs, bases),
                              Z.oracle_msm_affine(curve, raw, nlimbs, False, bases)), nlimbs
    allones = np.full((n, 4), Z.U64, np.uint64)
    assert np.array_equal(call(zk, curve, "jac", "std", "affine", allones, 4, bases),
                          Z.oracle_msm_affine(curve, allones, 4, False, bases))


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_skewed_digit_distribution(zk, curve):
    # a few scalars repeated many times (buckets whose segments span many accumulation chunks,
    # folded by the level kernels) mixed with random ones (segments inside one chunk or cut
    # across two neighbouring chunks, merged pairwise); window widths change the chunk layout
    n = 30000
    ks = Z.rand_fr(curve, n, 23500)
    few = Z.rand_fr(curve, 3, 23501)
    idx = np.arange(n)
    ks[idx % 3 == 0] = few[0]
    ks[idx % 7 == 1] = few[1]
    ks[: n // 10] = few[2]
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 23502))
    want = Z.oracle_msm_affine(curve, ks, 4, True, bases)
    L = zk.lib()
    try:
        for c in (0, 9, 13):
            L.zkg_set_msm_window(c)
            assert np.array_equal(call(zk, curve, "proj", "mont", "affine", ks, 4, bases), want), c
    finally:
        L.zkg_set_msm_window(0)


@pytest.mark.parametrize("curve", Z.CURVES)
def test_msm_deterministic_and_consistent_outputs(zk, curve):
    n = 20000
    ks = Z.rand_fr(curve, n, 24000)
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 24001))
    a = call(zk, curve, "proj", "mont", "affine", ks, 4, bases)
    for fam, kind in ENTRY:
        got = call(zk, curve, fam, "mont", kind, ks, 4, bases)
        assert np.array_equal(to_affine(curve, fam, kind, got), a)
        assert np.array_equal(call(zk, curve, fam, "mont", kind, ks, 4, bases), got)


def test_msm_bn254_2pow18_vs_oracle(zk):
    n = 1 << 18
    ks = Z.rand_fr(Z.BN254, n, 25000)
    bases = Z.gen_bases_cpu(Z.BN254, Z.rand_fr(Z.BN254, n, 25001))
    assert np.array_equal(call(zk, Z.BN254, "proj", "mont", "affine", ks, 4, bases),
                          Z.oracle_msm_affine(Z.BN254, ks, 4, True, bases))


def _full_size_identity(zk, curve, n, seed):
    """bases P_i = k_i G  =>  sum s_i P_i = (sum s_i k_i mod r) G: checks the 2^22 result
    without an oracle MSM of that size."""
    import torch
    r = Z.R[curve]
    ks = Z.rand_fr(curve, n, seed)
    ss = Z.rand_fr(curve, n, seed + 1)            # Montgomery scalars
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((n, 2 * Z.NLP[curve]), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(curve, n, d_k, d_b)
    torch.cuda.synchronize()
    sample = np.random.default_rng(seed).integers(0, n, 64)
    bh = d_b.cpu().numpy().view(np.uint64)
    assert np.array_equal(bh[sample], Z.gen_bases_cpu(curve, ks[sample]))
    d_s = torch.from_numpy(ss.view(np.int64)).cuda()
    got = zk.msm_device(curve, n, d_s, d_b, mont=True, kind=zk.OUT_AFFINE)
    sstd = Z.fr_from_mont_array(curve, ss)
    t = Z.fr_dot_std(curve, sstd, ks)   # sum s_i k_i mod r
    # spot-check the oracle's dot product with exact Python integers on a prefix
    assert Z.fr_dot_std(curve, sstd[:100], ks[:100]) == sum(
        Z.from_limbs(a) * Z.from_limbs(b) for a, b in zip(sstd[:100], ks[:100])) % r
    want = Z.gen_bases_cpu(curve, Z.ints_to_array([t], 4))[0]
    if t == 0:
        want = np.full(2 * Z.NLP[curve], Z.U64, np.uint64)
    assert np.array_equal(got, want)
    # the host-buffer drop-in path agrees with the device path
    assert np.array_equal(call(zk, curve, "proj", "mont", "affine", ss, 4, bh), got)


def test_msm_bn254_2pow22_scalar_identity(zk):
    _full_size_identity(zk, Z.BN254, 1 << 22, 26000)


def test_msm_bls12_381_2pow20_scalar_identity(zk):
    _full_size_identity(zk, Z.BLS12_381, 1 << 20, 27000)


def test_msm_bls12_381_2pow22_scalar_identity(zk):
    """the BLS12-381 configuration's size (bls12_381_G1_proj.c:598-605 at n = 2^22)"""
    _full_size_identity(zk, Z.BLS12_381, 1 << 22, 27100)


def test_msm_bls12_381_2pow22_fixed_window_16(zk):
    """the fixed c = 16 plain kernel of the BLS12-381 configuration, same identity"""
    L = zk.lib()
    prev = L.zkg_set_msm_window(16)
    try:
        _full_size_identity(zk, Z.BLS12_381, 1 << 22, 27200)
    finally:
        L.zkg_set_msm_window(prev)


def test_msm_rejects_bad_arguments(zk):
    L = zk.lib()
    out = np.zeros(12, np.uint64)
    s = np.zeros(8, np.uint64)
    b = np.zeros(16, np.uint64)
    assert L.zkg_msm(0, -1, Z.ptr(s), 4, 0, Z.ptr(b), 2, Z.ptr(out)) != 0
    assert L.zkg_msm(0, 1, Z.ptr(s), 3, 1, Z.ptr(b), 2, Z.ptr(out)) != 0   # mont needs 4 limbs
    assert L.zkg_msm(0, 1, Z.ptr(s), 0, 0, Z.ptr(b), 2, Z.ptr(out)) != 0
    assert L.zkg_msm(5, 1, Z.ptr(s), 4, 0, Z.ptr(b), 2, Z.ptr(out)) != 0
