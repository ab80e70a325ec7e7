"""Test helpers: loaders for the product library, the oracle and (when built) the reference C,
seeded input generation, and canonical comparisons.

The oracle (oracle/liboracle.so, our C restatement) and the reference C (oracle/_ref/libzkref.so)
are checkers only; they are never on the product path.
"""
import ctypes
import importlib.util
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "zikkurat-algebra_b200")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libzkref.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")

BN254, BLS12_381 = 0, 1
CURVES = (BN254, BLS12_381)
NAMES = {BN254: "bn128", BLS12_381: "bls12_381"}
NLP = {BN254: 4, BLS12_381: 6}
P = {
    BN254: 0x30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47,
    BLS12_381: 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab,
}
R = {
    BN254: 0x30644e72e131a029b85045b68181585d2833e84879b9709143e1f593f0000001,
    BLS12_381: 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001,
}
B_COEF = {BN254: 3, BLS12_381: 4}
GEN_STD = {
    BN254: (1, 2),
    BLS12_381: (0x17f1d3a73197d7942695638c4fa9ac0fc3688c4f9774b905a14e3a3f171bac586c55e83ff97a1aeffb3af00adb22c6bb,
                0x08b3f481e3aaa0f1a09e30ed741d8ae4fcf5e095d5d00af600db18cb2c04b3edd03cc744a2888ae40caa232946c5e7e1),
}
FFT_DOMAIN = {
    BN254: (28, 19103219067921713944291392827692070036145651957329286315305642004821462161904),
    BLS12_381: (32, 10238227357739495823651030575849232062558860180284477541189508159991286009131),
}
U64 = (1 << 64) - 1


def load_package():
    """Import zikkurat-algebra_b200 (a hyphenated directory) as module `zikkurat_algebra_b200`."""
    if "zikkurat_algebra_b200" in sys.modules:
        return sys.modules["zikkurat_algebra_b200"]
    spec = importlib.util.spec_from_file_location("zikkurat_algebra_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["zikkurat_algebra_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(
                os.path.join(ROOT, "oracle", "zkoracle.c")):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        L = ctypes.CDLL(ORACLE_SO)
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.oracle_msm_proj.argtypes = [i, i, vp, i, i, vp, vp, i]
        L.oracle_msm_proj.restype = i
        L.oracle_proj_to_affine.argtypes = [i, vp, vp]
        L.oracle_proj_add.argtypes = [i, vp, vp, vp]
        L.oracle_proj_to_jac.argtypes = [i, vp, vp]
        L.oracle_jac_to_affine.argtypes = [i, vp, vp]
        L.oracle_gen_bases.argtypes = [i, i, vp, vp]
        L.oracle_ntt.argtypes = [i, i, vp, vp, vp, i]
        L.oracle_ntt.restype = i
        L.oracle_eval_at.argtypes = [i, i, vp, vp, vp]
        L.oracle_ntt_shifted.argtypes = [i, i, vp, vp, vp, vp, i]
        L.oracle_ntt_shifted.restype = i
        L.oracle_ntt_asymmetric.argtypes = [i, i, i, vp, vp, vp, vp]
        L.oracle_ntt_asymmetric.restype = i
        L.oracle_field_op.argtypes = [i, i, i, i, vp, vp, vp]
        L.oracle_fr_dot_std.argtypes = [i, i, vp, vp, vp]
        L.oracle_msm_window.argtypes = [i]
        L.oracle_msm_window.restype = i
        L.oracle_msm_binary.argtypes = [i, i, vp, vp, vp]
        L.oracle_multi_msm_binary.argtypes = [i, i, i, vp, vp, vp]
        L.oracle_multi_msm_binary.restype = i
        L.oracle_g1_fft.argtypes = [i, i, i, vp, vp, vp, i]
        L.oracle_g1_fft.restype = i
        L.oracle_fr_op.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp]
        L.oracle_fr_op.restype = i
        L.oracle_fr_dot.argtypes = [i, i, vp, vp, vp]
        L.oracle_fr_sparse.argtypes = [i, i, i, vp, vp, vp, vp, vp]
        _oracle = L
    return _oracle


def reference():
    """The reference C compiled here (None when oracle/_ref was not built)."""
    if not os.path.exists(REF_SO):
        return None
    return ctypes.CDLL(REF_SO)


def ptr(a):
    # data_as keeps a reference to the array, so a temporary argument stays alive through the call
    return a.ctypes.data_as(ctypes.c_void_p)


# ------------------------------------------------------------------------ integers / limbs

def to_limbs(x, n):
    return np.array([(x >> (64 * k)) & U64 for k in range(n)], dtype=np.uint64)


def from_limbs(a):
    return sum(int(v) << (64 * k) for k, v in enumerate(np.asarray(a, dtype=np.uint64).tolist()))


def ints_to_array(xs, n):
    out = np.zeros((len(xs), n), dtype=np.uint64)
    for i, x in enumerate(xs):
        for k in range(n):
            out[i, k] = (x >> (64 * k)) & U64
    return out


def splitmix64(seed, n):
    """n outputs of SplitMix64 started at `seed` (vectorised)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & U64) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _lt_limbs(a, b_limbs):
    """vectorised a < b for a (n,4) uint64 and a constant b"""
    lt = np.zeros(a.shape[0], dtype=bool)
    eq = np.ones(a.shape[0], dtype=bool)
    for k in range(a.shape[1] - 1, -1, -1):
        bk = np.uint64(b_limbs[k])
        lt |= eq & (a[:, k] < bk)
        eq &= a[:, k] == bk
    return lt


def rand_fr(curve, n, seed):
    """n values uniform in [0, r) as (n, 4) uint64, by rejection sampling from SplitMix64 draws.
    (A uniform value below r is also a uniform Montgomery-form element.)"""
    r = R[curve]
    bits = r.bit_length()
    rl = to_limbs(r, 4)
    out = np.zeros((0, 4), dtype=np.uint64)
    s = seed
    while out.shape[0] < n:
        m = max(16, int((n - out.shape[0]) * 1.3) + 16)
        raw = splitmix64(s, 4 * m).reshape(m, 4)
        s = (s * 6364136223846793005 + 1442695040888963407) & U64
        raw[:, 3] &= np.uint64((1 << (bits - 192)) - 1)
        out = np.concatenate([out, raw[_lt_limbs(raw, rl)]])
    return np.ascontiguousarray(out[:n])


def gen_bases_cpu(curve, ks):
    """affine Montgomery k_i * G on the CPU with the oracle (chunks on host threads; ctypes
    releases the GIL during the call)"""
    from concurrent.futures import ThreadPoolExecutor
    ks = np.ascontiguousarray(ks, dtype=np.uint64)
    n = ks.shape[0]
    out = np.zeros((n, 2 * NLP[curve]), dtype=np.uint64)
    L = oracle()
    chunk = 4096
    def work(lo):
        hi = min(n, lo + chunk)
        kk = np.ascontiguousarray(ks[lo:hi])
        oo = np.zeros((hi - lo, 2 * NLP[curve]), dtype=np.uint64)
        L.oracle_gen_bases(curve, hi - lo, ptr(kk), ptr(oo))
        out[lo:hi] = oo
    with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as ex:
        list(ex.map(work, range(0, n, chunk)))
    return out


def fr_dot_std(curve, a_std, b_std):
    """sum a_i b_i mod r (standard-form inputs) with the oracle"""
    a = np.ascontiguousarray(a_std, dtype=np.uint64)
    b = np.ascontiguousarray(b_std, dtype=np.uint64)
    out = np.zeros(4, dtype=np.uint64)
    oracle().oracle_fr_dot_std(curve, a.shape[0], ptr(a), ptr(b), ptr(out))
    return from_limbs(out)


def fr_to_mont_array(curve, xs_std):
    xs_std = np.ascontiguousarray(xs_std, dtype=np.uint64)
    out = np.zeros_like(xs_std)
    oracle().oracle_field_op(curve, 1, 1, xs_std.shape[0], ptr(xs_std), None, ptr(out))
    return out


def fr_from_mont_array(curve, xs):
    xs = np.ascontiguousarray(xs, dtype=np.uint64)
    out = np.zeros_like(xs)
    oracle().oracle_field_op(curve, 1, 0, xs.shape[0], ptr(xs), None, ptr(out))
    return out


def ntt_large_cases():
    """The whole-vector NTT cases pinned by digests of the reference C's outputs
    (tests/golden/ntt_large_digests.json, made by tests/golden/make_golden.py ntt_large)."""
    import json
    with open(os.path.join(GOLDEN, "ntt_large_digests.json")) as f:
        return json.load(f)


def sha256(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def fft_gen(curve, m):
    mx, g = FFT_DOMAIN[curve]
    return to_limbs(pow(g, 1 << (mx - m), R[curve]) * (1 << 256) % R[curve], 4)


# --------------------------------------------------------------------------- oracle calls

def oracle_msm_affine(curve, scalars, nlimbs, mont, bases, window=0):
    scalars = np.ascontiguousarray(scalars, dtype=np.uint64)
    bases = np.ascontiguousarray(bases, dtype=np.uint64)
    n = bases.size // (2 * NLP[curve])
    proj = np.zeros(3 * NLP[curve], dtype=np.uint64)
    rc = oracle().oracle_msm_proj(curve, n, ptr(scalars), nlimbs, int(mont), ptr(bases), ptr(proj), window)
    assert rc == 0
    aff = np.zeros(2 * NLP[curve], dtype=np.uint64)
    oracle().oracle_proj_to_affine(curve, ptr(proj), ptr(aff))
    return aff


def oracle_ntt(curve, m, gen, src, inverse):
    src = np.ascontiguousarray(src, dtype=np.uint64)
    gen = np.ascontiguousarray(gen, dtype=np.uint64)
    out = np.zeros_like(src)
    assert oracle().oracle_ntt(curve, m, ptr(gen), ptr(src), ptr(out), int(inverse)) == 0
    return out


def oracle_ntt_shifted(curve, m, eta, gen, src, inverse):
    src = np.ascontiguousarray(src, dtype=np.uint64)
    out = np.zeros_like(src)
    assert oracle().oracle_ntt_shifted(curve, m, ptr(np.ascontiguousarray(eta, dtype=np.uint64)),
                                       ptr(np.ascontiguousarray(gen, dtype=np.uint64)), ptr(src), ptr(out),
                                       int(inverse)) == 0
    return out


def oracle_ntt_asymmetric(curve, ms, mt, gs, gt, src):
    src = np.ascontiguousarray(src, dtype=np.uint64)
    out = np.zeros((1 << mt, 4), dtype=np.uint64)
    assert oracle().oracle_ntt_asymmetric(curve, ms, mt, ptr(np.ascontiguousarray(gs, dtype=np.uint64)),
                                          ptr(np.ascontiguousarray(gt, dtype=np.uint64)), ptr(src), ptr(out)) == 0
    return out


def oracle_msm_binary(curve, coeffs, bases):
    """rows of byte coefficients (nrows, npoints) -> (nrows, 3*NLP) projective sums"""
    coeffs = np.ascontiguousarray(coeffs, dtype=np.uint8)
    bases = np.ascontiguousarray(bases, dtype=np.uint64)
    nrows, npoints = coeffs.shape
    out = np.zeros((nrows, 3 * NLP[curve]), dtype=np.uint64)
    if nrows == 1:
        oracle().oracle_msm_binary(curve, npoints, ptr(coeffs), ptr(bases), ptr(out))
    else:
        assert oracle().oracle_multi_msm_binary(curve, nrows, npoints, ptr(coeffs), ptr(bases), ptr(out)) == 0
    return out


def oracle_g1_fft(curve, jac, m, gen, src, inverse):
    src = np.ascontiguousarray(src, dtype=np.uint64)
    out = np.zeros_like(src)
    assert oracle().oracle_g1_fft(curve, int(jac), m, ptr(np.ascontiguousarray(gen, dtype=np.uint64)), ptr(src),
                                  ptr(out), int(inverse)) == 0
    return out


def scaled_points(curve, aff, lam, jac):
    """affine Montgomery points -> projective (x l, y l, l) or Jacobian (x l^2, y l^3, l) with the
    scale l (standard ints) in Montgomery form; (0,0) -> the reference's infinity"""
    nl = NLP[curve]
    p = P[curve]
    Rm = (1 << (64 * nl)) % p
    out = np.zeros((aff.shape[0], 3 * nl), np.uint64)
    for i in range(aff.shape[0]):
        x, y = from_limbs(aff[i, :nl]), from_limbs(aff[i, nl:])
        if x == 0 and y == 0:
            # projective infinity (0,1,0), Jacobian (1,1,0) (bn128_G1_proj.c:183, bn128_G1_jac.c:183)
            if jac:
                out[i, :nl] = to_limbs(Rm, nl)
            out[i, nl:2 * nl] = to_limbs(Rm, nl)
            continue
        l = lam[i] % p or 1
        X, Y = (x * l * l % p, y * l * l * l % p) if jac else (x * l % p, y * l % p)
        out[i, :nl] = to_limbs(X, nl)
        out[i, nl:2 * nl] = to_limbs(Y, nl)
        out[i, 2 * nl:] = to_limbs(l * Rm % p, nl)
    return out


def oracle_fr_op(curve, op, a=None, b=None, c=None, ka=None, kb=None, n=None, out=None):
    """the *_arr_mont_* operation `op` (ZKG_FR_* code) on (n, 4) Montgomery arrays"""
    arrs = [None if x is None else np.ascontiguousarray(x, dtype=np.uint64) for x in (a, b, c, ka, kb)]
    if n is None:
        n = arrs[0].shape[0]
    out = np.zeros((n, 4), np.uint64) if out is None else np.array(out, dtype=np.uint64, copy=True)
    ps = [None if x is None else ptr(x) for x in arrs]
    assert oracle().oracle_fr_op(curve, op, n, *ps, ptr(out)) == 0
    return out


def row_pointers(coeffs):
    """ctypes array of row pointers (const uint8_t **) into a C-contiguous (nrows, npoints) uint8 array"""
    nrows = coeffs.shape[0]
    arr = (ctypes.c_void_p * max(nrows, 1))()
    for r in range(nrows):
        arr[r] = coeffs.ctypes.data + r * coeffs.strides[0]
    return arr


def proj_to_affine(curve, proj):
    proj = np.ascontiguousarray(proj, dtype=np.uint64)
    aff = np.zeros(2 * NLP[curve], dtype=np.uint64)
    oracle().oracle_proj_to_affine(curve, ptr(proj), ptr(aff))
    return aff


def jac_to_affine(curve, jac):
    jac = np.ascontiguousarray(jac, dtype=np.uint64)
    aff = np.zeros(2 * NLP[curve], dtype=np.uint64)
    oracle().oracle_jac_to_affine(curve, ptr(jac), ptr(aff))
    return aff


# ------------------------------------------------- independent pure-Python group law (tiny)

def py_affine_std(curve, aff_mont):
    """Montgomery affine limbs -> (x, y) standard ints, or None for infinity (0xff.. or (0,0))."""
    nl = NLP[curve]
    x, y = from_limbs(aff_mont[:nl]), from_limbs(aff_mont[nl:])
    if x == (1 << (64 * nl)) - 1 or (x == 0 and y == 0):
        return None
    rinv = pow(1 << (64 * nl), -1, P[curve])
    return (x * rinv % P[curve], y * rinv % P[curve])


def py_add(curve, a, b):
    p = P[curve]
    if a is None:
        return b
    if b is None:
        return a
    if a[0] == b[0]:
        if (a[1] + b[1]) % p == 0:
            return None
        lam = 3 * a[0] * a[0] * pow(2 * a[1], -1, p) % p
    else:
        lam = (b[1] - a[1]) * pow(b[0] - a[0], -1, p) % p
    x3 = (lam * lam - a[0] - b[0]) % p
    return (x3, (lam * (a[0] - x3) - a[1]) % p)


def py_mul(curve, k, a):
    acc = None
    while k:
        if k & 1:
            acc = py_add(curve, acc, a)
        a = py_add(curve, a, a)
        k >>= 1
    return acc


def py_msm(curve, ks, pts):
    acc = None
    for k, pt in zip(ks, pts):
        acc = py_add(curve, acc, py_mul(curve, k, pt))
    return acc


def fr_dot_mod(a, b, r):
    """sum_i a_i b_i mod r for (n, 4) uint64 arrays, exact, in numpy (no oracle): 16-bit digit
    products (< 2^32) summed per column in uint64 over row chunks (< 2^58 per column)."""
    a16 = np.ascontiguousarray(a, dtype=np.uint64).view(np.uint16).reshape(-1, 16)
    b16 = np.ascontiguousarray(b, dtype=np.uint64).view(np.uint16).reshape(-1, 16)
    cols = [0] * 31
    step = 1 << 18
    for lo in range(0, a16.shape[0], step):
        A = a16[lo:lo + step].astype(np.uint64)
        B = b16[lo:lo + step].astype(np.uint64)
        for i in range(16):
            s = (A[:, i:i + 1] * B).sum(axis=0, dtype=np.uint64)
            for j in range(16):
                cols[i + j] += int(s[j])
    return sum(c << (16 * k) for k, c in enumerate(cols)) % r


def msm_identity_affine(curve, ks_std, scalars_mont):
    """Affine Montgomery encoding (all 0xff for the identity) of sum_i s_i (k_i G) computed as
    (sum_i s_i k_i mod r) G, for bases P_i = k_i G and Montgomery scalars s_i R. Pure Python and
    numpy: an independent check of a full-size MSM that needs no oracle MSM of that size."""
    r, p = R[curve], P[curve]
    nl = NLP[curve]
    t = fr_dot_mod(scalars_mont, ks_std, r) * pow(1 << 256, -1, r) % r
    pt = py_mul(curve, t, GEN_STD[curve])
    if pt is None:
        return np.full(2 * nl, U64, np.uint64)
    Rm = 1 << (64 * nl)
    return np.concatenate([to_limbs(pt[0] * Rm % p, nl), to_limbs(pt[1] * Rm % p, nl)])


# *_arr_mont_* function -> (ZKG_FR_* op, which inputs: a b c of the call, in-place flag)
FR_OPS = {
    "from_std": (0, "a"), "to_std": (1, "a"), "neg": (2, "a"), "sqr": (5, "a"), "inv": (7, "a"),
    "add": (3, "ab"), "sub": (4, "ab"), "mul": (6, "ab"), "div": (8, "ab"),
    "mul_add": (9, "abc"), "mul_sub": (10, "abc"),
    "neg_inplace": (2, "a"), "sqr_inplace": (5, "a"), "inv_inplace": (7, "a"),
    "add_inplace": (3, "ab"), "sub_inplace": (4, "ab"), "mul_inplace": (6, "ab"), "div_inplace": (8, "ab"),
    "sub_inplace_reverse": (4, "ba"),
    "powers": (14, ""), "mul_by_powers": (15, "a"),
    "scale": (11, "a"), "scale_inplace": (11, "a"),
    "Ax_plus_y": (12, "ab"), "Ax_plus_y_inplace": (12, "ab"),
    "Ax_plus_By": (13, "ab"), "Ax_plus_By_inplace": (13, "ab"),
}
