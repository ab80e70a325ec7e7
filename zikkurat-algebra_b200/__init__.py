"""zikkurat-algebra_b200: B200 host-side mirror of zikkurat-algebra's MSM and NTT interface.

The compute path is libzkb200.so (hand-written sm_100a CUDA kernels behind a C ABI,
include/zkb200.h). This module binds it with ctypes and mirrors the reference's Haskell
operator interface for the two hot paths, with numpy arrays standing in for FlatArray:

  reference (Haskell)                                   here
  ZK.Algebra.Class.Curve.msm        (Class/Curve.hs:92)  msm(curve, scalars_mont, bases)      -> projective
  msmStd                       (BN128/G1/Proj.hs:262)    msm_std(curve, scalars_std, bases)    -> projective
  Affine.msm                  (BN128/G1/Affine.hs:145)   msm_affine(curve, scalars_mont, bases)
  ZK.Algebra.Class.Poly.ntt / intt  (Class/Poly.hs:55-59) forward_ntt / inverse_ntt(subgroup, values)
  getFFTSubgroup                    (Class/FFT.hs:60-68) fft_subgroup(curve, m)

Arrays use the reference's memory layout: little-endian uint64 limbs, Montgomery form,
points as x|y (affine) or X|Y|Z. Errors raise ZkgError carrying zkg_last_error(); there is no
CPU fallback: if the shared library is missing the import of the binding fails.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzkb200.so")

BN254 = 0
BLS12_381 = 1
OUT_PROJ, OUT_JAC, OUT_AFFINE = 0, 1, 2

# limbs per Fp element, per curve
NLIMBS_P = {BN254: 4, BLS12_381: 6}
# field moduli (lib/cbits/curves/fields/mont/*_mont.c:20)
P_MOD = {
    BN254: 0x30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47,
    BLS12_381: 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab,
}
R_MOD = {
    BN254: 0x30644e72e131a029b85045b68181585d2833e84879b9709143e1f593f0000001,
    BLS12_381: 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001,
}
# FFT domains (codegen/src/Zikkurat/Generate.hs:143-144): (log2 size, generator in standard form)
FFT_DOMAIN = {
    BN254: (28, 19103219067921713944291392827692070036145651957329286315305642004821462161904),
    BLS12_381: (32, 10238227357739495823651030575849232062558860180284477541189508159991286009131),
}


ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_TIMEOUT = 1, 2, 3, 4, 5


class ZkgError(RuntimeError):
    """a failed library call; .status holds the zkg_status code"""

    def __init__(self, msg, status=None):
        super().__init__(msg)
        self.status = status


_lib = None


def lib():
    """The loaded libzkb200.so (ctypes.CDLL), with argument types declared."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libzkb200.so not built: run python zikkurat-algebra_b200/build.py (%s)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    u64p = ctypes.c_void_p
    i = ctypes.c_int
    L.zkg_msm.argtypes = [i, i, u64p, i, i, u64p, i, u64p]
    L.zkg_msm_device.argtypes = [i, i, u64p, i, i, u64p, i, u64p]
    L.zkg_ntt.argtypes = [i, i, u64p, u64p, u64p, i]
    L.zkg_ntt_device.argtypes = [i, i, u64p, u64p, u64p, i]
    L.zkg_g1_gen_mul_device.argtypes = [i, i, u64p, u64p]
    for f in ("zkg_msm", "zkg_msm_device", "zkg_ntt", "zkg_ntt_device", "zkg_g1_gen_mul_device",
              "zkg_last_status", "zkg_release_cache"):
        getattr(L, f).restype = ctypes.c_int
    L.zkg_last_error.restype = ctypes.c_char_p
    L.zkg_last_kernel_ms.restype = ctypes.c_float
    L.zkg_kernel_launches.restype = ctypes.c_uint64
    L.zkg_set_msm_window.argtypes = [i]
    L.zkg_set_msm_window.restype = i
    L.zkg_msm_window_for.argtypes = [i, i]
    L.zkg_msm_window_for.restype = i
    L.zkg_set_msm_parts.argtypes = [i]
    L.zkg_set_msm_parts.restype = i
    L.zkg_set_msm_tree.argtypes = [i, i]
    L.zkg_set_msm_tree.restype = i
    L.zkg_set_ntt_kmax.argtypes = [i]
    L.zkg_set_ntt_kmax.restype = i
    vp = ctypes.c_void_p
    L.zkg_batch_create.argtypes = [i, vp, i, ctypes.POINTER(vp)]
    L.zkg_batch_add_msm.argtypes = [vp, i, vp, vp]
    L.zkg_batch_add_ntt.argtypes = [vp, i, vp, vp, vp, i]
    L.zkg_batch_run.argtypes = [vp]
    L.zkg_batch_last_ms.argtypes = [vp]
    L.zkg_batch_last_ms.restype = ctypes.c_float
    L.zkg_batch_destroy.argtypes = [vp]
    L.zkg_batch_set_wait_limit.argtypes = [vp, ctypes.c_uint32, i]
    L.zkg_batch_set_wait_limit.restype = i
    L.zkg_batch_persistent.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_uint32)]
    L.zkg_batch_persistent.restype = i
    L.zkg_batch_set_mode.argtypes = [vp, i]
    L.zkg_batch_set_mode.restype = i
    L.zkg_server_create.argtypes = [i, vp, i, i, i, ctypes.c_size_t, i, ctypes.POINTER(vp)]
    L.zkg_server_submit.argtypes = [vp, i, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
    L.zkg_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    L.zkg_server_wait_for.argtypes = [vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    L.zkg_server_wait_for.restype = i
    L.zkg_server_inject_failure.argtypes = [vp, ctypes.c_long]
    L.zkg_server_inject_failure.restype = i
    L.zkg_server_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(i), ctypes.POINTER(ctypes.c_size_t)]
    L.zkg_server_destroy.argtypes = [vp]
    L.zkg_autotune_msm.argtypes = [i, vp, i, i, i, vp]
    L.zkg_autotune_ntt.argtypes = [i, i, i, vp]
    L.zkg_msm_tuned_window.argtypes = [i, i]
    L.zkg_msm_tuned_window.restype = i
    L.zkg_g1_fft.argtypes = [i, i, i, u64p, u64p, u64p, i]
    L.zkg_g1_fft_device.argtypes = [i, i, i, u64p, u64p, u64p, i]
    L.zkg_msm_binary.argtypes = [i, i, i, i, u64p, u64p, u64p]
    L.zkg_msm_binary_device.argtypes = [i, i, i, i, u64p, ctypes.c_size_t, u64p, u64p]
    L.zkg_fr_map.argtypes = [i, i, i, u64p, u64p, u64p, u64p, u64p, u64p]
    L.zkg_fr_map_device.argtypes = [i, i, i, u64p, u64p, u64p, u64p, u64p, u64p]
    L.zkg_fr_dot.argtypes = [i, i, u64p, u64p, u64p]
    L.zkg_fr_dot_device.argtypes = [i, i, u64p, u64p, u64p]
    L.zkg_fr_predicate.argtypes = [i, i, i, u64p, u64p, ctypes.POINTER(i)]
    L.zkg_fr_predicate_device.argtypes = [i, i, i, u64p, u64p, ctypes.POINTER(i)]
    L.zkg_fr_sparse_matrix_mul.argtypes = [i, i, i, u64p, u64p, u64p, u64p, u64p]
    L.zkg_fr_sparse_matrix_mul_device.argtypes = [i, i, i, u64p, u64p, u64p, u64p, i, u64p]
    L.zkg_bases_upload.argtypes = [i, vp, i, i, ctypes.POINTER(vp)]
    L.zkg_bases_destroy.argtypes = [vp]
    L.zkg_bases_count.argtypes = [vp]
    L.zkg_bases_count.restype = i
    L.zkg_msm_resident.argtypes = [vp, i, vp, i, i, i, vp]
    L.zkg_msm_resident_host.argtypes = [vp, i, vp, i, i, i, vp]
    L.zkg_batch_create_resident.argtypes = [vp, ctypes.POINTER(vp)]
    L.zkg_server_create_resident.argtypes = [vp, i, i, ctypes.c_size_t, i, ctypes.POINTER(vp)]
    for f in ("zkg_bases_upload", "zkg_bases_destroy", "zkg_msm_resident", "zkg_msm_resident_host",
              "zkg_batch_create_resident", "zkg_server_create_resident"):
        getattr(L, f).restype = ctypes.c_int
    for f in ("zkg_batch_create", "zkg_batch_add_msm", "zkg_batch_add_ntt", "zkg_batch_run", "zkg_batch_destroy",
              "zkg_server_create", "zkg_server_submit", "zkg_server_wait", "zkg_server_stats", "zkg_server_destroy",
              "zkg_autotune_msm", "zkg_autotune_ntt"):
        getattr(L, f).restype = ctypes.c_int
    _lib = L
    return L


def _check(status):
    if status != 0:
        raise ZkgError("zkb200 status %d: %s" % (status, lib().zkg_last_error().decode(errors="replace")), status)


def _ptr(a):
    # data_as keeps a reference to the array: a temporary argument stays alive through the call
    return a.ctypes.data_as(ctypes.c_void_p) if isinstance(a, np.ndarray) else ctypes.c_void_p(int(a))


def _c_u64(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a


# ------------------------------------------------------------------ integer <-> limb helpers

def to_limbs(x, n):
    return np.array([(x >> (64 * k)) & 0xFFFFFFFFFFFFFFFF for k in range(n)], dtype=np.uint64)


def from_limbs(a):
    return sum(int(v) << (64 * k) for k, v in enumerate(np.asarray(a, dtype=np.uint64).tolist()))


def fr_to_mont(curve, x):
    return to_limbs(x * (1 << 256) % R_MOD[curve], 4)


def fft_subgroup(curve, m):
    """Generator of the size-2^m subgroup of Fr (Montgomery limbs): g_max^(2^(max-m))
    (Class/FFT.hs:60-65 getFFTSubgroup)."""
    mx, g = FFT_DOMAIN[curve]
    if not 0 <= m <= mx:
        raise ValueError("m out of range for this curve's FFT domain")
    return fr_to_mont(curve, pow(g, 1 << (mx - m), R_MOD[curve]))


# --------------------------------------------------------------------------------- MSM

def _msm(curve, scalars, bases, mont, kind, nlimbs=None):
    scalars = _c_u64(scalars)
    bases = _c_u64(bases)
    nlp = NLIMBS_P[curve]
    n = bases.size // (2 * nlp)
    if nlimbs is None:
        nlimbs = scalars.size // n if n else 4
    if scalars.size < n * nlimbs:
        raise ValueError("not enough scalar limbs")
    out = np.zeros((2 if kind == OUT_AFFINE else 3) * nlp, dtype=np.uint64)
    _check(lib().zkg_msm(curve, n, _ptr(scalars), nlimbs, int(mont), _ptr(bases), kind, _ptr(out)))
    return out


def msm(curve, scalars_mont, bases):
    """sum k_i * P_i for Montgomery Fr scalars and affine bases; projective result (Z = 1)."""
    return _msm(curve, scalars_mont, bases, True, OUT_PROJ, 4)


def msm_std(curve, scalars_std, bases, nlimbs=None):
    return _msm(curve, scalars_std, bases, False, OUT_PROJ, nlimbs)


def msm_affine(curve, scalars, bases, mont=True, nlimbs=None):
    return _msm(curve, scalars, bases, mont, OUT_AFFINE, 4 if mont else nlimbs)


def msm_jac(curve, scalars, bases, mont=True, nlimbs=None):
    return _msm(curve, scalars, bases, mont, OUT_JAC, 4 if mont else nlimbs)


def msm_device(curve, n, d_scalars, d_bases, mont=True, nlimbs=4, kind=OUT_AFFINE):
    """MSM on device-resident inputs (raw device pointers or objects with data_ptr())."""
    sp = d_scalars.data_ptr() if hasattr(d_scalars, "data_ptr") else int(d_scalars)
    bp = d_bases.data_ptr() if hasattr(d_bases, "data_ptr") else int(d_bases)
    out = np.zeros((2 if kind == OUT_AFFINE else 3) * NLIMBS_P[curve], dtype=np.uint64)
    _check(lib().zkg_msm_device(curve, n, ctypes.c_void_p(sp), nlimbs, int(mont), ctypes.c_void_p(bp), kind,
                                _ptr(out)))
    return out


# --------------------------------------------------------------------------------- NTT

def _ntt(curve, m, gen, values, inverse):
    values = _c_u64(values)
    if values.size != 4 << m:
        raise ValueError("expected 2^m field elements")
    gen = _c_u64(gen)
    out = np.zeros_like(values)
    _check(lib().zkg_ntt(curve, m, _ptr(gen), _ptr(values), _ptr(out), int(inverse)))
    return out


def forward_ntt(curve, m, values, gen=None):
    """Evaluations y_k = sum_i x_i g^(i k) on the size-2^m subgroup (Montgomery in and out)."""
    return _ntt(curve, m, fft_subgroup(curve, m) if gen is None else gen, values, False)


def inverse_ntt(curve, m, values, gen=None):
    """Coefficients from evaluations on the size-2^m subgroup."""
    return _ntt(curve, m, fft_subgroup(curve, m) if gen is None else gen, values, True)


def ntt_device(curve, m, d_src, d_tgt, inverse=False, gen=None):
    gen = _c_u64(fft_subgroup(curve, m) if gen is None else gen)
    sp = d_src.data_ptr() if hasattr(d_src, "data_ptr") else int(d_src)
    tp = d_tgt.data_ptr() if hasattr(d_tgt, "data_ptr") else int(d_tgt)
    _check(lib().zkg_ntt_device(curve, m, _ptr(gen), ctypes.c_void_p(sp), ctypes.c_void_p(tp), int(inverse)))


def g1_gen_mul_device(curve, n, d_scalars_std, d_out):
    sp = d_scalars_std.data_ptr() if hasattr(d_scalars_std, "data_ptr") else int(d_scalars_std)
    op = d_out.data_ptr() if hasattr(d_out, "data_ptr") else int(d_out)
    _check(lib().zkg_g1_gen_mul_device(curve, n, ctypes.c_void_p(sp), ctypes.c_void_p(op)))


# ------------------------------------------------------- binary MSMs and the G1 group FFT

def _binary(curve, rows, bases, kind):
    """rows: (nrows, npoints) array of bytes (non-zero selects the base), or a list of such rows"""
    rows = [np.ascontiguousarray(r, dtype=np.uint8).reshape(-1) for r in rows]
    bases = _c_u64(bases)
    nlp = NLIMBS_P[curve]
    npoints = bases.size // (2 * nlp)
    if any(r.size != npoints for r in rows):
        raise ValueError("incompatible array dimensions")
    ptrs = (ctypes.c_void_p * max(len(rows), 1))(*[r.ctypes.data for r in rows])
    out = np.zeros((len(rows), (2 if kind == OUT_AFFINE else 3) * nlp), dtype=np.uint64)
    _check(lib().zkg_msm_binary(curve, kind, len(rows), npoints, ctypes.cast(ptrs, ctypes.c_void_p), _ptr(bases),
                                _ptr(out)))
    return out


def msm_binary(curve, bits, bases):
    """sum of the bases whose coefficient byte is non-zero; projective result (msmBinary,
    lib/src/ZK/Algebra/Curves/BN128/G1/Proj.hs:280)"""
    return _binary(curve, [bits], bases, OUT_PROJ)[0]


def binary_multi_msm(curve, rows, bases, affine=False):
    """one binary MSM per row over the same bases (binaryMultiMSM / binaryMultiMSM_,
    lib/src/ZK/Algebra/Curves/BN128/G1/Proj.hs:302,329)"""
    return _binary(curve, list(rows), bases, OUT_AFFINE if affine else OUT_PROJ)


def _g1_fft(curve, m, points, gen, inverse, jac):
    points = _c_u64(points)
    if points.size != 3 * NLIMBS_P[curve] << m:
        raise ValueError("expected 2^m points")
    gen = _c_u64(fft_subgroup(curve, m) if gen is None else gen)
    out = np.zeros_like(points)
    _check(lib().zkg_g1_fft(curve, int(jac), m, _ptr(gen), _ptr(points), _ptr(out), int(inverse)))
    return out


def forward_fft(curve, m, points, gen=None, jac=False):
    """group FFT of 2^m projective (or Jacobian) points, normalised output (forwardFFT,
    lib/src/ZK/Algebra/Curves/BN128/G1/Proj.hs:352)"""
    return _g1_fft(curve, m, points, gen, False, jac)


def inverse_fft(curve, m, points, gen=None, jac=False):
    """inverse group FFT (inverseFFT, lib/src/ZK/Algebra/Curves/BN128/G1/Proj.hs:365)"""
    return _g1_fft(curve, m, points, gen, True, jac)


def g1_fft_device(curve, m, d_src, d_tgt, inverse=False, gen=None, jac=False):
    gen = _c_u64(fft_subgroup(curve, m) if gen is None else gen)
    _check(lib().zkg_g1_fft_device(curve, int(jac), m, _ptr(gen), _dptr(d_src), _dptr(d_tgt), int(inverse)))


def msm_binary_device(curve, nrows, npoints, d_coeffs, ld, d_bases, d_out, kind=OUT_AFFINE):
    _check(lib().zkg_msm_binary_device(curve, kind, nrows, npoints, _dptr(d_coeffs), ld, _dptr(d_bases),
                                       _dptr(d_out)))


# ------------------------------------------------------------------ Fr vector operations

FR_OPS = {"from_std": 0, "to_std": 1, "neg": 2, "add": 3, "sub": 4, "sqr": 5, "mul": 6, "inv": 7, "div": 8,
          "mul_add": 9, "mul_sub": 10, "scale": 11, "Ax_plus_y": 12, "Ax_plus_By": 13, "powers": 14,
          "mul_by_powers": 15}


def fr_map(curve, op, a=None, b=None, c=None, coeff_a=None, coeff_b=None, n=None, out=None):
    """the *_arr_mont_* element-wise operation `op` (a name of FR_OPS) on (n, 4) Montgomery arrays
    (lib/src/ZK/Algebra/Curves/BN128/Array.hs)"""
    arrs = [None if x is None else _c_u64(x) for x in (a, b, c, coeff_a, coeff_b)]
    if n is None:
        n = arrs[0].size // 4
    out = np.zeros((n, 4), dtype=np.uint64) if out is None else out
    _check(lib().zkg_fr_map(curve, FR_OPS[op] if isinstance(op, str) else op, n,
                            *[None if x is None else _ptr(x) for x in arrs], _ptr(out)))
    return out


def dot_prod(curve, a, b):
    a, b = _c_u64(a), _c_u64(b)
    out = np.zeros(4, dtype=np.uint64)
    _check(lib().zkg_fr_dot(curve, a.size // 4, _ptr(a), _ptr(b), _ptr(out)))
    return out


def powers(curve, coeff_a, coeff_b, n):
    return fr_map(curve, "powers", coeff_a=coeff_a, coeff_b=coeff_b, n=n)


def batch_inverse(curve, a):
    return fr_map(curve, "inv", a)


def sparse_matrix_mul(curve, n_rows, rows, cols, coeffs, src):
    rows, cols, coeffs, src = (_c_u64(x) for x in (rows, cols, coeffs, src))
    out = np.zeros((n_rows, 4), dtype=np.uint64)
    _check(lib().zkg_fr_sparse_matrix_mul(curve, n_rows, rows.size, _ptr(rows), _ptr(cols), _ptr(coeffs), _ptr(src),
                                          _ptr(out)))
    return out


def last_kernel_ms():
    return float(lib().zkg_last_kernel_ms())


def kernel_launches():
    return int(lib().zkg_kernel_launches())


def _dptr(x):
    return ctypes.c_void_p(x.data_ptr() if hasattr(x, "data_ptr") else int(x))


# -------------------------------------------------------------------- resident base set

class Bases:
    """A base set uploaded to the device once (host numpy array or device tensor) and kept there
    in the MSM pipeline's form; msm() runs over its first n points."""

    def __init__(self, curve, bases, n=None, on_device=None):
        self.curve = curve
        self._h = ctypes.c_void_p()
        if on_device is None:
            on_device = not isinstance(bases, np.ndarray)
        if n is None:
            n = (bases.shape[0] if bases.ndim == 2 else bases.size // (2 * NLIMBS_P[curve]))
        self.n = int(n)
        p = _dptr(bases) if on_device else _ptr(_c_u64(bases))
        _check(lib().zkg_bases_upload(curve, p, self.n, int(on_device), ctypes.byref(self._h)))

    def msm(self, n, scalars, mont=True, nlimbs=4, kind=OUT_AFFINE):
        """scalars: device tensor (resident path) or host numpy array (copied each call)"""
        out = np.zeros((2 if kind == OUT_AFFINE else 3) * NLIMBS_P[self.curve], dtype=np.uint64)
        if isinstance(scalars, np.ndarray):
            sc = _c_u64(scalars)
            _check(lib().zkg_msm_resident_host(self._h, n, _ptr(sc), nlimbs, int(mont), kind, _ptr(out)))
        else:
            _check(lib().zkg_msm_resident(self._h, n, _dptr(scalars), nlimbs, int(mont), kind, _ptr(out)))
        return out

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().zkg_bases_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------- batched mode

class Batch:
    """Many MSMs (prefixes of one resident base set) and NTTs in one captured CUDA graph.
    Add requests with device buffers, then run() (first run captures, later runs replay)."""

    def __init__(self, curve, d_bases, n_bases=None, persistent=None):
        """d_bases: a device buffer of n_bases points, or a Bases set; persistent: True / False to
        choose the persistent-kernel form or graph branches (None: the library default, graph
        branches)"""
        self.curve = curve
        self._h = ctypes.c_void_p()
        self._keep = [d_bases]
        if isinstance(d_bases, Bases):
            _check(lib().zkg_batch_create_resident(d_bases.handle, ctypes.byref(self._h)))
        else:
            _check(lib().zkg_batch_create(curve, _dptr(d_bases), n_bases, ctypes.byref(self._h)))
        if persistent is not None:
            _check(lib().zkg_batch_set_mode(self._h, int(bool(persistent))))
        self.outputs = []

    def add_msm(self, n, d_scalars_mont):
        out = np.zeros(2 * NLIMBS_P[self.curve], dtype=np.uint64)
        self._keep += [d_scalars_mont, out]
        _check(lib().zkg_batch_add_msm(self._h, n, _dptr(d_scalars_mont), _ptr(out)))
        self.outputs.append(out)
        return out

    def add_ntt(self, m, d_src, d_tgt, inverse=False, gen=None):
        g = _c_u64(fft_subgroup(self.curve, m) if gen is None else gen)
        self._keep += [d_src, d_tgt, g]
        _check(lib().zkg_batch_add_ntt(self._h, m, _ptr(g), _dptr(d_src), _dptr(d_tgt), int(inverse)))

    def run(self):
        _check(lib().zkg_batch_run(self._h))
        return float(lib().zkg_batch_last_ms(self._h))

    def set_wait_limit(self, polls, inject_stall=False):
        """before the first run: bound of a pass-dependency wait; inject_stall for tests"""
        _check(lib().zkg_batch_set_wait_limit(self._h, int(polls), int(bool(inject_stall))))

    def persistent_info(self):
        """(runs the persistent kernel, its grid, its number of tasks), after the first run"""
        g, t = ctypes.c_int(), ctypes.c_uint32()
        r = lib().zkg_batch_persistent(self._h, ctypes.byref(g), ctypes.byref(t))
        return r == 1, g.value, t.value

    def close(self):
        if self._h:
            lib().zkg_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -------------------------------------------------------------------------- served mode

class Server:
    """KZG commit server over a resident base set: submit(values) -> ticket, wait(ticket)."""

    def __init__(self, curve, d_bases, n_bases, k_min, k_max, hbm_budget, slots):
        self.curve = curve
        self._h = ctypes.c_void_p()
        self._bases = d_bases
        self._pending = {}
        if isinstance(d_bases, Bases):
            _check(lib().zkg_server_create_resident(d_bases.handle, k_min, k_max, int(hbm_budget), slots,
                                                    ctypes.byref(self._h)))
        else:
            _check(lib().zkg_server_create(curve, _dptr(d_bases), n_bases, k_min, k_max, int(hbm_budget), slots,
                                           ctypes.byref(self._h)))

    def submit(self, k, values_host):
        """values_host: numpy or pinned torch tensor holding 2^k Montgomery Fr elements; kept
        alive until wait() returns."""
        out = np.zeros(2 * NLIMBS_P[self.curve], dtype=np.uint64)
        t = ctypes.c_uint64()
        vp = _ptr(values_host) if isinstance(values_host, np.ndarray) else _dptr(values_host)
        _check(lib().zkg_server_submit(self._h, k, vp, _ptr(out), ctypes.byref(t)))
        self._pending[t.value] = (out, values_host)
        return t.value

    def wait(self, ticket, timeout_ms=None):
        """(affine result, latency ms); raises ZkgError on a failed request (status in .status)
        or when timeout_ms passes first (status ZKG_ERR_TIMEOUT, the ticket stays valid)"""
        lat = ctypes.c_double()
        if timeout_ms is None:
            st = lib().zkg_server_wait(self._h, ticket, ctypes.byref(lat))
        else:
            st = lib().zkg_server_wait_for(self._h, ticket, float(timeout_ms), ctypes.byref(lat))
        if st != ERR_TIMEOUT:
            out, _ = self._pending.pop(ticket)
        _check(st)
        return out, lat.value

    def inject_failure(self, admission):
        """make the admission `admission` places from now fail on the host (failure-path tests)"""
        _check(lib().zkg_server_inject_failure(self._h, admission))

    def stats(self):
        c, mi, pb = ctypes.c_uint64(), ctypes.c_int(), ctypes.c_size_t()
        _check(lib().zkg_server_stats(self._h, ctypes.byref(c), ctypes.byref(mi), ctypes.byref(pb)))
        return {"completed": c.value, "max_inflight": mi.value, "peak_bytes": pb.value}

    def close(self):
        if self._h:
            lib().zkg_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune_msm(curve, d_bases, n_bases, log_min, log_max):
    chosen = np.zeros(log_max - log_min + 1, dtype=np.int32)
    _check(lib().zkg_autotune_msm(curve, _dptr(d_bases), n_bases, log_min, log_max, _ptr(chosen)))
    return {log_min + i: int(c) for i, c in enumerate(chosen)}


def autotune_ntt(curve, m_min, m_max):
    chosen = np.zeros(m_max - m_min + 1, dtype=np.int32)
    _check(lib().zkg_autotune_ntt(curve, m_min, m_max, _ptr(chosen)))
    return {m_min + i: int(c) for i, c in enumerate(chosen)}
