"""Drop-in entry points called from several host threads at once.

A Haskell program built with -threaded may call the generated C functions from several OS threads
at the same time (the FFI imports are `unsafe`, so each call runs on its caller's thread), and any C
user of lib/cbits may do the same: the reference is reentrant. Here four threads call the MSM, NTT
and Fr drop-ins concurrently, with pageable inputs large enough to go through the library's shared
page-locked staging and copy thread pool, and every result must equal the same call made alone.
"""
import ctypes
import threading

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu


def _host_bases(zk, curve, n, seed):
    """affine bases k_i G generated on the device, returned as a pageable host array"""
    import torch
    ks = Z.rand_fr(curve, n, seed)
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((n, 2 * Z.NLP[curve]), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(curve, n, d_k, d_b)
    return d_b.cpu().numpy().view(np.uint64).copy()


def _jobs(zk):
    L = zk.lib()
    jobs = []
    # MSMs through *_G1_proj_MSM_mont_coeff_affine_out; the 2^17 BN254 and 2^16 BLS12-381 base
    # arrays (8 MB, 6 MB) are staged through the page-locked slots
    for curve, n, seed in ((Z.BN254, 1 << 17, 1), (Z.BN254, 5000, 2), (Z.BLS12_381, 1 << 16, 3)):
        b = _host_bases(zk, curve, n, 47000 + seed)
        s = Z.rand_fr(curve, n, 47100 + seed)
        fn = getattr(L, "%s_G1_proj_MSM_mont_coeff_affine_out" % Z.NAMES[curve])

        def msm(fn=fn, n=n, s=s, b=b, nl=Z.NLP[curve]):
            out = np.zeros(2 * nl, np.uint64)
            fn(ctypes.c_int(n), Z.ptr(s), Z.ptr(b), Z.ptr(out), ctypes.c_int(4))
            return out
        jobs.append(("msm", curve, n, msm))
    # forward and inverse NTTs through *_poly_mont_ntt_{forward,inverse} (8 MB and 4 MB vectors)
    for curve, m, inverse, seed in ((Z.BN254, 18, False, 4), (Z.BLS12_381, 17, True, 5)):
        x = Z.rand_fr(curve, 1 << m, 47200 + seed)
        g = np.ascontiguousarray(zk.fft_subgroup(curve, m), dtype=np.uint64)
        fn = getattr(L, "%s_poly_mont_ntt_%s" % (Z.NAMES[curve], "inverse" if inverse else "forward"))

        def ntt(fn=fn, m=m, g=g, x=x):
            y = np.zeros_like(x)
            fn(ctypes.c_int(m), Z.ptr(g), Z.ptr(x), Z.ptr(y))
            return y
        jobs.append(("ntt", curve, m, ntt))
    # element-wise product through bn128_arr_mont_mul (two 8 MB operands)
    n = 1 << 18
    a, b = Z.rand_fr(Z.BN254, n, 47300), Z.rand_fr(Z.BN254, n, 47301)

    def mul(a=a, b=b, n=n):
        out = np.zeros_like(a)
        L.bn128_arr_mont_mul(ctypes.c_int(n), Z.ptr(a), Z.ptr(b), Z.ptr(out))
        return out
    jobs.append(("fr_mul", Z.BN254, n, mul))
    return jobs


def test_drop_in_calls_from_host_threads(zk):
    L = zk.lib()
    jobs = _jobs(zk)
    alone = []
    for name, curve, size, fn in jobs:
        alone.append(fn())
        assert L.zkg_last_status() == 0, (name, L.zkg_last_error())
    errors = []

    def worker(t):
        try:
            for rep in range(2):
                for k in range(len(jobs)):
                    j = (k + t) % len(jobs)   # each thread starts at a different job
                    name, curve, size, fn = jobs[j]
                    got = fn()
                    assert L.zkg_last_status() == 0, (name, L.zkg_last_error())   # per-thread status
                    assert np.array_equal(got, alone[j]), (t, rep, name, curve, size)
        except Exception as e:   # collected: an assertion in a thread would not fail the test
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    # and the calls made alone are right: the 5000-point MSM equals (sum s_i k_i) G
    assert jobs[1][0] == "msm" and jobs[1][2] == 5000
    want = Z.msm_identity_affine(Z.BN254, Z.rand_fr(Z.BN254, 5000, 47002), Z.rand_fr(Z.BN254, 5000, 47102))
    assert np.array_equal(alone[1], want)
