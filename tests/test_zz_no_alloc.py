"""GPU test of zkg_ntt_device_noalloc, the NTT entry point that allocates no memory.

It serves callers that cannot call cudaMalloc (a framework memory pool owns the device memory,
or the host application gives this library no device-memory quota). The test calls it through
the C ABI and requires its output to equal zkg_ntt_device's, bit for bit, on two calls in a row,
device free memory to stay unchanged across repeated calls, and calls made at the same time from
several host threads (which share the one static scratch array) to give each its own correct
result. This file is collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes
import threading

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu


def _lib(zk):
    L = zk.lib()
    f = L.zkg_ntt_device_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    f.restype = ctypes.c_int
    return L


@pytest.mark.parametrize("curve", Z.CURVES)
def test_noalloc_ntt_matches_allocating_entry_point(zk, curve):
    import torch
    L = _lib(zk)
    vp = ctypes.c_void_p
    for m in (0, 1, 3, 8, 9, 13, 16):
        x = Z.rand_fr(curve, 1 << m, 31000 + 17 * m + curve)
        gen = Z.fft_gen(curve, m)
        d_x = torch.from_numpy(x.view(np.int64)).cuda()
        for inverse in (0, 1):
            want = torch.empty_like(d_x)
            zk.ntt_device(curve, m, d_x, want, inverse=bool(inverse), gen=gen)
            torch.cuda.synchronize()
            for rep in range(2):   # two calls in a row share (and overwrite) the static scratch
                got = torch.full_like(d_x, -1)
                torch.cuda.synchronize()
                st = L.zkg_ntt_device_noalloc(curve, m, Z.ptr(gen), vp(d_x.data_ptr()), vp(got.data_ptr()), inverse)
                assert st == 0, L.zkg_last_error()
                assert torch.equal(got, want), (m, inverse, rep)


def test_noalloc_ntt_takes_no_device_memory_per_call(zk):
    import torch
    L = _lib(zk)
    vp = ctypes.c_void_p
    m = 16
    x = Z.rand_fr(Z.BN254, 1 << m, 32000)
    gen = Z.fft_gen(Z.BN254, m)
    d_x = torch.from_numpy(x.view(np.int64)).cuda()
    d_y = torch.empty_like(d_x)
    for inverse in (0, 1):   # first calls: address lookup and lazy loading of the kernels' code
        assert L.zkg_ntt_device_noalloc(0, m, Z.ptr(gen), vp(d_x.data_ptr()), vp(d_y.data_ptr()), inverse) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for inverse in (0, 1, 0, 1):
        assert L.zkg_ntt_device_noalloc(0, m, Z.ptr(gen), vp(d_x.data_ptr()), vp(d_y.data_ptr()), inverse) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # the result is still right after the scratch was reused by other calls
    want = Z.oracle_ntt(Z.BN254, m, gen, x, True)
    assert np.array_equal(d_y.cpu().numpy().view(np.uint64), want)


def test_noalloc_ntt_rejects_sizes_beyond_the_maximum(zk):
    import torch
    L = _lib(zk)
    vp = ctypes.c_void_p
    d_x = torch.zeros((1 << 17) * 4, dtype=torch.int64, device="cuda")
    d_y = torch.zeros_like(d_x)
    gen = Z.fft_gen(Z.BN254, 17)
    st = L.zkg_ntt_device_noalloc(0, 17, Z.ptr(gen), vp(d_x.data_ptr()), vp(d_y.data_ptr()), 0)
    assert st == 1   # ZKG_ERR_ARG
    assert b"2^16" in L.zkg_last_error()
    assert L.zkg_ntt_device_noalloc(0, 4, Z.ptr(gen), vp(d_x.data_ptr()), vp(d_x.data_ptr()), 0) == 1


def test_noalloc_ntt_concurrent_host_threads(zk):
    """Calls from four host threads at once, with different curves, sizes and directions, all
    share the static scratch; the library serialises them, so each output must still equal the
    allocating entry point's."""
    import torch
    L = _lib(zk)
    vp = ctypes.c_void_p
    cases = [(Z.BN254, 16, 0), (Z.BLS12_381, 14, 1), (Z.BN254, 9, 1), (Z.BLS12_381, 16, 0)]
    jobs = []
    for t, (curve, m, inverse) in enumerate(cases):
        x = Z.rand_fr(curve, 1 << m, 33000 + t)
        gen = Z.fft_gen(curve, m)
        d_x = torch.from_numpy(x.view(np.int64)).cuda()
        want = torch.empty_like(d_x)
        zk.ntt_device(curve, m, d_x, want, inverse=bool(inverse), gen=gen)
        jobs.append((curve, m, inverse, gen, d_x, want, torch.full_like(d_x, -1)))
    torch.cuda.synchronize()
    errors = []

    def run(job):
        curve, m, inverse, gen, d_x, _, got = job
        for _ in range(6):
            st = L.zkg_ntt_device_noalloc(curve, m, Z.ptr(gen), vp(d_x.data_ptr()), vp(got.data_ptr()), inverse)
            if st != 0:
                errors.append((curve, m, st))
                return

    ths = [threading.Thread(target=run, args=(j,)) for j in jobs]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    torch.cuda.synchronize()
    assert not errors, errors
    for curve, m, inverse, _, _, want, got in jobs:
        assert torch.equal(got, want), (curve, m, inverse)
