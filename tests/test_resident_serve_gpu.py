"""GPU tests of the resident base set (zkg_bases_*) and of the commit server's failure, deadline
and admission behaviour.

Resident base set: MSMs over prefixes of a set uploaded once (from host memory or from a device
buffer) must equal the plain device-path MSM on the same points, with device or host scalars,
and launch no more kernels than it; batches and servers built on the set must give the per-call
results. Server: a launch failure injected on the host must complete every ticket (no wait may
hang), a deadline wait must time out and leave the ticket valid, and a large request behind many
small ones must still be admitted.
"""
import ctypes

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu


def _bases(zk, curve, n, seed):
    import torch
    ks = Z.rand_fr(curve, n, seed)
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((n, 2 * Z.NLP[curve]), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(curve, n, d_k, d_b)
    torch.cuda.synchronize()
    return d_b


@pytest.mark.parametrize("curve", Z.CURVES)
def test_resident_bases_match_device_path(zk, curve):
    import torch
    nb = 1 << 16
    d_b = _bases(zk, curve, nb, 60000 + curve)
    bh = d_b.cpu().numpy().view(np.uint64).copy()
    sets = [zk.Bases(curve, bh), zk.Bases(curve, d_b, nb, on_device=True)]   # from host, from device
    L = zk.lib()
    for n in (0, 1, 7, 1000, nb // 2 + 3, nb):
        s = Z.rand_fr(curve, max(n, 1), 60100 + n)[:n] if n else np.zeros((0, 4), np.uint64)
        d_s = torch.from_numpy(np.ascontiguousarray(s).view(np.int64).reshape(-1, 4)).cuda() if n else \
            torch.zeros((1, 4), dtype=torch.int64, device="cuda")
        want = zk.msm_device(curve, n, d_s, d_b, mont=True)
        for B in sets:
            assert np.array_equal(B.msm(n, d_s), want), n
            if n:
                assert np.array_equal(B.msm(n, s), want), n   # host scalars
        # std scalars with 2 limbs and projective output
        if n:
            s2 = np.ascontiguousarray(s[:, :2])
            d_s2 = torch.from_numpy(s2.view(np.int64)).cuda()
            want2 = zk.msm_device(curve, n, d_s2, d_b, mont=False, nlimbs=2, kind=zk.OUT_PROJ)
            assert np.array_equal(sets[0].msm(n, d_s2, mont=False, nlimbs=2, kind=zk.OUT_PROJ), want2)
    # the resident path launches no more kernels than the device path (no per-call base handling)
    n = nb
    d_s = torch.from_numpy(Z.rand_fr(curve, n, 60200).view(np.int64)).cuda()
    l0 = L.zkg_kernel_launches()
    zk.msm_device(curve, n, d_s, d_b, mont=True)
    l1 = L.zkg_kernel_launches()
    sets[0].msm(n, d_s)
    l2 = L.zkg_kernel_launches()
    assert 0 < (l2 - l1) <= (l1 - l0)
    with pytest.raises(zk.ZkgError):
        sets[0].msm(nb + 1, d_s)
    for B in sets:
        B.close()


def test_batch_and_server_on_resident_bases(zk):
    import torch
    curve = Z.BN254
    nb = 1 << 14
    d_b = _bases(zk, curve, nb, 61000)
    B = zk.Bases(curve, d_b, nb, on_device=True)
    b = zk.Batch(curve, B)
    rng = np.random.default_rng(61100)
    msm_in = []
    for i in range(12):
        n = int(2 ** rng.uniform(4, 14))
        s = torch.from_numpy(Z.rand_fr(curve, n, 61200 + i).view(np.int64)).cuda()
        msm_in.append((n, s, b.add_msm(n, s)))
    for rep in range(2):
        b.run()
        for n, s, out in msm_in:
            assert np.array_equal(out, zk.msm_device(curve, n, s, d_b, mont=True)), (rep, n)
    b.close()
    srv = zk.Server(curve, B, nb, 4, 14, 1 << 30, 4)
    bh = d_b.cpu().numpy().view(np.uint64)
    for k in (4, 9, 14):
        v = torch.from_numpy(Z.rand_fr(curve, 1 << k, 61300 + k).view(np.int64)).pin_memory()
        out, _ = srv.wait(srv.submit(k, v))
        coef = zk.inverse_ntt(curve, k, v.numpy().view(np.uint64).reshape(-1, 4))
        assert np.array_equal(out, zk.msm_affine(curve, coef, bh[:1 << k], mont=True)), k
    srv.close()
    B.close()


def test_server_injected_failure_completes_every_ticket(zk):
    import torch
    curve = Z.BN254
    nb = 1 << 12
    d_b = _bases(zk, curve, nb, 62000)
    srv = zk.Server(curve, d_b, nb, 4, 12, 1 << 30, 2)
    vals = {k: torch.from_numpy(Z.rand_fr(curve, 1 << k, 62100 + k).view(np.int64)).pin_memory()
            for k in (8, 12)}
    good, _ = srv.wait(srv.submit(8, vals[8]))
    srv.inject_failure(3)   # the fourth admission from now fails on the host
    tickets = [srv.submit(12 if i % 3 == 0 else 8, vals[12 if i % 3 == 0 else 8]) for i in range(12)]
    ok, failed = 0, 0
    for i, t in enumerate(tickets):
        try:
            out, lat = srv.wait(t, timeout_ms=60000)
            ok += 1
            if i % 3:
                assert np.array_equal(out, good)
        except zk.ZkgError as e:
            assert e.status != zk.ERR_TIMEOUT, "a ticket was left hanging after the failure"
            failed += 1
    assert ok + failed == len(tickets)
    assert ok >= 3 and failed >= 1   # the three admissions before the failure completed
    with pytest.raises(zk.ZkgError):   # new submissions are refused after the failure
        srv.submit(8, vals[8])
    srv.close()


def test_server_deadline_and_large_request_admission(zk):
    import torch
    curve = Z.BN254
    nb = 1 << 16
    d_b = _bases(zk, curve, nb, 63000)
    # budget: one 2^16 request at a time; small requests fit beside each other
    L = zk.lib()
    h = ctypes.c_void_p()
    budget = 1 << 20
    while L.zkg_server_create(curve, ctypes.c_void_p(d_b.data_ptr()), nb, 6, 16, budget, 8, ctypes.byref(h)) != 0:
        budget = int(budget * 1.25)
    L.zkg_server_destroy(h)
    srv = zk.Server(curve, d_b, nb, 6, 16, budget, 8)
    v16 = torch.from_numpy(Z.rand_fr(curve, 1 << 16, 63100).view(np.int64)).pin_memory()
    v6 = torch.from_numpy(Z.rand_fr(curve, 1 << 6, 63101).view(np.int64)).pin_memory()
    t_small = [srv.submit(6, v6) for _ in range(4)]
    t_big = srv.submit(16, v16)
    t_more = [srv.submit(6, v6) for _ in range(60)]
    # a deadline of 0 ms on a request that cannot be finished yet returns a timeout, ticket valid
    early = set()
    try:
        srv.wait(t_more[-1], timeout_ms=0.0)
        early.add(t_more[-1])
    except zk.ZkgError as e:
        assert e.status == zk.ERR_TIMEOUT
    big, _ = srv.wait(t_big, timeout_ms=120000)
    for t in t_small + t_more:
        if t not in early:
            srv.wait(t, timeout_ms=120000)
    bh = d_b.cpu().numpy().view(np.uint64)
    coef = zk.inverse_ntt(curve, 16, v16.numpy().view(np.uint64).reshape(-1, 4))
    assert np.array_equal(big, zk.msm_affine(curve, coef, bh, mont=True))
    assert srv.stats()["completed"] == 65
    srv.close()
