"""GPU tests of the batched mode (one captured graph of many MSMs and NTTs) and the served commit
loop: every result must be byte-identical to the same request run alone on the per-call path,
and (for a sample) to the oracle."""
import ctypes
import threading

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


@pytest.mark.parametrize("persistent", (False, True))
@pytest.mark.parametrize("curve", Z.CURVES)
def test_batch_matches_per_call(zk, curve, persistent):
    import torch
    rng = np.random.default_rng(40000 + curve)
    nb = 1 << 14
    d_b = _bases(zk, curve, nb, 40100 + curve)
    b = zk.Batch(curve, d_b, nb, persistent=persistent)
    msm_in = []
    for i in range(24):
        n = int(2 ** rng.uniform(0, 14)) if i else 0      # includes an empty MSM
        s = torch.from_numpy(Z.rand_fr(curve, max(n, 1), 40200 + i).view(np.int64)).cuda()
        msm_in.append((n, s, b.add_msm(n, s)))
    ntt_in = []
    for i in range(10):
        m = int(rng.integers(1, 15))
        x = torch.from_numpy(Z.rand_fr(curve, 1 << m, 40300 + i).view(np.int64)).cuda()
        y = torch.empty_like(x)
        b.add_ntt(m, x, y, inverse=bool(i % 2))
        ntt_in.append((m, x, y, bool(i % 2)))
    for rep in range(2):   # second run replays the graph on new input contents
        if rep:
            for n, s, _ in msm_in:
                s.copy_(torch.from_numpy(Z.rand_fr(curve, s.shape[0], 41000 + n).view(np.int64)))
            for m, x, _, _ in ntt_in:
                x.copy_(torch.from_numpy(Z.rand_fr(curve, 1 << m, 41500 + m).view(np.int64)))
            torch.cuda.synchronize()
        b.run()
        for n, s, out in msm_in:
            alone = zk.msm_device(curve, n, s, d_b, mont=True)
            assert np.array_equal(out, alone), (rep, n)
        for m, x, y, inv in ntt_in:
            want = torch.empty_like(x)
            zk.ntt_device(curve, m, x, want, inverse=inv)
            torch.cuda.synchronize()
            assert torch.equal(y, want), (rep, m, inv)
    # spot check one batched MSM against the oracle
    n, s, out = max(msm_in, key=lambda t: t[0] if t[0] < 5000 else -1)
    sh = s.cpu().numpy().view(np.uint64)[:n]
    bh = d_b.cpu().numpy().view(np.uint64)[:n]
    assert np.array_equal(out, Z.oracle_msm_affine(curve, sh, 4, True, bh))
    b.close()


def test_batch_runs_one_persistent_kernel_with_bounded_waits(zk):
    """the batch's accumulation and NTT passes run in one persistent launch; a pass whose
    dependency never completes ends the run with ZKG_ERR_TIMEOUT after its bounded wait, and the
    device stays usable for the next batch"""
    import torch
    curve = Z.BN254
    nb = 1 << 12
    d_b = _bases(zk, curve, nb, 44000)
    def make(stall):
        b = zk.Batch(curve, d_b, nb, persistent=True)
        if stall:
            b.set_wait_limit(1 << 14, inject_stall=True)
        s = torch.from_numpy(Z.rand_fr(curve, nb, 44001).view(np.int64)).cuda()
        out = b.add_msm(nb, s)
        xs = [torch.from_numpy(Z.rand_fr(curve, 1 << m, 44010 + m).view(np.int64)).cuda() for m in (12, 17)]
        ys = [torch.empty_like(x) for x in xs]
        for m, x, y in zip((12, 17), xs, ys):
            b.add_ntt(m, x, y, inverse=(m == 17))
        return b, s, out, xs, ys
    b, s, out, xs, ys = make(True)
    with pytest.raises(zk.ZkgError) as e:
        b.run()
    assert e.value.status == zk.ERR_TIMEOUT
    b.close()
    b, s, out, xs, ys = make(False)
    b.run()
    persistent, grid, tasks = b.persistent_info()
    assert persistent and grid >= 1 and tasks > 0
    assert np.array_equal(out, zk.msm_device(curve, nb, s, d_b, mont=True))
    for m, x, y in zip((12, 17), xs, ys):
        want = torch.empty_like(x)
        zk.ntt_device(curve, m, x, want, inverse=(m == 17))
        torch.cuda.synchronize()
        assert torch.equal(y, want), m
    b.close()


@pytest.mark.parametrize("curve", Z.CURVES)
def test_server_results_same_alone_and_in_the_mix(zk, curve):
    import torch
    nb = 1 << 13
    d_b = _bases(zk, curve, nb, 42000 + curve)
    # budget for about two of the largest requests: admission has to wait for memory
    L = zk.lib()
    one = ctypes.c_void_p()
    # find the smallest budget the server accepts, then double it
    budget = 1 << 20
    while L.zkg_server_create(curve, ctypes.c_void_p(d_b.data_ptr()), nb, 4, 13, budget, 4, ctypes.byref(one)) != 0:
        budget *= 2
    L.zkg_server_destroy(one)
    srv = zk.Server(curve, d_b, nb, 4, 13, 2 * budget, 4)
    rng = np.random.default_rng(42100 + curve)
    reqs = []
    for i in range(40):
        k = int(rng.integers(4, 14))
        v = torch.from_numpy(Z.rand_fr(curve, 1 << k, 42200 + i).view(np.int64)).pin_memory()
        reqs.append((k, v))
    tickets = [None] * len(reqs)

    def submit(lo, hi):
        for j in range(lo, hi):
            tickets[j] = srv.submit(reqs[j][0], reqs[j][1])
    th = [threading.Thread(target=submit, args=(t * 10, t * 10 + 10)) for t in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["max_inflight"] >= 2          # requests overlapped on the device
    assert st["peak_bytes"] <= 2 * budget   # admission respected the HBM budget
    srv.close()
    bh = d_b.cpu().numpy().view(np.uint64)
    for (k, v), (out, lat) in zip(reqs, results):
        assert lat > 0
        vals = v.numpy().view(np.uint64).reshape(-1, 4)
        coef = zk.inverse_ntt(curve, k, vals)
        alone = zk.msm_affine(curve, coef, bh[:1 << k], mont=True)
        assert np.array_equal(out, alone), k
    # and one against the oracle end to end (iNTT + MSM)
    k, v = reqs[0]
    vals = v.numpy().view(np.uint64).reshape(-1, 4)
    coef = Z.oracle_ntt(curve, k, Z.fft_gen(curve, k), vals, True)
    assert np.array_equal(results[0][0], Z.oracle_msm_affine(curve, coef, 4, True, bh[:1 << k]))


def test_autotuners_pick_valid_choices_and_keep_results(zk):
    import torch
    nb = 1 << 12
    d_b = _bases(zk, Z.BN254, nb, 43000)
    ks = Z.rand_fr(Z.BN254, nb, 43001)
    bh = d_b.cpu().numpy().view(np.uint64)
    before = zk.msm_affine(Z.BN254, ks, bh)
    chosen = zk.autotune_msm(Z.BN254, d_b, nb, 8, 12)
    assert all(2 <= c <= 20 for c in chosen.values())
    assert zk.lib().zkg_msm_tuned_window(Z.BN254, 12) == chosen[12]
    assert np.array_equal(zk.msm_affine(Z.BN254, ks, bh), before)
    nt = zk.autotune_ntt(Z.BN254, 10, 12)
    assert all(6 <= k <= 11 for k in nt.values())
    x = Z.rand_fr(Z.BN254, 1 << 12, 43002)
    assert np.array_equal(zk.forward_ntt(Z.BN254, 12, x), Z.oracle_ntt(Z.BN254, 12, Z.fft_gen(Z.BN254, 12), x, False))


_CHILD_TUNE = r"""
import ctypes, json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, torch, zkutil as Z
zk = Z.load_package(); L = zk.lib()
mode = sys.argv[2]
c, l1, k1, pf = (ctypes.c_int() for _ in range(4))
if mode == "tune":
    n = 1 << 12
    ks = Z.rand_fr(Z.BN254, n, 43100)
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((n, 8), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(Z.BN254, n, d_k, d_b)
    torch.cuda.synchronize()
    zk.autotune_msm(Z.BN254, d_b, n, 11, 12)
    zk.autotune_ntt(Z.BN254, 12, 12)
r = L.zkg_msm_tuned_config(Z.BN254, 12, ctypes.byref(c), ctypes.byref(l1), ctypes.byref(k1), ctypes.byref(pf))
print(json.dumps([r, c.value, l1.value, k1.value, pf.value]))
"""


def test_autotune_results_persist_across_processes(tmp_path):
    """zkg_autotune_* with ZKG_TUNE_CACHE set writes the tuned settings; a new process with the
    same variable starts with them (the drop-in entry points then use them)"""
    import json
    import os
    import subprocess
    import sys
    cache = tmp_path / "tune.txt"
    env = dict(os.environ, ZKG_TUNE_CACHE=str(cache))
    here = os.path.dirname(os.path.abspath(__file__))
    run = lambda mode, e: json.loads(subprocess.run([sys.executable, "-c", _CHILD_TUNE, here, mode], env=e,
                                                    capture_output=True, text=True, check=True).stdout.strip().splitlines()[-1])
    tuned = run("tune", env)
    assert tuned[0] == 1 and 2 <= tuned[1] <= 20
    lines = cache.read_text().splitlines()
    assert any(l.startswith("msm 0 12 ") for l in lines) and any(l.startswith("ntt 0 12 ") for l in lines)
    assert run("read", env) == tuned
    fresh = dict(os.environ)
    fresh.pop("ZKG_TUNE_CACHE", None)
    assert run("read", fresh)[0] == 0
