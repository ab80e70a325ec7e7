"""The tuning and path-selection knobs change no result.

Each knob is read once from the environment when the library loads, so every setting runs in a
child process; its MSMs (host-buffer path, split into point-range parts where the setting asks),
NTTs and group FFTs must equal the default configuration's byte for byte:
  ZKB_MSM_DPF / ZKB_NTT_DPF / ZKB_G1_DPF = 0   products on the 32-bit integer path
  ZKB_MSM_PF = 0 / 3                           base prefetch into registers / three stages
  ZKB_MSM_L1, ZKB_MSM_K1                       chunk length, running-sum group size
  ZKB_MSM_PARTS, ZKB_MSM_PART_RATIO            host-buffer pipeline layout
  ZKB_MSM_WMAJOR = 0                           point-major digit histogram and scatter
  ZKB_MSM_DIGITS = 0                           window-major scatter re-deriving digits from the scalars
  ZKB_FR_DPF = 0                               Fr vector operations on 32-bit-limb products
  ZKB_FR_MAP_MODE = 1                          Fr single-product operations two elements per iteration
  ZKB_BATCH_PERSISTENT = 1                     batches as one persistent kernel instead of graph branches
  ZKB_DEVICE_CHECKS = 1                        device bounds checks on (valid inputs: no check fires)
  ZKB_MSM_TRACE = 1                            host-buffer MSM timeline printed to stderr
  ZKB_MSM_TREE, ZKB_MSM_TREE_B                 affine tree levels forced on these small MSMs
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import zkutil as Z

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

SETTINGS = [
    {"ZKB_MSM_DPF": "0", "ZKB_NTT_DPF": "0", "ZKB_G1_DPF": "0"},
    {"ZKB_MSM_PF": "0", "ZKB_MSM_L1": "37", "ZKB_MSM_K1": "4", "ZKB_MSM_PARTS": "4", "ZKB_MSM_PART_RATIO": "15"},
    {"ZKB_MSM_PF": "3", "ZKB_MSM_L1": "200", "ZKB_MSM_K1": "64", "ZKB_MSM_PARTS": "2", "ZKB_MSM_PART_RATIO": "40"},
    {"ZKB_MSM_PARTS": "3", "ZKB_MSM_L1": "16", "ZKB_MSM_K1": "2", "ZKB_FR_MAP_MODE": "1"},
    {"ZKB_MSM_WMAJOR": "0", "ZKB_FR_DPF": "0", "ZKB_BATCH_PERSISTENT": "1"},
    {"ZKB_DEVICE_CHECKS": "1", "ZKB_MSM_PARTS": "2", "ZKB_MSM_TRACE": "1"},
    {"ZKB_MSM_DIGITS": "0", "ZKB_DEVICE_CHECKS": "1"},
    {"ZKB_MSM_TREE": "5", "ZKB_MSM_TREE_B": "6", "ZKB_DEVICE_CHECKS": "1"},
]


def _inputs(curve):
    n = 3000
    ks = Z.rand_fr(curve, n, 31000 + curve)
    bases = Z.gen_bases_cpu(curve, Z.rand_fr(curve, n, 31100 + curve))
    vals = Z.rand_fr(curve, 1 << 10, 31200 + curve)
    nl = Z.NLP[curve]
    one = Z.to_limbs((1 << (64 * nl)) % Z.P[curve], nl)
    pts = np.concatenate([bases[:64], np.tile(one, (64, 1))], axis=1)
    return ks, bases, vals, pts


def compute_all():
    zk = Z.load_package()
    out = {}
    for curve in Z.CURVES:
        ks, bases, vals, pts = _inputs(curve)
        tag = Z.NAMES[curve]
        out[tag + "_msm"] = zk.msm_affine(curve, ks, bases)
        out[tag + "_msm_small"] = zk.msm_affine(curve, ks[:100], bases[:100])
        skew = ks.copy()   # long segments (repeated scalars) beside short ones
        skew[::3] = ks[0]
        skew[: len(ks) // 10] = ks[1]
        out[tag + "_msm_skew"] = zk.msm_affine(curve, skew, bases)
        out[tag + "_ntt"] = zk.forward_ntt(curve, 10, vals)
        out[tag + "_intt"] = zk.inverse_ntt(curve, 10, vals)
        out[tag + "_fft"] = zk.forward_fft(curve, 6, pts)
        L = zk.lib()
        rev = vals[::-1].copy()   # held in a name: a temporary's buffer could be freed before the call
        A, B = Z.to_limbs(12345, 4), Z.to_limbs(678, 4)
        for op in (6, 7, 15):   # mul, batch inverse, mul_by_powers
            o = np.zeros_like(vals)
            assert L.zkg_fr_map(curve, op, vals.shape[0], Z.ptr(vals), Z.ptr(rev), None, Z.ptr(A),
                                Z.ptr(B), Z.ptr(o)) == 0
            out[tag + "_fr%d" % op] = o
        # a batch: three MSMs against prefixes of the bases and three NTTs
        import torch
        d_b = torch.from_numpy(bases.view(np.int64)).cuda()
        b = zk.Batch(curve, d_b, bases.shape[0])
        outs = []
        for i, n in enumerate((100, 1000, 3000)):
            s = torch.from_numpy(np.ascontiguousarray(ks[:n]).view(np.int64)).cuda()
            outs.append((s, b.add_msm(n, s)))
        ys = []
        for m in (5, 10, 14):
            x = torch.from_numpy(Z.rand_fr(curve, 1 << m, 31300 + m).view(np.int64)).cuda()
            y = torch.empty_like(x)
            b.add_ntt(m, x, y, inverse=(m == 10))
            ys.append((x, y))
        b.run()
        for i, (_, o) in enumerate(outs):
            out[tag + "_batch_msm%d" % i] = o.copy()
        for i, (_, y) in enumerate(ys):
            out[tag + "_batch_ntt%d" % i] = y.cpu().numpy()
        b.close()
    return out


def _dump(path):
    np.savez(path, **compute_all())


@pytest.mark.parametrize("setting", range(len(SETTINGS)))
def test_knob_settings_change_no_result(zk, setting, tmp_path):
    want = compute_all()
    path = str(tmp_path / "knobs.npz")
    env = dict(os.environ)
    env.update(SETTINGS[setting])
    code = "import sys; sys.path.insert(0, %r); import test_knobs_gpu as T; T._dump(%r)" % (HERE, path)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    if SETTINGS[setting].get("ZKB_MSM_TRACE") == "1":
        assert "zkb msm trace" in r.stderr   # the host-buffer MSMs printed their timelines
    got = np.load(path)
    for k, v in want.items():
        assert np.array_equal(got[k], v), (SETTINGS[setting], k)
