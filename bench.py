"""Benchmark: BN254 G1 multi-scalar multiplication at n = 2^22 points on B200.

Workload (one step): sum_i s_i * P_i over n = 2^22 points, s_i uniform in Fr stored as Montgomery
limbs, P_i = k_i * G affine Montgomery with k_i uniform in Fr (seeded synthetic inputs, the
shapes and distributions of the reference's MSM configurations), affine output, bit-exact.
It is the call the reference's Haskell `msm` makes: bn128_G1_proj_MSM_mont_coeff_affine_out.

  value  points/s with inputs resident in HBM (zkg_msm_device), device-timed with CUDA events on
         the stream the kernels run on; inputs (402 MB) exceed L2 (126 MB)
  e2e    points/s through the drop-in C ABI with host (pinned) buffers: every step copies the
         scalars and bases host->device and reads the affine point back
  roofline  the bucket-accumulation kernel (k_msm_accum, ~80% of device time) against the
         measured FP64-pipe rate of this GPU (the field products' pipe), with the integer
         multiply-add (IMAD) equivalent beside it
  cpu_baseline  the reference's own C MSM (oracle/_ref, compiled from the reference sources) on
         the same 2^22 inputs, the points split into one contiguous range per host thread (the
         reference is single-threaded), partial sums added with the reference's own
         bn128_G1_proj_add
  ntt    BN254 Fr forward + inverse NTT at 2^24, device-resident (secondary figure)

Every full-size MSM result is checked against (sum_i s_i k_i mod r) G computed independently in
numpy / Python integers (bases P_i = k_i G).

--impl reference times the reference's CPU implementation on the same 2^22 workload (all host
threads, one contiguous point range each) and prints the same JSON line with "impl": "reference".
--details PATH writes the full records of the secondary configurations to a JSON file; the
printed line keeps their summary figures.

Multi-GPU (torchrun): every rank runs the same workload on its own GPU (replicas; the MSM path
has no exchange step); value = points of all ranks / max over ranks of the device time.
"""
import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import zkutil as Z  # noqa: E402  (input generation and package loader; oracle only in the CPU legs)

METRIC = "MSM points/s @2^22 BN254 G1 (bit-exact)"
IMAD_PER_MADD = 10 * 264   # XYZZ mixed addition: 8 multiplications + 2 squarings, 264 IMAD each (8x32-bit CIOS)
# The field products run on the FP64 pipe: 5 limbs of 52 bits, 2*5^2 = 50 limb products per
# Montgomery product (25 for a*b, 25 for m*p; the digits m_i are 64-bit integer products), each
# split exactly by 2 FMAs + 1 DADD; a squaring needs 15 + 25 = 40 limb products
FP64_PER_PRODUCT = 3 * 50
FP64_PER_SQUARE = 3 * 40
FP64_PER_MADD = 8 * FP64_PER_PRODUCT + 2 * FP64_PER_SQUARE
IMAD_PER_NTT_BFLY = 264
# FMA-pipe issue slots of one 8x32-bit Montgomery product: 128 mad.lo (1 slot) + 128 mad.hi (2 slots,
# measured at half the mad.lo rate on B200) + 8 (m = t0 * n0)
FMA_SLOTS_PER_MADD = 10 * (128 + 2 * 128 + 8)
# DRAM bytes (read + write) of one bucket-accumulation launch (k_msm_accum_w<BN254E, 384, 2>) by
# log2 n, from `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none
# -k regex:k_msm_accum -c 1` on `python bench.py --steps 2 --warmup 3 --no-extra --no-cpu --no-ntt
# --no-tune`; re-captured whenever the kernel changes
ACCUM_DRAM_BYTES = {22: 6.828788480e9}


def hbm_peak():
    """Measured HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json, else a fallback figure of an
    earlier measurement on B200."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--log-n", type=int, default=22)
    ap.add_argument("--no-ntt", action="store_true")
    ap.add_argument("--no-msm", action="store_true", help="only the NTT figure (for profiling)")
    ap.add_argument("--ntt-m", type=int, default=24)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip configurations 1, 3, 4 and 5")
    ap.add_argument("--details", default=None, help="write the full secondary records to this JSON file")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default settings; for profiling)")
    ap.add_argument("--config3-only", action="store_true",
                    help="only configuration 3 (BLS12-381 MSM at 2^22; for profiling its kernels)")
    ap.add_argument("--single-thread-ref", type=int, default=1,
                    help="reference arm: also time one single-thread 2^22 reference MSM (1) or not (0)")
    return ap.parse_args()


# --------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi sampling (every 20 ms, timestamped) of SM clock and throttle reasons; stop() keeps
    the samples taken inside the window [mark_begin(), mark_end()] when both were marked."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.f = None
        self.t0 = self.t1 = None

    def mark_begin(self):
        self.t0 = datetime.datetime.now()

    def mark_end(self):
        self.t1 = datetime.datetime.now()

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", delete=False)
            cmd = ["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits", "-lms", "20"]
            if self.gpu_id:
                cmd += ["-i", self.gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.seek(0)
        rows = [l.strip().split(",") for l in self.f.read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        if self.t0 is not None and self.t1 is not None:   # samples inside the marked window only
            pad = datetime.timedelta(milliseconds=25)
            inside = []
            for r in rows:
                try:
                    ts = datetime.datetime.strptime(r[0].strip(), "%Y/%m/%d %H:%M:%S.%f")
                except (ValueError, IndexError):
                    inside = rows   # unparsable timestamps: keep everything
                    break
                if self.t0 - pad <= ts <= self.t1 + pad:
                    inside.append(r)
            rows = inside
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[2]))
                mx.append(float(r[3]))
                pw.append(float(r[4]))
                for k, v in zip(names, r[6:10]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------- CPU reference

def _ref_msm_fns():
    """The reference C's MSM, projective add and affine conversion (oracle/_ref), or None."""
    ref = Z.reference()
    if ref is None:
        return None
    vp, ci = ctypes.c_void_p, ctypes.c_int
    msm = ref.bn128_G1_proj_MSM_mont_coeff_proj_out
    msm.argtypes = [ci, vp, vp, vp, ci]
    add = ref.bn128_G1_proj_add
    add.argtypes = [vp, vp, vp]
    aff = ref.bn128_G1_proj_to_affine
    aff.argtypes = [vp, vp]
    return msm, add, aff


def cpu_msm_all_cores(scal, bases, threads):
    """sum s_i P_i over all points on the host: one contiguous point range per thread, each
    range summed by the reference's own bn128_G1_proj_MSM_mont_coeff_proj_out (the reference is
    single-threaded), the partial sums added with bn128_G1_proj_add and converted by
    bn128_G1_proj_to_affine. Without oracle/_ref the oracle restatement runs instead (kind
    "port"). Returns (affine out, seconds, kind)."""
    n = scal.shape[0]
    bounds = [n * t // threads for t in range(threads + 1)]
    parts = np.zeros((threads, 12), np.uint64)
    fns = _ref_msm_fns()
    if fns is not None:
        msm, add, aff = fns
        kind = "reference"

        def one(t):
            lo, hi = bounds[t], bounds[t + 1]
            msm(hi - lo, ctypes.c_void_p(scal[lo:].ctypes.data), ctypes.c_void_p(bases[lo:].ctypes.data),
                ctypes.c_void_p(parts[t].ctypes.data), 4)
    else:
        kind = "port"
        O = Z.oracle()

        def one(t):
            lo, hi = bounds[t], bounds[t + 1]
            O.oracle_msm_proj(0, hi - lo, ctypes.c_void_p(scal[lo:].ctypes.data), 4, 1,
                              ctypes.c_void_p(bases[lo:].ctypes.data), ctypes.c_void_p(parts[t].ctypes.data), 0)
    ths = [threading.Thread(target=one, args=(t,)) for t in range(threads)]
    t0 = time.perf_counter()
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    acc = parts[0].copy()
    out = np.zeros(8, np.uint64)
    if fns is not None:
        for t in range(1, threads):
            add(Z.ptr(acc), Z.ptr(parts[t]), Z.ptr(acc))
        aff(Z.ptr(acc), Z.ptr(out))
    else:
        O = Z.oracle()
        for t in range(1, threads):
            nxt = np.zeros(12, np.uint64)
            O.oracle_proj_add(0, Z.ptr(acc), Z.ptr(parts[t]), Z.ptr(nxt))
            acc = nxt
        O.oracle_proj_to_affine(0, Z.ptr(acc), Z.ptr(out))
    return out, time.perf_counter() - t0, kind


def msm_inputs_host(log_n, seed):
    """the seeded 2^log_n BN254 workload on the host: k_i, Montgomery scalars, bases k_i G (bases
    by the oracle's fixed-base comb on host threads; input preparation, not timed)"""
    n = 1 << log_n
    ks = Z.rand_fr(Z.BN254, n, seed)
    sc = Z.rand_fr(Z.BN254, n, seed + 1)
    return ks, sc, Z.gen_bases_cpu(Z.BN254, ks)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = len(os.sched_getaffinity(0))
    n = 1 << args.log_n
    ks, sc, bases = msm_inputs_host(args.log_n, 0x5eed0001)
    want = Z.msm_identity_affine(Z.BN254, ks, sc)
    for _ in range(max(1, args.warmup)):
        out, _, kind = cpu_msm_all_cores(sc, bases, threads)
        assert np.array_equal(out, want), "reference MSM differs from (sum s_i k_i) G"
    times = []
    for _ in range(args.steps):
        out, t, kind = cpu_msm_all_cores(sc, bases, threads)
        times.append(t)
    assert np.array_equal(out, want)
    v = n / statistics.mean(times)
    single = None
    if args.single_thread_ref:
        out1, t1, _ = cpu_msm_all_cores(sc, bases, 1)
        assert np.array_equal(out1, want)
        single = {"seconds": t1, "points_per_s": n / t1,
                  "note": "one single-thread run of the whole 2^%d MSM (the reference as shipped), once" % args.log_n}
    what = "bn128_G1_proj_MSM_mont_coeff_proj_out (oracle/_ref, reference C)" if kind == "reference" else "oracle port"
    sample = ("per step: the whole 2^%d-point workload, one contiguous point range per host thread (%d) summed "
              "by the reference's %s, partials added with bn128_G1_proj_add, bn128_G1_proj_to_affine; result "
              "checked against (sum s_i k_i) G" % (args.log_n, threads, what))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64 limbs (exact integer, reference C)",
        "data": "synthetic: seeded k*G bases, uniform Fr Montgomery scalars",
        "config": {"workload": "BN254 G1 MSM n=2^%d, Montgomery scalars, affine out" % args.log_n,
                   "n_points": n, "host_threads": threads},
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "single_thread": single,
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- our arm

def gpu_uuid(torch, dev):
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def max_over_ranks(torch, dist, world, value, device="cuda"):
    """The largest of one float per rank: a multi-GPU job is as slow as its slowest rank."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms_max):
    """Units per second of the whole job: every rank processes units_per_rank in ms_max."""
    return world * units_per_rank / (ms_max * 1e-3)


def run_msm(args, zk, L, torch, stream, rank, world, dist, imad_peak, fp64_peak):
    n = 1 << args.log_n
    seed = 0x5eed0001 + 1000 * rank
    # inputs: bases P_i = k_i G (generated on the device), Montgomery scalars
    ks = Z.rand_fr(Z.BN254, n, seed)
    sc = Z.rand_fr(Z.BN254, n, seed + 1)
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((n, 8), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(Z.BN254, n, d_k, d_b)
    del d_k
    d_s = torch.from_numpy(sc.view(np.int64)).cuda()
    torch.cuda.synchronize()

    # the autotuner picks this size's window width, chunk length, running-sum group and prefetch
    # depth on the device (results never depend on them; the identity check below still holds)
    if not args.no_tune:
        zk.autotune_msm(Z.BN254, d_b, n, args.log_n, args.log_n)
    tc = [ctypes.c_int() for _ in range(4)]
    L.zkg_msm_tuned_config(Z.BN254, args.log_n, *[ctypes.byref(x) for x in tc])
    tuned = {"c": tc[0].value, "chunk_len": tc[1].value, "group": tc[2].value, "prefetch": tc[3].value}

    def step():
        return zk.msm_device(Z.BN254, n, d_s, d_b, mont=True, kind=zk.OUT_AFFINE)

    for _ in range(max(3, args.warmup)):
        ref_out = step()
    want = Z.msm_identity_affine(Z.BN254, ks, sc)
    assert np.array_equal(ref_out, want), "MSM result differs from (sum s_i k_i) G"
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(gpu_uuid(torch, torch.cuda.current_device()))
    clk.start()
    time.sleep(0.3)
    l0 = L.zkg_kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    phases = np.zeros(4)
    ph = (ctypes.c_float * 4)()
    clk.mark_begin()
    ev0.record(stream)
    for _ in range(args.steps):
        out = step()
        L.zkg_last_phase_ms(ph, 4)
        phases += np.array(ph[:4])
        assert np.array_equal(out, ref_out), "MSM result changed between steps"
    ev1.record(stream)
    torch.cuda.synchronize()
    clk.mark_end()
    launches = L.zkg_kernel_launches() - l0
    clocks = clk.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = max_over_ranks(torch, dist, world, ms)
    c, nwin, adds = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint64()
    L.zkg_msm_last_info(ctypes.byref(c), ctypes.byref(nwin), ctypes.byref(adds))

    # e2e through the drop-in C ABI (host buffers, pinned)
    h_s = torch.from_numpy(sc.view(np.int64)).pin_memory()
    h_b = d_b.cpu().pin_memory()
    h_out = np.zeros(8, np.uint64)
    fn = L.bn128_G1_proj_MSM_mont_coeff_affine_out
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    for _ in range(2):
        fn(n, ctypes.c_void_p(h_s.data_ptr()), ctypes.c_void_p(h_b.data_ptr()), Z.ptr(h_out), 4)
    assert np.array_equal(h_out, ref_out), "drop-in C ABI result differs from the device path"
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        fn(n, ctypes.c_void_p(h_s.data_ptr()), ctypes.c_void_p(h_b.data_ptr()), Z.ptr(h_out), 4)
    e1.record(stream)
    torch.cuda.synchronize()
    wall_e2e = (time.perf_counter() - w0) / args.steps
    e2e_ms = e0.elapsed_time(e1) / args.steps
    e2e_ms = max_over_ranks(torch, dist, world, e2e_ms)
    # the same call from pageable host arrays (what a Haskell caller passes), wall clock
    p_s, p_b = h_s.numpy().view(np.uint64).copy(), h_b.numpy().view(np.uint64).copy()
    fn(n, Z.ptr(p_s), Z.ptr(p_b), Z.ptr(h_out), 4)
    assert np.array_equal(h_out, ref_out), "drop-in result from pageable buffers differs"
    w0 = time.perf_counter()
    for _ in range(max(2, args.steps // 2)):
        fn(n, Z.ptr(p_s), Z.ptr(p_b), Z.ptr(h_out), 4)
    wall_pageable = (time.perf_counter() - w0) / max(2, args.steps // 2)
    del p_s, p_b

    # the reference C on the host cores, same inputs (rank 0, one GPU): a bounded sample of one
    # whole 2^22 MSM split over all host threads
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = len(os.sched_getaffinity(0))
        cpu_out, cpu_s, kind = cpu_msm_all_cores(sc, h_b.numpy().view(np.uint64), threads)
        assert np.array_equal(cpu_out, ref_out), "reference C result differs from the GPU result"
        cpu = {"value": n / cpu_s, "unit": "points/s", "cores": threads, "kind": kind,
               "sample": "one whole 2^%d MSM on the same inputs, one contiguous point range per host thread "
                         "through the reference's bn128_G1_proj_MSM_mont_coeff_proj_out, partials added with "
                         "bn128_G1_proj_add; result equal to the GPU's" % args.log_n}

    # roofline of the bucket-accumulation kernel
    accum_ms = phases[1] / args.steps
    accum_imad = float(adds.value) * IMAD_PER_MADD
    accum_fp64 = float(adds.value) * FP64_PER_MADD
    achieved = accum_fp64 / (accum_ms * 1e-3)
    # DRAM traffic of one k_msm_accum launch at this workload, from an ncu capture
    # (dram__bytes_read.sum + dram__bytes_write.sum); None for other sizes
    traffic = ACCUM_DRAM_BYTES.get(args.log_n)
    # the same launch against the measured throughput of the field product it is made of (10 per
    # mixed addition: 8 multiplications + 2 squarings, each one product call)
    L.zkg_product_probe.argtypes = [ctypes.c_int]
    L.zkg_product_probe.restype = ctypes.c_double
    prod_peak = L.zkg_product_probe(Z.BN254)
    prod_rate = float(adds.value) * 10 / (accum_ms * 1e-3)
    return {
        "tuned": tuned,
        "cpu_baseline": cpu,
        "n": n, "ms_max": ms_max, "value": whole_job_rate(n, world, ms_max), "c": c.value, "nwin": nwin.value,
        "e2e": {"value": whole_job_rate(n, world, e2e_ms), "unit": "points/s",
                "h2d_bytes_per_step": n * 32 + n * 64, "d2h_bytes_per_step": 64,
                "wall_ms_per_step": 1e3 * wall_e2e, "device_ms_per_step": e2e_ms,
                "pageable_host_buffers_wall_ms_per_step": 1e3 * wall_pageable},
        "roofline": {"kernel": "k_msm_accum_w<BN254E, 384, 2> (bucket mixed additions, exact-radix FP64-pipe field products)",
                     "bound": "fp64",
                     "achieved": achieved / 1e12, "peak": fp64_peak / 1e12, "unit": "T FP64 ops/s",
                     "frac": achieved / fp64_peak if fp64_peak > 0 else None,
                     "traffic": traffic, "launch_ms": accum_ms, "mixed_additions": int(adds.value),
                     "algorithmic_fp64_ops_per_launch": accum_fp64,
                     "peak_source": "measured: zkg_pipe_probe fma.rn.f64 (independent FMA chains on all SMs, this GPU)",
                     "convention": "8 Montgomery multiplications + 2 squarings per XYZZ mixed addition; a "
                                   "multiplication is 50 limb products of 52 x 52 bits (5 limbs), a squaring 40, each "
                                   "split exactly into high and low halves by 2 FMAs and 1 DADD = 150 / 120 FP64-pipe "
                                   "operations (carry handling, the digits m_i and the curve formulas' additions run "
                                   "on the integer ALU and are not counted)",
                     "product_ceiling": {"achieved": prod_rate / 1e9, "peak": prod_peak / 1e9, "unit": "G Fp products/s",
                                         "frac": prod_rate / prod_peak if prod_peak > 0 else None,
                                         "convention": "10 field products per mixed addition against zkg_product_probe "
                                                       "(the same exact-radix FP64 product in independent chains on "
                                                       "all SMs, this GPU)"},
                     "imad_equivalent": {"achieved": accum_imad / (accum_ms * 1e-3) / 1e12, "peak": imad_peak / 1e12,
                                         "unit": "TIMAD/s",
                                         "frac": accum_imad / (accum_ms * 1e-3) / imad_peak if imad_peak > 0 else None,
                                         "convention": "the same additions counted as 264 IMAD per product "
                                                       "(8x32-bit CIOS, 4w^2+w), against the measured mad.lo.u32 rate"}},
        "phases_ms": {"sort": phases[0] / args.steps, "accumulate": accum_ms,
                      "fold_levels": phases[2] / args.steps, "bucket_reduce": phases[3] / args.steps},
        "clocks": clocks, "gpu_launches": int(launches),
    }


def run_ntt(args, zk, torch, stream, seed, imad_peak, fp64_peak):
    m = args.ntt_m
    N = 1 << m
    x = torch.from_numpy(Z.rand_fr(Z.BN254, N, seed + 7).view(np.int64)).cuda()
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    for _ in range(2):
        zk.ntt_device(Z.BN254, m, x, y, inverse=False)
        zk.ntt_device(Z.BN254, m, y, z, inverse=True)
    torch.cuda.synchronize()
    assert torch.equal(z, x), "NTT round trip failed"
    f0, f1, f2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    reps = max(3, args.steps)
    f0.record(stream)
    for _ in range(reps):
        zk.ntt_device(Z.BN254, m, x, y, inverse=False)
    f1.record(stream)
    for _ in range(reps):
        zk.ntt_device(Z.BN254, m, y, z, inverse=True)
    f2.record(stream)
    torch.cuda.synchronize()
    fwd_ms, inv_ms = f0.elapsed_time(f1) / reps, f1.elapsed_time(f2) / reps
    alg_bytes = 2 * 32 * N   # one read and one write of the vector
    imad = (N // 2) * m * IMAD_PER_NTT_BFLY
    return {"m": m, "fwd_ms": fwd_ms, "inv_ms": inv_ms,
            "fwd_gbs_algorithmic": alg_bytes / (fwd_ms * 1e-3) / 1e9,
            "hbm_frac": alg_bytes / (fwd_ms * 1e-3) / 1e9 / hbm_peak()[0], "hbm_peak_source": hbm_peak()[1],
            "imad_equivalent_frac": imad / (fwd_ms * 1e-3) / imad_peak if imad_peak > 0 else None,
            "fp64_frac": (N // 2) * m * FP64_PER_PRODUCT / (fwd_ms * 1e-3) / fp64_peak if fp64_peak > 0 else None,
            "bound": "field products (FP64 pipe + integer ALU); HBM fraction reported as asked"}


def device_bases(zk, torch, curve, n, seed):
    ks = Z.rand_fr(curve, n, seed)
    d_k = torch.from_numpy(ks.view(np.int64)).cuda()
    d_b = torch.empty((n, 2 * Z.NLP[curve]), dtype=torch.int64, device="cuda")
    zk.g1_gen_mul_device(curve, n, d_k, d_b)
    torch.cuda.synchronize()
    return d_b


def time_msm_device(zk, torch, stream, curve, n, d_s, d_b, reps):
    out = zk.msm_device(curve, n, d_s, d_b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        assert np.array_equal(zk.msm_device(curve, n, d_s, d_b), out)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, out


def run_small_bn(args, zk, torch, stream):
    """configuration 1: plain BN254 MSM at 2^16 (device-resident and through the C ABI)"""
    n = 1 << 16
    d_b = device_bases(zk, torch, Z.BN254, n, 0x5eed0101)
    sc = Z.rand_fr(Z.BN254, n, 0x5eed0102)
    d_s = torch.from_numpy(sc.view(np.int64)).cuda()
    ms, out = time_msm_device(zk, torch, stream, Z.BN254, n, d_s, d_b, max(5, args.steps))
    bh = d_b.cpu().numpy().view(np.uint64)
    t0 = time.perf_counter()
    reps = max(5, args.steps)
    for _ in range(reps):
        assert np.array_equal(zk.msm_affine(Z.BN254, sc, bh), out)
    e2e = (time.perf_counter() - t0) / reps
    return {"n": n, "device_ms": ms, "points_per_s": n / (ms * 1e-3), "e2e_wall_ms": 1e3 * e2e,
            "e2e_points_per_s": n / e2e}


def run_bls(args, zk, L, torch, stream):
    """configuration 3: BLS12-381 MSM at 2^22, autotuned window vs fixed c = 16"""
    n = 1 << 22
    d_b = device_bases(zk, torch, Z.BLS12_381, n, 0x5eed0201)
    sc = Z.rand_fr(Z.BLS12_381, n, 0x5eed0202)
    d_s = torch.from_numpy(sc.view(np.int64)).cuda()
    want = Z.msm_identity_affine(Z.BLS12_381, Z.rand_fr(Z.BLS12_381, n, 0x5eed0201), sc)
    tuned = None if args.no_tune else zk.autotune_msm(Z.BLS12_381, d_b, n, 22, 22)[22]
    reps = max(3, args.steps // 2)
    ms_t, out_t = time_msm_device(zk, torch, stream, Z.BLS12_381, n, d_s, d_b, reps)
    prev = L.zkg_set_msm_window(16)
    ms_f, out_f = time_msm_device(zk, torch, stream, Z.BLS12_381, n, d_s, d_b, reps)
    L.zkg_set_msm_window(prev)
    assert np.array_equal(out_t, want), "autotuned BLS12-381 MSM differs from (sum s_i k_i) G"
    assert np.array_equal(out_f, want), "fixed c = 16 BLS12-381 MSM differs from (sum s_i k_i) G"
    del d_b, d_s
    return {"n": n, "tuned_c": tuned, "tuned_ms": ms_t, "tuned_points_per_s": n / (ms_t * 1e-3),
            "fixed_c16_ms": ms_f, "fixed_c16_points_per_s": n / (ms_f * 1e-3),
            "both_equal_sum_s_k_G": True}


def run_batched(args, zk, L, torch, stream):
    """configuration 4: 64 MSMs (n = floor(2^U), U ~ U[10, 20]) against one resident 2^20 base set
    and 64 NTTs (m uniform in 12..22, half inverse) as one captured graph, vs the per-call path"""
    rng = np.random.default_rng(0x5eed0301)
    nb = 1 << 20
    d_b = device_bases(zk, torch, Z.BN254, nb, 0x5eed0302)
    zk.autotune_msm(Z.BN254, d_b, nb, 10, 20)
    zk.autotune_ntt(Z.BN254, 12, 22)
    B = zk.Bases(Z.BN254, d_b, nb, on_device=True)   # resident: uploaded once, not per run
    b = zk.Batch(Z.BN254, B)
    msms, ntts = [], []
    for i in range(64):
        n = int(2 ** rng.uniform(10, 20))
        s = torch.from_numpy(Z.rand_fr(Z.BN254, n, 0x5eed0400 + i).view(np.int64)).cuda()
        msms.append((n, s, b.add_msm(n, s)))
    for i in range(64):
        m = int(rng.integers(12, 23))
        x = torch.from_numpy(Z.rand_fr(Z.BN254, 1 << m, 0x5eed0500 + i).view(np.int64)).cuda()
        y = torch.empty_like(x)
        b.add_ntt(m, x, y, inverse=bool(i % 2))
        ntts.append((m, x, y, bool(i % 2)))
    torch.cuda.synchronize()
    b.run()   # plan, capture, first replay
    reps = max(3, args.steps // 2)
    w0 = time.perf_counter()
    dev = [b.run() for _ in range(reps)]
    batched_s = (time.perf_counter() - w0) / reps
    batched_out = [o.copy() for _, _, o in msms]
    ntt_out = [y.clone() for _, _, y, _ in ntts]
    # the same batch in the library's other form: one persistent kernel draining a work queue of
    # accumulation blocks and NTT pass tiles (mode 1)
    def other_form(mode):
        b2 = zk.Batch(Z.BN254, B, persistent=mode)
        outs2 = [b2.add_msm(n, s) for n, s, _ in msms]
        y2 = [torch.empty_like(x) for _, x, _, _ in ntts]
        for (m, x, _, inv), yy in zip(ntts, y2):
            b2.add_ntt(m, x, yy, inverse=inv)
        b2.run()
        w0 = time.perf_counter()
        dev2 = [b2.run() for _ in range(reps)]
        wall = (time.perf_counter() - w0) / reps
        assert all(np.array_equal(o2, o) for o2, o in zip(outs2, batched_out)), "batch form %d differs" % mode
        assert all(torch.equal(a2, a) for a2, a in zip(y2, ntt_out)), "batch form %d NTT differs" % mode
        info = b2.persistent_info()
        b2.close()
        return wall, float(np.median(dev2)), info
    pers_s, pers_dev, (persistent, grid, tasks) = other_form(1)
    # per-call path: the same 128 requests one at a time; one untimed pass first (module loading,
    # plan and workspace growth), then the timed pass
    z = [torch.empty_like(x) for _, x, _, _ in ntts]

    def per_call(check):
        for (n, s, _), bo in zip(msms, batched_out):
            o = zk.msm_device(Z.BN254, n, s, d_b)
            if check:
                assert np.array_equal(o, bo), "batched MSM differs from per-call"
        for (m, x, _, inv), zz in zip(ntts, z):
            zk.ntt_device(Z.BN254, m, x, zz, inverse=inv)
        torch.cuda.synchronize()

    per_call(True)
    w0 = time.perf_counter()
    per_call(False)
    percall_s = time.perf_counter() - w0
    for zz, yo in zip(z, ntt_out):
        assert torch.equal(zz, yo), "batched NTT differs from per-call"

    # per-call with the bases resident (no per-call base handling): what batching itself buys
    def per_call_resident(check):
        for (n, s, _), bo in zip(msms, batched_out):
            o = B.msm(n, s)
            if check:
                assert np.array_equal(o, bo), "batched MSM differs from resident per-call"
        for (m, x, _, inv), zz in zip(ntts, z):
            zk.ntt_device(Z.BN254, m, x, zz, inverse=inv)
        torch.cuda.synchronize()

    per_call_resident(True)
    w0 = time.perf_counter()
    per_call_resident(False)
    percall_res_s = time.perf_counter() - w0
    pts = sum(n for n, _, _ in msms)
    els = sum(1 << m for m, _, _, _ in ntts)
    b.close()
    B.close()
    out = {"requests": 128, "msm_points": pts, "ntt_elements": els,
           "batched_req_per_s": 128 / batched_s, "batched_wall_ms": 1e3 * batched_s,
           "batched_graph_device_ms": float(np.median(dev)),
           "per_call_req_per_s": 128 / percall_s, "per_call_wall_ms": 1e3 * percall_s,
           "per_call_resident_req_per_s": 128 / percall_res_s,
           "speedup": percall_s / batched_s, "speedup_vs_resident_per_call": percall_res_s / batched_s,
           "persistent_kernel": {"used": persistent, "grid": grid, "tasks": tasks},
           "batched_form": "graph branches (NTTs on parallel streams beside the MSM pipeline)",
           "persistent_kernel_req_per_s": 128 / pers_s, "persistent_kernel_device_ms": pers_dev,
           "results_equal_per_call": True}
    # the reference C on the host, all cores: the same 128 requests from one queue (one request
    # per core at a time), each result compared with the batched one
    fns = _ref_fns()
    if fns is not None:
        rmsm, rfwd, rinv = fns
        threads = len(os.sched_getaffinity(0))
        bh = d_b.cpu().numpy().view(np.uint64)
        jobs = []
        for (n, s, _), bo in zip(msms, batched_out):
            sh = s.cpu().numpy().view(np.uint64)

            def job(n=n, sh=sh, bo=bo):
                o = np.zeros(8, np.uint64)
                rmsm(n, Z.ptr(sh), Z.ptr(bh), Z.ptr(o), 4)
                assert np.array_equal(o, bo), "reference MSM differs from the batched result"
            jobs.append((n * 20.0, job))
        for (m, x, _, inv), yo in zip(ntts, ntt_out):
            xh = x.cpu().numpy().view(np.uint64)
            yh = yo.cpu().numpy().view(np.uint64)
            g = zk.fft_subgroup(Z.BN254, m)

            def job(m=m, xh=xh, yh=yh, g=g, inv=inv):
                o = np.zeros_like(xh)
                (rinv if inv else rfwd)(m, Z.ptr(g), Z.ptr(xh), Z.ptr(o))
                assert np.array_equal(o, yh), "reference NTT differs from the batched result"
            jobs.append(((1 << m) * m / 2.0, job))
        wall, _ = cpu_pool(jobs, threads)
        out["cpu_baseline"] = {"value": 128 / wall, "unit": "req/s", "cores": threads, "kind": "reference",
                               "sample": "the same 128 requests on the reference C (oracle/_ref), one request "
                                         "per host thread at a time from a shared queue, results compared"}
    return out


def run_served(args, zk, L, torch, stream):
    """configuration 5: KZG commits (iNTT of 2^k values, k uniform in 12..22, then MSM against a
    resident 2^24-point base set) with Poisson arrivals, vs the per-call C ABI path"""
    nb = 1 << 24
    d_b = device_bases(zk, torch, Z.BN254, nb, 0x5eed0601)
    rng = np.random.default_rng(0x5eed0602)
    nreq = 192
    ks = [int(rng.integers(12, 23)) for _ in range(nreq)]
    vals = {k: torch.from_numpy(Z.rand_fr(Z.BN254, 1 << k, 0x5eed0700 + k).view(np.int64)).pin_memory()
            for k in sorted(set(ks))}
    budget = 24 << 30
    srv = zk.Server(Z.BN254, d_b, nb, 12, 22, budget, 8)
    # capacity: closed loop with everything submitted at once
    for k in sorted(set(ks)):
        srv.wait(srv.submit(k, vals[k]))
    t0 = time.perf_counter()
    tk = [srv.submit(k, vals[k]) for k in ks]
    outs = [srv.wait(t) for t in tk]
    cap = nreq / (time.perf_counter() - t0)
    ref = {k: None for k in set(ks)}
    for k, (o, _) in zip(ks, outs):
        ref[k] = o if ref[k] is None else ref[k]
        assert np.array_equal(o, ref[k])
    # open loop: Poisson arrivals at 80% of capacity
    lam = 0.8 * cap
    gaps = rng.exponential(1.0 / lam, nreq)
    t0 = time.perf_counter()
    tk = []
    for k, g in zip(ks, gaps):
        time.sleep(g)
        tk.append(srv.submit(k, vals[k]))
    lat = []
    for k, t in zip(ks, tk):
        o, ms = srv.wait(t)
        assert np.array_equal(o, ref[k]), "served commit changed between runs"
        lat.append(ms)
    served_s = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    # per-call path: iNTT and MSM through the host-buffer C ABI, one request at a time
    bh = d_b[: 1 << 22].cpu().numpy().view(np.uint64)
    t0 = time.perf_counter()
    for k in ks:
        coef = zk.inverse_ntt(Z.BN254, k, vals[k].numpy().view(np.uint64).reshape(-1, 4))
        o = zk.msm_affine(Z.BN254, coef, bh[: 1 << k], mont=True)
        assert np.array_equal(o, ref[k]), "served commit differs from per-call"
    percall = nreq / (time.perf_counter() - t0)
    # per-call path with the bases resident on the device (what continuous batching is compared
    # with): copy the values in, inverse NTT and MSM on device buffers, one request at a time
    d_vals = torch.empty(((1 << 22), 4), dtype=torch.int64, device="cuda")
    d_coef = torch.empty_like(d_vals)
    def resident_call(k):
        N = 1 << k
        d_vals[:N].copy_(vals[k].view(N, 4), non_blocking=True)
        zk.ntt_device(Z.BN254, k, d_vals[:N], d_coef[:N], inverse=True)
        return zk.msm_device(Z.BN254, N, d_coef[:N], d_b, mont=True)
    for k in sorted(set(ks)):
        assert np.array_equal(resident_call(k), ref[k]), "resident per-call commit differs from served"
    t0 = time.perf_counter()
    for k in ks:
        resident_call(k)
    percall_resident = nreq / (time.perf_counter() - t0)
    del d_vals, d_coef
    out = {"requests": nreq, "per_call_resident_commits_per_s": percall_resident, "resident_bases": nb, "hbm_budget_bytes": budget, "slots": 8,
           "poisson_rate_per_s": lam, "commits_per_s": nreq / served_s, "capacity_commits_per_s": cap,
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "max_inflight": st["max_inflight"], "peak_bytes": st["peak_bytes"],
           "per_call_commits_per_s": percall, "results_equal_per_call": True}
    # the reference C on the host: one commit (reference iNTT, then reference MSM) for every k in
    # 12..22 on its own thread, each compared with the served result; k is uniform, so the
    # reference's aggregate rate with one commit per core is cores / mean commit time
    fns = _ref_fns()
    if fns is not None:
        rmsm, _, rinv = fns
        threads = len(os.sched_getaffinity(0))
        kset = list(range(12, 23))
        jobs = []
        for k in kset:
            vh = (vals[k].numpy() if k in vals else Z.rand_fr(Z.BN254, 1 << k, 0x5eed0700 + k)).view(np.uint64)
            g = zk.fft_subgroup(Z.BN254, k)

            def job(k=k, vh=vh, g=g):
                coef = np.zeros_like(vh)
                rinv(k, Z.ptr(g), Z.ptr(vh), Z.ptr(coef))
                o = np.zeros(8, np.uint64)
                rmsm(1 << k, Z.ptr(coef), Z.ptr(bh), Z.ptr(o), 4)
                if k in ref:
                    assert np.array_equal(o, ref[k]), "reference commit differs from the served result"
            jobs.append((float(1 << k), job))
        _, times = cpu_pool(jobs, min(threads, len(jobs)))
        mean_t = float(np.mean(times))
        out["cpu_baseline"] = {"value": threads / mean_t, "unit": "commits/s", "cores": threads,
                               "kind": "reference", "mean_commit_s": mean_t,
                               "commit_s_by_k": {str(k): t for k, t in zip(kset, times)},
                               "sample": "one commit per k in 12..22 on the reference C (oracle/_ref), each on "
                                         "its own host thread, results compared; rate = cores / mean time"}
    return out


def cpu_pool(jobs, threads):
    """Runs jobs [(cost, fn)] on `threads` host threads from one shared queue, largest cost first
    (the reference C is single-threaded and releases the GIL inside ctypes calls). Returns the wall
    seconds and each job's seconds (in the given order)."""
    order = sorted(range(len(jobs)), key=lambda i: -jobs[i][0])
    times = [0.0] * len(jobs)
    lock = threading.Lock()
    nxt = [0]

    def worker():
        while True:
            with lock:
                if nxt[0] >= len(order):
                    return
                i = order[nxt[0]]
                nxt[0] += 1
            t = time.perf_counter()
            jobs[i][1]()
            times[i] = time.perf_counter() - t

    ths = [threading.Thread(target=worker) for _ in range(threads)]
    t0 = time.perf_counter()
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return time.perf_counter() - t0, times


def _ref_fns():
    ref = Z.reference()
    if ref is None:
        return None
    msm = ref.bn128_G1_proj_MSM_mont_coeff_affine_out
    msm.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    fwd, inv = ref.bn128_poly_mont_ntt_forward, ref.bn128_poly_mont_ntt_inverse
    fwd.argtypes = inv.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return msm, fwd, inv


def _cpu_timed(fn, reps=1):
    fn()   # warm-up
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    return (time.perf_counter() - t0) / reps


def run_next_rows(args, zk, L, torch, stream):
    """the widened rows, each against the reference's own C on the host (one thread, as the
    reference runs): G1 group FFT, binary multi-MSM, Fr vector operations"""
    ref = Z.reference()
    kind = "reference" if ref is not None else "port"
    out = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nl = 4
    one = Z.to_limbs((1 << 256) % Z.P[Z.BN254], nl)

    def proj_points(m, seed):
        n = 1 << m
        d_b = device_bases(zk, torch, Z.BN254, n, seed)
        d_p = torch.zeros((n, 3 * nl), dtype=torch.int64, device="cuda")
        d_p[:, :2 * nl] = d_b
        d_p[:, 2 * nl:] = torch.from_numpy(one.view(np.int64)).cuda()
        return d_p

    # --- G1 group FFT, BN254, m = 16 (device) and m = 8 (reference CPU sample)
    m = 16
    d_p = proj_points(m, 0x5eed0401)
    d_o = torch.empty_like(d_p)
    res = {}
    outs = {}
    for inv in (False, True):
        zk.g1_fft_device(Z.BN254, m, d_p, d_o, inverse=inv)
        e0.record(stream)
        zk.g1_fft_device(Z.BN254, m, d_p, d_o, inverse=inv)
        e1.record(stream)
        torch.cuda.synchronize()
        res["inverse_ms" if inv else "forward_ms"] = e0.elapsed_time(e1)
        outs[inv] = d_o.cpu().numpy().view(np.uint64).copy()
    hp = d_p.cpu().numpy().view(np.uint64)
    t0 = time.perf_counter()
    fwd = zk.forward_fft(Z.BN254, m, hp)
    res["forward_host_api_ms"] = 1e3 * (time.perf_counter() - t0)
    assert np.array_equal(fwd, outs[False])
    # inverse(forward(x)) == x (inputs are normalised, Z = 1)
    d_f = torch.from_numpy(fwd.view(np.int64)).cuda()
    zk.g1_fft_device(Z.BN254, m, d_f, d_o, inverse=True)
    torch.cuda.synchronize()
    assert np.array_equal(d_o.cpu().numpy().view(np.uint64), hp)
    bfly = m * (1 << m) // 2
    res["butterflies_per_s"] = bfly / (res["forward_ms"] * 1e-3)
    ms_cpu = 8
    small = d_p[: 1 << ms_cpu].cpu().numpy().view(np.uint64).copy()
    gen = np.ascontiguousarray(Z.fft_gen(Z.BN254, ms_cpu))
    tgt = np.zeros_like(small)
    if ref is not None:
        f = ref.bn128_G1_proj_fft_forward
        t = _cpu_timed(lambda: f(ctypes.c_int(ms_cpu), Z.ptr(gen), Z.ptr(small), Z.ptr(tgt)))
    else:
        t = _cpu_timed(lambda: Z.oracle_g1_fft(Z.BN254, 0, ms_cpu, gen, small, 0))
    res["cpu_baseline"] = {"butterflies_per_s": ms_cpu * (1 << ms_cpu) // 2 / t, "cores": 1, "kind": kind,
                           "sample": "bn128_G1_proj_fft_forward at m = %d" % ms_cpu}
    res["m"] = m
    out["g1_fft_bn254"] = res
    del d_p, d_o

    # --- binary multi-MSM, BN254, 64 rows x 2^18 points (device + host API); reference 64 x 2^12
    nrows, npts = 64, 1 << 18
    d_b = device_bases(zk, torch, Z.BN254, npts, 0x5eed0402)
    co = (Z.splitmix64(0x5eed0403, nrows * npts) & np.uint64(1)).astype(np.uint8).reshape(nrows, npts)
    d_co = torch.from_numpy(co).cuda()
    d_out = torch.empty((nrows, 2 * nl), dtype=torch.int64, device="cuda")
    zk.msm_binary_device(Z.BN254, nrows, npts, d_co, npts, d_b, d_out)
    e0.record(stream)
    zk.msm_binary_device(Z.BN254, nrows, npts, d_co, npts, d_b, d_out)
    e1.record(stream)
    torch.cuda.synchronize()
    dev_ms = e0.elapsed_time(e1)
    bh = d_b.cpu().numpy().view(np.uint64)
    zk.binary_multi_msm(Z.BN254, co, bh, affine=True)
    t0 = time.perf_counter()
    got = zk.binary_multi_msm(Z.BN254, co, bh, affine=True)
    host_ms = 1e3 * (time.perf_counter() - t0)
    assert np.array_equal(got, d_out.cpu().numpy().view(np.uint64))
    npc = 1 << 12
    cs = np.ascontiguousarray(co[:, :npc])
    bs = np.ascontiguousarray(bh[:npc])
    tgt = np.zeros((nrows, 2 * nl), np.uint64)
    if ref is not None:
        f = ref.bn128_G1_proj_multi_MSM_binary_coeff_affine_out
        rp = Z.row_pointers(cs)
        t = _cpu_timed(lambda: f(ctypes.c_int(nrows), ctypes.c_int(npc), rp, Z.ptr(bs), Z.ptr(tgt)))
    else:
        t = _cpu_timed(lambda: Z.oracle_msm_binary(Z.BN254, cs, bs))
    out["binary_multi_msm_bn254"] = {
        "rows": nrows, "points": npts, "device_ms": dev_ms, "host_api_ms": host_ms,
        "row_points_per_s": nrows * npts / (dev_ms * 1e-3),
        "cpu_baseline": {"row_points_per_s": nrows * npc / t, "cores": 1, "kind": kind,
                         "sample": "bn128_G1_proj_multi_MSM_binary_coeff_affine_out, %d rows x %d points" % (nrows, npc)}}
    del d_b, d_co, d_out

    # --- Fr vector operations, BN254, 2^22 elements (device + host API); reference at 2^20
    n = 1 << 22
    a, b = Z.rand_fr(Z.BN254, n, 0x5eed0404), Z.rand_fr(Z.BN254, n, 0x5eed0405)
    d_a = torch.from_numpy(a.view(np.int64)).cuda()
    d_bb = torch.from_numpy(b.view(np.int64)).cuda()
    d_o = torch.empty_like(d_a)
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    fr = {}
    hbm, _ = hbm_peak()
    for name, op, bytes_per in (("mul", 6, 96), ("inv", 7, 64)):
        for _ in range(3):
            assert L.zkg_fr_map_device(Z.BN254, op, n, P(d_a), P(d_bb), None, None, None, P(d_o)) == 0
        # kernel time: the library's events around its launches (best of 10 calls); call time:
        # CUDA events around 10 whole device-pointer calls on the stream (host overhead included)
        kern = []
        e0.record(stream)
        for _ in range(10):
            assert L.zkg_fr_map_device(Z.BN254, op, n, P(d_a), P(d_bb), None, None, None, P(d_o)) == 0
            kern.append(L.zkg_last_kernel_ms())
        e1.record(stream)
        torch.cuda.synchronize()
        call_ms = e0.elapsed_time(e1) / 10
        ms = float(np.median(kern))
        ho = np.zeros_like(a)
        t0 = time.perf_counter()
        assert L.zkg_fr_map(Z.BN254, op, n, Z.ptr(a), Z.ptr(b), None, None, None, Z.ptr(ho)) == 0
        host_ms = 1e3 * (time.perf_counter() - t0)
        assert np.array_equal(ho, d_o.cpu().numpy().view(np.uint64))
        nc = 1 << 20
        ac, bc, oc = np.ascontiguousarray(a[:nc]), np.ascontiguousarray(b[:nc]), np.zeros((nc, 4), np.uint64)
        if ref is not None:
            if op == 6:
                t = _cpu_timed(lambda: ref.bn128_arr_mont_mul(ctypes.c_int(nc), Z.ptr(ac), Z.ptr(bc), Z.ptr(oc)))
            else:
                t = _cpu_timed(lambda: ref.bn128_arr_mont_inv(ctypes.c_int(nc), Z.ptr(ac), Z.ptr(oc)))
        else:
            t = _cpu_timed(lambda: Z.oracle_fr_op(Z.BN254, op, ac, bc))
        fr[name] = {"n": n, "device_ms": ms, "device_call_ms": call_ms, "elements_per_s": n / (ms * 1e-3),
                    "hbm_frac_of_measured": (bytes_per * n / (ms * 1e-3)) / (hbm * 1e9), "host_api_ms": host_ms,
                    "cpu_baseline": {"elements_per_s": nc / t, "cores": 1, "kind": kind,
                                     "sample": "bn128_arr_mont_%s at 2^20" % name}}
    out["fr_vector_ops_bn254"] = fr
    return out


def our_arm(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    zk = Z.load_package()
    L = zk.lib()
    L.zkg_set_stream.argtypes = [ctypes.c_void_p]
    L.zkg_last_phase_ms.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.zkg_imad_probe.restype = ctypes.c_double
    L.zkg_msm_last_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    stream = torch.cuda.current_stream()
    L.zkg_set_stream(ctypes.c_void_p(stream.cuda_stream))
    imad_peak = L.zkg_imad_probe()
    L.zkg_pipe_probe.argtypes = [ctypes.c_int]
    L.zkg_pipe_probe.restype = ctypes.c_double
    pipes = {k: L.zkg_pipe_probe(i) / 1e12 for i, k in enumerate(("mad.lo.u32", "mad.hi.u32", "mad.wide.u32", "fma.rn.f64"))}

    fp64_peak = pipes["fma.rn.f64"] * 1e12
    if args.config3_only:
        args.no_msm = args.no_ntt = args.no_extra = True
    msm = None if args.no_msm else run_msm(args, zk, L, torch, stream, rank, world, dist, imad_peak, fp64_peak)
    ntt = None if args.no_ntt else run_ntt(args, zk, torch, stream, 0x5eed0001 + 1000 * rank, imad_peak, fp64_peak)
    extra = {}
    if args.config3_only and world == 1:
        extra["config3_bls12_381_2p22"] = run_bls(args, zk, L, torch, stream)
    if not args.no_extra and not args.no_msm and world == 1:
        extra["config1_bn254_2p16"] = run_small_bn(args, zk, torch, stream)
        extra["config3_bls12_381_2p22"] = run_bls(args, zk, L, torch, stream)
        extra["config4_batched"] = run_batched(args, zk, L, torch, stream)
        extra["config5_served"] = run_served(args, zk, L, torch, stream)
        extra["next_rows"] = run_next_rows(args, zk, L, torch, stream)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    line = {"metric": METRIC, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32 words; field products on 52-bit limbs in f64 (exact integer)",
            "data": "synthetic: seeded k*G bases (device-generated), uniform Fr Montgomery scalars"}
    details = {}
    tail = {}
    if msm is not None:
        roof = dict(msm["roofline"])
        imad = roof.pop("imad_equivalent")
        roof["product_ceiling"] = dict(roof["product_ceiling"])
        details["roofline_conventions"] = {"fp64": roof.pop("convention"), "imad": imad.pop("convention"),
                                           "product": roof["product_ceiling"].pop("convention"),
                                           "peak_source": roof.pop("peak_source")}
        line.update({
            "value": msm["value"], "ms_per_step": msm["ms_max"],
            "config": {"workload": "BN254 G1 MSM n=2^%d, Montgomery scalars, affine out "
                                   "(bn128_G1_proj_MSM_mont_coeff_affine_out)" % args.log_n,
                       "n_points": msm["n"], "window_c": msm["c"], "windows": msm["nwin"],
                       "autotuned": msm["tuned"],
                       "parallelism": "replicas x%d" % world,
                       "l2": "inputs 402 MB > 126 MB L2 (no flush needed)"},
            "e2e": msm["e2e"], "roofline": roof, "phases_ms": msm["phases_ms"],
            "cpu_baseline": msm["cpu_baseline"], "clocks": msm["clocks"], "gpu_launches": msm["gpu_launches"],
            "result_check": "equal to (sum s_i k_i mod r) G (numpy / Python integers) and, at N=1, to the "
                            "reference C on the same inputs"})
        tail["imad_equivalent"] = {k: imad[k] for k in ("achieved", "peak", "unit", "frac")}
    # secondary configurations: summary figures on the line, full records in --details
    if "config1_bn254_2p16" in extra:
        c1 = extra["config1_bn254_2p16"]
        line["config1_bn254_2p16"] = {"device_ms": c1["device_ms"], "e2e_wall_ms": c1["e2e_wall_ms"]}
    if "config4_batched" in extra:
        c4 = extra["config4_batched"]
        details["config4_batched"] = c4
        line["config4_batched"] = {k: c4.get(k) for k in ("batched_req_per_s", "per_call_req_per_s",
                                                          "per_call_resident_req_per_s", "speedup",
                                                          "batched_graph_device_ms", "persistent_kernel_req_per_s",
                                                          "results_equal_per_call")}
        if c4.get("cpu_baseline"):
            line["config4_batched"]["reference_cpu_req_per_s"] = c4["cpu_baseline"]["value"]
    if "config5_served" in extra:
        c5 = extra["config5_served"]
        details["config5_served"] = c5
        line["config5_served"] = {k: c5.get(k) for k in ("commits_per_s", "p50_ms", "p99_ms",
                                                         "per_call_commits_per_s",
                                                         "per_call_resident_commits_per_s",
                                                         "capacity_commits_per_s", "poisson_rate_per_s",
                                                         "max_inflight")}
        if c5.get("cpu_baseline"):
            line["config5_served"]["reference_cpu_commits_per_s"] = c5["cpu_baseline"]["value"]
    if "next_rows" in extra:
        details["next_rows"] = extra["next_rows"]
        nr = extra["next_rows"]
        line["next_rows"] = {"g1_fft_2p16_fwd_ms": nr["g1_fft_bn254"]["forward_ms"],
                             "binary_msm_64x2p18_ms": nr["binary_multi_msm_bn254"]["device_ms"],
                             "fr_mul_2p22_ms": nr["fr_vector_ops_bn254"]["mul"]["device_ms"],
                             "fr_mul_hbm_frac": nr["fr_vector_ops_bn254"]["mul"]["hbm_frac_of_measured"],
                             "fr_inv_2p22_ms": nr["fr_vector_ops_bn254"]["inv"]["device_ms"]}
    line["pipe_rates_T_per_s"] = pipes
    # kept last: the figures a reader of the end of the line looks for
    line.update(tail)
    if ntt is not None:
        line["ntt"] = ntt
    if "config3_bls12_381_2p22" in extra:
        line["config3_bls12_381_2p22"] = extra["config3_bls12_381_2p22"]
    if args.details:
        with open(args.details, "w") as f:
            json.dump(details, f, indent=1)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
