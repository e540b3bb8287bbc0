"""Benchmark of the B200 FFTLIB batched FFT hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the headline configuration): FFTLIB_fft1dBatched_i32fc_c32fc_o32fc,
FP32 complex-to-complex forward FFT, N = 4096 points, 8192 channels per GPU,
interleaved re/im, inputs iid U[-1, 1) from a fixed seed. A step is one
batched transform of the whole batch. Metric: HBM throughput in GB/s of
algorithmic bytes (16 bytes per point: read 8 + write 8), whole job.

* value: device-resident buffers, one `_kernelAsync` launch per step, timed
  with CUDA events on the launching stream (inputs 256 MiB > 126 MB L2).
* e2e: the same transform through the synchronous FFTLIB `_kernel` call with
  pinned host buffers, host->device and device->host copies inside the
  timed region (wall clock).
* roofline: achieved GB/s of the FFT kernel against the measured HBM copy
  bandwidth in MEASURED_PEAKS.json; traffic per launch from the committed
  ncu capture summary (profiles/).
* cpu_baseline: the reference's own _cn code (oracle/_ref, built from the
  reference sources with gcc -O3) on the host cores, on a bounded sample of
  the same workload.
* --impl reference: that reference CPU implementation alone, as the
  reference arm.

Multi-GPU (torchrun): every rank transforms its own 8192-channel batch
(weak scaling, no collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 4096
CHANNELS = 8192
METRIC = "batched FFT HBM GB/s (% peak); TC-DFT vs FP32-FFT speedup at ≤2e-6 rel err"
WORKLOAD = "fft1dBatched_i32fc_c32fc_o32fc c2c FP32 forward, N=4096 x 8192 channels"


REL_L2_BOUND = 2e-6  # FP32 paths against FP64 (relative L2)

# Parity checks of the timed outputs: every bench line carries them, and a
# line whose checks fail is printed with parity.ok false and the process
# exits non-zero.
PARITY_FAILURES = []


def parity_check(name, ok, value=None):
    if not ok:
        PARITY_FAILURES.append(f"{name}: {value}")
    return ok


def algo_bytes(n, ch):
    return 16.0 * n * ch


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_peaks():
    """The driver-measured peaks (hbm_gbs, bf16_tflops, ...) or {}."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def traffic_from_profile(kernel_tag):
    """Per-launch DRAM bytes of the kernel from the committed ncu summary
    (lines 'traffic <tag> <bytes>'), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(p):
            f = line.split()
            if len(f) >= 3 and f[0] == "traffic" and f[1] == kernel_tag:
                return float(f[2])
    except OSError:
        pass
    return None


class ClockSampler:
    """SM clock and throttle-reason samples taken during the timed region
    through NVML (every ~2 ms, plus one sample at entry and exit)."""

    REASONS = {  # NVML clocks-event-reason bits
        "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4,
    }

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.smax = None
        self._stop = threading.Event()
        self._nv = None

    def _sample(self):
        nv = self._nv
        try:
            self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            for name, bit in self.REASONS.items():
                if bits & bit:
                    self.reasons.add(name)
        except Exception:
            pass

    def _handle(self, nv):
        """NVML handle of the CUDA device (NVML ignores CUDA_VISIBLE_DEVICES):
        by UUID, else by PCI address, else by index."""
        import torch

        prop = torch.cuda.get_device_properties(self.index)
        uuid = getattr(prop, "uuid", None)
        if uuid is not None:
            try:
                return nv.nvmlDeviceGetHandleByUUID(f"GPU-{uuid}")
            except Exception:
                pass
        if hasattr(prop, "pci_bus_id"):
            try:
                addr = f"{getattr(prop, 'pci_domain_id', 0):08x}:{prop.pci_bus_id:02x}:{prop.pci_device_id:02x}.0"
                return nv.nvmlDeviceGetHandleByPciBusId(addr)
            except Exception:
                pass
        return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _loop(self):
        while not self._stop.is_set():
            self._sample()
            time.sleep(0.002)

    def __enter__(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            self._nv = nv
            self.h = self._handle(nv)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            self._sample()
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
        except Exception:
            self._nv = None
        return self

    def __exit__(self, *a):
        if self._nv:
            self._stop.set()
            self.t.join(timeout=2)
            self._sample()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def max_over_ranks(x: float, dist, device) -> float:
    """The largest of every rank's x (the job's time is its slowest rank's)."""
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput of weak-scaled replicas: the units all ranks
    processed over the slowest rank's time."""
    return units_per_rank * world / seconds_max


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_arm(args, world, rank):
    """The reference's own CPU implementation (_cn compiled from its sources)
    on all host threads: each step a bounded sample of the workload."""
    if rank != 0:
        return
    import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference _cn build) is not present"}))
        return
    sample = 256  # channels per step: ~64 MiB of the 8192-channel workload
    threads = O.host_threads()
    for _ in range(args.warmup):
        O.time_reference_c2c(N_POINTS, sample, threads, reps=1)
    times = [O.time_reference_c2c(N_POINTS, sample, threads, reps=1, seed=s)[0] for s in range(args.steps)]
    t = sum(times)
    gbs = algo_bytes(N_POINTS, sample) * args.steps / t / 1e9
    ms_full = (algo_bytes(N_POINTS, CHANNELS) / (gbs * 1e9)) * 1e3
    out = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 4), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_full, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_channels_per_step": sample, "parallelism": "host threads",
                   "ms_per_step_basis": f"extrapolated: the time of the {sample}-channel sample per step scaled "
                                        f"to {CHANNELS} channels (channels are independent)"},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} channels of N={N_POINTS} per step, reference "
                                   f"FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_cn built with gcc -O3"},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def our_arm(args, world, rank, local):
    import torch

    import c7x_fftlib_b200 as F

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n, ch = N_POINTS, args.channels
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    X = torch.rand(2 * n * ch, device="cuda", generator=g) * 2 - 1
    Y = torch.empty_like(X)
    W = torch.zeros(2 * n, device="cuda")
    b, bw = F.bp(F.FFTLIB_FLOAT32, 2 * n * ch), F.bp(F.FFTLIB_FLOAT32, 2 * n)
    base = F.KERNELS["c2c"]
    pb = F.pblock("c2c")
    F.check(F.fn(base + "_init")(F.ptr(X), b, F.ptr(W), bw, F.ptr(Y), b, n, ch, pb), "init")
    stream = torch.cuda.Stream()
    launch = F.fn("FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelAsync")
    sp = F.ptr(stream.cuda_stream)

    def step():
        st = launch(F.ptr(X), F.ptr(Y), n, ch, pb, sp)
        if st:
            F.check(st, "kernelAsync")

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist:
        ms = max_over_ranks(ms, dist, "cuda")
    ms_step = ms / args.steps
    per_gpu_gbs = algo_bytes(n, ch) / (ms_step * 1e-3) / 1e9
    value = job_rate(algo_bytes(n, ch), world, ms_step * 1e-3) / 1e9

    if args.quick:  # profiling runs: the timed launches only
        if dist:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"quick": True, "ms_per_step": ms_step, "GBps": value, "channels": ch}))
        return

    # spot check of the timed output: a few channels against numpy's FFT in FP64
    import numpy as np

    idx = [0, ch // 3, ch - 1]
    xs = X.view(ch, 2 * n)[idx].cpu().numpy().astype(np.float64)
    ys = Y.view(ch, 2 * n)[idx].cpu().numpy().astype(np.float64)
    want = np.fft.fft(xs[:, 0::2] + 1j * xs[:, 1::2], axis=1)
    got = ys[:, 0::2] + 1j * ys[:, 1::2]
    rel = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    parity_check("c2c_4096 sampled rel-L2", rel <= REL_L2_BOUND, rel)

    # end to end through the synchronous FFTLIB call with pinned host buffers
    e2e_steps = max(2, min(args.steps, 5))
    Xh = X.cpu().pin_memory()
    Yh = torch.empty_like(Xh).pin_memory()
    kern = F.fn(base + "_kernel")
    F.check(kern(F.ptr(Xh), b, F.ptr(W), bw, F.ptr(Yh), b, n, ch, pb), "kernel (host)")
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        F.check(kern(F.ptr(Xh), b, F.ptr(W), bw, F.ptr(Yh), b, n, ch, pb), "kernel (host)")
    e2e_s = time.perf_counter() - t0
    if dist:
        e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    e2e_gbs = job_rate(algo_bytes(n, ch) * e2e_steps, world, e2e_s) / 1e9

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    peak, peak_kind = measured_peak()
    traffic = traffic_from_profile("c2c_4096")
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(ms_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "numPoints": n, "numChannels_per_gpu": ch, "parallelism": f"replicas{world}",
                   "plan": F.describe_block(pb), "autotune": autotune_on(),
                   "l2": "inputs (256 MiB) larger than L2, no flush",
                   "transforms_per_s": round(ch * world / (ms_step * 1e-3), 1)},
        "roofline": {"bound": "hbm", "achieved": round(per_gpu_gbs, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(per_gpu_gbs / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic},
        "e2e": {"value": round(e2e_gbs, 2), "unit": "GB/s", "h2d_bytes_per_step": int(8 * n * ch),
                "d2h_bytes_per_step": int(8 * n * ch), "path": "FFTLIB _kernel, pinned host buffers"},
        "gpu_launches": args.steps,
        "parity": {"rel_l2_vs_fp64_sampled": rel, "bound": REL_L2_BOUND},
        "clocks": clk.summary(),
    }
    if world == 1:
        out["cpu_baseline"] = cpu_baseline()
        out["configs"] = secondary_configs(args)
    out["parity"]["ok"] = not PARITY_FAILURES
    if PARITY_FAILURES:
        out["parity"]["failures"] = PARITY_FAILURES
    print(json.dumps(out))
    if PARITY_FAILURES:
        sys.exit(1)


def autotune_on():
    v = os.environ.get("FFTLIB_B200_AUTOTUNE", "")
    return bool(v) and v != "0"


def _time_launches(torch, stream, fn, steps, warmup=3):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def mixed_lengths(count, seed, nmax=4096):
    """Lengths 12 * 2^a 3^b 5^c <= nmax, log N uniform on [log 12, log nmax]
    snapped to the nearest allowed length."""
    import numpy as np

    allowed = sorted({12 * (2 ** a) * (3 ** b) * (5 ** c) for a in range(12) for b in range(8) for c in range(6)
                      if 12 * (2 ** a) * (3 ** b) * (5 ** c) <= nmax})
    allowed = np.array(allowed)
    u = np.random.default_rng(seed).uniform(np.log(12), np.log(nmax), count)
    return allowed[np.abs(np.log(allowed)[None, :] - u[:, None]).argmin(axis=1)].astype(np.uint32)


def secondary_configs(args):
    """The other workloads of the benchmark configuration list, device
    buffers, CUDA events on the launching stream."""
    import numpy as np
    import torch

    import c7x_fftlib_b200 as F

    steps = max(5, min(args.steps, 20))
    stream = torch.cuda.Stream()
    sp = F.ptr(stream.cuda_stream)
    res = {}
    g = torch.Generator(device="cuda").manual_seed(7)

    # int16 c2c, N=1024 x 4096, inputs in [-2048, 2047], shift 2 per radix-4 stage
    n, ch = 1024, 4096
    x = torch.randint(-2048, 2048, (2 * n * ch,), device="cuda", dtype=torch.int16, generator=g)
    y = torch.empty_like(x)
    w = np.zeros(2 * n, np.int16)
    F.lib().FFTLIB_b200_tw_gen_i16(F.ptr(w), n)
    wd = torch.from_numpy(w).cuda()
    sh = torch.full((5,), 2, dtype=torch.int32, device="cuda")
    bx, bw, bs = F.bp(F.FFTLIB_INT16, 2 * n * ch), F.bp(F.FFTLIB_INT16, 2 * n), F.bp(F.FFTLIB_UINT32, 5)
    pb = F.pblock("i16")
    F.check(F.fn(F.KERNELS["i16"] + "_init")(F.ptr(x), bx, F.ptr(wd), bw, F.ptr(y), bx, F.ptr(sh), bs, n, ch, pb))
    k = F.fn("FFTLIB_b200_fft1dBatched_i16sc_c16sc_o16sc_kernelAsync")
    ms = _time_launches(torch, stream, lambda: k(F.ptr(x), F.ptr(wd), F.ptr(y), F.ptr(sh), 5, n, ch, pb, sp), steps)
    torch.cuda.synchronize()
    import oracle as O

    k16 = 16  # bit-exact sample: the first 16 channels against the oracle's restated _cn
    xs = x[: 2 * n * k16].cpu().numpy()
    exact16 = bool(np.array_equal(y[: 2 * n * k16].cpu().numpy(), O.fft_c2c_i16(xs, n, k16, [2] * 5)))
    parity_check("int16_c2c_1024 bit-exact sample", exact16)
    res["int16_c2c_n1024_x4096"] = {"plan": F.describe_block(pb), "ms": round(ms, 4),
                                     "GBps": round(8.0 * n * ch / ms / 1e6, 1),
                                     "transforms_per_s": round(ch / ms * 1e3, 1), "bit_exact_sample": exact16}

    # r2c then c2r, N=4096 x 8192 reals (128 MiB), outmode / inMode 0
    n, ch = 4096, 8192
    xr = torch.randn(n * ch, device="cuda", generator=g)
    yc = torch.empty(2 * (n // 2 + 1) * ch, device="cuda")
    xb = torch.empty_like(xr)
    b = F.bp(F.FFTLIB_FLOAT32, n * ch)
    pr, pc = F.pblock("r2c"), F.pblock("c2r")
    F.check(F.fn(F.KERNELS["r2c"] + "_init")(F.ptr(xr), b, F.ptr(xr), b, None, b, F.ptr(xr), b, F.ptr(yc), b, n, ch,
                                             0, pr))
    F.check(F.fn(F.KERNELS["c2r"] + "_init")(F.ptr(yc), b, F.ptr(yc), b, None, b, F.ptr(yc), b, F.ptr(xb), b, n, ch,
                                             0, pc))
    kr = F.fn("FFTLIB_b200_fft1dBatched_i32f_c32fc_o32fc_kernelAsync")
    kc = F.fn("FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32f_kernelAsync")
    ms_r = _time_launches(torch, stream, lambda: kr(F.ptr(xr), None, F.ptr(yc), n, ch, 0, pr, sp), steps)
    ms_c = _time_launches(torch, stream, lambda: kc(F.ptr(yc), None, F.ptr(xb), n, ch, 0, pc, sp), steps)
    bytes_rc = (4.0 * n + 8.0 * (n // 2 + 1)) * ch
    torch.cuda.synchronize()
    rt = float(torch.linalg.norm(xb - xr) / torch.linalg.norm(xr))
    idx = [0, ch // 2, ch - 1]
    xs = xr.view(ch, n)[idx].cpu().numpy().astype(np.float64)
    want = np.fft.rfft(xs, axis=1)
    got = yc.view(ch, n // 2 + 1, 2)[idx].cpu().numpy().astype(np.float64)
    fwd = float(np.linalg.norm(got[..., 0] + 1j * got[..., 1] - want) / np.linalg.norm(want))
    parity_check("r2c_4096 sampled rel-L2", fwd <= REL_L2_BOUND, fwd)
    parity_check("r2c->c2r round trip rel-L2", rt <= REL_L2_BOUND, rt)
    res["r2c_c2r_n4096_x8192"] = {"r2c_plan": F.describe_block(pr), "c2r_plan": F.describe_block(pc),
                                  "r2c_ms": round(ms_r, 4), "r2c_GBps": round(bytes_rc / ms_r / 1e6, 1),
                                  "c2r_ms": round(ms_c, 4), "c2r_GBps": round(bytes_rc / ms_c / 1e6, 1),
                                  "r2c_rel_l2_vs_fp64_sampled": fwd, "roundtrip_rel_l2": rt}

    # uneven lengths: 20,000 c2c transforms, 12 * 2^a 3^b 5^c <= 4096, log-uniform,
    # laid out grouped by length so per-length batched calls can run on the same memory
    lengths = np.sort(mixed_lengths(20000, seed=2024))[::-1].copy()
    total = int(lengths.sum())
    xm = torch.rand(2 * total, device="cuda", generator=g) * 2 - 1
    ym = torch.empty_like(xm)
    mb = F.MixedBatch(lengths)
    ms_graph = _time_launches(torch, stream, lambda: mb.exec(xm, ym, sp), steps)
    # every group in the single persistent kernel (runtime-radix passes)
    mbp = F.MixedBatch(lengths, persistent_only=True)
    ms_persistent = _time_launches(torch, stream, lambda: mbp.exec(xm, ym, sp), steps)
    mbp.close()
    ms_per = _time_launches(torch, stream, lambda: mb.exec_per_size(xm, ym, sp), steps)
    # the regular batched API, one call per length (fixed-size kernels where compiled)
    uniq, counts = np.unique(lengths, return_counts=True)
    calls = []
    off = 0
    for nn, cc in sorted(zip(uniq.tolist(), counts.tolist()), reverse=True):
        pbk = F.pblock("c2c")
        bb = F.bp(F.FFTLIB_FLOAT32, 2 * nn * cc)
        xs, ys = xm.data_ptr() + 8 * off, ym.data_ptr() + 8 * off
        F.check(F.fn(F.KERNELS["c2c"] + "_init")(F.ptr(xs), bb, F.ptr(xs), F.bp(F.FFTLIB_FLOAT32, 2 * nn), F.ptr(ys),
                                                 bb, nn, cc, pbk))
        calls.append((xs, ys, nn, cc, pbk))
        off += nn * cc
    ka = F.fn("FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelAsync")

    def per_length_api():
        for xs, ys, nn, cc, pbk in calls:
            ka(F.ptr(xs), F.ptr(ys), nn, cc, pbk, sp)

    ms_api = _time_launches(torch, stream, per_length_api, steps)
    # sampled check of the graph launch's output: the first and last
    # transform of every length against numpy's FP64 FFT
    mb.exec(xm, ym, sp)
    torch.cuda.synchronize()
    starts = np.concatenate([[0], np.cumsum(lengths.astype(np.int64))[:-1]])
    pick = sorted({int(np.argmax(lengths == u)) for u in uniq} |
                  {len(lengths) - 1 - int(np.argmax(lengths[::-1] == u)) for u in uniq})
    xh, yh = xm.cpu().numpy().astype(np.float64), ym.cpu().numpy().astype(np.float64)
    e2 = r2 = 0.0
    for i in pick:
        o, nn = int(starts[i]), int(lengths[i])
        xc = xh[2 * o: 2 * (o + nn)]
        want = np.fft.fft(xc[0::2] + 1j * xc[1::2])
        yc_ = yh[2 * o: 2 * (o + nn)]
        e2 += float(np.sum(np.abs(yc_[0::2] + 1j * yc_[1::2] - want) ** 2))
        r2 += float(np.sum(np.abs(want) ** 2))
    mixed_rel = (e2 / r2) ** 0.5
    parity_check("mixed_20000 sampled rel-L2", mixed_rel <= REL_L2_BOUND, mixed_rel)
    mbytes = 16.0 * total
    res["mixed_20000"] = {"lengths": len(uniq), "total_points": total,
                          "launch": "one graph: the length groups' persistent fixed-size kernels chained "
                                    "by programmatic dependent launch, largest and smallest groups in turn",
                          "persistent_graph_ms": round(ms_graph, 4),
                          "persistent_graph_GBps": round(mbytes / ms_graph / 1e6, 1),
                          "single_persistent_kernel_ms": round(ms_persistent, 4),
                          "single_persistent_kernel_GBps": round(mbytes / ms_persistent / 1e6, 1),
                          "per_length_same_kernel_ms": round(ms_per, 4),
                          "per_length_batched_api_ms": round(ms_api, 4),
                          "speedup_vs_per_length_api": round(ms_api / ms_graph, 3),
                          "rel_l2_vs_fp64_sampled": mixed_rel, "sampled_transforms": len(pick),
                          "transforms_per_s": round(20000 / ms_graph * 1e3, 1)}
    mb.close()
    res["tc_dft"] = tc_dft_configs(args, steps)
    res["fft1d_single"] = fft1d_single_configs(steps)
    res["int_dft"] = int_dft_configs(steps)
    res["linalg"] = linalg_configs(steps)
    return res


def int_dft_configs(steps):
    """The coordinator's integer paths (INT16 / INT32, bit-exact with the
    reference's natural C), on device buffers through execAsync: dftSmall,
    dftLarge and highRadix lengths with the rows of the tensor-core DFT
    configuration (2^20 rows up to 64 points, 16 M points per launch above).
    Bytes: one read and one write of 2 N values per row. ref_cn: the
    reference's natural C on one host core over 256 rows of the same data."""
    import time

    import numpy as np
    import torch

    import c7x_fftlib_b200 as F
    import oracle as O

    stream = torch.cuda.Stream()
    sp = F.ptr(stream.cuda_stream)
    out = {}
    for bits, n, rows in ((16, 16, 1 << 20), (16, 32, 1 << 20), (16, 256, 1 << 16), (16, 1024, 1 << 14),
                          (32, 8, 1 << 20), (32, 16, 1 << 20), (32, 64, 1 << 18)):
        dt = F.FFTLIB_INT16 if bits == 16 else F.FFTLIB_INT32
        tdt = torch.int16 if bits == 16 else torch.int32
        sh = [bits - 1] * 5 if n <= (32 if bits == 16 else 16) else [2, 2, 2, 2, 4]
        d = F.DftMma(n, rows, dtype=dt, interleave=1, shifts=sh)
        lim = (1 << (bits - 1)) - 1
        x0 = torch.randint(-lim, lim, (2 * n * rows,), dtype=torch.int64, device="cuda").to(tdt)
        x = x0.clone()
        y = torch.empty_like(x)
        ms = _time_launches(torch, stream, lambda: d.exec_async(x, y, sp), max(steps, 10))
        F.check(F.lib().FFTLIB_b200_FFT_fft_sync(sp), "sync")
        # bit-exact spot check against the oracle (highRadix overwrote x: rerun on a fresh copy)
        x.copy_(x0)
        d.exec_async(x, y, sp)
        F.check(F.lib().FFTLIB_b200_FFT_fft_sync(sp), "sync")
        k = min(rows, 64)
        xs = x0[: 2 * n * k].cpu().numpy()
        want = O.mma_exec(bits, n, k, 1, sh, xs)
        exact = bool(np.array_equal(y[: 2 * n * k].cpu().numpy(), want))
        parity_check(f"int{bits}_dft_{n} bit-exact sample", exact)
        entry = {"variant": O.mma_variant(bits, n, rows, 1), "rows": rows, "ms": round(ms, 4),
                 "GBps": round(2.0 * 2 * n * rows * (bits // 8) / ms / 1e6, 1),
                 "rows_per_s": round(rows / ms * 1e3, 1), "bit_exact_sample": exact}
        if O.ref_mma_available():
            kr = 256
            xr = x0[: 2 * n * kr].cpu().numpy()
            t0 = time.perf_counter()
            O.ref_mma_exec(bits, n, kr, 1, sh, xr)
            t_ref = time.perf_counter() - t0
            entry["ref_cn_rows_per_s"] = round(kr / t_ref, 1)
            entry["ref_cn_cores"] = 1
            entry["speedup_vs_ref_cn"] = round(entry["rows_per_s"] / entry["ref_cn_rows_per_s"], 1)
        out[f"int{bits}_n{n}"] = entry
        del x, x0, y
    return out


def linalg_configs(steps):
    """The integer matrix multiply FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX
    (bit-exact with the reference's natural C) on device buffers through
    execAsync: a square 4096^3 product and the DFT-shaped 2^20 x 64 x 64, for
    INT8, INT16 and INT32. MAC/s counts the M K N multiply-adds; bytes: A, B
    and C once. ref_cn: the reference's natural C on one host core over the
    first 16 rows of A."""
    import time

    import numpy as np
    import torch

    import c7x_fftlib_b200 as F
    import oracle as O

    stream = torch.cuda.Stream()
    sp = F.ptr(stream.cuda_stream)
    out = {}
    types = {8: (F.FFTLIB_INT8, torch.int8), 16: (F.FFTLIB_INT16, torch.int16), 32: (F.FFTLIB_INT32, torch.int32)}
    for bits in (8, 16, 32):
        dt, tdt = types[bits]
        lim = (1 << (bits - 1)) - 1
        for m, k, n in ((4096, 4096, 4096), (1 << 20, 64, 64)):
            a = torch.randint(-lim, lim, (m, k), dtype=torch.int64, device="cuda").to(tdt)
            b = torch.randint(-lim, lim, (k, n), dtype=torch.int64, device="cuda").to(tdt)
            c = torch.empty((m, n), dtype=tdt, device="cuda")
            shift = 2 * bits - 1
            mm = F.MatMul(m, k, n, dt, shift=shift)
            ms = _time_launches(torch, stream, lambda: mm.exec_async(a, b, c, sp), max(steps, 5))
            torch.cuda.synchronize()
            rs = 16
            a_s, b_h = a[:rs].cpu().numpy(), b.cpu().numpy()
            exact = bool(np.array_equal(c[:rs].cpu().numpy(), O.linalg_mm(bits, a_s, b_h, shift)))
            parity_check(f"linalg_int{bits}_{m}x{k}x{n} bit-exact sample", exact)
            entry = {"m": m, "k": k, "n": n, "ms": round(ms, 4),
                     "TMACps": round(m * k * n / ms / 1e9, 3),
                     "GBps": round((m * k + k * n + m * n) * (bits // 8) / ms / 1e6, 1),
                     "bit_exact_sample": exact}
            if O.ref_mma_available():
                t0 = time.perf_counter()
                O.ref_linalg_mm(bits, a_s, b_h, shift)
                t_ref = time.perf_counter() - t0
                entry["ref_cn_TMACps_1core"] = round(rs * k * n / t_ref / 1e12, 6)
                entry["speedup_vs_ref_cn"] = round(entry["TMACps"] / entry["ref_cn_TMACps_1core"], 1)
            out[f"int{bits}_{m}x{k}x{n}"] = entry
            del a, b, c
    return out


def fft1d_single_configs(steps):
    """Single-transform c2c (FFTLIB_fft1d_i32fc_c32fc_o32fc): the largest
    single-kernel length, the reference test list's largest length and two
    long lengths run as global passes. device_ms: the kernels alone (batched
    async entry with one channel, device buffers, CUDA events); e2e_ms: the
    synchronous FFTLIB_fft1d_i32fc_c32fc_o32fc_kernel on pinned host buffers
    (copies in and out included), wall clock per call; ref_cn_ms: the
    reference's natural-C single-transform kernel on one host core."""
    import time

    import numpy as np
    import torch

    import c7x_fftlib_b200 as F
    import oracle as O

    stream = torch.cuda.Stream()
    sp = F.ptr(stream.cuda_stream)
    out = {}
    base = F.KERNELS["1d_c2c"]
    for n in (16384, 78125, 1 << 20, 1 << 24):
        x = torch.rand(2 * n, device="cuda") * 2 - 1
        y = torch.empty_like(x)
        pb = F.pblock("c2c")
        bb = F.bp(F.FFTLIB_FLOAT32, 2 * n)
        F.check(F.fn(F.KERNELS["c2c"] + "_init")(F.ptr(x), bb, F.ptr(x), bb, F.ptr(y), bb, n, 1, pb))
        k = F.fn("FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelAsync")
        ms = _time_launches(torch, stream, lambda: k(F.ptr(x), F.ptr(y), n, 1, pb, sp), max(steps, 20))
        xh = torch.empty(2 * n, dtype=torch.float32, pin_memory=True)
        yh = torch.empty(2 * n, dtype=torch.float32, pin_memory=True)
        x0 = (torch.rand(2 * n) * 2 - 1)
        pb1 = F.pblock("1d_c2c")
        F.check(F.fn(base + "_init")(F.ptr(xh), bb, F.ptr(xh), bb, F.ptr(yh), bb, pb1))
        reps = 20 if n <= (1 << 20) else 5
        t_e2e = []
        for _ in range(reps + 2):
            xh.copy_(x0)  # the kernel may use pX as work buffer
            t0 = time.perf_counter()
            F.check(F.fn(base + "_kernel")(F.ptr(xh), bb, F.ptr(xh), bb, F.ptr(yh), bb, pb1))
            t_e2e.append(time.perf_counter() - t0)
        e2e_ms = float(np.median(t_e2e[2:])) * 1e3
        got = yh.numpy().astype(np.float64)
        want = np.fft.fft(x0.numpy().astype(np.float64).view(np.complex128))
        rel = float(np.linalg.norm(got.view(np.complex128) - want) / np.linalg.norm(want))
        parity_check(f"fft1d_{n} rel-L2", rel <= REL_L2_BOUND, rel)
        entry = {"plan": F.describe_plan(n), "device_ms": round(ms, 5),
                 "device_GBps": round(16.0 * n / ms / 1e6, 1), "e2e_ms": round(e2e_ms, 4),
                 "h2d_d2h_bytes": 16 * n, "rel_l2_vs_fp64": rel}
        if n <= 78125 and O.ref1d_available():
            xr = x0.numpy()
            w = O.ref_tw_gen_c2c(n)
            t_ref = []
            for _ in range(3):
                t0 = time.perf_counter()
                O.ref_fft1d_c2c_f32(xr, n, False, w)
                t_ref.append(time.perf_counter() - t0)
            entry["ref_cn_ms"] = round(float(np.median(t_ref)) * 1e3, 3)
            entry["ref_cn_cores"] = 1
            entry["e2e_speedup_vs_ref_cn"] = round(entry["ref_cn_ms"] / e2e_ms, 2)
        out[str(n)] = entry
        del x, y, xh, yh
    return out


def tc_flops(n: int) -> float:
    """Executed tensor-core FLOPs of one split-precision DFT of length n:
    3 FP16 products of the real-embedding GEMMs (one stage: rows x 2n x 2n;
    two stages n = n1 n2: n2 rows x (2 n1)^2 then n1 rows x (2 n2)^2)."""
    import c7x_fftlib_b200 as F  # noqa: F401

    two = {128: (16, 8), 256: (16, 16), 512: (32, 16), 1024: (32, 32), 2048: (64, 32), 4096: (64, 64)}
    if n in two:
        n1, n2 = two[n]
        return 3.0 * (2.0 * n2 * (2 * n1) ** 2 + 2.0 * n1 * (2 * n2) ** 2)
    return 3.0 * 2.0 * (2 * n) ** 2


def tc_dft_configs(args, steps):
    """Split-FP16 tensor-core DFT (the fft_c7xmma coordinator, funcStyle
    OPTIMIZED) against the CUDA-core FP32 FFT (funcStyle NATC) on the same
    inputs: 2^20 rows for n = 16..256 and n = 4096 x 8192. Relative L2 error
    of sampled rows against numpy's FP64 FFT."""
    import numpy as np
    import torch

    import c7x_fftlib_b200 as F

    peaks = measured_peaks()
    hbm = float(peaks.get("hbm_gbs") or 6650.0)
    tfl = float(peaks.get("bf16_tflops") or 1590.0)  # dense FP16 runs at the BF16 rate
    stream = torch.cuda.Stream()
    sp = F.ptr(stream.cuda_stream)
    out = {}
    g = torch.Generator(device="cuda").manual_seed(5)
    for n, batch in [(16, 1 << 20), (32, 1 << 20), (64, 1 << 20), (128, 1 << 20), (256, 1 << 20), (4096, 8192)]:
        x = torch.rand(2 * n * batch, device="cuda", generator=g) * 2 - 1
        y = torch.empty_like(x)
        yf = torch.empty_like(x)
        tc = F.DftMma(n, batch, F.FFTLIB_FUNCTION_OPTIMIZED)
        ff = F.DftMma(n, batch, F.FFTLIB_FUNCTION_NATC)
        with ClockSampler(torch.cuda.current_device()) as clk:
            ms_tc = _time_launches(torch, stream, lambda: tc.exec_async(x, y, sp), steps)
        ms_ff = _time_launches(torch, stream, lambda: ff.exec_async(x, yf, sp), steps)
        F.check(F.lib().FFTLIB_b200_FFT_fft_sync(sp), "sync")
        rows = np.random.default_rng(n).choice(batch, size=min(batch, 256), replace=False)
        xs = x.view(batch, 2 * n)[torch.from_numpy(rows).cuda()].cpu().numpy().astype(np.float64)
        ys = y.view(batch, 2 * n)[torch.from_numpy(rows).cuda()].cpu().numpy().astype(np.float64)
        want = np.fft.fft(xs[:, 0::2] + 1j * xs[:, 1::2], axis=1)
        rel = float(np.linalg.norm(ys[:, 0::2] + 1j * ys[:, 1::2] - want) / np.linalg.norm(want))
        parity_check(f"tc_dft_{n} sampled rel-L2", rel <= REL_L2_BOUND, rel)
        gbs = 16.0 * n * batch / ms_tc / 1e6
        tfs = tc_flops(n) * batch / ms_tc / 1e9
        out[str(n)] = {"rows": batch, "tc_ms": round(ms_tc, 4), "tc_GBps": round(gbs, 1),
                       "tc_hbm_frac": round(gbs / hbm, 3), "tc_tensor_TFLOPs": round(tfs, 1),
                       "tc_tensor_frac": round(tfs / tfl, 3),
                       "fft_ms": round(ms_ff, 4), "fft_GBps": round(16.0 * n * batch / ms_ff / 1e6, 1),
                       "tc_speedup_vs_fft": round(ms_ff / ms_tc, 3), "tc_rel_l2_vs_fp64": rel,
                       "tc_clocks": clk.summary()}
        del x, y, yf
    return out


def cpu_baseline():
    import oracle as O

    if not O.ref_available():
        return None
    sample = 512
    threads = O.host_threads()
    t, used = O.time_reference_c2c(N_POINTS, sample, threads, reps=5)
    t1, _ = O.time_reference_c2c(N_POINTS, 64, 1, reps=5)
    return {"value": round(algo_bytes(N_POINTS, sample) / t / 1e9, 4), "unit": "GB/s", "cores": used,
            "kind": "reference",
            "single_thread_value": round(algo_bytes(N_POINTS, 64) / t1 / 1e9, 4),
            "sample": f"{sample} channels of N={N_POINTS}, median of 5, reference _cn (gcc -O3), one thread per "
                      f"core; single_thread_value: 64 channels on one thread, median of 5"}


def run_case(args):
    """W warm-up and K timed launches of one kernel on device buffers; one
    JSON line with the per-launch time. For profiler captures and sweeps.
    Cases: tc:N:rows (tensor-core DFT), fft:N:rows (CUDA-core FFT through the
    coordinator), c2c:N:channels, r2c:N:channels, c2r:N:channels,
    i16:N:channels (fft1dBatched kernels), int16:N:rows / int32:N:rows (the
    coordinator's integer paths), mm8:N:M / mm16:N:M (LINALG multiply of an
    M x N by an N x N matrix), mixed:COUNT:SEED (uneven lengths, one graph
    launch)."""
    import numpy as np
    import torch

    import c7x_fftlib_b200 as F

    kind, n, batch = args.case.split(":")
    n, batch = int(n), int(batch)
    g = torch.Generator(device="cuda").manual_seed(1)
    stream = torch.cuda.current_stream()
    sp = F.ptr(stream.cuda_stream)
    nbytes = 16.0 * n * batch
    if kind in ("tc", "fft"):
        style = {"tc": F.FFTLIB_FUNCTION_OPTIMIZED, "fft": F.FFTLIB_FUNCTION_NATC}[kind]
        x = torch.rand(2 * n * batch, device="cuda", generator=g) * 2 - 1
        y = torch.empty_like(x)
        d = F.DftMma(n, batch, style)

        def launch():
            d.exec_async(x, y, sp)
    elif kind == "c2c":
        x = torch.rand(2 * n * batch, device="cuda", generator=g) * 2 - 1
        y = torch.empty_like(x)
        pb = F.pblock("c2c")
        bb = F.bp(F.FFTLIB_FLOAT32, 2 * n * batch)
        F.check(F.fn(F.KERNELS["c2c"] + "_init")(F.ptr(x), bb, F.ptr(x), F.bp(F.FFTLIB_FLOAT32, 2 * n), F.ptr(y),
                                                 bb, n, batch, pb))
        k = F.fn("FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelAsync")

        def launch():
            return k(F.ptr(x), F.ptr(y), n, batch, pb, sp)
    elif kind in ("r2c", "c2r"):
        nb = 4 * n + 8 * (n // 2 + 1)
        nbytes = float(nb) * batch
        xr = torch.randn(n * batch, device="cuda", generator=g)
        yc = torch.randn(2 * (n // 2 + 1) * batch, device="cuda", generator=g)
        b = F.bp(F.FFTLIB_FLOAT32, n * batch)
        pb = F.pblock(kind)
        src, dst = (xr, yc) if kind == "r2c" else (yc, xr)
        wk = torch.empty(n * batch, device="cuda")  # pXFFT: the global-pass lengths' work buffer
        F.check(F.fn(F.KERNELS[kind] + "_init")(F.ptr(src), b, F.ptr(src), b, None, b, F.ptr(src), b, F.ptr(dst), b,
                                                n, batch, 0, pb))
        k = F.fn("FFTLIB_b200_fft1dBatched_i32f_c32fc_o32fc_kernelAsync" if kind == "r2c"
                 else "FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32f_kernelAsync")

        def launch():
            return k(F.ptr(src), F.ptr(wk), F.ptr(dst), n, batch, 0, pb, sp)
    elif kind == "i16":
        nbytes = 8.0 * n * batch
        x = torch.randint(-2048, 2048, (2 * n * batch,), device="cuda", dtype=torch.int16, generator=g)
        y = torch.empty_like(x)
        w = np.zeros(2 * n, np.int16)
        F.lib().FFTLIB_b200_tw_gen_i16(F.ptr(w), n)
        wd = torch.from_numpy(w).cuda()
        ns = max(1, (n.bit_length() - 1 + 1) // 2)
        sh = torch.full((ns,), 2, dtype=torch.int32, device="cuda")
        bx = F.bp(F.FFTLIB_INT16, 2 * n * batch)
        pb = F.pblock("i16")
        F.check(F.fn(F.KERNELS["i16"] + "_init")(F.ptr(x), bx, F.ptr(wd), F.bp(F.FFTLIB_INT16, 2 * n), F.ptr(y), bx,
                                                 F.ptr(sh), F.bp(F.FFTLIB_UINT32, ns), n, batch, pb))
        k = F.fn("FFTLIB_b200_fft1dBatched_i16sc_c16sc_o16sc_kernelAsync")

        def launch():
            return k(F.ptr(x), F.ptr(wd), F.ptr(y), F.ptr(sh), ns, n, batch, pb, sp)
    elif kind in ("int16", "int32"):  # the coordinator's integer path, interleaved
        bits = int(kind[3:])
        dt = F.FFTLIB_INT16 if bits == 16 else F.FFTLIB_INT32
        tdt = torch.int16 if bits == 16 else torch.int32
        nbytes = 2.0 * 2 * n * batch * (bits // 8)
        d = F.DftMma(n, batch, dtype=dt, interleave=1, shifts=[2, 2, 2, 2, 4])
        x = torch.randint(-1000, 1000, (2 * n * batch,), dtype=torch.int64, device="cuda").to(tdt)
        y = torch.empty_like(x)

        def launch():
            d.exec_async(x, y, sp)
    elif kind in ("mm8", "mm16"):  # mmB:N:M -- LINALG multiply of M x N by N x N
        bits = int(kind[2:])
        dt = F.FFTLIB_INT8 if bits == 8 else F.FFTLIB_INT16
        tdt = torch.int8 if bits == 8 else torch.int16
        nbytes = float(2 * n * batch + n * n) * (bits // 8)
        a = torch.randint(-100, 100, (batch, n), dtype=torch.int64, device="cuda").to(tdt)
        bm = torch.randint(-100, 100, (n, n), dtype=torch.int64, device="cuda").to(tdt)
        c = torch.empty((batch, n), dtype=tdt, device="cuda")
        mm = F.MatMul(batch, n, n, dt, shift=bits)

        def launch():
            mm.exec_async(a, bm, c, sp)
    elif kind == "mixed":  # mixed:COUNT:SEED -- the uneven-length batch, one graph launch
        lengths = np.sort(mixed_lengths(n, seed=batch))[::-1].copy()
        total = int(lengths.sum())
        nbytes = 16.0 * total
        x = torch.rand(2 * total, device="cuda", generator=g) * 2 - 1
        y = torch.empty_like(x)
        mb = F.MixedBatch(lengths)

        def launch():
            mb.exec(x, y, sp)
    else:
        raise SystemExit(f"unknown case kind {kind}")
    for _ in range(args.warmup):
        st = launch()
        if isinstance(st, int):  # the C-ABI calls return their status
            F.check(st, args.case)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        launch()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"case": args.case, "ms": round(ms, 5), "GBps": round(nbytes / ms / 1e6, 1)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--channels", type=int, default=CHANNELS, help="channels per GPU (default: the workload's 8192)")
    ap.add_argument("--quick", action="store_true", help="time the kernel only (for profiler captures)")
    ap.add_argument("--autotune", type=int, choices=[0, 1], default=0,
                    help="1: every _init times its launch candidates (FFTLIB_B200_AUTOTUNE=1), with a fresh "
                         "cache file unless FFTLIB_B200_TUNE_CACHE names one")
    ap.add_argument("--case", default=None,
                    help="time one kernel only, for profiler captures: tc:N:batch (tensor-core DFT), "
                         "fft:N:batch (CUDA-core FFT through the same coordinator API)")
    args = ap.parse_args()
    if args.autotune:
        import tempfile

        os.environ["FFTLIB_B200_AUTOTUNE"] = "1"
        if "FFTLIB_B200_TUNE_CACHE" not in os.environ:
            os.environ["FFTLIB_B200_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="fftlib_tune_"), "tune.txt")
    if args.case:
        run_case(args)
        return
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        reference_arm(args, world, rank)
    else:
        our_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
