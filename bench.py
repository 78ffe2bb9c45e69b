#!/usr/bin/env python3
"""bench.py -- FP64-accurate GEMM throughput on B200: the Ozaki INT8 form beside the native FP64
form, at N = 16384 (the product MGXBench's per-rank block multiply computes, 1D-row-block/
mulmat_kernel.cu:39-92, at the size the headline metric is quoted on).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one C = A B of 16384 x 16384 x 16384 FP64 with wide-exponent inputs
(u * 2^e, u ~ U[-1,1), e ~ U{-20..20}), A and B resident in HBM (2 GiB each, larger than L2).
`value` is effective TFLOP/s = 2 N^3 / step time of the Ozaki INT8 form -- by default its CRT
form (Ozaki scheme II: scales and residues, one tensor-core product per modulus, CRT
recombination), `--form slices` for the digit-slice form -- valid only if its normwise error
against a double-double product (sampled rows) is <= 1e-15.  `e2e` is the same product through
the C ABI with pinned host buffers, host-to-device and device-to-host copies inside each step.
Under torchrun every rank computes its own independent product (weak scaling, no data-path
collective); the step time is the max over ranks.
`--impl reference` times MGXBench's arithmetic on the host cores instead: the oracle's
restatement of sharedABMultiply (one FMA chain per output) with all host threads, on a bounded
sample of rows of the same product.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FP64-accurate GEMM TFLOP/s @N=16384: Ozaki-INT8 vs native FP64 at ≤1e-15 err"
N_DEFAULT = 16384
EXP_RANGE = 20
ERROR_GATE = 1e-15
CHECK_ROWS = 256
# DRAM bytes (read + write) per launch of the dominant kernel at N = 16384, from one-pass ncu
# captures (dram__bytes_read.sum + dram__bytes_write.sum) of bench.py at full size:
# ozaki_gemm with s = 8 reads 83.69 GB and writes 2.15 GB; crt_gemm with q = 15 reads
# 48.43 GB and writes 4.03 GB.  (Counter captures now run at N = 8192, where crt_gemm moves
# 5.41 GB, 1.79x its algorithmic bytes; scaled by the algorithmic bytes that would be 21.7 GB
# at N = 16384, an underestimate because a modulus's operands outgrow L2, so the measured
# full-size figure is kept.)
OZAKI_GEMM_TRAFFIC_BYTES = 85.84e9
CRT_GEMM_TRAFFIC_BYTES = 52.46e9


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), d.get("hbm_gbs", 6650.0), "measured"
    return 1590.0, 1400.0, 6650.0, "fallback"


class ClockSampler:
    """SM clock, power and clock-event (throttle) reasons sampled during a timed region: through
    NVML every 10 ms where the binding is present, else nvidia-smi every 200 ms.  It only reads."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))
    PERIOD_S = 0.01

    def __init__(self, device_index: int, uuid: str | None = None):
        self.dev = device_index
        self.uuid = uuid
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, power W, reason bits)
        self.done = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        if self.uuid:
            for u in (self.uuid if self.uuid.startswith("GPU-") else "GPU-" + self.uuid, self.uuid):
                try:
                    return pynvml, pynvml.nvmlDeviceGetHandleByUUID(u)
                except Exception:
                    pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _poll(self):
        nv, h = self.nvml
        while not self.done.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                     nv.nvmlDeviceGetPowerUsage(h) / 1000.0,
                                     int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
            except Exception:
                pass
            self.done.wait(self.PERIOD_S)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.done.set()
            self.thread.join(timeout=2)
            sms = [x[0] for x in self.samples]
            power = [x[1] for x in self.samples]
            reasons = {name for name, bit in self.REASONS for x in self.samples if x[2] & bit}
            return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": self.max_mhz,
                    "power_w_max": max(power) if power else None, "samples": len(sms),
                    "source": f"NVML every {self.PERIOD_S * 1000:.0f} ms", "reasons": sorted(reasons)}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sms, maxes, power, reasons = [], [], [], set()
        names = [name for name, _ in self.REASONS]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxes) if maxes else None,
                "power_w_max": max(power) if power else None, "samples": len(sms),
                "source": "nvidia-smi every 200 ms", "reasons": sorted(reasons)}


def device_uuid(torch) -> str | None:
    """The current CUDA device's UUID (NVML names the same GPU by it whatever CUDA_VISIBLE_DEVICES is)."""
    try:
        return str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
    except Exception:
        return None


def cpu_reference_rate(n: int, budget_s: float, threads: int = 0):
    """Times the oracle's FMA-chain restatement of MGXBench's kernel on `rows` x n x n."""
    import numpy as np
    from oracle import oracle as O
    rng = np.random.default_rng(1)
    B = rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-EXP_RANGE, EXP_RANGE + 1, (n, n)))
    probe = 128
    A = rng.uniform(-1, 1, (probe, n))
    t0 = time.perf_counter()
    O.ab_multiply(A, B, threads=threads)
    dt = time.perf_counter() - t0
    rate = 2.0 * probe * n * n / dt
    rows = int(max(probe, min(4096, budget_s * rate / (2.0 * n * n))))
    return B, rows, rate


def ranks_reduce_max(dist, value: float, device) -> float:
    """Max of a per-rank number over all ranks: a multi-GPU step takes as long as its slowest
    rank.  `dist` is None for a single process."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def host_cpu_model() -> str:
    """The host CPU's model name (from /proc/cpuinfo), for the CPU baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    rank, _, world = env_rank()
    if rank != 0:
        return 0
    import numpy as np
    from oracle import oracle as O
    n = args.n
    threads = O.max_threads()
    B, rows, _ = cpu_reference_rate(n, args.ref_step_seconds, threads)
    rng = np.random.default_rng(2)
    A = rng.uniform(-1, 1, (rows, n)) * np.exp2(rng.integers(-EXP_RANGE, EXP_RANGE + 1, (rows, n)))
    for _ in range(args.warmup):
        O.ab_multiply(A, B, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.ab_multiply(A, B, threads=threads)
        times.append(time.perf_counter() - t0)
    step = sum(times) / len(times)
    value = 2.0 * rows * n * n / step / 1e12
    sample = (f"{rows} rows x {n} x {n} of the N={n} product per step (sequential FMA chain per output, "
              f"MGXBench's sharedABMultiply arithmetic), {threads} host threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dgemm_n{n}_wide_exp{EXP_RANGE}", "m": n, "n": n, "k": n,
                   "form": "reference FP64 FMA chain on host cores", "sample_rows": rows},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "port", "sample": sample,
                         "cpu_model": host_cpu_model(), "host_cpus": os.cpu_count()},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import mgxbench_b200 as mgx

    rank, local_rank, world = env_rank()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    n = args.n
    flop = 2.0 * n * n * n
    stream = torch.cuda.Stream()
    A = torch.empty((n, n), dtype=torch.float64, device="cuda")
    B = torch.empty((n, n), dtype=torch.float64, device="cuda")
    C = torch.empty((n, n), dtype=torch.float64, device="cuda")
    mgx.fill_matrix(A, 2, e_range=EXP_RANGE, seed=1000 + 2 * rank, stream=stream)
    mgx.fill_matrix(B, 2, e_range=EXP_RANGE, seed=1001 + 2 * rank, stream=stream)
    crt = args.form == "crt"
    splits = args.splits or mgx.ozaki_choose_splits(n, float(EXP_RANGE), ERROR_GATE)
    moduli = args.moduli or mgx.crt_choose_moduli(n, ERROR_GATE)
    if crt:
        ws = torch.empty(mgx.crt_workspace_size(n, n, n, moduli), dtype=torch.uint8, device="cuda")
    else:
        ws = torch.empty(mgx.ozaki_workspace_size(n, n, n, splits), dtype=torch.uint8, device="cuda")
    stream.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    def step():
        if crt:
            mgx.crt_split(A, B, moduli, ws, stream=stream)
            ev_g0.record(stream)
            mgx.crt_products(n, n, n, moduli, ws, stream=stream)
            ev_g1.record(stream)
            mgx.crt_combine(C, n, moduli, ws, stream=stream)
        else:
            mgx.ozaki_split(A, B, splits, ws, stream=stream)
            ev_g0.record(stream)
            mgx.ozaki_multiply(C, n, splits, ws, stream=stream)
            ev_g1.record(stream)

    ev_g0 = torch.cuda.Event(enable_timing=True)
    ev_g1 = torch.cuda.Event(enable_timing=True)
    int8_peak = mgx.peak_int8(1, 200000)
    for _ in range(args.warmup):
        step()
    stream.synchronize()

    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local_rank,
                           device_uuid(torch))
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_stop = torch.cuda.Event(enable_timing=True)
    gemm_ms = []
    t_start.record(stream)
    for _ in range(args.steps):
        step()
        ev_g1.synchronize()
        gemm_ms.append(ev_g0.elapsed_time(ev_g1))
    t_stop.record(stream)
    # (ev_g1.synchronize() waits for the products only; the next step's split is queued behind
    # the combine on the same stream, so the steps stay back to back on the GPU.)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    elapsed_ms = ranks_reduce_max(dist, t_start.elapsed_time(t_stop), "cuda")
    ms_per_step = elapsed_ms / args.steps
    value = world * flop / (ms_per_step * 1e-3) / 1e12

    # accuracy gate on sampled rows against the double-double product
    err = mgx.error_vs_dd(A, B, C, row_start=(n - CHECK_ROWS) // 2, row_count=CHECK_ROWS)
    status = mgx.device_status()
    valid = err["normwise"] <= ERROR_GATE and status == 0

    # native FP64 form on the same inputs
    native = {}
    if not args.skip_native:
        C2 = torch.empty_like(C)
        mgx.gemm_fp64(A, B, C2, stream=stream)
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = max(1, min(args.steps, 3))
        e0.record(stream)
        for _ in range(reps):
            mgx.gemm_fp64(A, B, C2, stream=stream)
        e1.record(stream)
        e1.synchronize()
        nat_ms = e0.elapsed_time(e1) / reps
        nerr = mgx.error_vs_dd(A, B, C2, row_start=(n - CHECK_ROWS) // 2, row_count=CHECK_ROWS)
        # the FP64 tensor-core peak, measured on this GPU by the library's DMMA loops (m16n8k8 / k16)
        fp64_peak = max(mgx.peak_fp64(3, 20000), mgx.peak_fp64(4, 20000))
        nat_tf = flop / (nat_ms * 1e-3) / 1e12
        native = {"tflops": nat_tf, "ms_per_step": nat_ms, "normwise_err": nerr["normwise"],
                  "max_rel_err": nerr["max_rel"], "meets_1e-15": nerr["normwise"] <= ERROR_GATE,
                  "fp64_peak_tflops": fp64_peak, "frac_of_fp64_peak": nat_tf / fp64_peak,
                  "kernel": "dgemm_kernel (DMMA m16n8k8, TMA, warp-specialised)"}
        del C2

    # the other Ozaki form on the same inputs (slices when the headline is the CRT form)
    other = {}
    if crt and not args.skip_native:
        C3 = torch.empty_like(C)
        ws_s = torch.empty(mgx.ozaki_workspace_size(n, n, n, splits), dtype=torch.uint8, device="cuda")
        mgx.gemm_ozaki(A, B, C3, splits=splits, workspace=_Ws(ws_s), stream=stream)
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = max(1, min(args.steps, 3))
        e0.record(stream)
        for _ in range(reps):
            mgx.gemm_ozaki(A, B, C3, splits=splits, workspace=_Ws(ws_s), stream=stream)
        e1.record(stream)
        e1.synchronize()
        s_ms = e0.elapsed_time(e1) / reps
        serr = mgx.error_vs_dd(A, B, C3, row_start=(n - CHECK_ROWS) // 2, row_count=CHECK_ROWS)
        other = {"form": "ozaki-int8 digit slices", "splits": splits, "tflops": flop / (s_ms * 1e-3) / 1e12,
                 "ms_per_step": s_ms, "normwise_err": serr["normwise"], "int8_products": splits * (splits + 1) // 2}
        del C3, ws_s
        torch.cuda.empty_cache()

    # end to end through the C ABI with pinned host buffers: mgx_gemm_host streams row panels of
    # A and column panels of B in; once panel pair t is on the device it computes the new row and
    # column strips of C (two products) and streams them back while the rest computes
    e2e = None
    if not args.skip_e2e:
        hA = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        hB = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        hC = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        hA.copy_(A)
        hB.copy_(B)
        probe_rows = [0, n // 2, n - 1]
        c_probe = C[probe_rows].cpu()
        del C
        torch.cuda.empty_cache()
        reps = max(1, min(args.steps, 3))
        form_id, form_arg = (mgx.FORM_CRT, moduli) if crt else (mgx.FORM_OZAKI, splits)
        del ws
        torch.cuda.empty_cache()
        mgx.gemm_host(hA, hB, hC, form=form_id, splits=form_arg, panels=args.panels, stream=stream)
        stream.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            mgx.gemm_host(hA, hB, hC, form=form_id, splits=form_arg, panels=args.panels, stream=stream)
        e1.record(stream)
        e1.synchronize()
        e2e_ms = ranks_reduce_max(dist, e0.elapsed_time(e1) / reps, "cuda")
        same = bool(torch.equal(hC[probe_rows].view(torch.int64), c_probe.view(torch.int64)))
        e2e = {"value": world * flop / (e2e_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": 2 * n * n * 8, "d2h_bytes_per_step": n * n * 8, "ms_per_step": e2e_ms,
               "bit_identical_to_device_result": same,
               "path": f"mgx_gemm_host via the C ABI: pinned host A, B in, C out; {args.panels} row panels of A x "
                       f"{args.panels} column panels of B; as each panel pair arrives, the new row and column strips "
                       f"of C are computed and copied back while the rest computes"}

    # roofline of the dominant kernel (crt_gemm, or ozaki_gemm for the slice form): int8 tensor
    # ops per launch / launch time.
    # The INT8 peak is not in MEASURED_PEAKS.json; it is measured here, on this GPU, by the
    # library's tcgen05 kind::i8 loop (M=128 N=128 K=32, operands resident in shared memory):
    # a short burst before the timed region, and a sustained figure -- one launch of about
    # 2.5 s, long enough for the 1 kW power cap to set the clock -- after it.  ozaki_gemm runs
    # ~100 ms launches back to back inside a long step, so the sustained figure is its ceiling.
    peak_sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local_rank,
                                device_uuid(torch))
    peak_sampler.start()
    time.sleep(0.3)
    int8_sustained = mgx.peak_int8(1, 60_000_000)
    peak_clocks = peak_sampler.stop()
    bf16_burst, bf16_sust, hbm, peak_kind = peaks()
    products = moduli if crt else splits * (splits + 1) // 2
    kp = (n + 31) // 32 * 32
    int8_ops = 2.0 * n * n * kp * products
    gemm_avg_ms = sum(gemm_ms) / len(gemm_ms)
    achieved = int8_ops / (gemm_avg_ms * 1e-3) / 1e12
    peak = int8_sustained
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": (CRT_GEMM_TRAFFIC_BYTES if crt else OZAKI_GEMM_TRAFFIC_BYTES) if n == N_DEFAULT else None,
                "kernel": "crt_gemm" if crt else "ozaki_gemm",
                "peak_note": (f"INT8 dense peak measured on this GPU by mgx_peak_int8 (tcgen05.mma kind::i8 "
                              f"128x128x32 loop): sustained over one ~2.5 s launch {int8_sustained:.0f} TOP/s (used), "
                              f"burst {int8_peak:.0f} TOP/s; 2 x the {peak_kind} bf16 cuBLAS burst would be "
                              f"{2 * bf16_burst:.0f}"),
                "peak_burst": int8_peak, "frac_of_burst": achieved / int8_peak,
                "frac_of_2x_bf16_burst": achieved / (2.0 * bf16_burst),
                "ops_per_launch": int8_ops, "int8_products": products, "launch_ms": gemm_avg_ms,
                "other_kernels_ms": ms_per_step - gemm_avg_ms}
    # The kernel runs at the 1 kW power cap; the peak loop holds a higher clock.  The fraction per
    # clock scales the peak to the SM clock sampled during the timed region.
    if peak_clocks.get("sm_mhz") and clocks.get("sm_mhz"):
        roofline["peak_sm_mhz"] = peak_clocks["sm_mhz"]
        roofline["timed_sm_mhz"] = clocks["sm_mhz"]
        roofline["frac_per_clock"] = achieved / peak * peak_clocks["sm_mhz"] / clocks["sm_mhz"]

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        try:
            from oracle import oracle as O
            threads = O.max_threads()
            Bh, rows, _ = cpu_reference_rate(n, args.cpu_seconds, threads)
            import numpy as np
            rng = np.random.default_rng(2)
            Ah = rng.uniform(-1, 1, (rows, n))
            t0 = time.perf_counter()
            O.ab_multiply(Ah, Bh, threads=threads)
            dt = time.perf_counter() - t0
            cpu = {"value": 2.0 * rows * n * n / dt / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                   "sample": f"{rows} rows x {n} x {n} of the N={n} product (oracle FMA-chain restatement of "
                             f"sharedABMultiply), {dt:.1f} s", "cpu_model": host_cpu_model(), "host_cpus": os.cpu_count()}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "TFLOP/s", "cores": 0, "kind": "port", "sample": f"failed: {exc}"}

    # CRT: row_scale, col_max, col_sumsq, col_scale, split_a, split_b, crt_gemm, crt_combine;
    # slices: row_exp, col_max, col_exp, split_a, split_b, ozaki_gemm
    launches_per_step = 8 if crt else 6
    line = {
        "metric": METRIC, "value": value if valid else 0.0, "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dgemm_n{n}_wide_exp{EXP_RANGE}", "m": n, "n": n, "k": n,
                   "form": "ozaki-int8-crt" if crt else "ozaki-int8-slices",
                   **({"moduli": moduli} if crt else {"splits": splits}),
                   "input": f"u*2^e, u~U[-1,1), e~U{{-{EXP_RANGE}..{EXP_RANGE}}}",
                   "l2": "inputs larger than L2 (2 GiB per matrix vs 126 MB)", "error_gate": ERROR_GATE,
                   "per_rank": "independent product per GPU (weak scaling)"},
        "valid": bool(valid),
        "accuracy": {"normwise": err["normwise"], "max_rel": err["max_rel"],
                     "max_componentwise": err["max_componentwise"], "rows_checked": err["rows_checked"],
                     "reference": "double-double product on the GPU"},
        "native_fp64": native,
        "ozaki_other_form": other or None,
        "speedup_vs_native_fp64": (value / native["tflops"]) if native else None,
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "gpu_launches": launches_per_step * args.steps,
    }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


class _Ws:
    """Adapter handing a preallocated workspace tensor to mgx.gemm_ozaki."""

    def __init__(self, t):
        self.t = t

    def get(self, nbytes):
        assert self.t.numel() >= nbytes
        return self.t


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_DEFAULT, help="matrix size (the metric is quoted at 16384)")
    ap.add_argument("--form", choices=["crt", "slices"], default="crt",
                    help="Ozaki form timed for `value`: CRT (scheme II, default) or digit slices")
    ap.add_argument("--moduli", type=int, default=0, help="CRT moduli (0 = chosen for the 1e-15 gate)")
    ap.add_argument("--splits", type=int, default=0, help="Ozaki slices (0 = chosen for the 1e-15 gate)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--ref-step-seconds", type=float, default=8.0, help="reference arm: seconds per step")
    ap.add_argument("--panels", type=int, default=32, help="row panels of A and column panels of B in the host-buffer (e2e) path")
    ap.add_argument("--skip-native", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("bench.py: at least 3 warm-up steps are required", file=sys.stderr)
        return 2
    _, _, world = env_rank()
    if args.gpus != world:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch N>1 with torch.distributed.run",
              file=sys.stderr)
        return 2
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
