#!/usr/bin/env python
"""Throughput of lvl1 TFHE gate bootstrapping on B200 (one JSON line).

A step is one batch of 4096 independent lvl1 gates drawn uniformly from
{NAND, AND, OR, XOR, XNOR, MUX} on random bits, with Ctxt<lvl1> inputs (key
switching, then blind rotation, then SampleExtract), through the engine's
C-ABI.  A MUX needs two blind rotations, so the unit is bootstraps/s
(binary gate = 1, MUX = 2).

  value  device-resident inputs, CUDA events around each step (L2 flushed
         between steps by a 256 MiB write), max over ranks
  e2e    the same through cufhe_gate_batch_host with pinned host buffers:
         H2D of the inputs and D2H of the outputs inside the timed region;
         consecutive batches alternate between two engine streams, so one
         batch's copies overlap the previous batch's bootstrapping

Usage: python bench.py [--gpus N] [--steps K] [--warmup W]
                       [--path all|fp64_kb|fp64_plain|int8_kb|int8_plain]
                       [--impl ours|reference]
The default measures both precision forms with both bootstrapping-key forms
on the same batch (FP64 FFNT with the KeyBundle key is the headline `value`;
each form's numbers are under `paths`, and `int8_vs_fp64` compares the two
precision forms on the same key form), then 1000 random NAND pairs with the
plain key (`nand1000`, with the CPU port timed on the same pairs), the FP64
form's rounding error against the exact form at lvl1 (`fp64_error_lvl1`),
and the sub-workloads (uneven circuits, circuit bootstrapping + lookup
tables, lvl02).  Under torchrun each rank runs its own batch on its own GPU
(weak scaling, no data-path collective: gates are independent).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "lvl1 NAND bootstraps/sec on 1 B200: INT8-exact vs FP64-FFNT; p50 gate latency"
UNIT = "bootstraps/s"
GATE_SET = [0, 4, 1, 8, 9, 12]  # NAND, AND, OR, XOR, XNOR, MUX
A100_PUBLISHED = 1.0 / 0.12e-3   # reference README: 0.12 ms/gate, lvl1 NAND FP64 + KeyBundle
# algorithmic work per bootstrap (lvl1): FP64 FFNT flops, INT8 tensor ops
FLOP_FP64 = {True: 287_744 * 318, False: 189_440 * 636}
# INT8: 2 ops per MAC x K = 4096 (4 digit rows x 1024) x M = 8192 (2 polys x
# 1024 coefficients x 4 key limbs) per GEMM; 636 GEMMs (plain) or 318 pairs x
# 3 keys (KeyBundle)
OPS_INT8 = {False: 2 * 636 * 4096 * 8192, True: 2 * 318 * 3 * 4096 * 8192}
PATHS = {"fp64_kb": ("fp64", True), "fp64_plain": ("fp64", False),
         "int8_kb": ("int8", True), "int8_plain": ("int8", False)}
NAND_PAIRS = 1000  # configs: plain lvl1 NAND, FP64 FFNT, no KeyBundle
# lvl2 (N = 2048, 1024-point transforms, 8 digit rows): per KeyBundle step
# 10 transforms x 5*1024*10 + twist/untwist 10*1024*6 + combine/MAC 8*2*1024*32
FLOP_FP64_LVL2_KB = (10 * 51_200 + 61_440 + 524_288) * 318
LVL02_BATCHES = (512, 2048, 8192)
# exact INT8 form at lvl02: K = 8 digit rows x 2048, M = 2 polys x 2048
# coefficients x 8 key limbs, 2 digit limbs, 636 steps (a MAC is 2 ops)
OPS_INT8_LVL2 = 2 * 636 * (8 * 2048) * (2 * 2048 * 8) * 2
OPS_INT8_LVL2_KB = 2 * 318 * 3 * (8 * 2048) * (2 * 2048 * 8) * 2  # KeyBundle: 3 keys per pair
LVL02_INT8_BATCH = 2048
WORKLOAD = ("lvl1 mixed-gate batch: 4096 independent gates uniform over "
            "NAND/AND/OR/XOR/XNOR/MUX, Ctxt<lvl1> I/O (IKS->BR->SampleExtract), "
            "n0=636 N=1024 l=2 Bgbit=8 IKS basebit=2 t=7, Torus32")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--path", choices=["all"] + list(PATHS), default="all")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-lvl02", action="store_true",
                    help="skip the lvl0->lvl2 NAND batches reported under the 'lvl02' key")
    ap.add_argument("--no-uneven", action="store_true",
                    help="skip the uneven-circuit workload reported under the 'uneven' key")
    ap.add_argument("--no-nand1000", action="store_true",
                    help="skip the 1000 random NAND pairs (plain key) under the 'nand1000' key")
    ap.add_argument("--no-error", action="store_true",
                    help="skip the lvl1 FP64-vs-exact error figures ('fp64_error_lvl1' key)")
    ap.add_argument("--no-cb", action="store_true",
                    help="skip the circuit-bootstrapping + lookup-table workload ('cb_lut' key)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in lanes-per-CTA rule instead of the autotuner's table")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def make_workload(rng, batch):
    gates = rng.choice(GATE_SET, size=batch).astype(np.int32)
    a, b, c = (rng.integers(0, 2, batch).astype(np.uint8) for _ in range(3))
    return gates, a, b, c


def bootstraps(gates):
    return int(gates.size + np.count_nonzero(gates == 12))


def common_config(batch, nb):
    """The `config` of both arms (same workload, same keys, same units)."""
    return {"workload": WORKLOAD, "gates_per_step": batch, "bootstraps_per_step": nb,
            "keybundle": True,
            "l2": ("GPU arm: flushed between timed steps (256 MiB write); CPU arm: no flush "
                   "(the keys exceed the host caches)"),
            "parallelism": "replicas: an independent gate batch per GPU"}


def max_over_ranks(torch, x: float, device) -> float:
    """Maximum of x over all ranks (identity without a process group)."""
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if torch.distributed.is_available() and torch.distributed.is_initialized() and \
            torch.distributed.get_world_size() > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.item()


def whole_job_rate(units_per_rank_step: int, world: int, steps: int, max_ms: float) -> float:
    """Units per second of the whole job: every rank processes its own batch
    each step (weak scaling); the slowest rank's device time sets the pace."""
    return units_per_rank_step * world * steps / (max_ms * 1e-3)


# ---------------------------------------------------------------- clocks ---
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r)
                          if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "reasons": reasons}


# ----------------------------------------------------------- reference arm ---
def cpu_gate_rate(seed, batch, keybundle=True):
    """Oracle port of the reference's CPU gate (FP64 FFNT restatement),
    OpenMP over gates on all host cores: the bench's own gate batch (same
    seed, size and gate mix as the GPU arm), timed once."""
    from cufhepp_b200 import client
    from oracle import oracle as O
    sk = client.SecretKey.generate(seed)
    ek = client.EvalKey.generate(sk, keybundle=keybundle)
    fft = O.FFT()
    bkf = O.bk_to_fft(fft, ek.bk)
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    gates, a, b, c = make_workload(rng, batch)
    cts = [client.encrypt_bits(sk, x, 1, seed=seed + i) for i, x in enumerate((a, b, c))]
    n_warm = min(batch, 2 * cores)
    O.gate_batch(gates[:n_warm], 1, *(x[:n_warm] for x in cts), bkf, ek.ksk, keybundle, O.FP64,
                 fft)
    t0 = time.perf_counter()
    O.gate_batch(gates, 1, *cts, bkf, ek.ksk, keybundle, O.FP64, fft)
    el = time.perf_counter() - t0
    return bootstraps(gates) / el, cores, (
        f"the full {batch}-gate batch of the workload ({bootstraps(gates)} bootstraps), once, "
        f"{el:.1f} s; FP64 FFNT, {'KeyBundle' if keybundle else 'plain'} key")


def cpu_gate2_rate(seconds, seed):
    """Oracle port of the lvl02 CPU gate (FP64 FFNT restatement at N = 2048,
    KeyBundle), OpenMP over gates on all host cores; bounded sample."""
    from cufhepp_b200 import client
    from oracle import oracle as O
    sk = client.SecretKey.generate(seed)
    ek = client.EvalKey02.generate(sk, keybundle=True)
    fft = O.FFT2()
    bkf = O.bk2_to_fft(fft, ek.bk)
    cores = os.cpu_count() or 1
    n = max(8, cores)
    rng = np.random.default_rng(seed)
    a, b = (rng.integers(0, 2, n).astype(np.uint8) for _ in range(2))
    cts = [client.encrypt_bits(sk, x, 0, seed=seed + i) for i, x in enumerate((a, b))]
    gates = np.zeros(n, np.int32)
    done = 0
    t0 = time.perf_counter()
    while True:
        O.gate2_batch(gates, cts[0], cts[1], None, bkf, ek.ksk, True, O.FP64, fft)
        done += n
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return {"value": done / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n}-NAND batches repeated for {el:.1f} s"}


def run_reference(args):
    """The reference's CPU gate (oracle port: TFHEpp, which the reference's
    CPU path calls, is absent) on the workload of our arm: every timed step
    is the whole --batch gate batch of the same seed and mix, KeyBundle key,
    OpenMP over gates on all host threads.  Warm-up steps run a short prefix
    of the batch (they only spin up the threads and fault in the key)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    from cufhepp_b200 import client
    from oracle import oracle as O
    sk = client.SecretKey.generate(args.seed)
    ek = client.EvalKey.generate(sk, keybundle=True)
    fft = O.FFT()
    bkf = O.bk_to_fft(fft, ek.bk)
    rng = np.random.default_rng(args.seed)
    gates, a, b, c = make_workload(rng, args.batch)
    cts = [client.encrypt_bits(sk, x, 1, seed=args.seed + i) for i, x in enumerate((a, b, c))]
    n_warm = min(args.batch, 2 * cores)
    for _ in range(args.warmup):
        O.gate_batch(gates[:n_warm], 1, *(x[:n_warm] for x in cts), bkf, ek.ksk, True, O.FP64,
                     fft)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        O.gate_batch(gates, 1, *cts, bkf, ek.ksk, True, O.FP64, fft)
        times.append(time.perf_counter() - t)
    nb = bootstraps(gates)
    value = nb * args.steps / sum(times)
    sample = (f"the full {args.batch}-gate batch ({nb} bootstraps) every step (FP64 FFNT, "
              f"KeyBundle), OpenMP over gates on {cores} host threads; warm-up steps run a "
              f"{n_warm}-gate prefix")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded keys, random bits", "impl": "reference",
        "config": common_config(args.batch, nb),
        "impl_detail": ("cpu: oracle port of the reference algorithm (reference not buildable: "
                        "TFHEpp submodule absent)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# -------------------------------------------------------------- our arm ---
def ncu_traffic(kernel: str):
    """DRAM bytes per launch recorded from an ncu capture in profiles/."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(rf"dram_bytes_per_launch\[{kernel}\]\s*=\s*([0-9.eE+]+)", f.read_text())
        if m:
            return float(m.group(1))
    return None


def run_path(args, path, torch, engine, client, P, sk, workload, rank, ws, flush):
    """One precision form with one bootstrapping-key form (PATHS[path]) on the
    bench's gate batch."""
    gates, a, b, c = workload
    form, kb = PATHS[path]
    ek = client.EvalKey.generate(sk, keybundle=kb)
    engine.initialize(ek)
    engine.set_precision(P.FP64_FFNT if form == "fp64" else P.INT8_EXACT)
    level = 1
    words = P.TLWE1_WORDS
    B = gates.size
    cts = [client.encrypt_bits(sk, x, level, seed=args.seed + 100 * rank + i)
           for i, x in enumerate((a, b, c))]
    dev_in = [engine.to_device(x) for x in cts]
    dev_out = engine.DeviceBuffer(B * words * 4)

    def step():
        engine.gate_batch(gates, B, level, dev_out, *dev_in)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    out = engine.from_device(dev_out, (B, words))
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    fails = int(np.count_nonzero(client.decrypt_bits(sk, out, level) != exp))

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    engine.profile_reset()
    engine.profile_enable(True)
    l0 = engine.kernel_launches()
    clk = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clk.start()
    # latency and per-kernel device time: one batch at a time
    for k in range(args.steps):
        ev[k][0].record()
        step()
        ev[k][1].record()
        flush.zero_()
    torch.cuda.synchronize()
    engine.profile_enable(False)
    kern = {}
    for cls, name in enumerate(engine.K_NAMES):
        ms, n = engine.profile_read(cls)
        if n:
            kern[name] = (ms, n)
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]

    # single-gate latency on an idle GPU (one NAND through cufhe_gate)
    lat = []
    L = engine.load()
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        engine.check(L.cufhe_gate(0, level, engine.dptr(dev_out), engine.dptr(dev_in[0]),
                                  engine.dptr(dev_in[1]), None, None), "gate")
        e1.record()
        torch.cuda.synchronize()
        lat.append(e0.elapsed_time(e1))

    # throughput: consecutive batches alternate between two engine streams
    # (each with its own workspace and output buffer), as a streaming caller
    # would, so one batch's partial last wave overlaps the next batch's first
    # kernels.  K whole batches, L2 flushed on a batch's stream before it
    # starts, events around all K, max over ranks.
    streams = [engine.Stream(0) for _ in range(2)]  # each rank sees its GPU as device 0
    tstreams = [torch.cuda.ExternalStream(st.cuda) for st in streams]
    dev_outs = [dev_out, engine.DeviceBuffer(B * words * 4)]
    for i in range(2):
        engine.gate_batch(gates, B, level, dev_outs[i], *dev_in, stream=streams[i])
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = engine.kernel_launches()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_done = torch.cuda.Event()
    t_start.record(tstreams[0])
    tstreams[1].wait_event(t_start)
    for k in range(args.steps):
        i = k & 1
        with torch.cuda.stream(tstreams[i]):
            flush.zero_()
        engine.gate_batch(gates, B, level, dev_outs[i], *dev_in, stream=streams[i])
    t_done.record(tstreams[1])
    tstreams[0].wait_event(t_done)
    t_end.record(tstreams[0])
    torch.cuda.synchronize()
    launches = engine.kernel_launches() - l0
    if ws > 1:
        torch.distributed.barrier()
    total_ms = max_over_ranks(torch, t_start.elapsed_time(t_end), "cuda")
    nb = bootstraps(gates)
    value = whole_job_rate(nb, ws, args.steps, total_ms)
    for i in range(2):
        got = engine.from_device(dev_outs[i], (B, words))
        fails += int(np.count_nonzero(client.decrypt_bits(sk, got, level) != exp))

    # e2e through the C-ABI with pinned host buffers.  Consecutive batches
    # alternate between two engine streams (each with its own device I/O
    # workspace and host output buffer), as a streaming caller would: batch
    # k+1's host->device copies overlap batch k's bootstrapping.  Every
    # batch's inputs and outputs still cross PCIe inside the timed region,
    # and L2 is flushed on a batch's stream before it starts.
    host_in = [np.ascontiguousarray(x) for x in cts]
    host_out = [np.empty((B, words), np.uint32) for _ in range(2)]
    for h in host_in + host_out:
        engine.check(engine.load().cufhe_host_register(engine._p(h), h.nbytes), "host_register")
    for i in range(2):
        engine.gate_batch_host(gates, level, *host_in, stream=streams[i], out=host_out[i])
    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    done = [torch.cuda.Event() for _ in range(2)]
    e_start.record(tstreams[0])
    tstreams[1].wait_event(e_start)
    for k in range(args.steps):
        i = k & 1
        with torch.cuda.stream(tstreams[i]):
            flush.zero_()
        engine.gate_batch_host(gates, level, *host_in, stream=streams[i], out=host_out[i])
    done[1].record(tstreams[1])
    tstreams[0].wait_event(done[1])
    e_end.record(tstreams[0])
    torch.cuda.synchronize()
    clocks = clk.stop()
    e2e_ms = max_over_ranks(torch, e_start.elapsed_time(e_end), "cuda")
    for i in range(2):
        fails += int(np.count_nonzero(client.decrypt_bits(sk, host_out[i], level) != exp))
    for h in host_in + host_out:
        engine.load().cufhe_host_unregister(engine._p(h))
    for st in streams:
        st.destroy()

    engine.cleanup()

    br = "br_fp64" if form == "fp64" else "br_int8"
    rl = None
    if br in kern:
        ms, n = kern[br]
        per_launch_s = ms * 1e-3 / n
        if form == "fp64":
            work = FLOP_FP64[bool(kb)] * nb
            peak = engine_peak_fp64(engine)
            rl = {"bound": "fp64", "achieved": work / per_launch_s / 1e12, "peak": peak,
                  "unit": "TFLOP/s", "frac": work / per_launch_s / 1e12 / peak,
                  "traffic": ncu_traffic("br_fp64_kb") if kb else None,
                  "kernel": "k_br_fp64 (FP64 FFNT blind rotation + SampleExtract)",
                  "work_per_launch": work,
                  "peak_source": "measured FP64 FMA probe on this GPU "
                                 "(cufhe_measure_fp64_peak; the peaks file has no FP64 figure)"}
        else:
            work = OPS_INT8[bool(kb)] * nb
            peak = engine_peak_int8(engine)
            rl = {"bound": "tensor", "achieved": work / per_launch_s / 1e12, "peak": peak,
                  "unit": "TOP/s", "frac": work / per_launch_s / 1e12 / peak,
                  "traffic": ncu_traffic("br_int8_kb" if kb else "br_int8"),
                  "kernel": ("INT8 blind rotation (decompose + tcgen05 Toeplitz GEMM per " +
                             ("KeyBundle pair, three keys)" if kb else "CMUX step)")),
                  "work_per_launch": work,
                  "peak_source": "measured tcgen05.mma.kind::i8 M128 N256 K32 probe on this GPU "
                                 "(cufhe_measure_int8_peak, random operands; the peaks file has "
                                 "no INT8 figure)"}
    if rl is not None:
        # where the launch time comes from, and the same work over the
        # throughput loop's own time per batch (which also holds the key
        # switch, about 1 % of it)
        rl["launch_time_source"] = (
            "CUDA events on the launching stream around every launch of the kernel in the "
            "one-batch-at-a-time timed loop (the p50 loop: batches back to back, L2 flushed "
            "between them), each launch alone on the GPU; in the throughput loop consecutive "
            "batches overlap on two streams, so per-launch event times there would include the "
            "sharing")
        rl["launches_timed"] = kern[br][1]
        rl["frac_over_throughput_loop_step"] = rl["work_per_launch"] / (
            total_ms / args.steps * 1e-3) / 1e12 / rl["peak"]
    res = {
        "value": value, "ms_per_step": total_ms / args.steps,
        "p50_gate_latency_ms": statistics.median(step_ms),
        "p99_gate_latency_ms": float(np.percentile(step_ms, 99)),
        "single_gate_latency_ms": statistics.median(lat),
        "decrypt_failures": fails, "gates_checked": 5 * B, "streams": 2,
        "e2e": {"value": whole_job_rate(nb, ws, args.steps, e2e_ms), "unit": UNIT,
                "h2d_bytes_per_step": int(sum(x.nbytes for x in cts)),
                "d2h_bytes_per_step": int(B * words * 4)},
        "gpu_launches": launches,
        "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kern.items()},
        "roofline": rl, "clocks": clocks, "bootstraps_per_step": nb, "keybundle": bool(kb),
    }
    return res


def run_nand1000(args, torch, engine, client, P, sk, rank, ws, flush):
    """configs: plain lvl1 NAND gate bootstrapping, FP64 FFNT, no KeyBundle:
    1000 uniform random bit pairs encrypted at +-1/8 (Ctxt<lvl1>, key
    switching then blind rotation), as one batch per step: device-resident
    inputs, CUDA events per step, L2 flushed between steps; the same through
    host buffers (e2e); a single NAND on the idle GPU; and the CPU port of the
    reference's gate timed on the same 1000 pairs."""
    from oracle import oracle as O
    ek = client.EvalKey.generate(sk, keybundle=False)
    engine.initialize(ek)
    engine.set_precision(P.FP64_FFNT)
    rng = np.random.default_rng(args.seed + 1000 + rank)
    n = NAND_PAIRS
    a, b = (rng.integers(0, 2, n).astype(np.uint8) for _ in range(2))
    cts = [client.encrypt_bits(sk, x, 1, seed=args.seed + 1100 + i) for i, x in enumerate((a, b))]
    din = [engine.to_device(x) for x in cts]
    dout = engine.DeviceBuffer(n * P.TLWE1_WORDS * 4)
    gates = np.zeros(n, np.int32)

    def step():
        engine.gate_batch(None, n, 1, dout, *din, uniform=P.NAND)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    fails = int(np.count_nonzero(
        client.decrypt_bits(sk, engine.from_device(dout, (n, P.TLWE1_WORDS)), 1) != 1 - (a & b)))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        ev[k][0].record()
        step()
        ev[k][1].record()
        flush.zero_()
    torch.cuda.synchronize()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    total = max_over_ranks(torch, sum(step_ms), "cuda")
    # e2e through the C-ABI from pinned host buffers (the two NAND inputs in,
    # the outputs back, every batch, inside the timed region).  Streaming:
    # consecutive batches alternate between two engine streams, so batch k+1's
    # copies overlap batch k's bootstrapping (as in the 4096-gate legs); and
    # one batch at a time, for the end-to-end batch latency.
    host_in = [np.ascontiguousarray(x) for x in cts]
    host_out = [np.empty((n, P.TLWE1_WORDS), np.uint32) for _ in range(2)]
    for h in host_in + host_out:
        engine.check(engine.load().cufhe_host_register(engine._p(h), h.nbytes), "host_register")
    streams = [engine.Stream(0) for _ in range(2)]
    tstreams = [torch.cuda.ExternalStream(st.cuda) for st in streams]
    for i in range(2):
        engine.gate_batch_host(None, 1, *host_in, stream=streams[i], uniform=P.NAND,
                               out=host_out[i])
    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    done = torch.cuda.Event()
    e_start.record(tstreams[0])
    tstreams[1].wait_event(e_start)
    for k in range(args.steps):
        i = k & 1
        with torch.cuda.stream(tstreams[i]):
            flush.zero_()
        engine.gate_batch_host(None, 1, *host_in, stream=streams[i], uniform=P.NAND,
                               out=host_out[i])
    done.record(tstreams[1])
    tstreams[0].wait_event(done)
    e_end.record(tstreams[0])
    torch.cuda.synchronize()
    e2e_total = max_over_ranks(torch, e_start.elapsed_time(e_end), "cuda")
    for i in range(2):
        fails += int(np.count_nonzero(client.decrypt_bits(sk, host_out[i], 1) != 1 - (a & b)))
    # the same streaming on the device alone (inputs resident), the figure the
    # streaming e2e compares with
    douts = [dout, engine.DeviceBuffer(n * P.TLWE1_WORDS * 4)]
    s_start = torch.cuda.Event(enable_timing=True)
    s_end = torch.cuda.Event(enable_timing=True)
    s_start.record(tstreams[0])
    tstreams[1].wait_event(s_start)
    for k in range(args.steps):
        i = k & 1
        with torch.cuda.stream(tstreams[i]):
            flush.zero_()
        engine.gate_batch(None, n, 1, douts[i], *din, uniform=P.NAND, stream=streams[i])
    done2 = torch.cuda.Event()
    done2.record(tstreams[1])
    tstreams[0].wait_event(done2)
    s_end.record(tstreams[0])
    torch.cuda.synchronize()
    stream_total = max_over_ranks(torch, s_start.elapsed_time(s_end), "cuda")
    for i in range(2):
        got = engine.from_device(douts[i], (n, P.TLWE1_WORDS))
        fails += int(np.count_nonzero(client.decrypt_bits(sk, got, 1) != 1 - (a & b)))
    e2e_lat = []
    for k in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(tstreams[0]):
            flush.zero_()
        e0.record(tstreams[0])
        engine.gate_batch_host(None, 1, *host_in, stream=streams[0], uniform=P.NAND,
                               out=host_out[0])
        e1.record(tstreams[0])
        torch.cuda.synchronize()
        e2e_lat.append(e0.elapsed_time(e1))
    fails += int(np.count_nonzero(client.decrypt_bits(sk, host_out[0], 1) != 1 - (a & b)))
    for h in host_in + host_out:
        engine.load().cufhe_host_unregister(engine._p(h))
    for st in streams:
        st.destroy()
    lat = []
    L = engine.load()
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        engine.check(L.cufhe_gate(P.NAND, 1, engine.dptr(dout), engine.dptr(din[0]),
                                  engine.dptr(din[1]), None, None), "gate")
        e1.record()
        torch.cuda.synchronize()
        lat.append(e0.elapsed_time(e1))
    engine.cleanup()
    out = {"metric": "lvl1 NAND bootstraps/s (1000 random pairs per batch)", "unit": UNIT,
           "workload": (f"{n} uniform random NAND bit pairs at +-1/8, Ctxt<lvl1> I/O, FP64 FFNT, "
                        "plain bootstrapping key (no KeyBundle), one batch per step"),
           "value": whole_job_rate(n, ws, args.steps, total), "ms_per_step": total / args.steps,
           "value_note": "one batch at a time (each step a whole 1000-gate batch alone)",
           "value_streaming": whole_job_rate(n, ws, args.steps, stream_total),
           "value_streaming_note": "consecutive batches alternating on two engine streams, "
                                   "inputs resident, as the 4096-gate legs' value",
           "p50_batch_latency_ms": statistics.median(step_ms),
           "single_gate_latency_ms": statistics.median(lat),
           "e2e": {"value": whole_job_rate(n, ws, args.steps, e2e_total), "unit": UNIT,
                   "h2d_bytes_per_step": int(cts[0].nbytes + cts[1].nbytes),
                   "d2h_bytes_per_step": int(host_out[0].nbytes),
                   "pinned_host_buffers": True, "streams": 2,
                   "p50_batch_latency_ms": statistics.median(e2e_lat)},
           "decrypt_failures": fails, "gates_checked": 6 * n, "dtype": "f64"}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        fft = O.FFT()
        bkf = O.bk_to_fft(fft, ek.bk)
        O.gate_batch(gates[:16], 1, cts[0][:16], cts[1][:16], None, bkf, ek.ksk, False, O.FP64,
                     fft)
        t0 = time.perf_counter()
        ref = O.gate_batch(gates, 1, cts[0], cts[1], None, bkf, ek.ksk, False, O.FP64, fft)
        el = time.perf_counter() - t0
        cpu_fails = int(np.count_nonzero(client.decrypt_bits(sk, ref, 1) != 1 - (a & b)))
        out["cpu_baseline"] = {"value": n / el, "unit": UNIT, "cores": os.cpu_count() or 1,
                               "kind": "port", "cpu_model": cpu_model(),
                               "sample": f"the same {n} NAND pairs, once ({el:.2f} s), FP64 FFNT, "
                                         "plain key, OpenMP over gates",
                               "decrypt_failures": cpu_fails}
    return out


def fp64_error_lvl1(args, engine, client, P, sk, count=4096):
    """The FP64 form's rounding against the exact product at lvl1, per key
    form: both forms rotate the same `count` lvl0 inputs (the exact INT8 form
    is bit-identical to the schoolbook oracle); reported are the largest
    coefficient difference after one step (CMUX step or KeyBundle pair), and
    after the full rotation the largest coefficient difference and the
    largest phase difference (Torus32 units).  Over a full rotation the two
    ciphertexts part ways once a +-1 difference changes a gadget digit, so
    there only the phase is a rounding figure."""
    rng = np.random.default_rng(args.seed + 2000)
    bits = rng.integers(0, 2, count).astype(np.uint8)
    x = client.encrypt_bits(sk, bits, 0, seed=args.seed + 2001)
    d_x = engine.to_device(x)
    d_acc = engine.DeviceBuffer(count * P.TRLWE1_WORDS * 4)
    res = {"inputs": count, "unit": "Torus32 units (2^-32)"}
    for kb in (True, False):
        engine.initialize(client.EvalKey.generate(sk, keybundle=kb))
        accs = {}
        try:
            for form, prec in (("exact", P.INT8_EXACT), ("fp64", P.FP64_FFNT)):
                engine.set_precision(prec)
                for steps in (1, -1):
                    engine.blind_rotate(d_x, count, P.MU32, steps, acc_out=d_acc)
                    accs[form, steps] = engine.from_device(d_acc, (count, P.TRLWE1_WORDS)).copy()
        finally:
            engine.set_precision(P.FP64_FFNT)
            engine.cleanup()

        def diff(a_, b_):
            return np.abs((a_ - b_).astype(np.uint32).view(np.int32).astype(np.int64))
        d1, dn = diff(accs["fp64", 1], accs["exact", 1]), diff(accs["fp64", -1], accs["exact", -1])
        ph = 0
        for i in np.flatnonzero(dn.any(axis=1)):  # identical rotations have identical phases
            ph = max(ph, int(diff(client.trlwe_phase(sk, accs["fp64", -1][i]),
                                  client.trlwe_phase(sk, accs["exact", -1][i])).max()))
        res["kb" if kb else "plain"] = {
            "one_step_max_coef_diff": int(d1.max()),
            "one_step_coefs_differing": int(np.count_nonzero(d1)),
            "full_rotation_max_coef_diff": int(dn.max()),
            "full_rotation_coefs_differing": int(np.count_nonzero(dn)),
            "full_rotations_differing": int(np.count_nonzero(dn.any(axis=1))),
            "full_rotation_max_phase_diff": ph,
            "full_rotation_max_phase_diff_log2": float(np.log2(max(ph, 1)))}
    return res


def run_lvl02(args, torch, engine, client, P, sk, rank, ws, flush):
    """configs: lvl0 -> lvl2 NAND gate bootstrapping (Ctxt<lvl0> I/O: pre-add,
    blind rotation to N = 2048, lvl2 -> lvl0 key switching), KeyBundle,
    batches of 512 / 2048 / 8192 gates; device-resident inputs, CUDA events,
    L2 flushed between steps."""
    ek = client.EvalKey02.generate(sk, keybundle=True)
    engine.initialize_lvl02(ek)
    engine.set_precision(P.FP64_FFNT)
    rng = np.random.default_rng(args.seed + 7 + rank)
    out = {}
    kern_share = None
    for B in LVL02_BATCHES:
        a, b = (rng.integers(0, 2, B).astype(np.uint8) for _ in range(2))
        cts = [client.encrypt_bits(sk, x, 0, seed=args.seed + 500 + i) for i, x in enumerate((a, b))]
        din = [engine.to_device(x) for x in cts]
        dout = engine.DeviceBuffer(B * P.TLWE0_WORDS * 4)
        for _ in range(max(args.warmup, 3)):
            engine.gate_batch(None, B, engine.LVL02, dout, *din, uniform=P.NAND)
        torch.cuda.synchronize()
        res = engine.from_device(dout, (B, P.TLWE0_WORDS))
        fails = int(np.count_nonzero(client.decrypt_bits(sk, res, 0) != (1 - (a & b))))
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        engine.profile_reset()
        engine.profile_enable(True)
        for k in range(args.steps):
            ev[k][0].record()
            engine.gate_batch(None, B, engine.LVL02, dout, *din, uniform=P.NAND)
            ev[k][1].record()
            flush.zero_()
        torch.cuda.synchronize()
        engine.profile_enable(False)
        kern = {}
        for cls, name in enumerate(engine.K_NAMES):
            ms, n = engine.profile_read(cls)
            if n:
                kern[name] = ms / args.steps
        step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
        total = max_over_ranks(torch, sum(step_ms), "cuda")
        out[str(B)] = {"value": whole_job_rate(B, ws, args.steps, total),
                       "ms_per_step": total / args.steps, "decrypt_failures": fails,
                       "kernel_ms_per_step": kern}
        kern_share = kern
    # single NAND on an idle GPU
    lat = []
    L = engine.load()
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        engine.check(L.cufhe_gate(P.NAND, engine.LVL02, engine.dptr(dout), engine.dptr(din[0]),
                                  engine.dptr(din[1]), None, None), "gate")
        e1.record()
        torch.cuda.synchronize()
        lat.append(e0.elapsed_time(e1))
    engine.cleanup_lvl02()
    int8 = run_lvl02_int8(args, torch, engine, client, P, sk, rank, ws, flush)
    big = str(LVL02_BATCHES[-1])
    br_ms = kern_share.get("br_fp64_lvl02") if kern_share else None
    rl = None
    if br_ms:
        work = FLOP_FP64_LVL2_KB * LVL02_BATCHES[-1]
        peak = engine_peak_fp64(engine)
        ach = work / (br_ms * 1e-3) / 1e12
        rl = {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
              "frac": ach / peak, "traffic": ncu_traffic("br_fp64_lvl02"),
              "kernel": "k_br2_fp64 (FP64 FFNT blind rotation to lvl2 + SampleExtract)",
              "work_per_launch": work,
              "peak_source": "measured FP64 FMA probe on this GPU"}
    return {"metric": "lvl0->lvl2->lvl0 NAND bootstraps/s", "unit": UNIT,
            "workload": ("NAND gates, Ctxt<lvl0> I/O, lvl2 N=2048 l=4 Bgbit=10 Torus64, "
                         "KeyBundle, lvl20 key switch basebit=2 t=7"),
            "batches": out, "value": out[big]["value"],
            "single_gate_latency_ms": statistics.median(lat), "roofline": rl,
            "dtype": "f64", "int8_exact": int8}


def run_lvl02_int8(args, torch, engine, client, P, sk, rank, ws, flush):
    """The exact INT8 form of the lvl02 gates with the KeyBundle key, as the
    FP64 leg (eight key limbs x two digit limbs, INT32 accumulation; three key
    GEMMs per pair): NAND batch of LVL02_INT8_BATCH gates timed like the FP64
    form (3 warm-up, events, L2 flush, bounded to a few steps: a batch takes
    about a second), and the FP64 form's phase error against it after full
    rotations of the same 64 inputs."""
    ek = client.EvalKey02.generate(sk, keybundle=True)
    engine.initialize_lvl02(ek)
    engine.set_precision(P.INT8_EXACT)
    rng = np.random.default_rng(args.seed + 17 + rank)
    B = LVL02_INT8_BATCH
    steps = min(args.steps, 3)
    try:
        a, b = (rng.integers(0, 2, B).astype(np.uint8) for _ in range(2))
        cts = [client.encrypt_bits(sk, x, 0, seed=args.seed + 600 + i) for i, x in enumerate((a, b))]
        din = [engine.to_device(x) for x in cts]
        dout = engine.DeviceBuffer(B * P.TLWE0_WORDS * 4)
        for _ in range(max(args.warmup, 3)):
            engine.gate_batch(None, B, engine.LVL02, dout, *din, uniform=P.NAND)
        torch.cuda.synchronize()
        res = engine.from_device(dout, (B, P.TLWE0_WORDS))
        fails = int(np.count_nonzero(client.decrypt_bits(sk, res, 0) != (1 - (a & b))))
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        engine.profile_reset()
        engine.profile_enable(True)
        for k in range(steps):
            ev[k][0].record()
            engine.gate_batch(None, B, engine.LVL02, dout, *din, uniform=P.NAND)
            ev[k][1].record()
            flush.zero_()
        torch.cuda.synchronize()
        engine.profile_enable(False)
        br_ms, _ = engine.profile_read(engine.K_NAMES.index("br_int8_lvl02"))
        total = max_over_ranks(torch, sum(e0.elapsed_time(e1) for e0, e1 in ev), "cuda")
        # FP64 rounding against the exact product: phase error after a full
        # rotation (Torus64 units; the masks diverge once a step's FP64 error
        # exceeds the lowest digit weight, so only the phase is comparable)
        n = 64
        x = client.encrypt_bits(sk, a[:n], 0, seed=args.seed + 700)
        d_x = engine.to_device(x)
        d_acc = engine.DeviceBuffer(n * P.TRLWE2_WORDS * 8)
        engine.blind_rotate_lvl02(d_x, n, P.MU64, -1, acc_out=d_acc)
        exact = engine.from_device(d_acc, (n, P.TRLWE2_WORDS), np.uint64).copy()
        engine.set_precision(P.FP64_FFNT)
        engine.blind_rotate_lvl02(d_x, n, P.MU64, -1, acc_out=d_acc)
        fp64 = engine.from_device(d_acc, (n, P.TRLWE2_WORDS), np.uint64)
        err = max(float(np.abs((client.trlwe64_phase(sk, fp64[i]) -
                                client.trlwe64_phase(sk, exact[i])).view(np.int64)
                               .astype(np.float64)).max()) for i in range(n))
    finally:
        engine.set_precision(P.FP64_FFNT)
        engine.cleanup_lvl02()
    work = OPS_INT8_LVL2_KB * B
    peak = engine_peak_int8(engine)
    ach = work / (br_ms / steps * 1e-3) / 1e12 if br_ms else None
    return {"batch": B, "value": whole_job_rate(B, ws, steps, total), "steps": steps,
            "ms_per_step": total / steps, "decrypt_failures": fails,
            "fp64_phase_error_log2_torus64": float(np.log2(max(err, 1.0))),
            "fp64_phase_error_rotations": n,
            "roofline": {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TOP/s",
                         "frac": ach / peak if ach else None,
                         "kernel": "INT8 blind rotation to lvl2 (decompose + tcgen05 Toeplitz "
                                   "GEMMs per KeyBundle pair)",
                         "keybundle": True,
                         "work_per_launch": work,
                         "peak_source": "measured tcgen05.mma.kind::i8 probe on this GPU"},
            "dtype": "int8 products, int32 accumulation, Torus64 recombination"}


def run_uneven(args, torch, engine, client, P, sk, ek, rank, ws, flush, ref_rate):
    """Uneven circuits: 256 seeded levelised random DAGs of 50-2000 gates
    (fan-in 2, gate types uniform over the ten binary gates, level widths
    log-uniform 1-64) plus 64 ripple-carry adders of width 8-64 on random
    operands, merged into one wire table of Ctxt<lvl1>; the engine levelises
    it into waves (cufhe_circuit_create) and runs the waves as one CUDA graph,
    directly, and as two groups of connected components on two streams
    (cufhe_circuit_create_split), the leg's value.  Timed with CUDA events per
    full run, L2 flushed between runs; every mode's outputs are decrypted."""
    from cufhepp_b200 import circuits as CI
    net = CI.uneven_workload(args.seed + 31 * rank)
    engine.initialize(ek)
    engine.set_precision(P.FP64_FFNT)
    rng = np.random.default_rng(args.seed + 3 + rank)
    bits = rng.integers(0, 2, net.inputs.size).astype(np.uint8)
    host = np.zeros((net.num_wires, P.TLWE1_WORDS), np.uint32)
    host[net.inputs] = client.encrypt_bits(sk, bits, 1, seed=args.seed + 900 + rank)
    wires = torch.from_numpy(host.view(np.int32)).cuda()
    c = engine.Circuit(1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out)
    # the same circuit as two groups of its connected components, each on a
    # stream of its own (cufhe_circuit_create_split)
    c2 = engine.Circuit(1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out, parts=2)
    waves, max_gates, max_lanes = c.info()
    wg, wl = c.wave_sizes()
    plain = CI.evaluate(net, bits)
    res = {}
    fails = 0
    for mode, circ, graph in (("graph", c, True), ("direct", c, False), ("split2_graph", c2, True)):
        wires.copy_(torch.from_numpy(host.view(np.int32)).cuda())
        for _ in range(max(args.warmup, 3) if graph else 1):
            circ.run(wires.data_ptr(), graph=graph)
        torch.cuda.synchronize()
        n = max(2, min(args.steps, 3))
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(n)]
        if ws > 1:
            torch.distributed.barrier()
        l0 = engine.kernel_launches()
        for k in range(n):
            ev[k][0].record()
            circ.run(wires.data_ptr(), graph=graph)
            ev[k][1].record()
            flush.zero_()
        torch.cuda.synchronize()
        ms = max_over_ranks(torch, sum(e0.elapsed_time(e1) for e0, e1 in ev), "cuda") / n
        res[mode] = {"ms_per_run": ms, "value": net.bootstraps() * ws / (ms * 1e-3),
                     "gates_per_s": net.gates * ws / (ms * 1e-3),
                     "gpu_launches_per_run": (engine.kernel_launches() - l0) / n}
        out = wires.cpu().numpy().view(np.uint32)
        fails += int(np.count_nonzero(client.decrypt_bits(sk, out[net.out], 1) != plain[net.out]))
    res["split2_graph"]["waves_per_group"] = c2.info()[0]
    c.destroy()
    c2.destroy()
    engine.cleanup()
    return {"metric": "uneven-circuit bootstraps/s (whole workload per run)", "unit": UNIT,
            "workload": ("256 levelised random DAGs (50-2000 gates, fan-in 2, widths log-uniform "
                         "1-64) + 64 ripple-carry adders (width 8-64, carry by Mux), Ctxt<lvl1>"),
            "gates": net.gates, "bootstraps": net.bootstraps(), "waves": waves,
            "max_wave_gates": max_gates, "max_wave_lanes": max_lanes,
            "median_wave_lanes": float(np.median(wl)),
            "value": res["split2_graph"]["value"],
            "value_note": "the circuit as two groups of its connected components on two streams "
                          "(cufhe_circuit_create_split, CUDA graphs); one stream: graph",
            "graph": res["graph"], "direct": res["direct"], "split2_graph": res["split2_graph"],
            "decrypt_failures": fails, "gates_checked": 3 * net.gates,
            "vs_full_batch_rate": res["split2_graph"]["value"] / ref_rate if ref_rate else None,
            "dtype": "f64"}


def run_cb(args, torch, engine, client, P, sk, ek1, rank, ws, flush, gates_wl):
    """Circuit bootstrapping + CMUX lookup tables: 1024 lvl0 bits circuit-
    bootstrapped to TRGSW<lvl1> (l = 3, Bgbit = 6; three lvl0 -> lvl2 blind
    rotations and six private key switches lvl2 -> lvl1, basebit 4, t 10, per
    bit), then 128 random 8-bit -> 8-bit tables evaluated by CMUX trees over
    them; alone, and on one stream beside a 4096-gate lvl1 batch on another."""
    cbk = client.CBKey.generate(sk)
    engine.initialize(ek1)
    engine.set_precision(P.FP64_FFNT)
    engine.initialize_lvl02(cbk.ek02)
    engine.initialize_cb(cbk)
    q, nbits = 128, 1024
    rng = np.random.default_rng(args.seed + 17 + rank)
    luts = rng.integers(0, 256, (q, 256)).astype(np.uint8)
    addr = rng.integers(0, 256, q)
    bits = np.array([(int(addr[t]) >> k) & 1 for t in range(q) for k in range(8)], np.uint8)
    d_x = engine.to_device(client.encrypt_bits(sk, bits, 0, seed=args.seed + 1700 + rank))
    d_t = engine.DeviceBuffer(nbits * 6 * P.TRLWE1_WORDS * 4)
    d_f = engine.DeviceBuffer(nbits * 6 * 2 * 512 * 16)
    d_o = engine.DeviceBuffer(q * 8 * P.TLWE1_WORDS * 4)
    gates, a, b, c = gates_wl
    cts = [engine.to_device(client.encrypt_bits(sk, x, 1, seed=args.seed + 1800 + i))
           for i, x in enumerate((a, b, c))]
    g_out = engine.DeviceBuffer(gates.size * P.TLWE1_WORDS * 4)
    sa, sb = engine.Stream(), engine.Stream()
    ta = torch.cuda.ExternalStream(sa.cuda)
    tb = torch.cuda.ExternalStream(sb.cuda)

    def cb_step():
        engine.circuit_bootstrap(d_x, nbits, d_t, sa)
        engine.trgsw_to_fft(engine.GADGET_CB, d_t, nbits, d_f, sa)
        engine.lut_eval(luts, d_f, P.MU32, d_o, sa)

    def gate_step():
        engine.gate_batch(gates, gates.size, 1, g_out, *cts, stream=sb)

    def timed(fn_a, fn_b, n):
        total = 0.0
        for _ in range(n):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            ea = torch.cuda.Event()
            eb = torch.cuda.Event()
            e0.record(ta)
            tb.wait_event(e0)
            if fn_a:
                fn_a()
            if fn_b:
                fn_b()
            ea.record(ta)
            eb.record(tb)
            ta.wait_event(eb)
            e1.record(ta)
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
            flush.zero_()
        return max_over_ranks(torch, total, "cuda") / n

    for _ in range(max(args.warmup, 3)):
        cb_step()
        gate_step()
    torch.cuda.synchronize()
    n = max(2, min(args.steps, 5))
    engine.profile_reset()
    engine.profile_enable(True)
    l0 = engine.kernel_launches()
    ms_cb = timed(cb_step, None, n)
    launches = (engine.kernel_launches() - l0) / n
    engine.profile_enable(False)
    kern = {}
    for cls, name in enumerate(engine.K_NAMES):
        kms, kn = engine.profile_read(cls)
        if kn:
            kern[name] = kms / n
    ms_gates = timed(None, gate_step, n)
    ms_mixed = timed(cb_step, gate_step, n)
    out = engine.from_device(d_o, (q, 8, P.TLWE1_WORDS))
    got = client.decrypt_bits(sk, out.reshape(-1, P.TLWE1_WORDS), 1).reshape(q, 8)
    want = np.array([[(int(luts[t][addr[t]]) >> k) & 1 for k in range(8)] for t in range(q)])
    fails = int(np.count_nonzero(got != want))
    nb = bootstraps(gates)
    sa.destroy()
    sb.destroy()
    engine.cleanup_cb()
    engine.cleanup_lvl02()
    engine.cleanup()
    return {"metric": "circuit-bootstrapped bits/s (1024 bits + 128 8-bit tables per step)",
            "unit": "bits/s",
            "workload": ("1024 lvl0 bits -> TRGSW<lvl1> (l=3, Bgbit=6) by 3 lvl0->lvl2 blind "
                         "rotations + 6 private key switches lvl2->lvl1 (basebit 4, t 10) per bit; "
                         "128 random 8-bit->8-bit tables by CMUX trees (255 CMUXes each)"),
            "value": nbits * ws / (ms_cb * 1e-3), "ms_per_step": ms_cb,
            "luts_per_s": q * ws / (ms_cb * 1e-3), "kernel_ms_per_step": kern,
            "gpu_launches_per_step": launches, "decrypt_failures": fails,
            "outputs_checked": q * 8,
            "mixed": {"gate_batch": f"{gates.size} lvl1 gates ({nb} bootstraps) on a second stream",
                      "ms_gates_alone": ms_gates, "ms_cb_alone": ms_cb, "ms_both": ms_mixed,
                      "overlap_saving": 1.0 - ms_mixed / (ms_gates + ms_cb)},
            "dtype": "f64 (blind rotations, CMUX) + integer (private key switching)"}


_PEAK = {}
PROBES = {}


def _probe(kind, fn, per_clk_name, per_clk_div):
    """Best of three runs of a throughput probe, with the SM clock sampled
    while the probes ran, so that the denominator can be checked against
    clock x SMs x units: `per_clk_name` is the probe's rate per SM per clock
    (FP64 FMAs, or INT8 multiply-adds counted as 2 ops: per_clk_div = 2)."""
    import torch
    clk = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clk.start()
    t0 = time.perf_counter()
    runs = [fn() for _ in range(3)]
    while time.perf_counter() - t0 < 1.2:  # at least ~6 clock samples
        runs.append(fn())
    c = clk.stop()
    best = max(runs)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    rec = {"value": best, "runs": len(runs), "sms": sms,
           "sm_mhz_median": c["sm_mhz"] if c else None,
           "clock_reasons": c["reasons"] if c else None}
    if c and c["sm_mhz"]:
        rec[per_clk_name] = best * 1e12 / per_clk_div / (sms * c["sm_mhz"] * 1e6)
    PROBES[kind] = rec
    return best


def engine_peak_fp64(engine):
    if "fp64" not in _PEAK:
        _PEAK["fp64"] = _probe("fp64_tflops", engine.measure_fp64_peak, "dfma_per_clk_per_sm", 2)
    return _PEAK["fp64"]


def engine_peak_int8(engine):
    if "int8" not in _PEAK:
        _PEAK["int8"] = _probe("int8_tops", engine.measure_int8_peak, "i8_macs_per_clk_per_sm", 2)
    return _PEAK["int8"]


def run_ours(args):
    ws, rank, local = dist_env()
    if ws > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    import torch
    from cufhepp_b200 import client, engine, params as P
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    rng = np.random.default_rng(args.seed + rank)
    workload = make_workload(rng, args.batch)
    sk = client.SecretKey.generate(args.seed)
    paths = list(PATHS) if args.path == "all" else [args.path]
    tuned = None
    if not args.no_autotune:
        ek_t = client.EvalKey.generate(sk, keybundle=True)
        engine.initialize(ek_t)
        tuned = engine.autotune()
        engine.cleanup()
    results = {}
    for p in paths:
        results[p] = run_path(args, p, torch, engine, client, P, sk, workload, rank, ws, flush)
    primary_name = paths[0]
    primary = results[primary_name]
    # the sub-workloads are measured by a single process (N = 1); under
    # torchrun every rank runs the headline batch only
    single = ws == 1
    nand = None
    if not args.no_nand1000 and single:
        nand = run_nand1000(args, torch, engine, client, P, sk, rank, ws, flush)
    err = None
    if not args.no_error and single:
        err = fp64_error_lvl1(args, engine, client, P, sk)
    uneven = None
    if not args.no_uneven and single:
        ek_u = client.EvalKey.generate(sk, keybundle=True)
        uneven = run_uneven(args, torch, engine, client, P, sk, ek_u, rank, ws, flush,
                            results["fp64_kb"]["value"] if "fp64_kb" in results else None)
    cb = None
    if not args.no_cb and single:
        cb = run_cb(args, torch, engine, client, P, sk, client.EvalKey.generate(sk, keybundle=True),
                    rank, ws, flush, workload)
    lvl02 = None
    if not args.no_lvl02 and single:
        lvl02 = run_lvl02(args, torch, engine, client, P, sk, rank, ws, flush)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, cores, sample = cpu_gate_rate(args.seed, args.batch, keybundle=PATHS[primary_name][1])
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
               "cpu_model": cpu_model()}
        if lvl02 is not None:
            lvl02["cpu_baseline"] = cpu_gate2_rate(min(args.cpu_seconds, 8.0), args.seed)
    if rank == 0:
        form, kb = PATHS[primary_name]
        line = {
            "metric": METRIC, "value": primary["value"], "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": primary["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if form == "fp64" else "int8",
            "data": "synthetic: seeded keys, random bits",
            "config": common_config(args.batch, primary["bootstraps_per_step"]),
            "headline_path": {"name": primary_name,
                              "form": {"fp64": "FP64 FFNT", "int8": "INT8 exact (tcgen05)"}[form],
                              "keybundle": kb},
            "p50_gate_latency_ms": primary["p50_gate_latency_ms"],
            "p99_gate_latency_ms": primary["p99_gate_latency_ms"],
            "single_gate_latency_ms": primary["single_gate_latency_ms"],
            "decrypt_failures": primary["decrypt_failures"],
            "roofline": primary["roofline"], "cpu_baseline": cpu, "e2e": primary["e2e"],
            "gpu_launches": primary["gpu_launches"], "clocks": primary["clocks"],
            "kernel_ms_per_step": primary["kernel_ms_per_step"],
            "vs_reference_a100_published": primary["value"] / A100_PUBLISHED,
            "peak_probes": PROBES,
        }
        line["config"]["keybundle"] = kb
        if len(paths) > 1:
            line["paths"] = {p: {k: results[p][k] for k in
                                 ("value", "ms_per_step", "p50_gate_latency_ms",
                                  "single_gate_latency_ms", "decrypt_failures", "roofline",
                                  "kernel_ms_per_step", "keybundle", "e2e", "gpu_launches")}
                             for p in paths}
            ratio = {}
            for tag in ("kb", "plain"):
                if f"int8_{tag}" in results and f"fp64_{tag}" in results:
                    ratio[tag] = results[f"int8_{tag}"]["value"] / results[f"fp64_{tag}"]["value"]
            line["int8_vs_fp64"] = ratio
        if nand is not None:
            line["nand1000"] = nand
        if err is not None:
            line["fp64_error_lvl1"] = err
        if lvl02 is not None:
            line["lvl02"] = lvl02
        if uneven is not None:
            line["uneven"] = uneven
        if cb is not None:
            line["cb_lut"] = cb
        if not single:
            line["sub_workloads"] = ("measured at N = 1 only (nand1000, fp64_error_lvl1, uneven, "
                                     "cb_lut, lvl02)")
        line["br_lanes_per_cta"] = (
            {"source": "autotuner (cufhe_autotune)", "table": tuned} if tuned
            else {"source": "built-in rule"})
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
