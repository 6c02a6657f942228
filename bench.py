"""Benchmark: sharded RS encode + 128-erasure recover, n=256, k=128, 64 KiB
shards (the reference's bandwidth case), on B200.

One step = encode of one codeword (k*L read, t*L written) + recover of t
uniformly random erasures of one codeword ((n-t)*L read, t*L written); the
metric counts n*L bytes per operation (shards read + shards written).
Inputs rotate over enough codewords that every step reads data that is not
in L2.  Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
  python bench.py --workload {small,batched,serving,large}   (other configs)

--impl reference times the reference's CPU algorithm instead: the reference
is a Rust crate and no Rust toolchain exists here, so its GFNI kernel
(rs/src/kernel/gfni_kernel.rs) and codec sequence (rs/src/codec.rs) are timed
as their C restatement in oracle/gfni_baseline.c, on all host cores.
"""
from __future__ import annotations

import argparse
import math
import threading
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SHARDS, T_PARITY, SHARD_LEN = 256, 128, 65536
METRIC = "encode & recover GB/s (% of HBM peak)"
WORKLOAD = "n=256 k=128 t=128, 64 KiB shards: encode + recover of 128 random erasures (one codeword each)"


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of each kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []  # (perf_counter when read, line)
        self.window = (None, None)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return

        def read():
            for line in self.proc.stdout:
                self.lines.append((time.perf_counter(), line))

        self.reader = threading.Thread(target=read, daemon=True)
        self.reader.start()

    def mark(self, begin: bool):
        """Marks the start or the end of the timed region (host clock)."""
        b, e = self.window
        self.window = (time.perf_counter(), e) if begin else (b, time.perf_counter())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.reader.join(timeout=5)
        b, e = self.window
        inside = [ln for ts, ln in self.lines if b is not None and e is not None and b <= ts <= e + 0.15]
        rows = inside or [ln for _, ln in self.lines]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in rows:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "in_timed_region": bool(inside)}


_PER_PAIR = None


def cpu_per_pair() -> float:
    """Seconds for one encode + one recover on one host thread (probed once)."""
    global _PER_PAIR
    if _PER_PAIR is None:
        from oracle import oracle

        n, t, L = N_SHARDS, T_PARITY, SHARD_LEN
        probe_e = oracle.gfni_throughput("encode", n, t, L, 1, 1)
        probe_r = oracle.gfni_throughput("recover", n, t, L, 1, 1)
        _PER_PAIR = n * L / probe_e + n * L / probe_r
    return _PER_PAIR


def host_cpu() -> dict:
    """Model and vector features of the host cores the CPU baseline runs on."""
    model, flags = "unknown", set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                key, _, val = line.partition(":")
                key = key.strip()
                if key == "model name" and model == "unknown":
                    model = val.strip()
                elif key == "flags" and not flags:
                    flags = set(val.split())
    except OSError:
        pass
    return {"cpu": model, "gfni": "gfni" in flags, "avx512f": "avx512f" in flags}


def cpu_baseline(seconds: float, threads: int):
    """GFNI restatement of the reference's kernel + codec on host cores, on a
    bounded sample of the same workload (same n, t, L): about `seconds` of
    work, at least one encode and one recover per thread."""
    from oracle import oracle

    n, t, L = N_SHARDS, T_PARITY, SHARD_LEN
    iters = max(1, int(seconds / max(cpu_per_pair(), 1e-6) / 2))
    enc = oracle.gfni_throughput("encode", n, t, L, iters, threads, 42)
    rec = oracle.gfni_throughput("recover", n, t, L, iters, threads, 43)
    combined = 2.0 / (1.0 / enc + 1.0 / rec)  # same mix as one GPU step: one encode + one recover
    sample = f"{iters} encodes + {iters} recovers of one n=256 t=128 L=64KiB codeword per thread, {threads} threads"
    return combined / 1e9, enc / 1e9, rec / 1e9, sample


def max_over_ranks(value: float, world: int, device) -> float:
    """The largest of one number over all ranks (the slowest rank's time);
    every rank takes part and gets the result."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gbs(bytes_per_rank_step: float, world: int, steps: int, max_seconds: float) -> float:
    """Whole-job throughput: all ranks' bytes over the slowest rank's time."""
    return world * bytes_per_rank_step * steps / max_seconds / 1e9


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    vals = []
    enc = rec = 0.0
    sample = ""
    # Each step is a sample of about min(2 s, 90 s / steps) of CPU work (at
    # least one encode + one recover per thread); samples are taken until
    # `steps` are done or 90 s of wall time have passed (at least 3), so the
    # run stays within a few minutes for any --steps.
    per_step = min(2.0, 90.0 / max(1, args.steps))
    for _ in range(min(args.warmup, 3)):
        cpu_baseline(per_step, threads)
    t0 = time.perf_counter()
    samples = 0
    while samples < args.steps and (samples < 3 or time.perf_counter() - t0 < 90.0):
        v, enc, rec, sample = cpu_baseline(per_step, threads)
        vals.append(v)
        samples += 1
    wall = time.perf_counter() - t0
    sample = f"{samples} samples of {sample}"
    value = statistics.median(vals)
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * wall / samples, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": N_SHARDS, "k": N_SHARDS - T_PARITY, "t": T_PARITY,
                   "shard_len": SHARD_LEN, "erasures": T_PARITY},
        "encode_gbs": round(enc, 3), "recover_gbs": round(rec, 3),
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": sample + " (C restatement of rs/src/kernel/gfni_kernel.rs; no Rust toolchain)",
                         **host_cpu()},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="afrs", choices=["afrs", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serial", action="store_true", help="encode and recover of a step on one stream")
    ap.add_argument("--pairs", type=int, default=2, help="stream pairs the steps go to round-robin")
    ap.add_argument("--no-graphs", action="store_true", help="launch eagerly instead of replaying CUDA graphs")
    ap.add_argument("--e2e-pairs", type=int, default=3, help="host thread pairs (encode + recover) of the e2e line")
    ap.add_argument("--workload", default="codeword", choices=["codeword", "small", "batched", "serving", "large", "kernels"])
    ap.add_argument("--shard-len", type=int, default=0, help="--workload large: shard length (default 4 MiB)")
    ap.add_argument("--priority", default="none", choices=["none", "recover", "encode"],
                    help="give this operation's streams the higher CUDA stream priority")
    ap.add_argument("--work-cap", type=int, default=0,
                    help="scratch cap (bytes) of the device-path contexts (afrs_ctx_set_work_cap; 0 = default)")
    ap.add_argument("--host-mode", default="auto", choices=["auto", "staged", "direct"],
                    help="how the e2e line's host-buffer calls move data (afrs_ctx_set_staging)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "codeword":
        import bench_workloads  # noqa: E402  (secondary configurations)

        return bench_workloads.run(args.workload, args)

    import numpy as np
    import torch
    import torch.distributed as dist

    import __graft_entry__

    afrs = __graft_entry__.load_package()
    from oracle import oracle

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    n, t, L = N_SHARDS, T_PARITY, SHARD_LEN
    k = n - t
    op_bytes = n * L
    # 16 codewords per role: 16 * (16 MiB encode + 16 MiB recover) = 512 MiB > L2
    # (24 when the stream pairs do not divide 16).
    pairs = 1 if args.serial else args.pairs
    R = 16 if 16 % pairs == 0 else 8 * pairs
    rng = np.random.default_rng(1234 + rank)
    msg0 = oracle.random_bytes(k * L, 42 + rank)
    par0 = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg0, par0, L)
    cw0 = np.concatenate([par0, msg0])
    enc_bufs, rec_bufs, patterns = [], [], []
    dev = torch.device("cuda", local)
    for r in range(R):
        m = torch.from_numpy(oracle.random_bytes(k * L, 1000 + r) if r else msg0).to(dev)
        enc_bufs.append((m, torch.zeros(t * L, dtype=torch.uint8, device=dev)))
        pos = sorted(rng.choice(n, t, replace=False).tolist())
        rx = cw0.copy()
        for p in pos:
            rx[p * L:(p + 1) * L] = 0
        rec_bufs.append(torch.from_numpy(rx).to(dev))
        patterns.append(pos)
    # One context per operation and stream pair: with overlap, the encode of
    # one codeword and the recover of another run concurrently on two streams,
    # and consecutive steps go round-robin to `pairs` such stream pairs (a
    # context's scratch serves one operation at a time).  `pairs` divides R,
    # so the steps that reuse a codeword buffer stay on one pair, in order.
    stream = torch.cuda.current_stream(dev)
    overlap = not args.serial
    S = pairs
    assert R % S == 0, "--pairs must divide the number of rotating codewords"
    codec_e = [afrs.Codec(n, t, device=local, context=afrs.Context(local)) for _ in range(S)]
    codec_r = [afrs.Codec(n, t, device=local, context=afrs.Context(local)) for _ in range(S)]
    if args.work_cap:
        for cdc in codec_e + codec_r:
            cdc.ctx.set_work_cap(args.work_cap)
    pe = -1 if args.priority == "encode" else 0
    pr = -1 if args.priority == "recover" else 0
    s_enc = [torch.cuda.Stream(dev, priority=pe) if overlap else stream for _ in range(S)]
    s_rec = [torch.cuda.Stream(dev, priority=pr) if overlap else stream for _ in range(S)]

    def enc_call(r):
        m, p = enc_bufs[r]
        codec_e[r % S].encode_parity(m, p, L)

    def rec_call(r):
        codec_r[r % S].recover_erasure_shards(rec_bufs[r], None, L, patterns[r])

    for i in range(max(args.warmup, S)):
        with torch.cuda.stream(s_enc[i % S]):
            enc_call(i % R)
        with torch.cuda.stream(s_rec[i % S]):
            rec_call(i % R)
    torch.cuda.synchronize()
    # correctness of the measured path on codeword 0
    assert (enc_bufs[0][1].cpu().numpy() == par0).all(), "encode mismatch vs oracle"
    assert (rec_bufs[0].cpu().numpy() == cw0).all(), "recover mismatch vs oracle"

    # CUDA graphs: each operation on each of the R codewords is captured once
    # (the erasure locator of its pattern is computed on the host at capture)
    # and replayed, so the timed steps carry no host launch overhead.
    use_graphs = not args.no_graphs
    launches_per_step = None
    if use_graphs:
        cap = torch.cuda.Stream(dev)
        g_enc, g_rec = [], []
        l0 = afrs.lib().afrs_kernel_launches()
        for r in range(R):
            ge, gr = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
            with torch.cuda.graph(ge, stream=cap):
                enc_call(r)
            with torch.cuda.graph(gr, stream=cap):
                rec_call(r)
            g_enc.append(ge)
            g_rec.append(gr)
        launches_per_step = (afrs.lib().afrs_kernel_launches() - l0) / R

    def step(i, ev=None):
        se, sr = s_enc[i % S], s_rec[i % S]
        with torch.cuda.stream(se):
            if ev is not None:
                ev[0].record(se)
            g_enc[i % R].replay() if use_graphs else enc_call(i % R)
            if ev is not None:
                ev[1].record(se)
        with torch.cuda.stream(sr):
            if ev is not None:
                ev[2].record(sr)
            g_rec[i % R].replay() if use_graphs else rec_call(i % R)
            if ev is not None:
                ev[3].record(sr)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()

    # One graph per rotation of the R codewords (both operations of every
    # step on the pairs' streams, forked from and joined back into the
    # capture stream): the timed steps then cost one host launch per R steps.
    g_rot = None
    if use_graphs and overlap:
        g_rot = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(dev)
        with torch.cuda.graph(g_rot, stream=cap):
            for x in s_enc + s_rec:
                x.wait_stream(cap)
            for i in range(R):
                with torch.cuda.stream(s_enc[i % S]):
                    enc_call(i)
                with torch.cuda.stream(s_rec[i % S]):
                    rec_call(i)
            for x in s_enc + s_rec:
                cap.wait_stream(x)
        g_rot.replay()
        torch.cuda.synchronize()

    full_rot = args.steps // R if g_rot is not None else 0
    n_step = args.steps - full_rot * R  # steps replayed one by one, with events
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(n_step)]
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)

    def timed_region(events):
        """Exactly args.steps steps between two events on `stream`, with a
        barrier and a device synchronisation on both sides."""
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        for x in s_enc + s_rec:
            x.wait_stream(stream)
        with torch.cuda.stream(stream):
            for _ in range(full_rot):
                g_rot.replay()
        for x in s_enc + s_rec:
            x.wait_stream(stream)
        for i in range(n_step):
            step(i, evs[i] if events else None)
        for x in s_enc + s_rec:
            stream.wait_stream(x)
        end.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return start.elapsed_time(end)

    # The timed region (exactly args.steps steps) is repeated until the
    # repetitions cover at least 0.5 s of device time, so that a short region
    # is not a single noisy sample and the clock sampler sees the GPU under
    # load; the reported time is the median region.
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = afrs.lib().afrs_kernel_launches()
    clocks.mark(True)
    region_ms = [timed_region(True)]
    launches = afrs.lib().afrs_kernel_launches() - launches0
    repeats = int(min(5000, max(1, math.ceil(500.0 / max(region_ms[0], 1e-3)))))
    if world > 1:  # every rank repeats the region the same number of times
        rep_t = torch.tensor([repeats], dtype=torch.int64, device=dev)
        dist.all_reduce(rep_t, op=dist.ReduceOp.MAX)
        repeats = int(rep_t.item())
    for _ in range(repeats - 1):
        region_ms.append(timed_region(False))
    clocks.mark(False)
    if use_graphs:
        launches = int(round(launches_per_step * args.steps))  # kernel nodes replayed per region
    clk = clocks.stop()
    assert (enc_bufs[0][1].cpu().numpy() == par0).all(), "encode mismatch after the timed steps"
    assert (rec_bufs[0].cpu().numpy() == cw0).all(), "recover mismatch after the timed steps"
    elapsed_ms = statistics.median(region_ms)
    enc_ms = [e[0].elapsed_time(e[1]) for e in evs]
    rec_ms = [e[2].elapsed_time(e[3]) for e in evs]
    in_step = bool(enc_ms and rec_ms)
    elapsed_ms = max_over_ranks(elapsed_ms, world, dev)

    ms_per_step = elapsed_ms / args.steps
    value = aggregate_gbs(2 * op_bytes, world, args.steps, elapsed_ms * 1e-3)
    enc_avg = statistics.mean(enc_ms) if in_step else None
    rec_avg = statistics.mean(rec_ms) if in_step else None

    # Roofline of the dominant operation: with several operations sharing the
    # GPU in the timed steps, each one's event-timed duration includes the
    # sharing, so the operations are also timed one at a time (same graphs and
    # inputs, CUDA events on the launching stream).
    def isolated_ms(run_op, reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            for i in range(3):
                run_op(i)
            a.record(stream)
            for i in range(reps):
                run_op(i)
            b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    reps = max(16, min(args.steps, 400))
    enc_iso = isolated_ms(lambda i: g_enc[i % R].replay() if use_graphs else enc_call(i % R), reps)
    rec_iso = isolated_ms(lambda i: g_rec[i % R].replay() if use_graphs else rec_call(i % R), reps)
    peak, peak_kind = measured_peak_gbs()
    dom = "recover" if rec_iso >= enc_iso else "encode"
    dom_ms = max(enc_iso, rec_iso)
    achieved = op_bytes / (dom_ms * 1e-3) / 1e9
    achieved_in_steps = (op_bytes / ((rec_avg if dom == "recover" else enc_avg) * 1e-3) / 1e9) if in_step else None
    traffic = profile_traffic().get(dom)

    # End to end through the public host-buffer API (pinned host memory):
    # every step copies its inputs in and its results out.  A storage node
    # serves many stripes at once, so `e2e_pairs` pairs of host threads (one
    # encoding, one recovering, each through its own context and its own
    # codeword buffers; the C calls release the GIL) run their steps back to
    # back, and the value is all their steps over the wall time of the run.
    # With --serial one thread runs encode then recover per step.
    P = args.e2e_pairs if overlap else 1
    h_msg = torch.from_numpy(msg0).pin_memory().numpy()
    h_rx_src = rec_bufs[0].cpu().numpy().copy()
    pos0 = patterns[0]
    for p in pos0:
        h_rx_src[p * L:(p + 1) * L] = 0
    h_pars = [torch.zeros(t * L, dtype=torch.uint8).pin_memory().numpy() for _ in range(P)]
    h_rxs = [torch.from_numpy(h_rx_src).pin_memory().numpy() for _ in range(P)]
    e2e_codecs = [(codec_e[i], codec_r[i]) if i < S else
                  (afrs.Codec(n, t, device=local, context=afrs.Context(local)),
                   afrs.Codec(n, t, device=local, context=afrs.Context(local))) for i in range(P)]
    e2e_steps = max(3, min(args.steps, 150))
    mode = {"auto": afrs._lib.AFRS_HOST_AUTO, "staged": afrs._lib.AFRS_HOST_STAGED,
            "direct": afrs._lib.AFRS_HOST_DIRECT}[args.host_mode]
    for pair in e2e_codecs:
        for cdc in pair:
            afrs.codec._check(afrs.lib().afrs_ctx_set_staging(cdc.ctx.handle, 0, 0, mode), "afrs_ctx_set_staging")

    def e2e_encode(i):
        e2e_codecs[i][0].encode_parity(h_msg, h_pars[i], L)

    def e2e_recover(i):
        # The decoder reads only the surviving shards and rewrites the erased
        # ones, so repeated steps on one buffer move the same bytes.
        e2e_codecs[i][1].recover_erasure_shards(h_rxs[i], None, L, pos0)

    for i in range(P):
        for _ in range(2):
            e2e_encode(i)
            e2e_recover(i)
        assert (h_pars[i] == par0).all() and (h_rxs[i] == cw0).all(), "host-API result mismatch"

    def staged():
        import ctypes

        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        afrs.lib().afrs_staged_bytes(ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def worker(fn, i):
        for _ in range(e2e_steps):
            fn(i)

    s0 = staged()
    t0 = time.perf_counter()
    if overlap:
        workers = [threading.Thread(target=worker, args=(fn, i)) for i in range(P) for fn in (e2e_encode, e2e_recover)]
        for w in workers:
            w.start()
        for w in workers:
            w.join()
    else:
        for _ in range(e2e_steps):
            e2e_encode(0)
            e2e_recover(0)
    e2e_time = time.perf_counter() - t0
    s1 = staged()
    for i in range(P):
        assert (h_pars[i] == par0).all() and (h_rxs[i] == cw0).all(), "host-API result mismatch"
    e2e_total = P * e2e_steps
    e2e_time = max_over_ranks(e2e_time, world, dev)
    e2e_value = aggregate_gbs(2 * op_bytes, world, e2e_total, e2e_time)
    h2d_step, d2h_step = (s1[0] - s0[0]) // e2e_total, (s1[1] - s0[1]) // e2e_total

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, ce, cr, sample = cpu_baseline(args.cpu_seconds, threads)
        cpu = {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample,
               "encode_gbs": round(ce, 3), "recover_gbs": round(cr, 3), **host_cpu()}

    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "k": k, "t": t, "shard_len": L, "erasures": t,
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "work_cap": args.work_cap or None,
                   "stream_priority": args.priority,
                   "overlap": (f"encode and recover of a step on two streams; steps round-robin over {S} "
                               "stream pairs (own contexts)") if overlap else "encode then recover on one stream",
                   "launch": ("one CUDA graph per rotation of the codewords (all streams), replayed"
                              if g_rot is not None else "CUDA graph per operation and codeword, replayed")
                   if use_graphs else "eager",
                   "l2": f"inputs rotate over {R} encode + {R} recover codewords ({R * 2 * op_bytes >> 20} MiB > 126 MB L2)"},
        "encode_gbs": round(op_bytes / (enc_iso * 1e-3) / 1e9, 2),
        "recover_gbs": round(op_bytes / (rec_iso * 1e-3) / 1e9, 2),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes": op_bytes,
                     "timing": f"{dom} alone, {reps} graph replays, mean {dom_ms * 1e3:.1f} us",
                     "achieved_while_sharing_gpu": round(achieved_in_steps, 2) if in_step else None},
        "cpu_baseline": cpu,
        "clocks": clk,
        "e2e": {"value": round(e2e_value, 3), "unit": "GB/s",
                "h2d_bytes_per_step": int(h2d_step), "d2h_bytes_per_step": int(d2h_step),
                "steps": e2e_total,
                "how": (f"host-buffer API, page-locked buffers, staging {args.host_mode}; {P} pairs of host threads "
                        "(encode, recover), own contexts and codewords, steps back to back; wall time") if overlap
                       else "host-buffer API, page-locked buffers; encode then recover per step, one thread"},
        "gpu_launches": int(launches),
        "timed_regions": {"count": len(region_ms), "median_ms": round(statistics.median(region_ms), 5),
                          "min_ms": round(min(region_ms), 5), "max_ms": round(max(region_ms), 5),
                          "how": f"each region {args.steps} steps between CUDA events, repeated to >= 0.5 s; "
                                 "value and ms_per_step from the median region (max over ranks)"},
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
