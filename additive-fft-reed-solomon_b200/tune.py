"""Route tuner: measures, on the GPU it runs on, which kernel family serves
each per-call shape fastest, and writes the route table the library compiles
in (csrc/route_table.inc, read by csrc/route.cu).

For every encode shape (n, t), recover shape n and shard-length bucket
(L = 64 B, 128 B, ..., 4 MiB: bucket b covers 64 * 2^(b-1) < L <= 64 * 2^b)
it times, at the bucket's largest length, each route the C ABI can force
(afrs_ctx_set_route): the one-launch generic kernel, the specialised
kernels, for t <= 16 encodes with more than one chunk both layouts of the
specialised kernel, and for the shapes it covers (encodes with t = 32, 64;
recovers with n = 32 .. 128) the specialised kernels fused into one launch.  A call is timed as CUDA-graph replays of 10 calls on
device buffers (no host overhead), best of 3.  The fastest route wins; the
built-in rule's route is kept when it is within 3 % of the fastest.
Codewords above --max-bytes are not measured (the table entry stays -1 and
the built-in rule decides).

    python additive-fft-reed-solomon_b200/tune.py [--out PATH] [--json PATH]

then rebuild the library (make -C additive-fft-reed-solomon_b200/csrc).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
BUCKETS = 17  # L <= 64 B .. L <= 4 MiB; must match csrc/route_table.inc


def _package():
    name = "afrs_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def builtin_encode_route(n, t, L):
    """The library's rule where the table has no entry (csrc/afrs_capi.cu
    generic_encode_wins, csrc/special.cuh enc_small_split)."""
    if n * L <= (4 << 20) and ((t == 16 and n >= 32) if t <= 16 else n <= 64):
        return 0
    if t <= 16 and n // t - 1 > 1 and (t < 16 or (L + 1023) // 1024 <= 128):
        return 2
    return 1


def builtin_recover_route(n, L):
    return 0 if n == 16 and n * L <= (4 << 20) else 1


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=os.path.join(HERE, "csrc", "route_table.inc"))
    ap.add_argument("--json", default=None, help="also write every timing here")
    ap.add_argument("--max-bytes", type=int, default=256 << 20, help="largest codeword measured (n * L)")
    ap.add_argument("--reps", type=int, default=10)
    args = ap.parse_args()

    import torch

    afrs = _package()
    lib = afrs._lib
    dev = torch.device("cuda", 0)
    ctx = afrs.Context(0)
    big = torch.zeros(args.max_bytes, dtype=torch.uint8, device=dev)
    big2 = torch.zeros(args.max_bytes // 2, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(call):
        call()
        call()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            for _ in range(args.reps):
                call()
        g.replay()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(3):
            ev_a.record(stream)
            with torch.cuda.stream(stream):
                g.replay()
            ev_b.record(stream)
            ev_b.synchronize()
            best = min(best, ev_a.elapsed_time(ev_b) * 1e3 / args.reps)
        del g
        return best  # microseconds per call

    def choose(times, default):
        best = min(times, key=times.get)
        if default in times and times[default] <= 1.03 * times[best]:
            return default
        return best

    enc = [[[-1] * BUCKETS for _ in range(9)] for _ in range(9)]
    rec = [[-1] * BUCKETS for _ in range(9)]
    log = []
    t0 = time.time()
    for ln in range(1, 9):
        n = 1 << ln
        for b in range(BUCKETS):
            L = 64 << b
            if n * L > args.max_bytes:
                break
            # recover: e = n/2 erasures at spread positions (t = n/2)
            t = n // 2
            rx = big[:n * L]
            pos = list(range(0, n, 2))
            codec = afrs.Codec(n, t, context=ctx)
            times = {}
            for route in (0, 1, 3) if 32 <= n <= 128 else (0, 1):
                ctx.set_route(route + lib.AFRS_ROUTE_GENERIC)
                times[route] = timed(lambda: codec.recover_erasure_shards(rx, None, L, pos))
            rec[ln][b] = choose(times, builtin_recover_route(n, L))
            log.append({"op": "recover", "n": n, "L": L, "us": times, "route": rec[ln][b]})
            for lt in range(0, ln):
                t = 1 << lt
                msg, par = big[:(n - t) * L], big2[:t * L]
                codec = afrs.Codec(n, t, context=ctx)
                routes = (0, 1, 2) if t <= 16 and n // t - 1 > 1 else (0, 1)
                if t in (32, 64):
                    routes += (3,)
                times = {}
                for route in routes:
                    ctx.set_route(route + lib.AFRS_ROUTE_GENERIC)
                    times[route] = timed(lambda: codec.encode_parity(msg, par, L))
                enc[ln][lt][b] = choose(times, builtin_encode_route(n, t, L))
                log.append({"op": "encode", "n": n, "t": t, "L": L, "us": times, "route": enc[ln][lt][b]})
        print(f"n={n} done ({time.time() - t0:.0f} s)", flush=True)
    ctx.set_route(lib.AFRS_ROUTE_TABLE)

    name = torch.cuda.get_device_name(dev)
    lines = [
        "// Route table of the per-call kernels (see route.cu), written by",
        f"// additive-fft-reed-solomon_b200/tune.py on {name}: the fastest of the routes",
        "// timed at each bucket's largest shard length (CUDA-graph replays, best of 3);",
        "// -1 = not measured.  Regenerate with",
        "//   python additive-fft-reed-solomon_b200/tune.py",
        f"constexpr int kRouteBuckets = {BUCKETS};  // L <= 64, <= 128, ..., <= 4 MiB",
        "// [log2 n][log2 t][bucket]: 0 generic, 1 specialised, 2 specialised with split chunks,",
        "// 3 specialised in one launch",
        f"const int8_t kEncRoute[9][9][{BUCKETS}] = {{",
    ]
    for ln in range(9):
        lines.append("    {" + ", ".join("{" + ", ".join(str(v) for v in enc[ln][lt]) + "}" for lt in range(9)) + "},")
    lines += ["};", "// [log2 n][bucket]: 0 generic, 1 specialised, 3 specialised in one launch",
              f"const int8_t kRecRoute[9][{BUCKETS}] = {{"]
    for ln in range(9):
        lines.append("    {" + ", ".join(str(v) for v in rec[ln]) + "},")
    lines.append("};")
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    if args.json:
        with open(args.json, "w") as f:
            json.dump({"device": name, "reps": args.reps, "entries": log}, f)
    print(f"wrote {args.out} ({len(log)} entries, {time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
