#!/usr/bin/env python
"""Headline benchmark: symmetric-heap all-reduce GB/s on one B200.

Workload (the plain-method GPU configuration): 64 emulated PEs, 2^20
elements per PE, in a 4 GiB symmetric heap (64 slices x 64 MiB):
  float32 SUM  (values N(0,1)),
  float64 MAX  (values uniform in [-1e6, 1e6]),
  int64   XOR  (uniform random bits),
each in the recursive-doubling and the Rabenseifner combine order.
One step = these 6 reductions.  Algorithmic bytes per reduction are
2*P*N*sizeof(T) (every source read once, every dest written once), so a
step moves 5 GiB.  Every launch reads >= 256 MiB, more than the 126 MB
L2, so no flush is needed between iterations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference's own CPU implementation of the same
reductions (its src/shcoll/src code, compiled unmodified into
oracle/_ref and run over emulated PEs on the host cores) on a bounded
sample of the workload.  Under torchrun, every rank runs its own
independent 64-PE team on its own GPU (weak scaling, no data-path
collective); rank 0 prints one JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "osss-ucx_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "reduce/alltoall GB/s vs HBM peak; batched ops/s + p99 latency vs per-call"
P = 64
N = 1 << 20
HEAP = 64 << 20
OPS = [("sum", "float32", np.float32), ("max", "float64", np.float64), ("xor", "int64", np.int64)]
ALGOS = ["rec_dbl", "rabenseifner"]
FALLBACK_HBM = 6650.0


def workload_desc(n_gpus):
    return {"workload": f"allreduce over 64 emulated PEs x {N} elems/PE: f32 sum N(0,1), "
                        "f64 max U(-1e6,1e6), i64 xor U(bits); rec_dbl and rabenseifner orders",
            "npes": P, "nelems_per_pe": N, "heap_bytes": P * HEAP,
            "ops": [f"{d}:{o}" for o, d, _ in OPS], "algos": ALGOS,
            "l2": "inputs larger than L2 (>= 256 MiB read per launch), no flush",
            "parallelism": f"{n_gpus} independent 64-PE teams, one per GPU"}


def inputs(seed_base=0, which=(0, 1, 2)):
    import gen
    make = [lambda: gen.normal(np.float32, P, N, 21 + seed_base),
            lambda: gen.uniform(np.float64, P, N, 22 + seed_base, -1e6, 1e6),
            lambda: gen.uniform_int(np.int64, P, N, 23 + seed_base)]
    return [make[i]() if i in which else None for i in range(3)]


def alg_bytes(npes, n, dt):
    return 2 * npes * n * np.dtype(dt).itemsize


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU: the reference's own shcoll code over emulated PEs
# ---------------------------------------------------------------------------
_CPU_INPUTS = {}


def cpu_reference_times(n_sample=N, warmup=1, iters=3):
    """Per-iteration seconds of one step (the 3 ops x 2 orders) of the
    reference's own shcoll code on P=64 emulated PEs (one pinned pthread
    each) with n_sample elements per PE.  Returns (step_seconds[iters],
    bytes_per_step, description, kind)."""
    import oracle
    if n_sample not in _CPU_INPUTS:
        _CPU_INPUTS[n_sample] = inputs_small(n_sample)
    xs = _CPU_INPUTS[n_sample]
    tnames = {"float32": "float", "float64": "double", "int64": "int64"}
    step = np.zeros(iters)
    nbytes = 0
    if oracle.Reference.available:
        R, kind = oracle.Reference(), "reference"
        for (op, dt, npdt), x in zip(OPS, xs):
            for algo in ALGOS:
                _, times = R.reduce(algo, op, x, tname=tnames[dt], warmup=warmup, iters=iters,
                                    pin=True)
                step += times
                nbytes += alg_bytes(P, n_sample, npdt)
        desc = (f"full workload: 64 emulated PEs (pinned pthreads) x {n_sample} elems/PE, "
                f"3 ops x 2 orders per step; the reference's src/shcoll/src code compiled "
                f"unmodified (oracle/_ref); {iters} timed steps after {warmup} warm-up")
    else:
        rs, kind = oracle.Restatement(), "port"
        for (op, dt, npdt), x in zip(OPS, xs):
            for algo in ALGOS:
                for _ in range(warmup):
                    rs.reduce(algo, op, x)
                for k in range(iters):
                    t0 = time.perf_counter()
                    rs.reduce(algo, op, x)
                    step[k] += time.perf_counter() - t0
                nbytes += alg_bytes(P, n_sample, npdt)
        desc = f"C restatement (oracle/shcoll_oracle.c), single thread, 64 PEs x {n_sample} elems/PE"
    return step, nbytes, desc, kind


def inputs_small(n):
    import gen
    return [gen.normal(np.float32, P, n, 21), gen.uniform(np.float64, P, n, 22, -1e6, 1e6),
            gen.uniform_int(np.int64, P, n, 23)]


def run_reference_arm(args, rank):
    if rank != 0:
        return
    step, nbytes, desc, kind = cpu_reference_times(warmup=args.warmup, iters=args.steps)
    value = nbytes / float(np.median(step)) / 1e9
    cores = os.cpu_count() or 1 if kind == "reference" else 1
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GB/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(float(np.median(step)) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64+i64", "data": "synthetic (seeded per PE)",
            "config": workload_desc(args.gpus),
            "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": cores, "kind": kind,
                             "sample": desc},
            "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "config1": config1_cpu_reference()}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def max_over_ranks(ms, dist, device):
    """The job's time for a step: the slowest rank's (every rank runs its
    own team on its own GPU, so the job is done when the last one is)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gbs(bytes_per_rank_step, steps, world, ms):
    """Whole-job throughput: the bytes all ranks moved over the job's time."""
    return bytes_per_rank_step * steps * world / (ms / 1e3) / 1e9


def main():
    global N
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--case", action="append", default=[],
                    help="time only dtype:op:algo (repeatable), e.g. float32:sum:rec_dbl")
    ap.add_argument("--heap-mb", type=int, default=HEAP >> 20, help="heap slice per PE (MiB)")
    ap.add_argument("--nelems", type=int, default=N, help="elements per PE")
    ap.add_argument("--workload", default="reduce",
                    choices=["reduce", "movement", "batch", "serve", "span"],
                    help="reduce (headline), movement (alltoall/alltoalls/fcollect/AMO), "
                         "batch (4096 reductions over 512 teams of 2048 PEs), serve "
                         "(open-loop request stream over 256 PEs) or span (the kernels of a "
                         "team spanning 8 GPUs, the 8 arenas emulated on one GPU)")
    ap.add_argument("--serve-requests", type=int, default=100000)
    ap.add_argument("--serve-rate", type=float, default=200000.0, help="arrivals per second")
    ap.add_argument("--serve-percall", type=int, default=20000,
                    help="requests replayed through the per-call entry points")
    ap.add_argument("--batch-npes", type=int, default=2048)
    ap.add_argument("--batch-teams", type=int, default=512)
    ap.add_argument("--batch-reductions", type=int, default=4096)
    ap.add_argument("--batch-tune", default="auto", choices=["auto", "off"],
                    help="batch workload: the autotuner (auto, the default) or the heuristic plan")
    ap.add_argument("--movement-npes", type=int, default=128,
                    help="movement workload: PEs (128 is the configuration; 64 keeps profiling "
                         "captures to a few GB)")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the config1/movement/batch/serve/span sub-objects of the default line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    if args.workload != "reduce":
        fn = {"movement": run_movement, "batch": run_batch, "serve": run_serve,
              "span": run_span}[args.workload]
        line = fn(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import __graft_entry__
    __graft_entry__.build_library()
    import b200shm as B
    N = args.nelems
    B.init(P, args.heap_mb << 20)
    team = (0, 1, P)
    calls = [(op, dt, algo, i, npdt) for i, (op, dt, npdt) in enumerate(OPS) for algo in ALGOS]
    if args.case:
        calls = [c for c in calls if f"{c[1]}:{c[0]}:{c[2]}" in args.case]
        if not calls:
            raise SystemExit("no reduction matches --case " + ",".join(args.case))
    used = sorted({c[3] for c in calls})
    xs = inputs(seed_base=rank * 100, which=used)
    dst = B.malloc(max(xs[i][0].nbytes for i in used))
    srcs = [None] * 3
    for i in used:
        srcs[i] = B.malloc(xs[i][0].nbytes)
        B.put_rows(srcs[i], xs[i], team=team)
    calls = [(op, dt, algo, srcs[i], npdt, i) for op, dt, algo, i, npdt in calls]
    stream_ptr = B.stream()
    s = torch.cuda.ExternalStream(stream_ptr)
    step_bytes = sum(alg_bytes(P, N, c[4]) for c in calls)

    def step(evs=None):
        for j, (op, dt, algo, so, _, _) in enumerate(calls):
            if evs is not None:
                evs[j][0].record(s)
            B.reduce(op, dt, algo, dst, so, N, team=team, stream=stream_ptr)
            if evs is not None:
                evs[j][1].record(s)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    B.quiet()
    barrier()

    per_call = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                 for _ in calls] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = B.launch_count()
    start.record(s)
    for k in range(args.steps):
        step(per_call[k])
    end.record(s)
    B.quiet()
    launches = B.launch_count() - launches0
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(start.elapsed_time(end), dist, "cuda")
    value = job_gbs(step_bytes, args.steps, world, ms)

    # per-kernel durations (the reduce kernel of each (dtype, op, order))
    durs = {}
    for j, (op, dt, algo, _, npdt, _) in enumerate(calls):
        d = [per_call[k][j][0].elapsed_time(per_call[k][j][1]) for k in range(args.steps)]
        durs[f"{dt}:{op}:{algo}"] = (float(np.mean(d)), alg_bytes(P, N, npdt))
    dom = max(durs, key=lambda k: durs[k][0])
    dom_ms, dom_bytes = durs[dom]
    peak, peak_kind = peaks()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "reduce_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(dom)

    # e2e: host buffers in, reduce, host buffers out, through the C ABI
    e2e = None
    if args.e2e_steps > 0:
        pinned_in = {i: torch.from_numpy(xs[i]).pin_memory() for i in used}
        pinned_out = {i: torch.empty(xs[i].shape, dtype=pinned_in[i].dtype).pin_memory()
                      for i in used}
        h2d = d2h = 0

        def e2e_step():
            nonlocal h2d, d2h
            h2d = d2h = 0
            for op, dt, algo, so, npdt, i in calls:
                nb = xs[i][0].nbytes
                rc = B.lib.b200shm_reduce_host(B.OPS.index(op), B.DTYPES.index(dt),
                                               B.ALGOS.index(algo), 0, 1, P,
                                               pinned_out[i].data_ptr(), nb,
                                               pinned_in[i].data_ptr(), nb, dst, so, N,
                                               stream_ptr)
                if rc:
                    raise B.B200Error(rc, B.lib.b200shm_last_error().decode())
                h2d += P * nb
                d2h += P * nb
        e2e_step()
        B.quiet()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.e2e_steps):
            e2e_step()
        e1.record(s)
        B.quiet()
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
        # the transfer bound: the same bytes in and out over PCIe with no
        # reduction, the two directions on two streams at once
        dev_in = {i: torch.empty(xs[i].shape, dtype=pinned_in[i].dtype, device="cuda")
                  for i in used}
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

        def copy_step():
            for _, _, _, _, _, i in calls:
                with torch.cuda.stream(s_in):
                    dev_in[i].copy_(pinned_in[i], non_blocking=True)
                with torch.cuda.stream(s_out):
                    pinned_out[i].copy_(dev_in[i], non_blocking=True)
        copy_step()
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(s)
        for st_ in (s_in, s_out):
            st_.wait_event(c0)
        for _ in range(args.e2e_steps):
            copy_step()
        for st_ in (s_in, s_out):
            s.wait_stream(st_)
        c1.record(s)
        torch.cuda.synchronize()
        cms = max_over_ranks(c0.elapsed_time(c1), dist, "cuda")
        del dev_in
        e2e = {"value": round(job_gbs(step_bytes, args.e2e_steps, world, ems), 3),
               "unit": "GB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "steps": args.e2e_steps, "ms_per_step": round(ems / args.e2e_steps, 3),
               "path": "b200shm_reduce_host (pinned host rows in and out; copy in, reduce and "
                       "copy out pipelined in chunks on three streams)",
               "transfer_bound": {"copy_only_ms_per_step": round(cms / args.e2e_steps, 3),
                                  "frac": round(cms / ems, 4),
                                  "what": "the same host->device and device->host bytes with no "
                                          "reduction, both directions at once (pinned memory)"}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        step_s, nbytes, desc, kind = cpu_reference_times()
        cpu = {"value": round(nbytes / float(np.median(step_s)) / 1e9, 4), "unit": "GB/s",
               "cores": (os.cpu_count() or 1) if kind == "reference" else 1, "kind": kind,
               "sample": desc, "seconds_per_step": round(float(np.median(step_s)), 4)}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    extras = {}
    if world == 1 and not args.headline_only and not args.case and N == 1 << 20:
        # the other configurations, each in its own arena, after the headline
        B.finalize()
        for name, fn in (("config1", run_config1), ("movement", run_movement),
                         ("batch", run_batch), ("serve", run_serve), ("span", run_span)):
            t0 = time.perf_counter()
            try:
                extras[name] = fn(args, world, rank, local)
            except Exception as e:  # the headline line is printed whatever happens here
                extras[name] = {"error": "%s: %s" % (type(e).__name__, e)}
                if B.initialized():
                    B.finalize()
            extras[name]["run_seconds"] = round(time.perf_counter() - t0, 1)
    line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64+i64", "data": "synthetic (seeded per PE: N(0,1), U(+-1e6), U(bits))",
            "config": workload_desc(world),
            "roofline": {"bound": "hbm", "kernel": f"k_reduce {dom}", "achieved": round(achieved, 1),
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_kind": peak_kind, "traffic": traffic,
                         "bytes_per_launch": dom_bytes, "avg_launch_ms": round(dom_ms, 4)},
            "per_kernel_ms": {k: round(v[0], 4) for k, v in durs.items()},
            "per_kernel_gbs": {k: round(v[1] / (v[0] / 1e3) / 1e9, 1) for k, v in durs.items()},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk}
    line.update(extras)
    print(json.dumps(line), flush=True)

# ---------------------------------------------------------------------------
# config 1: 8 PEs, int32 sum reduce + fcollect64 + barrier_all, latency
# ---------------------------------------------------------------------------
def config1_cpu_reference(reps=300):
    """The reference's own shcoll code for config 1 over 8 emulated PEs on
    the host: median microseconds per call (None without oracle/_ref)."""
    import gen
    import oracle
    if not oracle.Reference.available:
        return None
    x, fc = gen.config1_inputs()
    R = oracle.Reference()
    out = np.zeros_like(x)
    _, t_red = R.run(oracle.K_REDUCE_TEAM, "shcoll_int32_sum_reduce_rec_dbl", x, out,
                     nelems=1024, warmup=20, iters=reps, pin=True)
    out = np.zeros((8, 8 * 256), np.int64)
    _, t_fc = R.run(oracle.K_SIZED, "shcoll_fcollect64_bruck_inplace", fc, out, nelems=256,
                    warmup=20, iters=reps, pin=True)
    _, t_bar = R.run(oracle.K_BARRIER_ALL, "shcoll_barrier_all_binomial_tree",
                     np.zeros((8, 8), np.uint8), np.zeros((8, 8), np.uint8), warmup=20,
                     iters=reps, pin=True)
    m = [float(np.median(t)) * 1e6 for t in (t_red, t_fc, t_bar)]
    return {"int32_sum_reduce_us": round(m[0], 2), "fcollect64_us": round(m[1], 2),
            "barrier_all_us": round(m[2], 2), "sequence_us": round(sum(m), 2),
            "kind": "reference", "cores": 8,
            "sample": "the reference's src/shcoll/src code (oracle/_ref) over 8 emulated PEs "
                      "(pinned pthreads); median of %d calls between host barriers" % reps}


def launch_floor_us(reps=300):
    """The platform's floor under any blocking GPU call: one launch of an
    empty kernel and a stream synchronisation, through the CUDA driver API
    from ctypes (the way the C entry points are timed).  The kernel is a
    one-instruction PTX entry loaded with cuModuleLoadData."""
    import ctypes
    import torch
    torch.cuda.init()
    torch.zeros(1, device="cuda")  # the primary context is current
    cu = ctypes.CDLL("libcuda.so.1")
    ptx = (b".version 8.0\n.target sm_90\n.address_size 64\n"
           b".visible .entry b200_empty()\n{\n\tret;\n}\n\0")
    mod, fn, strm = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    if cu.cuModuleLoadData(ctypes.byref(mod), ctypes.c_char_p(ptx)) != 0:
        return None
    if cu.cuModuleGetFunction(ctypes.byref(fn), mod, b"b200_empty") != 0:
        return None
    if cu.cuStreamCreate(ctypes.byref(strm), 1) != 0:
        return None
    launch, sync = cu.cuLaunchKernel, cu.cuStreamSynchronize
    launch.argtypes = [ctypes.c_void_p] + [ctypes.c_uint] * 7 + [ctypes.c_void_p] * 3
    sync.argtypes = [ctypes.c_void_p]

    def one():
        launch(fn, 1, 1, 1, 32, 1, 1, 0, strm, None, None)
        sync(strm)
    for _ in range(20):
        one()
    t = []
    for _ in range(reps):
        t0 = time.perf_counter()
        one()
        t.append(time.perf_counter() - t0)
    cu.cuStreamDestroy_v2(strm)
    cu.cuModuleUnload(mod)
    return round(float(np.median(t)) * 1e6, 2)


def run_config1(args, world, rank, local, reps=300):
    """The reference's CPU-runnable configuration on the GPU: 8 PEs, team
    WORLD, int32 sum_reduce of 1024 elements (rec_dbl, the default), then
    fcollect64 of 256 int64 per PE, then barrier_all (binomial tree).  These
    are latency-bound; reported in microseconds per call, timed on the host
    around the C entry points: blocking calls (launch + synchronisation
    each, what an OpenSHMEM call costs) and the three stream-ordered with
    one synchronisation; next to the reference's own shcoll code over 8
    emulated PEs on the host."""
    import __graft_entry__
    __graft_entry__.build_library()
    import b200shm as B
    import gen
    x, fc = gen.config1_inputs()
    B.init(8, 4 << 20)
    team = (0, 1, 8)
    try:
        src, dst = B.malloc(4096), B.malloc(4096)
        fs, fd = B.malloc(2048), B.malloc(16384)
        B.put_rows(src, x, team=team)
        B.put_rows(fs, fc, team=team)
        s_ptr = B.stream()

        # the C entry points called directly (arguments converted once), so
        # the figures are the engine's per-call cost, not the binding's
        L = B.lib
        r_args = (B.OPS.index("sum"), B.DTYPES.index("int32"), B.ALGOS.index("rec_dbl"), 0, 1, 8,
                  dst, src, 1024)
        bar_algo = B.BARRIER_ALGOS.index("binomial_tree")

        def red(stream=None):
            if L.b200shm_reduce(*r_args, stream):
                raise B.B200Error(-1, L.b200shm_last_error().decode())

        def fcol(stream=None):
            if L.b200shm_fcollect(0, 1, 8, fd, fs, 2048, stream):
                raise B.B200Error(-1, L.b200shm_last_error().decode())

        def bar(stream=None):
            if L.b200shm_barrier(bar_algo, 0, 1, 8, stream):
                raise B.B200Error(-1, L.b200shm_last_error().decode())

        def seq():
            red(), fcol(), bar()

        def seq_ordered():
            red(s_ptr), fcol(s_ptr), bar(s_ptr)
            B.quiet()

        def med_us(fn):
            for _ in range(20):
                fn()
            t = []
            for _ in range(reps):
                t0 = time.perf_counter()
                fn()
                t.append(time.perf_counter() - t0)
            return round(float(np.median(t)) * 1e6, 2)

        gpu = {"int32_sum_reduce_us": med_us(red), "fcollect64_us": med_us(fcol),
               "barrier_all_us": med_us(bar), "sequence_blocking_us": med_us(seq),
               "sequence_stream_ordered_us": med_us(seq_ordered),
               "launch_sync_floor_us": launch_floor_us(reps),
               "floor_what": "an empty kernel launched and its stream synchronised (CUDA "
                             "driver API through ctypes): the least any blocking GPU call "
                             "costs on this host"}
        red(), fcol()
        z = np.load(os.path.join(ROOT, "tests", "golden", "config1.npz"))
        exact = (B.get_rows(dst, 4096, np.int32, team=team).tobytes() == z["reduce_out"].tobytes()
                 and B.get_rows(fd, 16384, np.int64, team=team).tobytes() ==
                 z["fcollect_out"].tobytes())
    finally:
        B.finalize()
    cpu = config1_cpu_reference(reps)
    return {"workload": "config1: 8 PEs, int32 sum_reduce 1024 + fcollect64 256 + barrier_all",
            "unit": "us per call (median of %d)" % reps, "gpu": gpu, "cpu_reference": cpu,
            "bit_exact_vs_golden": bool(exact)}


# ---------------------------------------------------------------------------
# data movement (the 128-PE configuration)
# ---------------------------------------------------------------------------
def movement_cpu_reference():
    """The reference's shcoll copies at the configuration's sizes over 128
    emulated PEs, one timed call each (a bounded sample)."""
    import gen
    import oracle
    if not oracle.Reference.available:
        return None
    R = oracle.Reference()
    PM = 128
    res = {}
    x = gen.uniform_int(np.int64, PM, 4096, 33)
    out = np.zeros((PM, PM * 4096), np.int64)
    _, t = R.run(oracle.K_SIZED, "shcoll_fcollect64_bruck_inplace", x, out, nelems=4096, pin=True)
    res["fcollect64"] = (PM * 4096 * 8 + PM * PM * 4096 * 8) / t[0] / 1e9
    del x, out
    x = gen.uniform_int(np.uint8, PM, PM * 65536, 31)
    out = np.zeros_like(x)
    _, t = R.run(oracle.K_TEAM_COPY, "shcoll_alltoallmem_shift_exchange_barrier", x, out,
                 nelems=65536, pin=True)
    res["alltoallmem"] = 2 * PM * PM * 65536 / t[0] / 1e9
    del x, out
    x = gen.uniform_int(np.int64, PM, PM * 4096 * 3, 32)
    out = np.zeros((PM, PM * 4096 * 2), np.int64)
    _, t = R.run(oracle.K_ALLTOALLS_SIZED, "shcoll_alltoalls64_shift_exchange_barrier", x, out,
                 nelems=4096, a=2, b=3, pin=True)
    res["alltoalls64"] = 2 * PM * PM * 4096 * 8 / t[0] / 1e9
    return {"value": {k: round(v, 3) for k, v in res.items()}, "unit": "GB/s",
            "cores": os.cpu_count() or 1, "kind": "reference",
            "sample": "one call of each at the full size over 128 emulated PEs (pinned "
                      "pthreads), the reference's src/shcoll/src code (oracle/_ref)"}


def run_movement(args, world, rank, local):
    """128 emulated PEs: alltoallmem of 64 KiB per PE pair (uint8),
    alltoalls64 with dst stride 2 / src stride 3 over 4096 int64 per pair,
    fcollect64 of 4096 int64 per PE, and 2^20 int64 fetch-adds on 2^20
    counters per PE at uniformly random (PE, offset).  Each op is timed on
    its own with CUDA events over --steps launches, then its result is
    checked bit for bit against the oracle."""
    import torch
    import __graft_entry__
    __graft_entry__.build_library()
    import b200shm as B
    import gen
    import oracle
    rs = oracle.Restatement()
    PM, BLK, NS, NF, NOPS, NCNT = args.movement_npes, 64 << 10, 4096, 4096, 1 << 20, 1 << 20
    # 128 PEs (the configuration): 12 GiB arena, 76 MiB of objects per PE;
    # fewer PEs (profiling captures): the same per-pair sizes in a smaller arena
    B.init(PM, (96 if PM > 64 else 64) << 20)
    team = (0, 1, PM)
    s_ptr = B.stream()
    st = torch.cuda.ExternalStream(s_ptr)
    x_a2a = gen.uniform_int(np.uint8, PM, PM * BLK, 31)
    x_as = gen.uniform_int(np.int64, PM, PM * NS * 3, 32)
    x_fc = gen.uniform_int(np.int64, PM, NF, 33)
    a2a_s, a2a_d = B.malloc(PM * BLK), B.malloc(PM * BLK)
    B.put_rows(a2a_s, x_a2a, team=team)
    as_s, as_d = B.malloc(PM * NS * 3 * 8), B.malloc(PM * NS * 2 * 8)
    B.put_rows(as_s, x_as, team=team)
    B.memset(as_d, 0, PM * NS * 2 * 8, team=team)
    fc_s, fc_d = B.malloc(NF * 8), B.malloc(PM * NF * 8)
    B.put_rows(fc_s, x_fc, team=team)
    cnt = B.malloc(NCNT * 8)
    B.memset(cnt, 0, NCNT * 8, team=team)
    rng = np.random.default_rng(34)
    pe = rng.integers(0, PM, NOPS).astype(np.int32)
    idx = rng.integers(0, NCNT, NOPS).astype(np.int64)
    off = (cnt + idx * 8).astype(np.uint64)
    req = B.malloc(NOPS * (4 + 8 + 8 + 8) + 4096)  # request arrays live in PE 0's slice
    o_pe, o_off, o_val, o_f = req, req + NOPS * 4, req + NOPS * 12, req + NOPS * 20
    for o, arr in ((o_pe, pe), (o_off, off), (o_val, np.ones(NOPS, np.int64))):
        B.put_rows(o, arr.reshape(1, -1).view(np.uint8), team=(0, 1, 1))
    d = {k: B.ptr(0, o) for k, o in (("pe", o_pe), ("off", o_off), ("val", o_val), ("f", o_f))}
    ops = {
        "alltoallmem": (lambda: B.alltoall(a2a_d, a2a_s, BLK, team=team, stream=s_ptr),
                        2 * PM * PM * BLK, "GB/s", "k_alltoall"),
        "alltoalls64": (lambda: B.alltoalls(as_d, as_s, 2, 3, NS, 8, team=team, stream=s_ptr),
                        2 * PM * PM * NS * 8, "GB/s", "k_alltoalls"),
        "fcollect64": (lambda: B.fcollect(fc_d, fc_s, NF * 8, team=team, stream=s_ptr),
                       PM * NF * 8 + PM * PM * NF * 8, "GB/s", "k_fcollect"),
        "atomic_fetch_add": (lambda: B.amo_batch("fetch_add", "int64", NOPS, d["pe"], d["off"],
                                                 d["val"], None, d["f"], stream=s_ptr),
                             NOPS, "Mops/s", "k_amo"),
    }
    peak, peak_kind = peaks()
    traffic = {}
    tpath = os.path.join(ROOT, "profiles", "movement_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f)
    # the write bound of fcollect64, which writes P x P x N x 8 bytes and
    # reads P x N x 8: the driver's memset of the same dest rows, timed alike
    def memset_fc():
        B.memset(fc_d, 0, PM * NF * 8, team=team, stream=s_ptr)
    for _ in range(args.warmup):
        memset_fc()
    B.quiet()
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record(st)
    for _ in range(args.steps):
        memset_fc()
    w1.record(st)
    B.quiet()
    memset_ms = w0.elapsed_time(w1) / args.steps
    res = {}
    launches0 = B.launch_count()
    runs = args.warmup + args.steps
    for name, (fn, units, unit, kern) in ops.items():
        for _ in range(args.warmup):
            fn()
        B.quiet()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            fn()
        e1.record(st)
        B.quiet()
        ms = e0.elapsed_time(e1) / args.steps
        rate = units / (ms / 1e3) / (1e9 if unit == "GB/s" else 1e6)
        res[name] = {"kernel": kern, "ms": round(ms, 4), "value": round(rate, 1), "unit": unit}
        if unit == "GB/s":
            res[name]["roofline"] = {"bound": "hbm", "achieved": round(rate, 1), "peak": peak,
                                     "unit": "GB/s", "frac": round(rate / peak, 4),
                                     "bytes_per_launch": units, "traffic": traffic.get(name)}
        else:
            res[name]["gbs_at_16B_per_op"] = round(units * 16 / (ms / 1e3) / 1e9, 1)
            res[name]["traffic"] = traffic.get(name)
    launches = B.launch_count() - launches0
    res["fcollect64"]["write_bound"] = {
        "memset_ms": round(memset_ms, 4),
        "memset_gbs": round(PM * PM * NF * 8 / (memset_ms / 1e3) / 1e9, 1),
        "frac": round(memset_ms / res["fcollect64"]["ms"], 4),
        "what": "cudaMemset2DAsync of the same dest rows (writes only), against fcollect64's time"}
    # bit-exact checks of each op's last result against the oracle
    got = B.get_rows(a2a_d, PM * BLK, np.uint8, team=team)
    res["alltoallmem"]["bit_exact"] = got.tobytes() == rs.alltoall(x_a2a).tobytes()
    del got
    got = B.get_rows(as_d, PM * NS * 2 * 8, np.int64, team=team)
    want = rs.alltoalls(x_as, np.zeros((PM, PM * NS * 2), np.int64), 2, 3, NS)
    res["alltoalls64"]["bit_exact"] = got.tobytes() == want.tobytes()
    del got, want
    got = B.get_rows(fc_d, PM * NF * 8, np.int64, team=team)
    res["fcollect64"]["bit_exact"] = got.tobytes() == rs.fcollect(x_fc).tobytes()
    final = B.get_rows(cnt, NCNT * 8, np.int64, team=team)
    fetched = B.get_rows(o_f, NOPS * 8, np.int64, team=(0, 1, 1))[0]
    hist = np.bincount(pe.astype(np.int64) * NCNT + idx, minlength=PM * NCNT)
    ok = np.array_equal(final.reshape(-1), runs * hist)
    key = pe.astype(np.int64) * NCNT + idx  # the last run's fetches: a permutation per counter
    order = np.lexsort((fetched, key))
    ks, fs = key[order], fetched[order]
    starts = np.r_[0, np.flatnonzero(np.diff(ks)) + 1]
    rank_in = np.arange(NOPS) - np.repeat(starts, np.diff(np.r_[starts, NOPS]))
    ok = ok and np.array_equal(fs, (runs - 1) * hist[ks] + rank_in)
    res["atomic_fetch_add"]["bit_exact"] = bool(ok)
    B.finalize()
    cpu = movement_cpu_reference() if PM == 128 and not args.no_cpu_baseline else None
    return {"workload": "movement", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "peak_gbs": peak, "peak_kind": peak_kind,
            "config": {"npes": PM, "alltoallmem_block": BLK, "alltoalls": "int64 dst=2 sst=3 n=4096",
                       "fcollect64_nelems": NF, "amo": "2^20 fetch_add int64 on 2^20 counters/PE",
                       "l2": "every copy moves >= 512 MiB (> L2); the AMO counters span 1 GiB"},
            "results": res, "gpu_launches": launches, "cpu_baseline": cpu}


# ---------------------------------------------------------------------------
# the span kernels: a team of 64 members over 8 GPUs (8 per GPU)
# ---------------------------------------------------------------------------
def run_span(args, world, rank, local, G=8, L=8, NC=1 << 23, FB=256 << 10, AB=256 << 10):
    """The cross-GPU kernels of a team spanning G=8 GPUs with L=8 members on
    each, as rank 0 runs them -- b200shm_span_combine (the butterfly's
    cross-GPU levels over 8 partial vectors of 2^23 float32, SUM, written to
    the 8 local members), b200shm_span_fcollect (64 blocks of 256 KiB) and
    b200shm_span_alltoall (64 x 8 blocks of 256 KiB) -- with the 8 ranks'
    arenas emulated as disjoint slice ranges of one 64-PE arena (rank g's
    members are PEs 8g..8g+7), so every load is a local HBM load.  Across
    GPUs 7/8 of the loads cross NVLink instead.  Timed with CUDA events,
    checked against the oracle (the combine is rank 0's rec_dbl result over
    the 8 partials)."""
    import torch
    import __graft_entry__
    __graft_entry__.build_library()
    import b200shm as B
    import gen
    import oracle
    rs = oracle.Restatement()
    P = G * L
    B.init(P, 128 << 20)  # 8 GiB: 113 MiB of objects per PE
    try:
        slice_ = B.heap_slice()
        base = B.heap_base()
        bases = [base + g * L * slice_ for g in range(G)]
        local_team = (0, 1, L)
        s_ptr = B.stream()
        st = torch.cuda.ExternalStream(s_ptr)
        part, dst = B.malloc(NC * 4), B.malloc(NC * 4)
        xs = gen.normal(np.float32, G, NC, 41)
        for g in range(G):  # rank g's partial in its member 0 (PE 8g)
            B.put_rows(part, xs[g:g + 1], team=(g * L, 1, 1))
        partials = [B.ptr(g * L, part) for g in range(G)]
        fsrc, fdst = B.malloc(FB), B.malloc(P * FB)
        asrc, adst = B.malloc(P * AB), B.malloc(P * AB)
        fx = gen.uniform_int(np.uint8, P, FB, 42)
        ax = gen.uniform_int(np.uint8, P, P * AB, 43)
        B.put_rows(fsrc, fx, team=(0, 1, P))
        B.put_rows(asrc, ax, team=(0, 1, P))
        peak, peak_kind = peaks()
        ops = {
            "combine_f32_sum": (lambda: B.span_combine("sum", "float32", G, 0, partials, dst, NC,
                                                       team=local_team, stream=s_ptr),
                                (G + L) * NC * 4, "k_span_combine"),
            "fcollect": (lambda: B.span_fcollect(G, 0, bases, fdst, fsrc, FB, team=local_team,
                                                 stream=s_ptr),
                         P * FB + L * P * FB, "k_span_fcollect"),
            "alltoall": (lambda: B.span_alltoall(G, 0, bases, adst, asrc, AB, team=local_team,
                                                 stream=s_ptr),
                         2 * L * P * AB, "k_span_alltoall"),
        }
        traffic = {}
        tpath = os.path.join(ROOT, "profiles", "span_traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                traffic = json.load(f)
        res = {}
        launches0 = B.launch_count()
        for name, (fn, nbytes, kern) in ops.items():
            for _ in range(args.warmup):
                fn()
            B.quiet()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(args.steps):
                fn()
            e1.record(st)
            B.quiet()
            ms = e0.elapsed_time(e1) / args.steps
            gbs = nbytes / (ms / 1e3) / 1e9
            res[name] = {"kernel": kern, "ms": round(ms, 4), "bytes_per_launch": nbytes,
                         "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak,
                                      "unit": "GB/s", "frac": round(gbs / peak, 4),
                                      "traffic": traffic.get(name)}}
        launches = B.launch_count() - launches0
        want = rs.reduce("rec_dbl", "sum", xs)[0]
        got = B.get_rows(dst, NC * 4, np.float32, team=local_team)
        res["combine_f32_sum"]["bit_exact"] = all(r.tobytes() == want.tobytes() for r in got)
        del got
        want = rs.fcollect(fx)[:L]
        got = B.get_rows(fdst, P * FB, np.uint8, team=local_team)
        res["fcollect"]["bit_exact"] = got.tobytes() == want.tobytes()
        want = rs.alltoall(ax)[:L]
        got = B.get_rows(adst, P * AB, np.uint8, team=local_team)
        res["alltoall"]["bit_exact"] = got.tobytes() == want.tobytes()
    finally:
        B.finalize()
    return {"workload": "span", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "config": {"ranks": G, "members_per_rank": L, "combine": "2^23 float32 SUM",
                       "fcollect_block": FB, "alltoall_block": AB,
                       "arenas": "8 ranks emulated as slice ranges of one arena (local loads)",
                       "l2": "each launch moves >= 144 MiB (> L2)"},
            "peak_gbs": peak, "peak_kind": peak_kind, "results": res, "gpu_launches": launches}


# ---------------------------------------------------------------------------
# batching: 4096 reductions over 512 teams of 2048 PEs
# ---------------------------------------------------------------------------
INT_OPS = ["and", "or", "xor", "min", "max", "sum", "prod"]
BATCH_ES = {"int32": 4, "int64": 8, "float32": 4, "float64": 8}


def batch_workload(seed=4, PB=2048, NT=512, NR=4096):
    """512 teams split_strided from 2048 PEs (sizes power-law in [2, 256],
    p(s) ~ s^-2, strides cycling 1/2/4, packed along the PEs), 4096
    reductions: team uniform, nelems log-uniform in [16, 2^18], dtype uniform
    over int32/int64/float32/float64, op uniform over the 7 ops for ints and
    sum/prod/min/max for floats.  Buffers sit at team-symmetric offsets (the
    same offset in every member), the largest teams placed first, which
    keeps the busiest PE's share of the heap smallest."""
    rng = np.random.default_rng(seed)
    u = rng.random(NT)
    sizes = np.clip((1.0 / (0.5 - u * (0.5 - 1 / 256))).astype(int), 2, min(256, PB))
    teams, pos = [], 0
    for k, sz in enumerate(sizes):
        stride = [1, 2, 4][k % 3]
        while stride > 1 and (int(sz) - 1) * stride + 1 > PB:
            stride //= 2  # only for arenas smaller than the configuration's 2048 PEs
        span = (int(sz) - 1) * stride + 1
        teams.append((pos % (PB - span + 1), stride, int(sz)))
        pos += span
    reds = []
    for _ in range(NR):
        t = int(rng.integers(NT))
        n = int(np.exp(rng.uniform(np.log(16), np.log(2 ** 18))))
        dt = ["int32", "int64", "float32", "float64"][int(rng.integers(4))]
        op = (INT_OPS[int(rng.integers(7))] if dt.startswith("int")
              else ["sum", "prod", "min", "max"][int(rng.integers(4))])
        reds.append((t, n, dt, op))
    need = np.zeros(NT, np.int64)
    for t, n, dt, _ in reds:
        need[t] += 2 * ((n * BATCH_ES[dt] + 255) // 256 * 256)
    top = np.zeros(PB, np.int64)
    base = np.zeros(NT, np.int64)
    for t in np.argsort(-sizes, kind="stable"):
        st, sd, sz = teams[t]
        mem = st + np.arange(sz) * sd
        base[t] = top[mem].max()
        top[mem] = base[t] + need[t]
    cur = base.copy()
    items = []
    for t, n, dt, op in reds:
        nb = (n * BATCH_ES[dt] + 255) // 256 * 256
        items.append(dict(op=op, dtype=dt, algo="rec_dbl", team=teams[t], src=int(cur[t]),
                          dest=int(cur[t] + nb), nelems=n))
        cur[t] += 2 * nb
    return items, int(top.max()), sizes


def run_batch(args, world, rank, local):
    """The batching configuration: the same 4096 reductions issued as 4096
    b200shm_reduce calls, and as one planned batch replayed as a CUDA graph.
    Inputs are generated on the device (b200shm_fill_uniform: ints in
    [-1000, 1000], floats in [-1, 1], [0.999, 1.001] for PROD)."""
    import torch
    import __graft_entry__
    __graft_entry__.build_library()
    import b200shm as B
    PB = args.batch_npes
    items, heap_need, sizes = batch_workload(PB=PB, NT=args.batch_teams, NR=args.batch_reductions)
    B.init(PB, heap_need + (2 << 20))
    region = B.malloc(heap_need)
    for k, it in enumerate(items):
        it["src"] += region
        it["dest"] += region
        lo, hi = ((-1000, 1000) if it["dtype"].startswith("int") else
                  (0.999, 1.001) if it["op"] == "prod" else (-1.0, 1.0))
        B.fill_uniform(it["src"], it["dtype"], it["nelems"], 1000 + k, lo, hi, team=it["team"])
    B.quiet()
    s_ptr = B.stream()
    st = torch.cuda.ExternalStream(s_ptr)
    total_bytes = sum(2 * it["team"][2] * it["nelems"] * BATCH_ES[it["dtype"]] for it in items)
    sample = list(range(0, len(items), 64))

    def snap():
        return [B.get_rows(items[k]["dest"], items[k]["nelems"] * BATCH_ES[items[k]["dtype"]],
                           np.uint8, team=items[k]["team"]).tobytes() for k in sample]

    def per_call():
        for it in items:
            B.reduce(it["op"], it["dtype"], it["algo"], it["dest"], it["src"], it["nelems"],
                     team=it["team"], stream=s_ptr)

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        B.quiet()
        return e0.elapsed_time(e1) / reps

    per_call()
    B.quiet()
    want = snap()
    pc_ms = timed(per_call, max(1, min(args.steps, 5)))
    # the heuristic plan first (the tuner's cache is still empty), then the
    # tuned plan, which starts from the heuristic and keeps only what made
    # the whole batch faster
    heur = B.Batch(B.make_descs(items), B.BATCH_GRAPH | B.BATCH_NO_TUNE)
    for _ in range(args.warmup):
        heur.run(s_ptr)
    B.quiet()
    h_ms = timed(lambda: heur.run(s_ptr), args.steps)
    heur.close()
    flags = B.BATCH_GRAPH | (0 if args.batch_tune == "auto" else B.BATCH_NO_TUNE)
    t0 = time.perf_counter()
    descs = B.make_descs(items)
    batch = B.Batch(descs, flags)
    plan_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        batch.run(s_ptr)
    B.quiet()
    launches0 = B.launch_count()
    b_ms = timed(lambda: batch.run(s_ptr), args.steps)
    launches = (B.launch_count() - launches0) / args.steps
    match = snap() == want
    peak, peak_kind = peaks()
    line = {"metric": METRIC, "workload": "batch", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup,
            "config": {"npes": PB, "teams": args.batch_teams, "team_size_alpha": 2,
                       "team_size_mean": round(float(sizes.mean()), 2),
                       "team_size_max": int(sizes.max()), "reductions": len(items),
                       "nelems": "log-uniform [16, 2^18]", "dtypes": "int32/int64/float32/float64",
                       "ops": "7 ops on ints, sum/prod/min/max on floats", "algo": "rec_dbl",
                       "heap_per_pe_bytes": heap_need + (2 << 20)},
            "batched": {"ms": round(b_ms, 4), "ops_per_s": round(len(items) / (b_ms / 1e3), 1),
                        "gbs": round(total_bytes / (b_ms / 1e3) / 1e9, 1),
                        "frac_of_hbm": round(total_bytes / (b_ms / 1e3) / 1e9 / peak, 4),
                        "form": "CUDA graph: one persistent kernel per (type, op, order) group "
                                "on 4 side streams + MIN/MAX replay",
                        "plan_seconds": round(plan_s, 2), "autotune": args.batch_tune,
                        "heuristic_plan_ms": round(h_ms, 4),
                        "tuned_vs_heuristic": round(h_ms / b_ms, 3),
                        "lanes_histogram": np.bincount([d.lanes for d in descs],
                                                       minlength=9).tolist()},
            "per_call": {"ms": round(pc_ms, 4), "ops_per_s": round(len(items) / (pc_ms / 1e3), 1),
                         "gbs": round(total_bytes / (pc_ms / 1e3) / 1e9, 1),
                         "form": "%d b200shm_reduce calls, stream-ordered" % len(items)},
            "speedup": round(pc_ms / b_ms, 2), "alg_bytes": total_bytes,
            "hbm_floor_ms": round(total_bytes / (peak * 1e9) * 1e3, 4), "peak_kind": peak_kind,
            "batch_matches_per_call": bool(match), "gpu_launches_per_batch": launches}
    batch.close()
    B.finalize()
    return line


# ---------------------------------------------------------------------------
# serving: an open-loop request stream over 256 PEs
# ---------------------------------------------------------------------------
SERVE_KINDS = ["reduce", "fcollect", "alltoall", "put", "get", "amo"]


def serve_ring_bytes(slice_bytes):
    """Bytes per PE of the dest ring of the serving stream (the slice after
    the source regions and counters, less 2 MiB)."""
    ring0 = (2 * (16 << 20) + 4096 * 8 + 4095) // 4096 * 4096
    return slice_bytes - ring0 - (2 << 20)


def serve_workload(nreq, rate, seed=6, PS=256, slice_bytes=256 << 20, slots=256):
    """nreq requests with Poisson arrivals at `rate`/s: kind uniform over
    reduce/fcollect/alltoall/put/get/atomic, payload (bytes each PE
    receives) log-uniform in [8 B, 4 MiB], dtype uniform over
    int32/int64/float32/float64, team uniform over 64 teams of 4 PEs
    (PEs 4k..4k+3); reduce algorithm rec_dbl; atomics are int64 fetch-adds of
    1 on 4096 counters per PE.  Sources are read from two 16 MiB regions per
    PE (float32 and float64 values uniform in [-1, 1]); every request gets
    its own dest at team-symmetric offsets of a ring that no two of any
    `slots` consecutive requests share."""
    rng = np.random.default_rng(seed)
    SRC, NCTR = 16 << 20, 4096
    src32, src64, ctr = 0, SRC, 2 * SRC
    ring0 = (ctr + NCTR * 8 + 4095) // 4096 * 4096
    ring_bytes = serve_ring_bytes(slice_bytes)
    assert ring_bytes == slice_bytes - ring0 - (2 << 20)
    arrival = np.cumsum(rng.exponential(1.0 / rate, nreq))
    arrival -= arrival[0]
    payload = np.exp(rng.uniform(np.log(8), np.log(4 << 20), nreq)).astype(np.int64)
    items, needs = [], []
    pos = 0
    for k in range(nreq):
        kind = SERVE_KINDS[int(rng.integers(6))]
        t = int(rng.integers(64))
        team = (4 * t, 1, 4)
        pl = int(payload[k])
        if kind == "amo":
            items.append(dict(kind="amo", op="fetch_add", dtype="int64", pe=int(rng.integers(PS)),
                              dest=ctr + 8 * int(rng.integers(NCTR)), value=1, bytes=8))
            continue
        dt = ["int32", "int64", "float32", "float64"][int(rng.integers(4))]
        es = 4 if dt.endswith("32") else 8
        region = src32 if es == 4 else src64
        ne = max(1, pl // es)  # payload in whole elements of the dtype
        if kind == "reduce":
            n = ne
            nb, sb = n * es, n * es
        elif kind in ("fcollect", "alltoall"):
            n = max(1, ne // 4) * es
            nb, sb = 4 * n, (n if kind == "fcollect" else 4 * n)
        else:
            n = ne * es
            nb, sb = n, n
        so = region + int(rng.integers(0, (SRC - sb) // 16 + 1)) * 16
        need = (nb + 255) // 256 * 256
        if pos + need > ring_bytes:
            pos = 0
        d = ring0 + pos
        pos += need
        needs.append(need)
        it = dict(kind=kind, team=team, src=so, dest=d, n=n, bytes=nb)
        if kind == "reduce":
            op = (INT_OPS[int(rng.integers(7))] if dt.startswith("int")
                  else ["sum", "prod", "min", "max"][int(rng.integers(4))])
            it.update(op=op, dtype=dt, algo="rec_dbl")
        elif kind in ("put", "get"):
            it.update(team=(4 * t + int(rng.integers(4)), 1, 1), pe=int(rng.integers(PS)))
        items.append(it)
    # no two of any `slots` consecutive ring users share a byte: a window's
    # needs (plus at most one wrap's waste, < 4 MiB) stay under one lap
    c = np.concatenate([[0], np.cumsum(needs)])
    w = min(slots, len(needs))
    assert len(needs) == 0 or (c[w:] - c[:-w]).max() <= ring_bytes - (8 << 20), "ring too small"
    return items, arrival


def run_serve(args, world, rank, local):
    """The serving configuration: the open-loop stream through the serving
    loop (latency from each request's arrival to its observed completion
    word), the same stream saturating (all arrivals at 0), and the per-call
    entry points (one blocking call per request, in arrival order) on the
    first --serve-percall requests of the stream."""
    import __graft_entry__
    __graft_entry__.build_library()
    import b200shm as B
    PS, SL, SLOTS = 256, 256 << 20, 256
    items, arrival = serve_workload(args.serve_requests, args.serve_rate, PS=PS, slice_bytes=SL,
                                    slots=SLOTS)
    B.init(PS, SL)
    base = B.malloc(SL - (2 << 20))
    B.fill_uniform(base, "float32", (16 << 20) // 4, 11, -1.0, 1.0)
    B.fill_uniform(base + (16 << 20), "float64", (16 << 20) // 8, 12, -1.0, 1.0)
    B.memset(base + (32 << 20), 0, 4096 * 8)
    B.quiet()
    for it in items:
        it["dest"] += base
        if "src" in it:
            it["src"] += base
    reqs = B.make_requests(items)
    small = np.array([it["bytes"] <= 64 << 10 for it in items])

    def pct(lat, mask=None):
        x = lat if mask is None else lat[mask]
        return {"p50_us": round(float(np.percentile(x, 50)) * 1e6, 2),
                "p99_us": round(float(np.percentile(x, 99)) * 1e6, 2),
                "p999_us": round(float(np.percentile(x, 99.9)) * 1e6, 2)}

    # admission by heap bytes: the heap the stream's requests write into is
    # the dest ring of every PE; admitted, incomplete requests may hold all of it
    budget = serve_ring_bytes(SL) * PS
    srv = B.Server(queue_slots=SLOTS, heap_budget=budget)
    warm = min(2000, len(items))
    srv.replay(B.make_requests(items[:warm]), arrival[:warm])  # warm-up stream
    launches0 = B.launch_count()
    t0 = time.perf_counter()
    lat, fetched = srv.replay(reqs, arrival)
    wall = time.perf_counter() - t0
    launches = B.launch_count() - launches0
    # device clock stamps of the last queue-full of requests (still in their slots)
    first = warm + len(items) - SLOTS
    tr = np.array([srv.trace(t) for t in range(first, warm + len(items))], dtype=np.float64)
    stages = {"mirrored_to_claimed_us_p50": round(float(np.median(tr[:, 1] - tr[:, 0])) / 1e3, 2),
              "claimed_to_done_us_p50": round(float(np.median(tr[:, 2] - tr[:, 1])) / 1e3, 2),
              "requests": SLOTS}
    last = float(np.max(arrival + lat))
    t0 = time.perf_counter()
    lat_sat, _ = srv.replay(reqs, np.zeros(len(items)))
    sat_s = float(np.max(lat_sat))
    srv.stop()
    npc = min(args.serve_percall, len(items))
    pc_reqs = B.make_requests(items[:npc])
    lat_pc, _ = B.replay(pc_reqs, arrival[:npc])
    pc_last = float(np.max(arrival[:npc] + lat_pc))
    lat_pc_sat, _ = B.replay(pc_reqs, np.zeros(npc))
    pc_sat_s = float(np.max(lat_pc_sat))
    B.replay_ordered(pc_reqs[:min(npc, 2000)])  # warm-up
    ord_s, _ = B.replay_ordered(pc_reqs)
    total_bytes = int(sum(it["bytes"] for it in items))
    line = {"metric": METRIC, "workload": "serve", "n_gpus": world,
            "config": {"npes": PS, "arena_gib": PS * SL / 2 ** 30, "teams": "64 x 4 PEs",
                       "requests": len(items), "arrival": "Poisson", "rate_per_s": args.serve_rate,
                       "mix": "uniform over reduce/fcollect/alltoall/put/get/atomic",
                       "payload": "log-uniform [8 B, 4 MiB] received per PE",
                       "dtypes": "int32/int64/float32/float64", "queue_slots": SLOTS,
                       "admission": "by heap bytes written (device counter)",
                       "heap_budget_bytes": budget},
            "served": {"latency_all": pct(lat), "latency_le_64KiB": pct(lat, small),
                       "ops_per_s": round(len(items) / last, 1),
                       "offered_per_s": round(len(items) / float(arrival[-1]), 1),
                       "saturated_ops_per_s": round(len(items) / sat_s, 1),
                       "saturated_gbs_received": round(total_bytes / sat_s / 1e9, 2),
                       "kernel_launches": launches, "wall_s": round(wall, 3),
                       "device_stages": stages},
            "per_call": {"requests": npc, "latency_all": pct(lat_pc),
                         "latency_le_64KiB": pct(lat_pc, small[:npc]),
                         "ops_per_s": round(npc / pc_last, 1),
                         "saturated_ops_per_s": round(npc / pc_sat_s, 1),
                         "form": "one blocking b200shm_* call per request, in arrival order"},
            "per_call_stream_ordered": {
                "requests": npc, "ops_per_s": round(npc / ord_s, 1),
                "form": "the same per-call entry points issued back to back on one stream, "
                        "one synchronisation at the end (b200shm_serve_replay_ordered)"},
            "amo_fetch_adds": int(sum(1 for it in items if it["kind"] == "amo"))}
    line["speedup_saturated_ops"] = round(line["served"]["saturated_ops_per_s"] /
                                          line["per_call"]["saturated_ops_per_s"], 2)
    line["speedup_saturated_ops_vs_stream_ordered"] = round(
        line["served"]["saturated_ops_per_s"] / line["per_call_stream_ordered"]["ops_per_s"], 2)
    B.finalize()
    return line


if __name__ == "__main__":
    main()
