"""Benchmark of the disparity hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload full|small]

One step = the whole path on one rectified pair: predict_auto (probe + up to
three StereoNet passes, FP32) followed by lr_refine with refine_disparity's
parameters (R=10, 9x7 census, P1=12, P2=150, tol=2; both views, bit-exact).
Default workload: the 450x375 uint8 pair (8-15 slanted planes, disparities
0-80 px, ~10% occluded, ~20% low texture).  Metric: refined Mpix/s, i.e.
W*H of every pair processed / device time.  Multi-GPU runs are replicas (the
path shards by pairs, no collective): every rank refines its own pair, the
step time is the max over ranks, value = ranks x W*H x K / that time.

``value`` times the device path with the images already in HBM (L2 flushed
by a 256 MB write before every step, outside the timed events); ``e2e`` times
the same step through the public pipeline from pinned host buffers (H2D of
both images and D2H of the refined disparity + status inside the events).
``roofline`` is the SGM aggregation kernel (the dominant kernel): algorithmic
bytes 48*K per pixel per view (uint16 C read + S read + S write per path, 8
paths) x 2 views x W*H over its CUDA-event duration, against the measured HBM
copy bandwidth.  ``cpu_baseline`` times the FP64 C port of the reference
(oracle/) on the host cores over a bounded sample.

``--impl reference`` times that CPU port alone (rank 0; other ranks exit).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "refined Mpix/s per B200 (bit-exact)"
UNIT = "Mpix/s"
PARAMS = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
TOL = 2.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="full",
                    choices=["full", "small", "batched", "refine_disparity", "read_image",
                             "train", "band"])
    ap.add_argument("--pairs", type=int, default=256, help="pairs of the batched workload")
    ap.add_argument("--batch", type=int, default=64, help="crops per step of the train workload")
    ap.add_argument("--band-pairs", type=int, default=48,
                    help="held-out 640x480 pairs of the band workload")
    ap.add_argument("--cpu-leg", default=None, choices=["pair", "refpy", "batch16"],
                    help=argparse.SUPPRESS)          # child process: one CPU baseline leg
    ap.add_argument("--clock-sampler", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--pci", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--threads", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="bound on the CPU-baseline sample")
    return ap.parse_args()


def make_pair(pkg, workload):
    if workload == "small":
        return pkg.synth.config_small(), "160x120 u8 pair, 3-6 slanted planes, 2-30 px"
    return (pkg.synth.config_full(),
            "450x375 u8 pair, 8-15 slanted planes, 0-80 px, ~10% occluded, ~20% low texture")


def pair_config(desc, world):
    """The `config` of the single-pair workloads: identical in both arms."""
    return {"workload": "%s: predict_auto + lr_refine (R=10, 9x7 census, P1=12, P2=150, "
                        "tol=2)" % desc,
            "pairs_per_step_per_gpu": 1, "parallelism": "replicas x%d" % world}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


# ------------------------------------------------------------------ CPU
# The CPU legs run in child processes, so the measured process maps only the
# product library (the oracle's shared object never loads beside it).
def cpu_port_run(pair, net, seconds, threads):
    """Time the FP64 C port (oracle/) of predict_auto + lr_refine on the host
    cores: whole pairs until `seconds` have passed (at least one).  Runs in
    the calling process (the reference arm and the child leg use it)."""
    import __graft_entry__
    orc = __graft_entry__.load_oracle()
    orc.set_threads(threads)
    L, R = pair.gray("left").ravel(), pair.gray("right").ravel()
    n, t0 = 0, time.perf_counter()
    while True:
        df, _, _, _ = orc.predict_auto(net, L, R, pair.W, pair.H)
        orc.lr_refine(L, R, df, pair.W, pair.H, tol=TOL, **PARAMS)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return n, el


def _child(argv, timeout):
    """Run bench.py in a child process and return its last JSON line."""
    r = subprocess.run([sys.executable, os.path.abspath(__file__)] + argv, capture_output=True,
                       text=True, timeout=timeout, cwd=REPO)
    lines = [ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        raise RuntimeError("CPU leg %s failed (rc %d): %s" % (argv, r.returncode,
                                                             r.stderr.strip()[-400:]))
    return json.loads(lines[-1])


def cpu_port_leg(workload, seconds, threads):
    """cpu_port_run of the workload's pair in a child process."""
    d = _child(["--cpu-leg", "pair", "--workload", workload, "--cpu-seconds", str(seconds),
                "--threads", str(threads)], timeout=600 + 4 * seconds)
    return d["pairs"], d["seconds"]


REF_SRC_ENV = "SV_REFERENCE_SRC"


def reference_source():
    """Path of the reference's own stereonet.py if this machine has one:
    $SV_REFERENCE_SRC, or baseline/_ref/stereonet.py.  None otherwise."""
    for c in (os.environ.get(REF_SRC_ENV), os.path.join(REPO, "baseline", "_ref", "stereonet.py")):
        if c and os.path.isfile(c):
            return c
    return None


def reference_cpython_leg():
    """The reference's own lr_refine under this interpreter, one call on the
    160x120 pair (about 3.4 s under CPython 3.12), in a child process; or why
    it could not run."""
    src = reference_source()
    if src is None:
        return {"available": False,
                "why": "reference source not on box (stereonet.py is not pip-installable: no "
                       "setup.py or pyproject.toml; set %s to a copy)" % REF_SRC_ENV}
    try:
        d = _child(["--cpu-leg", "refpy"], timeout=900)
    except (RuntimeError, subprocess.TimeoutExpired) as e:
        return {"available": False, "why": str(e)[:300]}
    d["available"] = True
    return d


def cpu_leg_main(args):
    """Child-process body of the CPU legs (prints one JSON line)."""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    if args.cpu_leg == "pair":
        pair, _ = make_pair(pkg, args.workload)
        net = pkg.weights.load_model()
        n, el = cpu_port_run(pair, net, args.cpu_seconds, args.threads or (os.cpu_count() or 1))
        print(json.dumps({"pairs": n, "seconds": el}))
        return
    if args.cpu_leg == "batch16":
        net = pkg.weights.load_model()
        orc = __graft_entry__.load_oracle()
        orc.set_threads(args.threads or (os.cpu_count() or 1))
        pairs = pkg.synth.config_batched(n=16, seed=3)
        t0 = time.perf_counter()
        done, mpix = 0, 0.0
        for p in pairs:
            L, R = p.gray("left").ravel(), p.gray("right").ravel()
            df, _, _, _ = orc.predict_auto(net, L, R, p.W, p.H)
            orc.lr_refine(L, R, df, p.W, p.H, tol=TOL, **PARAMS)
            done += 1
            mpix += p.W * p.H / 1e6
            if time.perf_counter() - t0 >= args.cpu_seconds and done >= 4:
                break
        print(json.dumps({"pairs": done, "mpix": mpix, "seconds": time.perf_counter() - t0}))
        return
    # refpy: exec the reference (as its own test harness does) and time lr_refine
    import platform
    src = reference_source()
    code = open(src).read().replace("if __name__ == '__main__':", "if False:").replace(
        'if __name__ == "__main__":', "if False:")
    SN = {"__name__": "stereonet_ref"}
    exec(compile(code, src, "exec"), SN)
    pair = pkg.synth.config_small()
    W, H = pair.W, pair.H
    L = [float(v) for v in pair.gray("left").ravel()]
    R = [float(v) for v in pair.gray("right").ravel()]
    d0 = [float(v) for v in pair.disp.ravel()]
    t0 = time.perf_counter()
    SN["lr_refine"](L, R, d0, W, H, tol=TOL, **PARAMS)
    el = time.perf_counter() - t0
    print(json.dumps({"value": round(W * H / el / 1e6, 6), "unit": UNIT, "cores": 1,
                      "interpreter": "%s %s" % (platform.python_implementation(),
                                                platform.python_version()),
                      "sample": "the reference's own lr_refine (R=10, 9x7, P1=12, P2=150, tol=2) "
                                "once on the 160x120 pair, ground-truth disp0, %.2f s" % el,
                      "pypy": "unavailable (no pypy3 on this machine)"}))


# --------------------------------------------------------------- clocks
# Read-only NVML sampling of the SM clock and the clock-event reasons at
# about 1 ms, in a child process so the launching thread shares no GIL time
# with it.  nvidia-smi (100 ms) is the fallback when NVML is unavailable.
_REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}


def clock_sampler_main(args):
    """Child body: append 't_ms,sm_mhz,reason_bits' lines to args.clock_sampler
    until terminated; the first line is '#max,<max sm MHz>'."""
    import signal
    import pynvml
    pynvml.nvmlInit()
    h = None
    if args.pci:
        try:
            h = pynvml.nvmlDeviceGetHandleByPciBusId(args.pci)
        except pynvml.NVMLError:
            h = None
    if h is None:
        h = pynvml.nvmlDeviceGetHandleByIndex(0)
    get_r = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
        pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
    stop = []
    signal.signal(signal.SIGTERM, lambda *a: stop.append(1))
    with open(args.clock_sampler, "w", buffering=1) as f:
        f.write("#max,%d\n" % pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        t0 = time.perf_counter()
        while not stop:
            sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
            f.write("%.3f,%d,%d\n" % (1e3 * (time.perf_counter() - t0), sm, get_r(h)))
            time.sleep(0.001)


class ClockSampler:
    """SM clock / clock-event reasons during the timed region (see above)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.kind = None

    def _pci(self):
        try:
            import torch
            p = torch.cuda.get_device_properties(self.index)
            return "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        except Exception:
            return None

    def __enter__(self):
        try:
            import pynvml  # noqa: F401
            argv = [sys.executable, os.path.abspath(__file__), "--clock-sampler", self.path]
            pci = self._pci()
            if pci:
                argv += ["--pci", pci]
            self.proc = subprocess.Popen(argv, stdout=subprocess.DEVNULL,
                                         stderr=subprocess.DEVNULL)
            self.kind = "nvml"
            t0 = time.time()
            while time.time() - t0 < 20:                  # until the first sample lands
                if os.path.exists(self.path) and open(self.path).read().count("\n") >= 2:
                    break
                if self.proc.poll() is not None:
                    raise OSError("NVML sampler exited")
                time.sleep(0.01)
        except (ImportError, OSError):
            if self.proc is not None and self.proc.poll() is None:
                self.proc.kill()
            try:
                self.f = open(self.path, "w")
                self.proc = subprocess.Popen(
                    ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                     "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                    stderr=subprocess.DEVNULL)
                self.kind = "nvidia-smi"
            except OSError:
                self.proc = None
        self.t_enter = time.perf_counter()
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.kind == "nvidia-smi":
                self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"]}
        sm, mx, reasons = [], None, set()
        if self.kind == "nvml":
            for line in open(self.path):
                p = line.strip().split(",")
                if p[0] == "#max":
                    mx = float(p[1])
                    continue
                if len(p) != 3:
                    continue
                sm.append(float(p[1]))
                for nm, bit in _REASON_BITS.items():
                    if int(p[2]) & bit:
                        reasons.add(nm)
        else:
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = float(p[2])
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "source": self.kind, "reasons": sorted(reasons)}


def hbm_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def sgm_traffic(K, N):
    """DRAM bytes per SGM launch from the committed ncu summary, scaled to
    this launch's pixel count (traffic grows with the pixels swept)."""
    p = os.path.join(REPO, "profiles", "ncu_sgm_group_450x375.md")
    if not os.path.exists(p):
        return None
    per_px = None
    for line in open(p):
        if line.startswith("dram_bytes_per_view_pixel:"):
            per_px = float(line.split(":")[1])
    return None if per_px is None else per_px * 2 * N


# ------------------------------------------------------------- our arm
def run_ours(args, rank, world, local):
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    lib = pkg._lib.load()
    net = pkg.weights.load_model()
    pair, desc = make_pair(pkg, args.workload)
    W, H, N = pair.W, pair.H, pair.W * pair.H
    K = 2 * PARAMS["R"] + 1
    pipe = pkg.pipeline.PairPipeline(W, H, net, **PARAMS, tol=TOL)
    hl = torch.from_numpy(pair.left.ravel()).pin_memory()
    hr = torch.from_numpy(pair.right.ravel()).pin_memory()
    pipe.left.copy_(hl)
    pipe.right.copy_(hr)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stages = pipe.refiner.STAGES
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(stages) + 1)]
          for _ in range(args.steps)]
    t0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    pe = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]

    def step(i=None):
        """One pair through predict_auto + lr_refine; with i, predict_auto's
        end and lr_refine's stages record events (outside the timed region
        only; predict_auto returns once its last pass is done, so pe[i]
        marks the end of its GPU work, not the host's next call)."""
        if i is None:
            pipe.run_device()
        else:
            pipe.predict()
            pe[i].record()
            pipe.refiner.run_timed(pipe.left, pipe.right, pipe.disp0, pipe.out, pipe.status, ev[i])

    # everything runs on the pipeline's own stream (captured passes replay as
    # graphs there); events are recorded on that stream
    sm = torch.cuda.stream(pipe.stream)
    with sm:
        for _ in range(args.warmup):
            step()
        pipe.refiner.data_status()
    torch.cuda.synchronize()

    # ---- device-resident timed region
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.sv_launch_count()
    with ClockSampler(local) as clk, torch.cuda.stream(pipe.stream):
        for i in range(args.steps):
            flush.zero_()
            t0[i].record()
            step()
            t1[i].record()
        torch.cuda.synchronize()
    launches = lib.sv_launch_count() - launches0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = sum(t0[i].elapsed_time(t1[i]) for i in range(args.steps))

    # ---- stage breakdown: the same steps again with lr_refine's stage
    # events (outside the timed region; predict_auto timed whole)
    with torch.cuda.stream(pipe.stream):
        for i in range(args.steps):
            flush.zero_()
            t0[i].record()
            step(i)
        torch.cuda.synchronize()
    stage_ms = [sum(ev[i][s].elapsed_time(ev[i][s + 1]) for i in range(args.steps)) / args.steps
                for s in range(len(stages))]
    pred_ms = sum(t0[i].elapsed_time(pe[i]) for i in range(args.steps)) / args.steps
    ms = pkg.shard.max_over_ranks(ms, device="cuda")
    value = world * N * args.steps / (ms / 1e3) / 1e6

    # ---- end to end through the public pipeline from pinned host buffers
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for _ in range(2):
        pipe.run_host(hl, hr)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        with torch.cuda.stream(pipe.stream):
            flush.zero_()
            e0[i].record()
        pipe.run_host(hl, hr)
        e1[i].record(pipe.stream)
    torch.cuda.synchronize()
    ems = sum(e0[i].elapsed_time(e1[i]) for i in range(args.steps))
    ems = pkg.shard.max_over_ranks(ems, device="cuda")
    evalue = world * N * args.steps / (ems / 1e3) / 1e6

    result = None
    if rank == 0:
        peak, peak_kind = hbm_peak()
        sgm_ms = stage_ms[stages.index("sgm")]
        alg = 48 * K * N * 2                      # both views in one launch
        achieved = alg / (sgm_ms / 1e3) / 1e9
        traffic = sgm_traffic(K, N)
        cpu = None
        if world == 1:
            threads = os.cpu_count() or 1
            n, el = cpu_port_leg(args.workload, args.cpu_seconds, threads)
            cpu = {"value": round(n * N / el / 1e6, 6), "unit": UNIT, "cores": threads,
                   "kind": "port",
                   "sample": "%d whole pairs (%s) through the FP64 C port of predict_auto + "
                             "lr_refine, %.1f s, OpenMP over %d threads (child process)"
                             % (n, desc, el, threads),
                   "reference_cpython": reference_cpython_leg()}
        dram_gbs = None if traffic is None else traffic / (sgm_ms / 1e3) / 1e9
        result = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "u8/u64/int32 integer refinement, f64 subpixel+LR, f32 network",
            "data": "synthetic (seeded generator; reference weights stereonet_weights.txt)",
            "config": pair_config(desc, world),
            "l2": "flushed before every step (256 MB write, untimed)",
            "work": {"work_size": list(pipe.work_size), "work_trace": pipe.work_trace},
            "stages_ms": {"predict_auto": round(pred_ms, 4),
                          **{s: round(v, 4) for s, v in zip(stages, stage_ms)}},
            # lr_refine alone (its stage events), both views + LR check per pair
            "refine_only_mpix_s": round(N / (sum(stage_ms) / 1e3) / 1e6, 3),
            # achieved = the algorithmic SGM bytes (48*K per pixel per view:
            # u16 costs read, path costs read and written per path) / the SGM
            # stage time; a pair's working set is L2-resident,
            # so the DRAM bytes ncu measures are far fewer (dram_frac)
            "roofline": {"kernel": "%s (8 paths x 2 views)" % pkg.refine.sgm_kernel_name(),
                         "bound": "hbm",
                         "basis": "algorithmic bytes (working set L2-resident)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind
                         if peak_kind == "measured" else "fallback",
                         "algorithmic_bytes_per_launch": alg,
                         "traffic": traffic,
                         "dram_frac": None if dram_gbs is None else round(dram_gbs / peak, 4)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(evalue, 3), "unit": UNIT,
                    "h2d_bytes_per_step": pipe.h2d_bytes(),
                    "d2h_bytes_per_step": pipe.d2h_bytes()},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


# --------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return None
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    net = pkg.weights.load_model()
    pair, desc = make_pair(pkg, args.workload)
    N = pair.W * pair.H
    threads = os.cpu_count() or 1
    budget = max(1.0, args.cpu_seconds / max(1, args.steps + args.warmup))
    for _ in range(min(args.warmup, 1)):
        cpu_port_run(pair, net, 0.0, threads)
    n_tot, t_tot = 0, 0.0
    for _ in range(args.steps):
        n, el = cpu_port_run(pair, net, budget, threads)
        n_tot += n
        t_tot += el
    value = n_tot * N / t_tot / 1e6
    sample = ("%d whole pairs (%s) through the FP64 C port of the reference's predict_auto + "
              "lr_refine (bit-identical to stereonet.py on the golden fixtures), OpenMP over "
              "%d threads" % (n_tot, desc, threads))
    return {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * t_tot / n_tot, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": pair_config(desc, world),
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_batched(args, rank, world, local):
    """The batched workload: 256 pairs of uneven sizes (200x150..1400x1100,
    max disparity 10-200 px), sharded over ranks by pixel count.  A step is
    the whole path for every pair -- predict_auto with its work-width
    decisions on the device, then lr_refine -- replayed from one CUDA graph
    (batch.NetBatch), images already in HBM; e2e adds the H2D of every
    image and the D2H of every refined disparity and status."""
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    net = pkg.weights.load_model()
    pairs = pkg.synth.config_batched(n=args.pairs, seed=3)
    mine = pkg.shard.shard([p.W * p.H for p in pairs], rank, world)
    pairs = [pairs[i] for i in mine]
    nb = pkg.batch.NetBatch([(p.W, p.H) for p in pairs], net, **PARAMS, tol=TOL)
    hl = [torch.from_numpy(p.left.ravel()).pin_memory() for p in pairs]
    hr = [torch.from_numpy(p.right.ravel()).pin_memory() for p in pairs]
    ho = [torch.empty(p.W * p.H, dtype=torch.float64).pin_memory() for p in pairs]
    hs = [torch.empty(p.W * p.H, dtype=torch.uint8).pin_memory() for p in pairs]
    for i in range(len(pairs)):
        nb.left[i].copy_(hl[i])
        nb.right[i].copy_(hr[i])
    N = nb.pixels
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            nb.run()
        nb.data_status()
    torch.cuda.synchronize()

    def timed(fn, steps):
        t0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        t1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for i in range(steps):
                flush.zero_()
                t0[i].record()
                fn()
                t1[i].record()
        torch.cuda.synchronize()
        return [t0[i].elapsed_time(t1[i]) for i in range(steps)]

    lib = pkg._lib.load()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = lib.sv_launch_count()
    with ClockSampler(local) as clk:
        times = timed(nb.run, args.steps)
    launches = lib.sv_launch_count() - l0
    ms = pkg.shard.max_over_ranks(sum(times), device="cuda")
    value = world * N * args.steps / (ms / 1e3) / 1e6
    # the network alone (same graph without the refinement), for the stage split
    pred_ms = statistics.median(timed(nb.predict, max(3, args.steps // 2)))

    def e2e_step():
        for i in range(len(pairs)):
            nb.left[i].copy_(hl[i], non_blocking=True)
            nb.right[i].copy_(hr[i], non_blocking=True)
        nb.run()
        for i in range(len(pairs)):
            ho[i].copy_(nb.out[i], non_blocking=True)
            hs[i].copy_(nb.status[i], non_blocking=True)

    ems = pkg.shard.max_over_ranks(sum(timed(e2e_step, args.steps)), device="cuda")
    evalue = world * N * args.steps / (ems / 1e3) / 1e6
    traces = nb.traces()
    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return None
    peak, peak_kind = hbm_peak()
    K = 2 * PARAMS["R"] + 1
    step_ms = ms / args.steps
    ref_ms = step_ms - pred_ms
    alg = 2350 * N                       # whole refinement, both views + LR, per left pixel
    achieved = alg / (ref_ms / 1e3) / 1e9
    cpu = None
    if world == 1:
        threads = os.cpu_count() or 1
        d = _child(["--cpu-leg", "batch16", "--cpu-seconds", str(args.cpu_seconds),
                    "--threads", str(threads)], timeout=3600)
        cpu = {"value": round(d["mpix"] / d["seconds"], 6), "unit": UNIT, "cores": threads,
               "kind": "port",
               "sample": "the first %d pairs of the same seeded batch (%.2f Mpix) through the "
                         "FP64 C port of predict_auto + lr_refine, %.1f s, OpenMP over %d threads "
                         "(child process)" % (d["pairs"], d["mpix"], d["seconds"], threads)}
    passes = [len(t[0]) for t in traces]
    res = {
        "metric": "refined Mpix/s per B200, batched predict_auto + lr_refine (bit-exact)",
        "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(step_ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "u8/u64/int32 integer refinement, f64 subpixel+LR, f32 network",
        "data": "synthetic (seeded generator; reference weights stereonet_weights.txt)",
        "config": {"workload": "%d pairs of uneven sizes 200x150..1400x1100, max disparity "
                               "10-200 px: predict_auto + lr_refine (R=10, 9x7 census, P1=12, "
                               "P2=150, tol=2), one CUDA graph per step" % args.pairs,
                   "pairs_per_step_per_gpu": len(pairs), "parallelism": "replicas x%d" % world},
        "l2": "flushed before every step (256 MB write, untimed); the batch is larger than L2",
        "stages_ms": {"predict_auto": round(pred_ms, 3), "lr_refine": round(ref_ms, 3)},
        "passes_per_pair": {str(k): passes.count(k) for k in sorted(set(passes))},
        "pixels_per_step_per_gpu": N,
        "roofline": {"kernel": "batched lr_refine (census, band costs, 8-path SGM, WTA, LR: 7 "
                               "launches)", "bound": "hbm",
                     "basis": "algorithmic bytes, 2350 B per left pixel at K = %d" % K,
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": alg, "traffic": None},
        "cpu_baseline": cpu,
        "e2e": {"value": round(evalue, 3), "unit": UNIT,
                "h2d_bytes_per_step": int(sum(2 * p.W * p.H for p in pairs)),
                "d2h_bytes_per_step": int(sum(9 * p.W * p.H for p in pairs))},
        "gpu_launches": int(launches), "clocks": clk.summary(),
    }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return res


def run_band(args, rank, world, local):
    """The learned-band workload on held-out 640x480 pairs (disparities
    30-150 px, thin bars, 30% low texture): every method after the same FP32
    predict_auto -- the fixed +-10 band, the no-net rule, the learned band
    (weights/band_weights.npz) and full-range SGM -- scored against the
    generator's ground truth (EPE, bad2 = share of valid pixels off by more
    than 2 px) and timed per pair with CUDA events.  One rank."""
    if rank != 0:
        return None
    # the harness's own eval command in a child process (its generator pool
    # spawns workers that import the harness as a script)
    rep = tempfile.mktemp(suffix=".json")
    harness = os.path.join(REPO, "from-scratch-stereo-vision_b200", "band_train.py")
    with ClockSampler(local) as clk:
        r = subprocess.run([sys.executable, harness, "eval", "--pairs", str(args.band_pairs),
                            "--report", rep], capture_output=True, text=True, timeout=3600,
                           cwd=REPO)
    if r.returncode != 0:
        raise RuntimeError("band evaluation failed: %s" % r.stderr.strip()[-600:])
    res = json.load(open(rep))["test"]
    os.unlink(rep)
    TEST_SEED0, DMAX = 3_000_000, 160
    acc = {k: {m: round(v, 6) if isinstance(v, float) else v for m, v in res[k].items()}
           for k in ("fixed_pm10", "rule_no_net", "learned", "full_range")}
    return {
        "metric": "learned-band refined Mpix/s per B200 (640x480, incl. predict_auto)",
        "value": round(res["learned"]["mpix_s"], 3), "unit": "Mpix/s", "n_gpus": 1,
        "steps": args.band_pairs, "warmup": 2,
        "ms_per_step": round(640 * 480 / res["learned"]["mpix_s"] / 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 network, bf16 band net (tensor cores), integer refinement",
        "data": "synthetic (seeded held-out pairs, seeds from %d)" % TEST_SEED0,
        "config": {"workload": "%d held-out 640x480 pairs, disparities 30-150 px, 1-3 bars "
                               "2-6 px, 30%% low texture; band search 0..%d" % (args.band_pairs,
                                                                              DMAX),
                   "pairs_per_step_per_gpu": 1, "parallelism": "replicas x1"},
        "accuracy": acc,
        "cpu_baseline": None, "e2e": None, "clocks": clk.summary(),
    }


def pseudo_rgb(pair):
    """An RGB image for plane_snap's SLIC: the left gray level and two smooth
    transforms of it, interleaved, in [0, 1] (as read_image returns)."""
    import numpy as np
    g = pair.left.astype(np.float64) / 255.0
    h, w = g.shape
    yy, xx = np.mgrid[0:h, 0:w]
    rgb = np.stack([g, 0.5 * g + 0.5 * (xx / max(1, w - 1)), 1.0 - 0.7 * g * (yy / max(1, h - 1))],
                   axis=-1)
    return (np.round(rgb * 255.0) / 255.0).ravel()


def run_refdisp(args, rank, world, local):
    """The refine_disparity workload: the 450x375 pair with an RGB image;
    a step is predict_auto and refine_disparity (lr_refine, plane_snap on
    the left-right-consistent pixels, 3x3 median; stereonet.py:5865-5883),
    from images in HBM."""
    import ctypes
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    lib = pkg._lib.load()
    net = pkg.weights.load_model()
    pair = pkg.synth.config_full()
    W, H, N = pair.W, pair.H, pair.W * pair.H
    rgb_h = pseudo_rgb(pair)
    rgb = torch.from_numpy(rgb_h).cuda()
    pipe = pkg.pipeline.PairPipeline(W, H, net, **PARAMS, tol=TOL)
    hl = torch.from_numpy(pair.left.ravel()).pin_memory()
    hr = torch.from_numpy(pair.right.ravel()).pin_memory()
    pipe.left.copy_(hl)
    pipe.right.copy_(hr)
    prm = pkg.refine._params(**PARAMS)
    need = lib.sv_refine_disparity_workspace_size(W, H, ctypes.byref(prm), 12)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    out = torch.empty(N, dtype=torch.float64, device="cuda")
    st = torch.empty(N, dtype=torch.uint8, device="cuda")
    hout = torch.empty(N, dtype=torch.float64).pin_memory()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())                         # noqa: E731
    s = pipe.stream.cuda_stream

    def refdisp():
        pkg._lib.check(lib.sv_refine_disparity(vp(pipe.left), vp(pipe.right), pipe.code, vp(rgb),
                                               vp(pipe.disp0), W, H, TOL, ctypes.byref(prm), 1, 12,
                                               1.0, 0.4, vp(out), vp(st), vp(ws), need, s),
                       "refine_disparity")

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    with torch.cuda.stream(pipe.stream):
        for _ in range(args.warmup):
            pipe.predict()
            refdisp()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.sv_launch_count()
    with ClockSampler(local) as clk, torch.cuda.stream(pipe.stream):
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record()
            pipe.predict()
            ev[i][1].record()
            refdisp()
            ev[i][2].record()
        torch.cuda.synchronize()
    launches = lib.sv_launch_count() - launches0
    ms = sum(ev[i][0].elapsed_time(ev[i][2]) for i in range(args.steps))
    st_pred = sum(ev[i][0].elapsed_time(ev[i][1]) for i in range(args.steps)) / args.steps
    st_ref = sum(ev[i][1].elapsed_time(ev[i][2]) for i in range(args.steps)) / args.steps
    # lr_refine alone on the same disparity, for the post-processing share
    with torch.cuda.stream(pipe.stream):
        for _ in range(3):
            pipe.refine()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            pipe.refine()
        e1.record()
        torch.cuda.synchronize()
    st_lr = e0.elapsed_time(e1) / args.steps
    ms = pkg.shard.max_over_ranks(ms, device="cuda")
    value = world * N * args.steps / (ms / 1e3) / 1e6
    # end to end: pinned host images in, refined disparity out, every step
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    with torch.cuda.stream(pipe.stream):
        for i in range(args.steps):
            flush.zero_()
            e0[i].record()
            pipe.left.copy_(hl, non_blocking=True)
            pipe.right.copy_(hr, non_blocking=True)
            pipe.predict()
            refdisp()
            hout.copy_(out, non_blocking=True)
            e1[i].record()
        torch.cuda.synchronize()
    ems = sum(e0[i].elapsed_time(e1[i]) for i in range(args.steps))
    ems = pkg.shard.max_over_ranks(ems, device="cuda")
    evalue = world * N * args.steps / (ems / 1e3) / 1e6
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    import __graft_entry__ as ge
    orc = ge.load_oracle()
    orc.set_threads(threads)
    L, R = pair.gray("left").ravel(), pair.gray("right").ravel()
    t0 = time.time()
    n = 0
    while n < 1 or time.time() - t0 < min(args.cpu_seconds, 20.0):
        df = orc.predict_auto(net, L, R, W, H)[0]
        orc.refine_disparity(L, R, rgb_h, df, W, H, **PARAMS, tol=TOL)
        n += 1
    el = time.time() - t0
    return {"metric": "refine_disparity Mpix/s per B200 (bit-exact post-processing)",
            "value": round(value, 3), "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 network, integer refinement, f64 planes and median",
            "data": "synthetic (seeded generator; pseudo-RGB from the left image)",
            "config": {"workload": "450x375 pair: predict_auto + refine_disparity (lr_refine R=10, "
                                   "plane_snap step 12 thr 1 min_inl 0.4, 3x3 median)",
                       "l2": "flushed before every step (256 MB write, untimed)",
                       "parallelism": "replicas x%d" % world},
            "stages_ms": {"predict_auto": round(st_pred, 4), "refine_disparity": round(st_ref, 4),
                          "of_which_lr_refine": round(st_lr, 4),
                          "of_which_plane_snap_and_median": round(st_ref - st_lr, 4)},
            "cpu_baseline": {"value": round(n * N / el / 1e6, 6), "unit": "Mpix/s",
                             "cores": threads, "kind": "port",
                             "sample": "%d whole pairs through the FP64 C port of predict_auto + "
                                       "refine_disparity, %.1f s, OpenMP over %d threads"
                                       % (n, el, threads)},
            "e2e": {"value": round(evalue, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 2 * N,
                    "d2h_bytes_per_step": 8 * N},
            "gpu_launches": int(launches), "clocks": clk.summary()}


def run_image(args, rank, world, local):
    """The input-image workload: both views of the 450x375 pair as 8-bit
    RGB PNGs held in host memory; a step decodes them (inflate + row
    filters on the host, stereonet.py:3335-3496) and forms the FP64 gray and
    RGB images on the GPU (read_png, stereonet.py:3499-3601)."""
    import ctypes
    import numpy as np
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from importlib import import_module
    image = import_module(pkg.__name__ + ".image")
    lib = pkg._lib.load()
    pair = pkg.synth.config_full()
    W, H, N = pair.W, pair.H, pair.W * pair.H
    views = []
    for g in (pair.left, pair.right):
        q = g.astype(np.int64)
        rgb = np.stack([q, np.clip(q + 17, 0, 255), np.clip(255 - q // 2, 0, 255)], -1)
        # 8-bit RGB, all five row filters in turn, zlib level 6 (dynamic
        # Huffman blocks), as image tools write
        views.append(pkg.synth.make_png(W, H, 8, 2, rgb.reshape(H, W * 3).tolist(),
                                        (0, 1, 2, 3, 4), 6)[0])
    s = torch.cuda.Stream()
    descs = [pkg._lib.RawImage() for _ in views]
    for d, v in zip(descs, views):
        pkg._lib.check(lib.sv_image_info(v, len(v), ctypes.byref(d)), "sv_image_info")
    nraw = [d.stride * d.height for d in descs]
    raw_h = [torch.empty(n, dtype=torch.uint8).pin_memory() for n in nraw]
    raw_d = [torch.empty(n, dtype=torch.uint8, device="cuda") for n in nraw]
    gray = [torch.empty(N, dtype=torch.float64, device="cuda") for _ in views]
    rgbd = [torch.empty(3 * N, dtype=torch.float64, device="cuda") for _ in views]
    done = [torch.cuda.Event() for _ in views]
    vp = lambda t: ctypes.c_void_p(t.data_ptr())                         # noqa: E731
    host_ms = []

    nv = len(views)
    c_data = (ctypes.c_char_p * nv)(*views)
    c_sizes = (ctypes.c_size_t * nv)(*[len(v) for v in views])
    c_raw = (ctypes.c_void_p * nv)(*[r.data_ptr() for r in raw_h])
    c_rb = (ctypes.c_size_t * nv)(*nraw)
    c_desc = (pkg._lib.RawImage * nv)(*descs)

    def step(timed_host=False):
        # the views decode concurrently on two host threads (the library's
        # batch call), then copy and convert on the stream
        for k in range(nv):
            done[k].synchronize()              # the previous copy out of raw_h[k] is over
        t0 = time.perf_counter()
        pkg._lib.check(lib.sv_image_decode_batch(nv, c_data, c_sizes, c_raw, c_rb, c_desc, None,
                                                 nv), "decode")
        if timed_host:
            host_ms.append((time.perf_counter() - t0) * 1e3)
        for k in range(nv):
            raw_d[k].copy_(raw_h[k], non_blocking=True)
            done[k].record()
            pkg._lib.check(lib.sv_raw_to_float(vp(raw_d[k]), ctypes.byref(c_desc[k]), vp(gray[k]),
                                               vp(rgbd[k]), s.cuda_stream), "raw_to_float")

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(s):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = lib.sv_launch_count()
    with ClockSampler(local) as clk, torch.cuda.stream(s):
        for i in range(args.steps):
            flush.zero_()
            e0[i].record()
            step(timed_host=True)
            e1[i].record()
        torch.cuda.synchronize()
    launches = lib.sv_launch_count() - launches0
    ms = sum(e0[i].elapsed_time(e1[i]) for i in range(args.steps))
    ms = pkg.shard.max_over_ranks(ms, device="cuda")
    value = world * 2 * N * args.steps / (ms / 1e3) / 1e6
    # the conversion kernel alone: raw samples (3 B/px) read, FP64 gray + rgb
    # (32 B/px) written
    with torch.cuda.stream(s):
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record()
        for _ in range(args.steps):
            lib.sv_raw_to_float(vp(raw_d[0]), ctypes.byref(c_desc[0]), vp(gray[0]), vp(rgbd[0]),
                                s.cuda_stream)
        k1.record()
        torch.cuda.synchronize()
    kms = k0.elapsed_time(k1) / args.steps
    # end to end through the public API: both files -> numpy FP64 gray and
    # rgb back on the host (the reference's return values)
    tmpd = tempfile.mkdtemp()
    paths = []
    for k, v in enumerate(views):
        paths.append(os.path.join(tmpd, "view%d.png" % k))
        with open(paths[-1], "wb") as f:
            f.write(v)
    x0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    x1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for _ in range(2):
        image.read_images(paths, out="numpy")
    for i in range(args.steps):
        x0[i].record()
        image.read_images(paths, out="numpy")
        x1[i].record()
    torch.cuda.synchronize()
    import shutil
    shutil.rmtree(tmpd, ignore_errors=True)
    ems = sum(x0[i].elapsed_time(x1[i]) for i in range(args.steps))
    ems = pkg.shard.max_over_ranks(ems, device="cuda")
    evalue = world * 2 * N * args.steps / (ems / 1e3) / 1e6
    if rank != 0:
        return None
    # CPU baseline: the oracle's restatement (zlib inflate + Python/numpy
    # row filters + numpy FP64) on the same two files
    sys.path.insert(0, REPO)
    from oracle import image_oracle
    t0 = time.time()
    n = 0
    while n < 1 or time.time() - t0 < min(args.cpu_seconds, 20.0):
        for v in views:
            image_oracle.read_png_bytes(v)
        n += 1
    el = time.time() - t0
    peak, peak_src = hbm_peak()
    kbytes = (3 + 32) * N
    achieved = kbytes / (kms / 1e3) / 1e9
    return {"metric": "decoded Mpix/s per B200 (PNG -> FP64 gray + RGB, bit-exact)",
            "value": round(value, 3), "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8 samples, f64 images",
            "data": "synthetic (the seeded 450x375 pair as RGB PNGs, zlib level 6, filters 0-4)",
            "config": {"workload": "read_image of both views of the 450x375 pair (%d + %d PNG "
                                   "bytes)" % (len(views[0]), len(views[1])),
                       "l2": "flushed before every step (256 MB write, untimed)",
                       "parallelism": "replicas x%d" % world},
            "stages_ms": {"host_decode_both_views_2_threads": round(statistics.median(host_ms), 4),
                          "raw_to_float_kernel_per_view": round(kms, 4)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                         "peak_source": peak_src, "kernel": "k_raw_to_float",
                         "note": "35 B/px algorithmic (3 read, 32 written); the step is bound "
                                 "by the host decode"},
            "cpu_baseline": {"value": round(n * 2 * N / el / 1e6, 6), "unit": "Mpix/s",
                             "cores": 1, "kind": "port",
                             "sample": "%d x both views through the oracle's restatement (zlib "
                                       "inflate, Python row filters, numpy FP64), %.1f s"
                                       % (n, el)},
            "e2e": {"value": round(evalue, 3), "unit": "Mpix/s",
                    "h2d_bytes_per_step": sum(nraw), "d2h_bytes_per_step": 2 * 32 * N,
                    "api": "read_images([left.png, right.png], out='numpy')"},
            "gpu_launches": int(launches), "clocks": clk.summary()}


def run_train(args, rank, world, local):
    """The training workload: a step is train_grads over a batch of 96x64
    crops (the crop size of the reference's harness, train_parallel.py:33)
    with the batch mean of the per-sample gradients, then Adam.step -- what
    the harness does with one CPU process per sample (train_parallel.py
    144-156)."""
    import numpy as np
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from importlib import import_module
    train = import_module(pkg.__name__ + ".train")
    lib = pkg._lib.load()
    net = pkg.weights.load_model()
    B, W, H = args.batch, 96, 64
    crops = [pkg.synth.make_pair(9000 + 1000 * rank + k, W, H, 2.0, 36.0, n_planes=(2, 4),
                                 lowtex_frac=0.3, bars=1) for k in range(B)]
    hl = torch.from_numpy(np.stack([c.gray("left") for c in crops]).astype(np.float32)).pin_memory()
    hr = torch.from_numpy(np.stack([c.gray("right") for c in crops]).astype(np.float32)).pin_memory()
    hd = torch.from_numpy(np.stack([c.disp for c in crops]).astype(np.float32)).pin_memory()
    hv = torch.from_numpy(np.stack([c.valid for c in crops]).astype(np.uint8)).pin_memory()
    dl, dr, dd, dv = (t.cuda() for t in (hl, hr, hd, hv))
    t = train.Trainer(net, lr=1.0e-4)
    s = torch.cuda.Stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(s):
        for _ in range(args.warmup):
            t.step(dl, dr, dd, dv)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = lib.sv_launch_count()
    with ClockSampler(local) as clk, torch.cuda.stream(s):
        for i in range(args.steps):
            flush.zero_()
            e0[i].record()
            t.step(dl, dr, dd, dv)
            e1[i].record()
        torch.cuda.synchronize()
    launches = lib.sv_launch_count() - launches0
    ms = sum(e0[i].elapsed_time(e1[i]) for i in range(args.steps))
    ms = pkg.shard.max_over_ranks(ms, device="cuda")
    value = world * B * args.steps / (ms / 1e3)
    # end to end: the batch from pinned host memory, the losses back
    x0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    x1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    hloss = torch.empty(B, dtype=torch.float64).pin_memory()
    with torch.cuda.stream(s):
        for i in range(args.steps):
            flush.zero_()
            x0[i].record()
            for dst, src in ((dl, hl), (dr, hr), (dd, hd), (dv, hv)):
                dst.copy_(src, non_blocking=True)
            loss = t.step(dl, dr, dd, dv)
            hloss.copy_(loss, non_blocking=True)
            x1[i].record()
        torch.cuda.synchronize()
    ems = sum(x0[i].elapsed_time(x1[i]) for i in range(args.steps))
    ems = pkg.shard.max_over_ranks(ems, device="cuda")
    evalue = world * B * args.steps / (ems / 1e3)
    if rank != 0:
        return None
    import __graft_entry__ as ge
    orc = ge.load_oracle()
    t0 = time.time()
    n = 0
    while n < 1 or time.time() - t0 < min(args.cpu_seconds, 20.0):
        c = crops[n % B]
        orc.train_grads(net, c.gray("left"), c.gray("right"), c.disp, c.valid, W, H)
        n += 1
    el = time.time() - t0
    return {"metric": "StereoNet training samples/s per B200 (train_grads + Adam, 96x64 crops)",
            "value": round(value, 1), "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 activations and gradients, f64 parameters and Adam",
            "data": "synthetic (seeded 96x64 crops, disparities 2-36 px, a thin bar, 30% low "
                    "texture)",
            "config": {"workload": "batch of %d crops 96x64 per step, reference checkpoint "
                                   "(12/6/12/8)" % B,
                       "l2": "flushed before every step (256 MB write, untimed)",
                       "parallelism": "replicas x%d" % world},
            "cpu_baseline": {"value": round(n / el, 3), "unit": "samples/s", "cores": 1,
                             "kind": "port",
                             "sample": "%d crops through the FP64 C port of train_grads, %.1f s, "
                                       "1 thread" % (n, el)},
            "e2e": {"value": round(evalue, 1), "unit": "samples/s",
                    "h2d_bytes_per_step": int(B * W * H * (4 * 3 + 1)),
                    "d2h_bytes_per_step": 8 * B},
            "gpu_launches": int(launches), "clocks": clk.summary()}


def main():
    args = parse()
    if args.clock_sampler:
        return clock_sampler_main(args)
    if args.cpu_leg:
        return cpu_leg_main(args)
    rank, world, local = dist_env()
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    elif args.workload == "batched":
        res = run_batched(args, rank, world, local)
    elif args.workload == "refine_disparity":
        res = run_refdisp(args, rank, world, local)
    elif args.workload == "read_image":
        res = run_image(args, rank, world, local)
    elif args.workload == "train":
        res = run_train(args, rank, world, local)
    elif args.workload == "band":
        res = run_band(args, rank, world, local)
    else:
        res = run_ours(args, rank, world, local)
    if res is not None and rank == 0:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
