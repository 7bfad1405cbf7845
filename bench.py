"""Benchmark of the nhswps time step on B200: member-steps/s at ng=256, nz=16.

Workload: the single-run configuration, ng=256 horizontal, nz=16 layers (17
levels), starting from the vstrip PV strip with a seeded N(0, 1e-3) perturbation
of q per grid point (delta = gamma = 0); one step = one predictor-corrector
``advance`` (main_invert + psolve + source, three times).  Synthetic data: there
is no dataset.  All fields (>= 8.9 MB each, ~0.5 GB working set) exceed the
126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed|fp32]
    python bench.py --impl reference ...   (CPU FP64 oracle on the host cores)

Multi-GPU: one ensemble per rank (replicas, weak scaling); the only collectives
are the timing barrier and the max-over-ranks reduction.  Launched under torchrun,
or as `python bench.py --gpus N`, which starts the N ranks itself.
"""
import argparse
import ctypes
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "shallow-water_b200")
NG, NZ = 256, 16
METRIC = "member-steps/s at ng=256 nz=16"
UNIT = "member-steps/s"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum, ncu) of one tile pass
# at ng=256 by (precision, planes per launch), averaged over two forward and two
# reverse passes of the transform micro-benchmark.  Reads are the plane data.  At
# 102 planes the written planes mostly stay in the 126 MB L2 until after the
# kernel; at 816 and 1632 planes most of them reach DRAM within it.
# Keys: (bytes per value of the pass, planes per launch).
FFT_PASS_DRAM_BYTES = {(4, 102): 26.86e6, (8, 102): 60.4e6, (8, 408): 377.3e6,
                       (4, 816): 377.7e6, (4, 1632): 805.9e6,
                       (8, 816): 803.5e6, (8, 1632): 1658.8e6}
PRECISIONS = ("fp64", "mixed", "fp32")


def load_package():
    if "shallow_water_b200" in sys.modules:
        return sys.modules["shallow_water_b200"]
    spec = importlib.util.spec_from_file_location(
        "shallow_water_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["shallow_water_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def initial_fields(ng, nz, seed, vstrip_fn):
    """vstrip PV strip replicated over the levels + N(0, 1e-3) (seeded); delta = gamma = 0."""
    qq2 = vstrip_fn(ng)
    rng = np.random.default_rng(seed)
    q3 = np.tile(qq2, nz + 1) + rng.normal(0.0, 1.0e-3, size=ng * ng * (nz + 1))
    z3 = np.zeros_like(q3)
    return q3, z3, z3.copy()


def algorithmic_bytes_per_step(ng, nz, sweeps, w_fft, corr_sweeps=0.0):
    """Algorithmic bytes of one advance step (member): one plane read + one plane
    write per 2-D transform of the reference's decomposition, plus the float64
    Thomas traffic per pressure sweep.  sweeps = psolve sweeps of the step in the
    precision w_fft (bytes per value); corr_sweeps = float32 correction sweeps of
    SW_MIXED (4-byte transforms, float32 Thomas input and correction)."""
    n2 = ng * ng
    ffts = 3 * (63 * nz + 47) + sweeps * (7 * nz + 1)
    fixed = ffts * 2 * n2 * w_fft + sweeps * (4 * nz + 2) * n2 * 8
    corr = corr_sweeps * ((7 * nz + 1) * 2 * n2 * 4 + (nz + 1) * n2 * 4 + (2 * nz - 1) * n2 * 8 + 2 * nz * n2 * 4)
    return fixed + corr


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons while running:
    through NVML every 20 ms when it is available (the GPU found by its PCI bus id,
    so that CUDA_VISIBLE_DEVICES renumbering does not matter), else through
    nvidia-smi every 200 ms.  Read-only: no setting of the GPU is touched."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.rows = []  # (sm_mhz, max_mhz, set of reason names)
        self._stop = threading.Event()
        self._th = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _run(self):
        try:
            nv, h = self._nvml_handle()
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.source = "nvml"
            while not self._stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), {k for k, b in bits.items() if r & b}))
                self._stop.wait(0.02)
            return
        except Exception:
            self.source = "nvidia-smi"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    c = [x.strip() for x in out.stdout.strip().split(",")]
                    if c[1].replace(".", "").isdigit() and c[2].replace(".", "").isdigit():
                        reasons = {n for k, n in enumerate(self.NAMES)
                                   if len(c) > 5 + k and c[5 + k].lower().startswith("active")}
                        self.rows.append((float(c[1]), float(c[2]), reasons))
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._th = threading.Thread(target=self._run, daemon=True)
        self._th.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._th.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "source": self.source}
        reasons = set()
        for _, _, r in self.rows:
            reasons |= r
        return {"sm_mhz": float(np.median([r[0] for r in self.rows])), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted(reasons), "samples": len(self.rows), "source": self.source}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def oracle_sample(steps, threads=None, warmup=1):
    """Time `steps` oracle advance steps at ng=256, nz=16 on the host cores, after
    `warmup` untimed steps (the first step's pressure solve starts from zero
    pressure and needs more sweeps than the steps after it)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    if threads:
        orc.set_num_threads(threads)
    q3, d3, g3 = initial_fields(NG, NZ, 1, orc.vstrip)
    sp, st = orc.initial_state(NG, NZ, q3, d3, g3)
    for _ in range(warmup):
        status, _, _ = orc.advance(sp, st, ggen=True)
        if status:
            raise RuntimeError("oracle advance failed: %d" % status)
    t0 = time.perf_counter()
    for _ in range(steps):
        status, _, _ = orc.advance(sp, st, ggen=True)
        if status:
            raise RuntimeError("oracle advance failed: %d" % status)
    dt = time.perf_counter() - t0
    return steps / dt, orc.num_threads(), dt


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, 2))
    warm = 1 if args.warmup > 0 else 0
    rate, cores, dt = oracle_sample(steps, warmup=warm)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "nhswps advance, ng=%d nz=%d, batched ensemble, vstrip + N(0,1e-3) q "
                               "(seed per member), delta=gamma=0" % (NG, NZ),
                   "ng": NG, "nz": NZ, "members_per_gpu": args.members, "precision": "fp64",
                   "note": "CPU members run one after another, so member-steps/s is the one-member rate"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "%d advance step(s), after %d untimed, of the FP64 C restatement of the "
                                   "reference (the Rust reference cannot be built here: no cargo), OpenMP over "
                                   "levels" % (steps, warm)},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(x, world, device="cpu"):
    """Maximum of a per-rank float over all ranks (identity for one rank)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, t_local, world, device="cpu"):
    """Whole-job units/s for independent replicas: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / max_over_ranks(t_local, world, device)


def time_fft_pass(sw, sp, planes, w_fft, reps=20, launches=2):
    """Average duration of one batched 2-D transform pass over `planes` planes,
    CUDA events on the library's stream; returns (seconds per launch, bytes per launch).
    `launches`: kernel launches per 2-D transform (2 tile passes, or 1 single-pass
    cluster launch)."""
    import torch
    L = sw._native.lib()
    stream_ptr = ctypes.c_void_p()
    sw._native.check(L.sw_stream(sp.ctx, ctypes.byref(stream_ptr)))
    stream = torch.cuda.ExternalStream(stream_ptr.value)
    dt = torch.float64 if w_fft == 8 else torch.float32
    planes = min(planes, sp.set_fft_chunk(planes))  # one launch per pass
    fbuf = torch.randn(planes * NG * NG, dtype=dt, device="cuda")
    obuf = torch.empty_like(fbuf)
    torch.cuda.synchronize()
    for _ in range(3):
        sw._native.check(L.sw_fft2d_dev(sp.ctx, 0, planes, ctypes.c_void_p(fbuf.data_ptr()), ctypes.c_void_p(obuf.data_ptr())))
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for r in range(reps):
        d = r & 1
        src, dst = (fbuf, obuf) if d == 0 else (obuf, fbuf)
        sw._native.check(L.sw_fft2d_dev(sp.ctx, d, planes, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr())))
    k1.record(stream)
    torch.cuda.synchronize()
    per_launch_s = k0.elapsed_time(k1) / 1e3 / (launches * reps)
    return per_launch_s, 2 * planes * NG * NG * w_fft


def fft_only(sw, sp, args, w_fft):
    launches = 1 if args.fft_single_pass else 2
    per, nbytes = time_fft_pass(sw, sp, args.planes, w_fft, reps=args.steps, launches=launches)
    peak, kind = measured_peak()
    print(json.dumps({"fft_pass_us": per * 1e6, "bytes_per_launch": nbytes, "gbs": nbytes / per / 1e9,
                      "frac": nbytes / per / 1e9 / peak, "planes": args.planes, "precision": args.precision,
                      "tile": sp.set_fft_tile(0), "launches_per_transform": launches,
                      "transform_us": per * launches * 1e6}))
    return 0


def prec_code(sw, name):
    return {"fp64": sw.SW_FP64, "mixed": sw.SW_MIXED, "fp32": sw.SW_FP32}[name]


def run_arm(sw, args, precision, rank, world, local, full=True, relax=None):
    """Build an ensemble context, warm up, time `steps` advance steps on the device
    (CUDA events on the library's stream) and, when `full`, the end-to-end C-ABI
    loop with host buffers and the top kernel.  Returns a dict of results and the
    member-0 prognostic fields after warmup + steps."""
    import torch
    L = sw._native.lib()
    prec = prec_code(sw, precision)
    w_fft = 4 if prec == sw.SW_FP32 else 8
    M = args.members
    sp = sw.Spectral(NG, NZ, precision=prec, nmembers=M, device=local)
    sw._native.check(L.sw_set_graphs(sp.ctx, 1 if args.graphs == "on" else 0))
    if relax is not None:
        sw._native.check(L.sw_set_psolve_relax(sp.ctx, relax))
    fft_pre = fft_step = None
    if full:  # the top kernel's pass over one member's 102 planes, timed on this context's stream
        chunk = sp.set_fft_chunk(0)
        fft_pre = time_fft_pass(sw, sp, 6 * (NZ + 1), w_fft)
        sp.set_fft_chunk(chunk)
    tune = sp.autotune() if args.autotune == "on" else None
    if full:  # and at the planes per launch the step's batched transforms use (the chunk)
        chunk = sp.set_fft_chunk(0)
        fft_step = (chunk,) + time_fft_pass(sw, sp, chunk, w_fft)
        sp.set_fft_chunk(chunk)
    qq2 = sw.vstrip.pv_strip(NG)
    for m in range(M):
        q3, d3, g3 = initial_fields(NG, NZ, args.seed0 + rank * M + m, lambda ng: qq2)
        sw.nhswps.initial_state(sp, q3, d3, g3, member=m, invert=False)
    sw.nhswps.main_invert_all(sp)
    st = sw.State(sp, member=0)
    stream_ptr = ctypes.c_void_p()
    sw._native.check(L.sw_stream(sp.ctx, ctypes.byref(stream_ptr)))
    stream = torch.cuda.ExternalStream(stream_ptr.value)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        sw._native.check(L.sw_advance(sp.ctx, 1, 1))
    sw.nhswps.diag_history(sp)
    n0, n1 = ctypes.c_longlong(), ctypes.c_longlong()
    c0, c1 = (ctypes.c_longlong * 2)(), (ctypes.c_longlong * 2)()
    barrier()
    torch.cuda.synchronize()
    sw._native.check(L.sw_kernel_launches(sp.ctx, ctypes.byref(n0)))
    sw._native.check(L.sw_sweep_counts(sp.ctx, c0))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # the K steps are queued as graph launches without a host round trip between
        # them (sw_advance_async); one sw_sync after the end event collects the status
        e0.record(stream)
        sw._native.check(L.sw_advance_async(sp.ctx, args.steps, 1))
        e1.record(stream)
        sw._native.check(L.sw_sync(sp.ctx))
        torch.cuda.synchronize()
    barrier()
    sw._native.check(L.sw_kernel_launches(sp.ctx, ctypes.byref(n1)))
    sw._native.check(L.sw_sweep_counts(sp.ctx, c1))
    ms = e0.elapsed_time(e1)
    t_local = ms / 1e3
    ref_sweeps = (c1[0] - c0[0]) / args.steps
    corr_sweeps = (c1[1] - c0[1]) / args.steps
    res = {
        "precision": precision, "w_fft": w_fft, "ms": ms, "t_local": t_local,
        "value": replica_throughput(args.steps * M, t_local, world, "cuda"),
        "launches": int(n1.value - n0.value), "sweeps": ref_sweeps + corr_sweeps,
        "sweeps_float64": ref_sweeps, "sweeps_correction": corr_sweeps, "clocks": clk.summary(),
        "tune": tune,
        "snapshot": {k: st.get(k).ravel(order="F") for k in ("qs", "ds", "gs", "pn")},
    }
    if full and args.e2e == "on":
        n3 = sp.n3 * M
        fidx = sw._native.FIELD_INDEX
        # the state makes a round trip through host memory every step: each step
        # uploads what the previous step downloaded, so the run follows one trajectory
        pinned = {k: torch.empty(n3, dtype=torch.float64, pin_memory=True) for k in ("qs", "ds", "gs", "pn")}
        outs = pinned
        for k in pinned:
            sw._native.check(L.sw_state_get_all(sp.ctx, fidx[k], ctypes.cast(pinned[k].data_ptr(), sw._native._dp), n3))
        e2e_steps = max(2, min(args.steps, 10))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for k, buf in pinned.items():
                sw._native.check(L.sw_state_set_all(sp.ctx, fidx[k], ctypes.cast(buf.data_ptr(), sw._native._dp), n3))
            sw._native.check(L.sw_advance(sp.ctx, 1, 1))
            for k, buf in outs.items():
                sw._native.check(L.sw_state_get_all(sp.ctx, fidx[k], ctypes.cast(buf.data_ptr(), sw._native._dp), n3))
        torch.cuda.synchronize()
        e2e_seq = time.perf_counter() - t0
        res["e2e"] = {"value": replica_throughput(e2e_steps * M, e2e_seq, world, "cuda"), "unit": UNIT,
                      "h2d_bytes_per_step": 4 * n3 * 8, "d2h_bytes_per_step": 4 * n3 * 8, "steps": e2e_steps,
                      "mode": "one context, each copy and step waited for; each step uploads the state "
                              "the previous step downloaded"}
        if M >= 2 and M % 2 == 0:
            pipe = e2e_pipelined(sw, L, args, M, prec, local, rank, tune, e2e_steps, world, barrier)
            res["e2e_sequential"] = res["e2e"]
            res["e2e"] = pipe
    if full:
        res["fft"] = {"planes": fft_step[0], "per_launch_s": fft_step[1], "bytes": fft_step[2],
                      "one_member": {"planes": 6 * (NZ + 1), "per_launch_s": fft_pre[0], "bytes": fft_pre[1]}}
    sp.close()
    torch.cuda.synchronize()
    return res


def e2e_pipelined(sw, L, args, M, prec, local, rank, tune, steps, world, barrier):
    """End-to-end member-steps/s through the C ABI with host buffers: the ensemble
    as two contexts of M/2 members on their own streams.  Every step of every
    member uploads qs, ds, gs, pn from pinned host memory (sw_state_set_all_async),
    advances (sw_advance_async) and downloads qs, ds, gs, pn (sw_state_get_all_async)
    into the same buffers, which the next step uploads, so the run follows one
    trajectory through host memory.  The two groups' steps alternate on the device
    (each step waits for the other group's previous step through an event), so one
    group's downloads and uploads run while the other group computes; left to the
    scheduler, the two steps interleave, finish together and leave the device idle
    while both groups copy.  Timed on the host clock from the first copy to the
    sync that completes the last download."""
    import torch
    fidx = sw._native.FIELD_INDEX
    half = M // 2
    groups = []
    qq2 = sw.vstrip.pv_strip(NG)
    for g in range(2):
        sp = sw.Spectral(NG, NZ, precision=prec, nmembers=half, device=local)
        if tune:
            sw._native.check(L.sw_set_fft_overlap(sp.ctx, tune["overlap"], None))
            sp.set_fft_tile(tune["tile"])
            sp.set_fft_chunk(tune["chosen"])
        for j in range(half):
            q3, d3, g3 = initial_fields(NG, NZ, args.seed0 + rank * M + g * half + j, lambda ng: qq2)
            sw.nhswps.initial_state(sp, q3, d3, g3, member=j, invert=False)
        sw.nhswps.main_invert_all(sp)
        sw._native.check(L.sw_advance(sp.ctx, 1, 1))  # captures the step graph
        n3 = sp.n3 * half
        ins = {k: torch.empty(n3, dtype=torch.float64, pin_memory=True) for k in ("qs", "ds", "gs", "pn")}
        outs = ins  # stream order: a step's download lands before the next step's upload reads it
        for k, buf in ins.items():
            sw._native.check(L.sw_state_get_all(sp.ctx, fidx[k], ctypes.cast(buf.data_ptr(), sw._native._dp), n3))
        groups.append((sp, n3, ins, outs))
    dp = sw._native._dp
    streams = []
    for sp, _, _, _ in groups:
        sptr = ctypes.c_void_p()
        sw._native.check(L.sw_stream(sp.ctx, ctypes.byref(sptr)))
        streams.append(torch.cuda.ExternalStream(sptr.value))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prev = None  # the last queued step's completion event
    for _ in range(steps):
        for (sp, n3, ins, outs), stream in zip(groups, streams):
            for k, buf in ins.items():
                sw._native.check(L.sw_state_set_all_async(sp.ctx, fidx[k], ctypes.cast(buf.data_ptr(), dp), n3))
            # the groups' steps alternate: each waits for the other group's step, so
            # that one group's copies run while the other group computes
            if prev is not None:
                stream.wait_event(prev)
            sw._native.check(L.sw_advance_async(sp.ctx, 1, 1))
            prev = torch.cuda.Event()
            prev.record(stream)
            for k, buf in outs.items():
                sw._native.check(L.sw_state_get_all_async(sp.ctx, fidx[k], ctypes.cast(buf.data_ptr(), dp), n3))
    for sp, _, _, _ in groups:
        sw._native.check(L.sw_sync(sp.ctx))
    secs = time.perf_counter() - t0
    nall = sum(g[1] for g in groups)
    for g in groups:
        g[0].close()
    return {"value": replica_throughput(steps * M, secs, world, "cuda"), "unit": UNIT,
            "h2d_bytes_per_step": 4 * nall * 8, "d2h_bytes_per_step": 4 * nall * 8, "steps": steps,
            "mode": "two contexts of M/2 members on their own streams; their steps alternate (event-ordered), "
                    "so one group's copies overlap the other's step; one sync at the end"}


def drift(sw, args, rank, local):
    """Energy and PV drift of one member over args.drift steps, FP64 and mixed.

    Every 50 steps: the savegrid energies (ekin, epot, etot) and the domain-mean
    PV anomaly of each level (the k = 0 mode of qs, which the spectral update
    conserves: diss(0) = 1).  Reports the relative drift of etot (hyperdiffusion
    dissipates energy, so the FP64 drift is the physical reference for the mixed
    one), the largest change of the mean PV, and the final mixed-vs-FP64
    differences."""
    if rank != 0:
        return 0
    import torch
    L = sw._native.lib()
    qq2 = sw.vstrip.pv_strip(NG)
    q3, d3, g3 = initial_fields(NG, NZ, 1, lambda ng: qq2)
    out = {"mode": "drift", "workload": "nhswps, one member, ng=%d nz=%d, vstrip + N(0,1e-3) q, delta=gamma=0"
                                         % (NG, NZ), "steps": args.drift, "ng": NG, "nz": NZ}
    finals = {}
    for prec_name in PRECISIONS:
        sp = sw.Spectral(NG, NZ, precision=prec_code(sw, prec_name), device=local)
        st = sw.nhswps.initial_state(sp, q3, d3, g3)
        sw.nhswps.psolve(st)  # z, w and p of the initial state, so that its energies are complete
        rec = []
        t0 = time.perf_counter()
        done = 0
        while True:
            e = sw.nhswps.energy(st)
            qs = st.get("qs")
            rec.append((done, float(e[2]), [float(qs[0, 0, iz]) for iz in range(NZ + 1)], float(e[0]), float(e[1])))
            if done >= args.drift:
                break
            n = min(50, args.drift - done)
            sw._native.check(L.sw_advance(sp.ctx, n, 1))
            done += n
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e0 = rec[0][1]
        pv0 = np.array(rec[0][2])
        pvmax = max(float(np.max(np.abs(np.array(r[2]) - pv0))) for r in rec)
        out[prec_name] = {
            "etot_start": e0, "etot_end": rec[-1][1], "etot_rel_drift": (rec[-1][1] - e0) / e0,
            "etot_max_rel_dev": max(abs(r[1] - e0) for r in rec) / abs(e0),
            "ekin_end": rec[-1][3], "epot_end": rec[-1][4],
            "pv_mean_max_abs_change": pvmax, "pv_mean_scale": float(np.max(np.abs(pv0))) if np.any(pv0) else 0.0,
            "wall_s": wall, "steps_per_s": args.drift / wall,
            "etot_every_50": [r[1] for r in rec],
        }
        finals[prec_name] = {k: st.get(k).ravel(order="F") for k in ("qs", "ds", "gs")}
        sp.close()
    for name in ("mixed", "fp32"):
        out[name + "_vs_fp64_after"] = {k: float(np.linalg.norm(finals[name][k] - finals["fp64"][k]) /
                                                max(np.linalg.norm(finals["fp64"][k]), 1e-300))
                                        for k in ("qs", "ds", "gs")}
        out["etot_%s_minus_fp64_rel" % name] = ((out[name]["etot_end"] - out["fp64"]["etot_end"]) /
                                               abs(out["fp64"]["etot_end"]))
    print(json.dumps(out), flush=True)
    return 0


def uneven(sw, args, rank, world, local):
    """Ensemble of members with uneven grids: ng from {64, 96, 128, 192, 256}, nz
    from {4, 8, 16}, drawn with a fixed seed, as one sw_ensemble: members of one
    (ng, nz) share a batched context, and a step of every member is one CUDA graph
    launch whose branches are the groups' steps.  Timed with CUDA events around the
    queued steps on the ensemble's stream."""
    import torch
    rng = np.random.default_rng(2024 + rank)
    draws = [(int(rng.choice([64, 96, 128, 192, 256])), int(rng.choice([4, 8, 16]))) for _ in range(args.uneven)]
    prec = prec_code(sw, args.precision)
    ens = sw.nhswps.Ensemble([d[0] for d in draws], [d[1] for d in draws], precision=prec, device=local)
    strips = {}
    for k, (ng, nz) in enumerate(draws):
        if ng not in strips:
            strips[ng] = sw.vstrip.pv_strip(ng)
        q3, d3, g3 = initial_fields(ng, nz, 100 + k, lambda n: strips[ng])
        ens.initial_state(k, q3, d3, g3)
    ens.invert_all()
    groups = {}
    for k, key in enumerate(draws):
        groups.setdefault(key, []).append(k)
    if args.autotune == "on":
        seen = set()
        for k in range(len(draws)):
            sp, _ = ens.member(k)
            if id(sp) not in seen:
                seen.add(id(sp))
                sp.autotune()
    ens.advance(args.warmup)  # the first step captures the combined graph
    torch.cuda.synchronize()
    es = torch.cuda.ExternalStream(ens.stream())
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(es)
        ens.advance_async(args.steps)
        stop.record(es)
        ens.sync()
        torch.cuda.synchronize()
    secs = start.elapsed_time(stop) / 1e3
    secs = max_over_ranks(secs, world, "cuda")
    points = sum(len(m) * ng * ng * (nz + 1) for (ng, nz), m in groups.items())
    if rank == 0:
        line = {
            "metric": "member-steps/s, uneven ensemble", "value": world * args.uneven * args.steps / secs,
            "unit": "member-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True, "scaling": "weak",
            "dtype": {"fp64": "f64", "mixed": "f64+f32", "fp32": "f32+f64"}[args.precision], "data": "synthetic",
            "config": {"workload": "uneven ensemble: %d members, ng in {64,96,128,192,256}, nz in {4,8,16} "
                                   "(seeded draw), vstrip + N(0,1e-3) q per member; one graph launch per step "
                                   "of every member" % args.uneven,
                       "groups": [{"ng": ng, "nz": nz, "members": len(m)} for (ng, nz), m in sorted(groups.items())],
                       "precision": args.precision},
            "grid_point_steps_per_s": world * points * args.steps / secs,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ens.close()
    return 0


def kernels(sw, args, rank, local):
    """Standalone kernels on device buffers, timed with CUDA events (reps launches
    after 3 warm-ups): forfft/revfft at n in {32, 96, 160, 256, 384, 512} over
    17 n columns, float64 and float32, N(0,1) input (seed 2); batched tridiagonal
    solves, 65,536 systems of 17 unknowns, diagonal U[2,4], off-diagonals
    U[-1,1], right-hand side N(0,1) (seed 3).  Algorithmic bytes: one read and
    one write of the batch per transform; a, b, c, d read and x written once per
    tridiagonal solve."""
    if rank != 0:
        return 0
    import torch
    L = sw._native.lib()
    peak, peak_kind = measured_peak()
    reps = max(5, args.steps)
    s = torch.cuda.Stream()
    sp = ctypes.c_void_p(s.cuda_stream)
    rows = []

    def timed(fn):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    rng = np.random.default_rng(2)
    for n in (32, 96, 160, 256, 384, 512):
        m = 17 * n
        for prec_name, prec, dt in (("fp64", sw.SW_FP64, torch.float64), ("fp32", sw.SW_FP32, torch.float32)):
            x = torch.from_numpy(rng.standard_normal(m * n)).to(dt).cuda()
            xp = ctypes.c_void_p(x.data_ptr())
            nbytes = 2 * m * n * x.element_size()
            for name, f in (("forfft", L.sw_forfft_dev), ("revfft", L.sw_revfft_dev)):
                t = timed(lambda: sw._native.check(f(m, n, xp, prec, sp)))
                rows.append({"kernel": name, "n": n, "columns": m, "precision": prec_name, "us": t * 1e6,
                             "gbs": nbytes / t / 1e9, "frac": nbytes / t / 1e9 / peak})
    rng = np.random.default_rng(3)
    n, nsys = 17, 65536
    arrs = [torch.from_numpy(v).cuda() for v in (rng.uniform(-1, 1, (n, nsys)), rng.uniform(2, 4, (n, nsys)),
                                                  rng.uniform(-1, 1, (n, nsys)), rng.standard_normal((n, nsys)))]
    xo = torch.empty_like(arrs[0])
    ptrs = [ctypes.c_void_p(v.data_ptr()) for v in arrs] + [ctypes.c_void_p(xo.data_ptr())]
    t = timed(lambda: sw._native.check(L.sw_tridiag_batched(n, nsys, *ptrs, sp)))
    nbytes = 5 * n * nsys * 8
    rows.append({"kernel": "tridiag_batched", "n": n, "systems": nsys, "precision": "fp64", "us": t * 1e6,
                 "gbs": nbytes / t / 1e9, "frac": nbytes / t / 1e9 / peak})
    print(json.dumps({"mode": "kernels", "peak_gbs": peak, "peak_kind": peak_kind, "reps": reps,
                      "note": "inputs below the 126 MB L2 for small n: the smaller cases partly run from L2",
                      "rows": rows}), flush=True)
    return 0


def accuracy(sw, args, rank, local):
    """Mixed vs FP64 on one member at (--ng, --nz) after --steps steps from the
    same vstrip + N(0,1e-3) initial state: rel-L2 of each prognostic field and of
    h = z(nz)/HBAR - 1, and the step rates."""
    if rank != 0:
        return 0
    import torch
    L = sw._native.lib()
    qq2 = sw.vstrip.pv_strip(NG)
    q3, d3, g3 = initial_fields(NG, NZ, args.seed0, lambda ng: qq2)
    res, rates = {}, {}
    for prec_name in PRECISIONS:
        sp = sw.Spectral(NG, NZ, precision=prec_code(sw, prec_name), device=local)
        st = sw.nhswps.initial_state(sp, q3, d3, g3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sw._native.check(L.sw_advance(sp.ctx, args.steps, 1))
        rates[prec_name] = args.steps / (time.perf_counter() - t0)
        f = {k: st.get(k).ravel(order="F") for k in ("qs", "ds", "gs", "pn", "u", "z")}
        f["h"] = f["z"][-NG * NG:] / 0.4 - 1.0
        res[prec_name] = f
        sp.close()
    err = {name: {k: float(np.linalg.norm(res[name][k] - res["fp64"][k]) / max(np.linalg.norm(res["fp64"][k]), 1e-300))
                  for k in res["fp64"]} for name in ("mixed", "fp32")}
    print(json.dumps({"mode": "accuracy", "ng": NG, "nz": NZ, "steps": args.steps,
                      "workload": "one member, vstrip + N(0,1e-3) q, delta=gamma=0",
                      "mixed_rel_l2_vs_fp64": err["mixed"], "fp32_rel_l2_vs_fp64": err["fp32"],
                      "steps_per_s_incl_first_graph_capture": rates}), flush=True)
    return 0


def free_port():
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def relaunch(n):
    """`--gpus N` without a torchrun environment: start N ranks of this same command
    line under torch.distributed.run (one process per GPU, rendezvous on 127.0.0.1)
    and return their exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % n,
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def rank_check(args, rank, world):
    """--rank-check: each rank joins a gloo process group (CPU) and rank 0 prints
    the ranks and world size that the launch produced; no GPU work."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    t = torch.tensor([rank], dtype=torch.int64)
    got = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(got, t)
    if rank == 0:
        print(json.dumps({"mode": "rank-check", "world_size": world, "gpus": args.gpus,
                          "ranks": [int(g.item()) for g in got]}), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


def main():
    global NG, NZ, METRIC
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=list(PRECISIONS),
                    help="precision of the timed (headline) path: mixed = float64 with float32 pressure "
                         "correction sweeps (the 1e-5 contract); fp32 = float32 transforms and work fields")
    ap.add_argument("--members", type=int, default=16, help="ensemble members per GPU (one batched context)")
    ap.add_argument("--compare", default="on", choices=["on", "off"],
                    help="also time the other precision on the same ensemble and report the ratio and the "
                         "mixed-vs-FP64 rel-L2 after the timed steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fft-only", action="store_true",
                    help="only time the batched 2-D transform pass (for profiling the top kernel)")
    ap.add_argument("--planes", type=int, default=None, help="planes of the --fft-only pass (default 6*(nz+1))")
    ap.add_argument("--fft-single-pass", action="store_true",
                    help="--fft-only: the single-pass cluster transform (n = 256) instead of the two tile passes")
    ap.add_argument("--fft-tile", type=int, default=0, choices=[0, 16, 32],
                    help="columns per tile of the --fft-only pass at ng=256 (0: the precision's default)")
    ap.add_argument("--ng", type=int, default=NG, help="horizontal grid (the headline workload is 256)")
    ap.add_argument("--nz", type=int, default=NZ, help="layers (the headline workload is 16)")
    ap.add_argument("--kernels", action="store_true",
                    help="time the standalone kernels: forfft/revfft at n in {32,...,512} (17n columns, FP64 and "
                         "FP32) and the batched tridiagonal solve (65,536 x 17)")
    ap.add_argument("--seed0", type=int, default=1, help="seed of member 0 (member m uses seed0 + m)")
    ap.add_argument("--accuracy", action="store_true",
                    help="run one member --steps steps in FP64 and in the mixed path at (--ng, --nz) and report "
                         "their rel-L2 differences (the ng=512 nz=32 sweep)")
    ap.add_argument("--drift", type=int, default=0, metavar="STEPS",
                    help="instead of timing: run one member STEPS steps in FP64 and in the mixed path and "
                         "report energy and PV drift")
    ap.add_argument("--uneven", type=int, default=0, metavar="MEMBERS",
                    help="time an ensemble of MEMBERS members with ng drawn from {64,96,128,192,256} and nz "
                         "from {4,8,16}: one batched context per (ng, nz) group, groups run concurrently")
    ap.add_argument("--autotune", default="on", choices=["on", "off"],
                    help="time the 2-D transform tile-width, launch-chunk and two-stream pipeline candidates "
                         "before warm-up and "
                         "keep the fastest")
    ap.add_argument("--e2e", default="on", choices=["on", "off"],
                    help="also measure the end-to-end loop through the C ABI with host buffers (off: for "
                         "profiling runs)")
    ap.add_argument("--rank-check", action="store_true",
                    help="only start the ranks (gloo, CPU) and print their ranks and world size")
    ap.add_argument("--psolve-relax", type=float, default=None, metavar="OMEGA",
                    help="relaxation factor of the pressure iteration of the benchmarked arm (default 1, the "
                         "reference's iteration)")
    ap.add_argument("--graphs", default="on", choices=["on", "off"],
                    help="run each step as one CUDA graph (on) or host-driven (off; same kernels, for profiling)")
    args = ap.parse_args()
    NG, NZ = args.ng, args.nz
    METRIC = "member-steps/s at ng=%d nz=%d" % (NG, NZ)
    if args.planes is None:
        args.planes = 6 * (NZ + 1)

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args.gpus)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.rank_check:
        return rank_check(args, rank, world)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    sw = load_package()
    if args.fft_only:
        prec = prec_code(sw, args.precision)
        # the intermediate holds 6 (nz+1) planes per member: enough members for --planes
        nmem = max(1, -(-args.planes // (6 * (NZ + 1))))
        sp = sw.Spectral(NG, NZ, precision=prec, nmembers=nmem, device=local)
        if args.fft_tile:
            sp.set_fft_tile(args.fft_tile)
        if args.fft_single_pass:
            sw._native.check(sw._native.lib().sw_set_fft_single_pass(sp.ctx, 1, None))
        return fft_only(sw, sp, args, 4 if prec == sw.SW_FP32 else 8)
    if args.kernels:
        return kernels(sw, args, rank, local)
    if args.accuracy:
        return accuracy(sw, args, rank, local)
    if args.drift:
        return drift(sw, args, rank, local)
    if args.uneven:
        return uneven(sw, args, rank, world, local)

    main_arm = run_arm(sw, args, args.precision, rank, world, local, full=True, relax=args.psolve_relax)
    arms = {args.precision: main_arm}
    if args.compare == "on":
        # every rank runs the same arms in the same order (the barriers inside match)
        for name in PRECISIONS:
            if name not in arms:
                arms[name] = run_arm(sw, args, name, rank, world, local, full=False)

    M = args.members
    w_fft = main_arm["w_fft"]
    peak, peak_kind = measured_peak()
    fft = main_arm["fft"]
    achieved = fft["bytes"] / fft["per_launch_s"] / 1e9
    one = fft["one_member"]
    achieved_one = one["bytes"] / one["per_launch_s"] / 1e9
    traffic = FFT_PASS_DRAM_BYTES.get((w_fft, fft["planes"])) if NG == 256 else None
    traffic_one = FFT_PASS_DRAM_BYTES.get((w_fft, one["planes"])) if NG == 256 else None
    step_bytes = algorithmic_bytes_per_step(NG, NZ, main_arm["sweeps_float64"], w_fft, main_arm["sweeps_correction"])
    step_gbs = step_bytes * (args.steps * M / main_arm["t_local"]) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, dt = oracle_sample(1)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "1 advance step at ng=%d nz=%d (one member), after 1 untimed, of the FP64 C "
                         "restatement (OpenMP over levels); %.1f s" % (NG, NZ, dt)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": main_arm["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main_arm["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "mixed": "f64+f32", "fp32": "f32+f64"}[args.precision], "data": "synthetic",
            "config": {"workload": "nhswps advance, ng=%d nz=%d, batched ensemble, vstrip + N(0,1e-3) q "
                                   "(seed per member), delta=gamma=0" % (NG, NZ),
                       "ng": NG, "nz": NZ, "members_per_gpu": M, "precision": args.precision,
                       "parallelism": "replicas" if world > 1 else "single", "l2": "inputs larger than L2",
                       "psolve_sweeps_per_step": main_arm["sweeps"],
                       "psolve_sweeps_per_step_float64": main_arm["sweeps_float64"],
                       "psolve_sweeps_per_step_float32_correction": main_arm["sweeps_correction"],
                       "timing": "K graph-launched steps queued without host round trips, CUDA events on the "
                                 "library's stream",
                       "precision_note": {"fp64": "float64 throughout",
                                          "mixed": "float64 fields and most transforms; float32 correction "
                                                   "sweeps after each solve's float64 reference sweep (stop rule "
                                                   "1e-7), and float32 transforms for the dealiased products "
                                                   "and filters of the pressure set-up and of source",
                                          "fp32": "float32 transforms and work fields; not within 1e-5 on "
                                                  "delta/gamma at ng=256"}[args.precision],
                       "psolve_relax": args.psolve_relax if args.psolve_relax is not None else 1.0,
                       "fft_autotune": main_arm["tune"]},
            "e2e": main_arm.get("e2e"),
            "e2e_sequential": main_arm.get("e2e_sequential"),
            "gpu_launches": main_arm["launches"],
            "roofline": {"bound": "hbm", "kernel": "k_fft_pass_r (batched 2-D transform pass, %d planes per "
                                                   "launch: the step's chunk)" % fft["planes"],
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "one_member_pass": {"planes": one["planes"], "achieved": achieved_one,
                                             "frac": achieved_one / peak, "traffic": traffic_one},
                         "step_algorithmic_gbs": step_gbs, "step_frac": step_gbs / peak},
            "cpu_baseline": cpu,
            "clocks": main_arm["clocks"],
        }
        if all(name in arms for name in PRECISIONS):
            fp64 = arms["fp64"]
            cmp = {"after_steps": args.warmup + args.steps, "fp64_value": fp64["value"],
                   "fp64_sweeps_per_step": fp64["sweeps"], "fp64_clocks": fp64["clocks"]}
            for name in ("mixed", "fp32"):
                a = arms[name]
                cmp[name + "_value"] = a["value"]
                cmp[name + "_over_fp64"] = a["value"] / fp64["value"]
                cmp[name + "_sweeps_per_step"] = {"float64": a["sweeps_float64"], "float32_correction":
                                                  a["sweeps_correction"]}
                cmp[name + "_rel_l2_vs_fp64"] = {k: float(np.linalg.norm(a["snapshot"][k] - fp64["snapshot"][k]) /
                                                          max(np.linalg.norm(fp64["snapshot"][k]), 1e-300))
                                                 for k in ("qs", "ds", "gs", "pn")}
            line["compare"] = cmp
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
