#!/usr/bin/env python3
"""Benchmark: zone-updates/s of AstroFD's per-step RHS on the B200.

Workload (default): RMHD 256^3 magnetised jet, Gamma = 4/3, WENO5 + "hlld"
(HLLC hydro + HLLE field), SSPRK3, resistivity 1e-4, two-temperature
(TEI_TAU 0.1) and cooling (lambda 0.01), NG = 3, 11 variables.  One "step" is
one iteration of the reference driver loop (solvers/srhd3d_mpi_muscl.py:276-326):
ghost fill, SSPRK3 step, ghost fill, cooling, two-temperature.  dt = CFL dx
with CFL 0.35 (the reference uses amax = 1 for RMHD).

Arms
  default            mixed precision (float32 reconstruction/Riemann, float64
                     state / RK / con2prim) on the GPU; also times the plain
                     float64 GPU path for the speed-up in the same line.
  --impl reference   the reference algorithm on the host cores (the C port of
                     the reference's Numba kernels, all threads), on a bounded
                     x-slab sample of the same state.

Timing: CUDA events on the launching stream around exactly K steps after W
warm-up steps, barrier + synchronize on both sides, max over ranks.  Every
array (1.6 GB each) is larger than the 126 MB L2, so no explicit flush.
With --gpus N (default --decomp slab) the ranks hold the x-slabs of one jet of
N n x n x n cells (weak scaling: n^3 cells per GPU): once per step each rank
swaps NG = 3 ghost layers with its x-neighbours over NCCL (send/recv, the
reference driver's exchange), the first rank drives the nozzle and the last
the +x outflow.  --decomp replicas runs N independent blocks instead.  value =
N x per-rank work / max time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from astrofd_b200.driver import STABLE, DriverStep, norms as _norms, rho_l1_arms  # noqa: E402

METRIC = "zone-updates/s 256^3 RMHD (mixed+learned c2p vs FP64 plain, L1<1e-4)"
UNIT = "zone-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--flux-mode", default="conservative", choices=["conservative", "reference"])
    ap.add_argument("--boundaries", default="baseline", choices=["baseline", "reference"],
                    help="baseline: outflow on every face but the nozzle and a toroidal "
                         "B_phi(r) jet field on the ambient Bx (the configuration as "
                         "specified); reference: the reference driver's periodic y/z, "
                         "fixed ambient inlet and By = B0 s")
    ap.add_argument("--decomp", default="slab", choices=["slab", "replicas"],
                    help="with --gpus N > 1: x-slabs of one jet with a ghost exchange per "
                         "step, or N independent blocks")
    ap.add_argument("--halo", default="step", choices=["step", "stage"],
                    help="with --decomp slab: exchange the ghost layers once per step (the "
                         "reference driver) or after every RK stage as well (the ranks then "
                         "compute exactly what one block would)")
    ap.add_argument("--graph", action="store_true",
                    help="replay CUDA graphs of one driver iteration in the timed steps "
                         "(kernel-class times then come from profiled steps after them)")
    ap.add_argument("--segment", type=int, default=8,
                    help="time the steps in segments of at most this many, each from the "
                         "state after the warm-up (restored untimed), so every timed step "
                         "lies in the jet's sane window; 0: one segment")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the untimed accuracy runs of the bench line")
    ap.add_argument("--workload", default="c5", choices=["c5", "c1", "c2", "c3"],
                    help="c5: the headline 256^3 RMHD jet (this line's contract); c1, c2, "
                         "c3: the other named jets at their own sizes (zone-updates/s of "
                         "their driver loops, float64 and, for c2/c3, mixed precision)")
    ap.add_argument("--stage-kernel", default="split", choices=["fused", "split"],
                    help="fused: one kernel per SSPRK stage (TMA tiles, faces and update "
                         "together); split: per-direction face passes, then the update")
    ap.add_argument("--no-fp64", action="store_true", help="skip the float64 comparison arm")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-x-cells", type=int, default=4,
                    help="x-slab thickness of the bounded CPU sample")
    ap.add_argument("--c2p-net", default=None,
                    help="learned con2prim weights (.npz); default: the packaged network")
    ap.add_argument("--no-learned", action="store_true",
                    help="headline arm without the learned con2prim guess")
    ap.add_argument("--validate-srhd", action="store_true",
                    help="with --validate-steps: the SRHD jet (PPM + HLLC, SSPRK3, v 0.995)")
    ap.add_argument("--c2p-batch", type=int, default=0, metavar="STATES",
                    help="learned con2prim on a batch of sampled states (2^24 for the "
                         "batch config) against the full float64 Newton, then exit")
    ap.add_argument("--c2p-jet", action="store_true",
                    help="with --c2p-batch: states of a 128^3 jet run instead of the sampler")
    ap.add_argument("--validate-steps", type=int, default=0,
                    help="instead of timing: run this many steps of mixed+learned, plain "
                         "float64, float64 with a 1e-12 density perturbation and the two "
                         "halves of the mixed+learned path (mixed faces with the "
                         "reference's con2prim start, float64 faces with the learned "
                         "start) in lockstep, and report density L1 errors against plain "
                         "float64 and conservative-mode mass drift")
    ap.add_argument("--validate-every", type=int, default=10,
                    help="with --validate-steps: report the errors every this many steps")
    ap.add_argument("--jet-v", type=float, default=0.995, help="jet three-velocity")
    ap.add_argument("--sigma-jet", type=float, default=0.5,
                    help="jet magnetisation (toroidal field); 0: unmagnetised jet")
    ap.add_argument("--sigma-amb", type=float, default=0.01,
                    help="ambient magnetisation (uniform Bx); 0: unmagnetised medium")
    return ap.parse_args()


# ------------------------------------------------------------------ ranks --
def dist_init(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        # one process per GPU over NCCL; gloo where there is no GPU (the CPU
        # tests of this rank logic).  The timeout ends a rank whose peer died.
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
    return rank, world, local


def slab_domain(args, world):
    """The x-slab of this rank in a jet of world x n cells along x, or None
    (one GPU, or independent replicas)."""
    if world <= 1 or args.decomp != "slab":
        return None
    from astrofd_b200.slabs import SlabDomain
    return SlabDomain(args.n * world, 3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during timing:
    every 20 ms through NVML's read-only queries, or every 200 ms from
    nvidia-smi where NVML is unavailable.  The GPU is addressed by its PCI
    bus id, which does not depend on CUDA_VISIBLE_DEVICES."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.nvml = []
        self.stop = None
        self.source = None
        try:
            import torch
            pr = torch.cuda.get_device_properties(index)
            self.bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        except Exception:
            self.bus = str(index)

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByPciBusId(self.bus.encode())
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.stop = threading.Event()

            def poll():
                while not self.stop.is_set():
                    try:
                        self.nvml.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), mx,
                                          pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)))
                    except Exception:
                        pass
                    self.stop.wait(0.02)

            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            self.source = "nvml"
            return self
        except Exception:
            self.stop = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.bus}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.source = "nvidia-smi"
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.stop is not None:
            self.stop.set()
            self.t.join(timeout=2)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.nvml:
            sm = [s for s, _, _ in self.nvml]
            reasons = sorted({k for _, _, r in self.nvml for k, b in self.BITS.items() if r & b})
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(self.nvml[0][1]),
                    "reasons": reasons, "samples": len(sm), "source": "nvml, 20 ms"}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ------------------------------------------------------------------- GPU ---
def time_arm(args, world, prec, pr_host, cfgs, profile, learned=False):
    import ctypes as C
    import torch
    from astrofd_b200 import _lib
    from astrofd_b200.core import rmhd_core
    core, noz, src = cfgs
    cfg = dict(core, PRECISION=prec, FLUX_MODE=args.flux_mode,
               C2P_GUESS="learned" if learned else "reference", STAGE_KERNEL=args.stage_kernel)
    rmhd_core.configure(cfg)
    if learned:
        from astrofd_b200 import learned_c2p
        rmhd_core.set_c2p_network(learned_c2p.load(args.c2p_net or learned_c2p.DATA))
    step = DriverStep(args.n, 3, core, noz, src, slab_domain(args, world), args.halo)
    a = torch.from_numpy(pr_host).to("cuda")
    b = torch.empty_like(a)
    for _ in range(args.warmup):
        a, b, _ = step(a, b)
    L = _lib.load()
    # --graph: one driver iteration is a fixed sequence of kernels on fixed
    # buffers (no host-drawn nozzle perturbation in this workload): capture
    # a -> b and b -> a as CUDA graphs and replay them.  Slab runs (NCCL
    # exchange in the step) launch eagerly.
    graphs, per_iter, graph_note = None, 0, "eager launches"
    if args.graph and step.slab is None:
        try:
            torch.cuda.synchronize()
            g1, g2 = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
            l0 = L.astro_launch_count()
            with torch.cuda.graph(g1):
                step(a, b)
            per_iter = L.astro_launch_count() - l0
            with torch.cuda.graph(g2):
                step(b, a)
            graphs = (g1, g2)
            graph_note = f"CUDA graphs of one driver iteration ({per_iter} kernels), replayed"
        except Exception as e:  # capture unsupported here: time eager launches
            graphs, graph_note = None, f"eager launches (graph capture failed: {e})"[:200]
            torch.cuda.synchronize()
    rmhd_core.c2p_stats(reset=True)
    stream = torch.cuda.current_stream()
    prof_ms = np.zeros(5)
    prof_n = np.zeros(5, dtype=np.int64)
    # eager timed steps of the profiled arm: an event after every launch
    # (astro_prof_start/stop), read after each timed segment, so the
    # kernel-class times are those of the timed steps, with no host
    # synchronisation among them
    session = profile and graphs is None
    # Segments of at most --segment steps, each from the state reached after
    # the warm-up (restored, untimed, between segments): the jet's flow stays
    # sane for the first ~13 driver steps at 256^3 and then blows up (the
    # reference scheme's own behaviour), so every timed step is one of steps
    # warmup+1 .. warmup+segment.  The time is the sum of the segments' CUDA
    # event times.
    seg = args.segment if 0 < args.segment < args.steps else args.steps
    saved = (a.clone(), b.clone()) if seg < args.steps else None
    barrier(world)
    torch.cuda.synchronize()
    l0 = L.astro_launch_count()
    ms_local, done, segments = 0.0, 0, 0
    with ClockSampler(torch.cuda.current_device()) as clk:
        while done < args.steps:
            if saved is not None and done > 0:
                a.copy_(saved[0])
                b.copy_(saved[1])
            m = min(seg, args.steps - done)
            if session:
                _lib.check(L.astro_prof_start(64 * m + 64, C.c_void_p(stream.cuda_stream)),
                           "astro_prof_start")
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(m):
                if graphs is not None:
                    graphs[i % 2].replay()
                    a, b = b, a
                else:
                    a, b, _ = step(a, b)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_local += e0.elapsed_time(e1)
            if session:
                kt = _lib.AstroKernelTimes()
                _lib.check(L.astro_prof_stop(C.byref(kt)), "astro_prof_stop")
                prof_ms += np.array([kt.ms[i] for i in range(5)])
                prof_n += np.array([kt.launches[i] for i in range(5)])
            done += m
            segments += 1
    barrier(world)
    launches = (L.astro_launch_count() - l0) if graphs is None else per_iter * args.steps
    ms = max_over_ranks(ms_local, world)
    finite = bool(torch.isfinite(a).all().item())
    stats = rmhd_core.c2p_stats(reset=True)
    state = a
    prof_steps, times_from = (args.steps, "the timed steps") if session else (0, None)
    if profile and not session:
        # graph replay: per-kernel-class times from a few more steps after the
        # timed ones (astro_step_profiled synchronises after every step)
        state = a.clone()
        prof_steps = max(1, min(args.steps, 3))
        times_from = f"{prof_steps} profiled steps after the timed ones"
        for _ in range(prof_steps):
            a, b, t = step(a, b, profile=True)
            prof_ms += np.array(t[0])
            prof_n += np.array(t[1])
    if graphs is not None:
        del graphs
    return dict(ms=ms, launches=int(launches), prof_ms=prof_ms, prof_n=prof_n,
                prof_steps=prof_steps, clocks=clk.summary(), finite=finite, state=state,
                c2p=stats, launch_mode=graph_note, times_from=times_from, segments=segments,
                segment=seg)


def time_e2e(args, world, prec, pr_host, cfgs, learned=False):
    """Public API with host buffers: every step uploads its input block from
    pinned host memory and reads its result back into pinned host memory.
    The blocks are independent, so the copies are double-buffered on two copy
    streams: the upload of step k+1 and the read-back of step k-1 overlap the
    compute of step k (full-duplex PCIe), and every step's two copies lie
    inside the timed region."""
    import torch
    from astrofd_b200.core import rmhd_core
    core, noz, src = cfgs
    rmhd_core.configure(dict(core, PRECISION=prec, FLUX_MODE=args.flux_mode,
                             C2P_GUESS="learned" if learned else "reference",
                             STAGE_KERNEL=args.stage_kernel))
    if learned:
        from astrofd_b200 import learned_c2p
        rmhd_core.set_c2p_network(learned_c2p.load(args.c2p_net or learned_c2p.DATA))
    step = DriverStep(args.n, 3, core, noz, src, slab_domain(args, world), args.halo)
    host_in = torch.from_numpy(pr_host).pin_memory()
    host_out = [torch.empty_like(host_in).pin_memory() for _ in range(2)]
    dev_in = [torch.empty(host_in.shape, dtype=torch.float64, device="cuda") for _ in range(2)]
    dev_out = [torch.empty_like(dev_in[0]) for _ in range(2)]
    comp = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event()
    computed, uploaded, read = [ev(), ev()], [ev(), ev()], [ev(), ev()]
    for i in range(2):  # all buffers free
        computed[i].record(comp)
        read[i].record(comp)

    def run(k0, k, start=None):
        if start is not None:
            up.wait_event(start)
        for s in range(k0, k0 + k):
            i = s % 2
            up.wait_event(computed[i])          # dev_in[i] no longer in use
            with torch.cuda.stream(up):
                dev_in[i].copy_(host_in, non_blocking=True)
            uploaded[i].record(up)
            comp.wait_event(uploaded[i])
            comp.wait_event(read[i])            # dev_out[i] read back already
            step(dev_in[i], dev_out[i])
            computed[i].record(comp)
            down.wait_event(computed[i])
            with torch.cuda.stream(down):
                host_out[i].copy_(dev_out[i], non_blocking=True)
            read[i].record(down)
        comp.wait_event(read[(k0 + k - 1) % 2])
        comp.wait_event(read[(k0 + k - 2) % 2])

    run(0, max(2, min(args.warmup, 2)))
    # enough steps that filling and draining the copy pipeline (one upload
    # before the first step, one read-back after the last) is amortised
    k = min(max(args.steps, 8), 16)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(comp)
    run(0, k, start=e0)
    e1.record(comp)
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    nbytes = host_in.numel() * 8
    # the link floor: one step's upload and read-back run concurrently,
    # nothing else on the GPU
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    torch.cuda.synchronize()
    f0.record(comp)
    for _ in range(reps):
        up.wait_stream(comp)
        down.wait_stream(comp)
        with torch.cuda.stream(up):
            dev_in[0].copy_(host_in, non_blocking=True)
        with torch.cuda.stream(down):
            host_out[0].copy_(dev_out[0], non_blocking=True)
        comp.wait_stream(up)
        comp.wait_stream(down)
    f1.record(comp)
    torch.cuda.synchronize()
    return dict(ms=ms, steps=k, h2d=nbytes, d2h=nbytes, link_ms=f0.elapsed_time(f1) / reps)


# ------------------------------------------------------------------- CPU ---
def cpu_sample(args, steps, warmup):
    """The reference algorithm (C port of the Numba kernels) on the host cores:
    the same driver iteration on an x-slab of the same state."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config
    n, ng, xc = args.n, 3, args.cpu_x_cells
    core, noz, src = rmhd_jet_config(n, ng, boundaries=args.boundaries)
    # the reference's own arithmetic (loop-carried x-face speeds, its resistive
    # handling), whatever flux mode the GPU arm runs
    cfg = dict(core, FLUX_MODE="reference")
    P = O.params_from_config("rmhd", cfg)
    pr = rmhd_jet(n, ng, x_cells=xc)
    d = 1.0 / n
    dt = core["CFL"] * d
    rng = np.random.default_rng(1234)

    def bcs(a):
        if noz.get("YZ_BOUNDARY") == "outflow":
            O.apply_outflow_yz(a, ng)
        else:
            O.apply_periodic_yz(a, ng)
        O.apply_outflow_right_x(a, ng)
        O.apply_nozzle_left_x(a, d, d, d, n, n, 0.5, 0.5, rng, noz)

    def one(a):
        bcs(a)
        a = O.step(P, a, d, d, d, dt, 3)
        bcs(a)
        O.apply_cooling_heating(a, dt, src)
        O.apply_two_temperature(a, dt, src)
        return a

    for _ in range(warmup):
        pr = one(pr)
    t0 = time.perf_counter()
    for _ in range(steps):
        pr = one(pr)
    sec = time.perf_counter() - t0
    zones = xc * n * n * steps
    return dict(value=zones / sec, cores=O.num_threads(), kind="port",
                sample=f"{steps} driver steps on a {xc}x{n}x{n} x-slab of the {n}^3 state "
                       f"(C port of the reference's Numba kernels, OpenMP)")


# ------------------------------------------------------------------ main ---
KERNELS = {0: "k_face (float32 reconstruction + Riemann, one direction)",
           1: "k_update (flux divergence + SSPRK3 combination)",
           3: "k_c2p_learned (tcgen05 MLP guess + Newton polish)"}


def _hbm_peak():
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    return float(json.load(open(pk)).get("hbm_gbs", 6650.0)) if os.path.exists(pk) else 6650.0


def roofline(args, prof_ms, prof_n, prec, learned, sm_mhz=None):
    """Dominant kernel class of the timed steps and its achieved bandwidth in
    ALGORITHMIC bytes (the unique bytes the kernel must move) per launch."""
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    peak = float(peaks.get("hbm_gbs", 6650.0))
    which = "measured" if "hbm_gbs" in peaks else "fallback"
    cls = max((0, 1, 3), key=lambda c: prof_ms[c])
    nlaunch = max(int(prof_n[cls]), 1)
    avg_s = prof_ms[cls] / nlaunch / 1e3
    n, ng, nv, nm, npas = args.n, 3, 11, 9, 2
    N = n + 2 * ng
    rs = 4 if prec == "mixed" else 8
    if cls == 0:
        # one direction: every face reads one new column of the nm primitives
        # (the float32 copy in mixed precision) and writes its nm fluxes
        units, per_unit = (n + 1) * n * n, nm * rs + nm * rs
    elif cls == 1:
        # every cell: 3 flux buffers, pr0 (nv), pr_k psi + passives, U_{k-1}
        # (stages 2-3), U_k, the next primitives (all nv, or the non-main ones
        # when the learned con2prim writes the main ones)
        u_in = 2.0 / 3.0 * nm * 8
        u_out = nm * 8 if learned else 2.0 / 3.0 * nm * 8
        dst = (nv - nm) * 8 if learned else nv * 8
        units, per_unit = N ** 3, 3 * nm * rs + nv * 8 + (npas + 1) * 8 + u_in + u_out + dst
    else:
        # U in, primitives out, and in mixed precision the float32 copy of the
        # primitives for the next stage's faces (written in 2 of 3 stages)
        units, per_unit = N ** 3, 2 * nm * 8 + (2.0 / 3.0 * nm * rs if prec == "mixed" else 0)
    achieved = units * per_unit / avg_s / 1e9
    traffic, tdata = None, {}
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        tdata = json.load(open(tf))
        traffic = tdata.get(f"{prec}:{cls}:{n}")
    out = {"bound": "hbm", "kernel": KERNELS[cls], "achieved": round(achieved, 1),
           "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
           "traffic": traffic, "peak_source": which,
           "bytes_per_launch": int(units * per_unit), "avg_launch_ms": round(avg_s * 1e3, 4),
           "class_share": round(float(prof_ms[cls] / max(prof_ms.sum(), 1e-30)), 3)}
    if cls == 0 and prec == "mixed" and "fp32_flop_per_face" in tdata and sm_mhz:
        # the pipe that binds the face kernel: float32 arithmetic.  FLOP per
        # face from ncu's instruction counters, over the float32 peak of
        # this GPU at the clock sampled during the timed steps (128 lanes x 2
        # FLOP per SM per clock)
        import torch
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        flops = units * tdata["fp32_flop_per_face"] / avg_s / 1e12
        fpk = sms * 128 * 2 * sm_mhz * 1e6 / 1e12
        out["pipe"] = {"pipe": "fp32", "flop_per_face": tdata["fp32_flop_per_face"],
                       "achieved": round(flops, 2), "peak": round(fpk, 1), "unit": "TFLOP/s",
                       "frac": round(flops / fpk, 3), "clock_mhz": sm_mhz}
    return out


def validate_srhd(args):
    """Accuracy of the mixed-precision SRHD jet (PPM + HLLC, SSPRK3, v_jet
    0.995, CFL 0.4 with the reference's amax rule) against plain float64, with
    the float64 perturbation floor beside it."""
    import torch
    from astrofd_b200.core import boundary, nozzle, srhd_core
    from astrofd_b200.workloads import srhd_jet, srhd_jet_config
    n, K, ng = args.n, args.validate_steps, 3
    core, noz = srhd_jet_config(n, ng, vjet=0.995, recon="ppm", riemann="hllc", rk_order=3,
                                boundaries=args.boundaries)
    d = 1.0 / n
    yz = boundary.apply_outflow_yz if noz.get("YZ_BOUNDARY") == "outflow" else \
        boundary.apply_periodic_yz

    def run(prec, perturb=0.0):
        srhd_core.configure(dict(core, PRECISION=prec, FLUX_MODE=args.flux_mode))
        pr = srhd_jet(n, ng)
        if perturb:
            pr[0] *= 1.0 + perturb * np.random.default_rng(5).standard_normal(pr[0].shape)
        a = torch.from_numpy(pr).cuda()
        rng = np.random.default_rng(1234)
        N = a.shape[1]

        def bcs(t):
            yz(t, ng)
            boundary.apply_outflow_right_x(t, ng)
            nozzle.apply_nozzle_left_x(t, d, d, d, n, n, 0.5, 0.5, rng, noz)
        for _ in range(K):
            dt = core["CFL"] * d / max(srhd_core.max_char_speed(a, N, N, N), 1e-12)
            bcs(a)
            a = srhd_core.step_ssprk3(a, d, d, d, dt)
            bcs(a)
        return a

    ref = run("fp64")
    out = {"validate_steps": K, "grid": n, "physics": "srhd ppm/hllc ssprk3",
           "flux_mode": args.flux_mode, "boundaries": args.boundaries,
           "mixed_vs_fp64": _norms(run("mixed"), ref, ng),
           "fp64_perturbed_1e-12_vs_fp64": _norms(run("fp64", 1e-12), ref, ng)}
    print(json.dumps(out), flush=True)


def validate(args):
    """Accuracy protocol of the mixed + learned path against plain float64
    (rho_l1_arms), then the mass change of one conservative float64 step."""
    import torch
    from astrofd_b200.core import rmhd_core
    from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config
    n, K = args.n, args.validate_steps
    out = rho_l1_arms(n, K, args.jet_v, args.sigma_jet, args.sigma_amb, args.boundaries,
                      args.flux_mode, args.c2p_net, args.validate_every, args.stage_kernel)
    core, _, _ = rmhd_jet_config(n, 3, boundaries=args.boundaries)
    # mass: sum(D) of the conserved state, before and after one conservative
    # float64 step of a state with nothing crossing the faces of the update
    # region (ambient at rest there)
    rmhd_core.configure(dict(core, PRECISION="fp64", FLUX_MODE="conservative",
                             C2P_GUESS="reference"))
    a = torch.from_numpy(rmhd_jet(n, 3)).cuda()
    a[1:4] = 0.0  # medium at rest outside the moving cube
    c = slice(n // 2 - n // 8, n // 2 + n // 8)
    a[0, c, c, c] = 0.1
    a[1, c, c, c] = 0.995
    d = 1.0 / n
    W = lambda q: 1.0 / torch.sqrt(1.0 - (q[1] ** 2 + q[2] ** 2 + q[3] ** 2))
    m0 = (a[0] * W(a)).sum().item()
    b = rmhd_core.step_ssprk3(a, d, d, d, core["CFL"] * d)
    out["mass_rel_change_one_conservative_step"] = abs((b[0] * W(b)).sum().item() - m0) / m0
    print(json.dumps(out), flush=True)


def c2p_batch(args):
    """Learned con2prim on sampled states (rho log-uniform [1e-4, 10], p
    [1e-6, 10], W [1, 50], isotropic v and B, sigma log-uniform [1e-3, 10],
    Gamma 4/3): Newton steps after the guess, fallback rate, relative error of
    the primitives against the full float64 Newton, and states/s of the
    learned path, the same solver from the analytic start, and the
    reference's con2prim."""
    import torch
    from astrofd_b200 import learned_c2p as LC
    N = args.c2p_batch
    e = LC.c2p_engine()
    if args.c2p_jet:
        from astrofd_b200.train_c2p_mlp import harvest_jet
        prim = harvest_jet(n=128, steps=12, per_snapshot=-(-N // 4), seed=7)[:, :N].contiguous()
        e = LC.c2p_engine(p_max=2.0)  # the jet's P_MAX
    else:
        prim = torch.as_tensor(LC.sample_primitives(N, 2024), device="cuda")
    U = e.p2c_array(prim)
    N = U.shape[1]
    params = torch.as_tensor(LC.load(args.c2p_net or LC.DATA), dtype=torch.float32).cuda()

    # one result buffer for every timed call, so that no call waits on the
    # caching allocator for a fresh 1.2 GB block
    qbuf = torch.empty_like(U)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / reps

    ref, ms_ref = timed(lambda: e.c2p_array(U))
    out = {"config": f"c2p batch, {N} " + ("states of a 128^3 jet run" if args.c2p_jet
                                           else "sampled states"), "states": N}
    p = e.p
    ref_root = LC.residual(U, ref, p.gamma, p.p_max, p.v_max) < 1e-8
    for name, prm in (("learned", params), ("analytic_start", None)):
        torch.cuda.empty_cache()
        (q, st), ms = timed(lambda: LC.c2p_learned(e, U, prm, max_polish=2, out=qbuf))
        rel = ((q[:5] - ref[:5]).abs() / ref[:5].abs().clamp_min(1e-300)).amax(0)
        n = st["cells"]
        # states off the reference's result: where both results solve the
        # reference's equation (other roots of f(Z) when v.B != 0), where only
        # this path found a root (the reference fell back to its hydro
        # solve), and misses (this path's result is no root)
        off = rel > 1e-6
        root = LC.residual(U, q, p.gamma, p.p_max, p.v_max) < 1e-8
        miss = off & ~root
        within = [LC.c2p_learned(e, U, prm, max_polish=k)[1]["learned_polish"] / n
                  for k in (0, 1)] + [st["learned_polish"] / n]
        out[name] = {"states_per_s": N / (ms / 1e3), "ms": ms,
                     "newton_steps_per_state": st["polish_steps"] / max(n, 1),
                     "polished_within_0_1_2": within,
                     "polish_step_histogram": {"0": within[0], "1": within[1] - within[0],
                                               "2": within[2] - within[1],
                                               "fallback": st["learned_fallback"] / n},
                     "polished_within_2": st["learned_polish"] / n,
                     "fallback_rate": st["learned_fallback"] / n,
                     "off_reference": {"other_root": float((off & root & ref_root).double().mean()),
                                       "root_where_reference_fell_back":
                                           float((off & root & ~ref_root).double().mean()),
                                       "miss": float(miss.double().mean())},
                     "max_rel_err_misses": float(rel[miss].max()) if bool(miss.any()) else 0.0,
                     "max_rel_err_all": float(rel.max()),
                     "p999_rel_err": float(torch.quantile(rel[::max(1, N // 1000000)].float(), 0.999)),
                     "frac_rel_err_gt_1e-6": float(off.double().mean()),
                     "status": st["status"]}
        # release this arm's arrays before the next arm's timed calls, so that
        # those do not wait on the allocator freeing cached blocks
        del q, rel, off, root, miss
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    out["reference_c2p"] = {"states_per_s": N / (ms_ref / 1e3), "ms": ms_ref}
    print(json.dumps(out), flush=True)


NAMED = {
    "c1": dict(physics="srhd", n=64, ng=2, steps=10, desc="SRHD 64^3, MUSCL-minmod + HLLE, "
               "SSPRK2, CFL 0.4, v_jet 0.99", scheme=dict(), precisions=("fp64",)),
    "c2": dict(physics="srhd", n=128, ng=3, steps=50, desc="SRHD 128^3, PPM + HLLC, SSPRK3, "
               "CFL 0.4, v_jet 0.995", scheme=dict(vjet=0.995, recon="ppm", riemann="hllc",
                                                     rk_order=3),
               precisions=("fp64", "mixed")),
    "c3": dict(physics="rmhd", n=128, ng=3, steps=50, desc="RMHD 128^3, Gamma 4/3, WENO5 + "
               "hlld, SSPRK3, CFL 0.35, v_jet 0.99, sigma_jet 0.5, ambient sigma 0.01",
               precisions=("fp64", "mixed", "mixed+learned")),
}


def named_config(args):
    """Zone-updates/s of a named jet's driver loop at its own size: W
    untimed steps, then K steps (the configuration's step count, or --steps
    when smaller) between CUDA events.  SRHD takes the reference driver's CFL
    rule each step (max_char_speed read back to the host:
    solvers/srhd3d_mpi_muscl.py:276-283); RMHD its fixed amax = 1."""
    import torch
    from astrofd_b200 import learned_c2p
    from astrofd_b200.core import boundary, nozzle, rmhd_core, srhd_core
    from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config, srhd_jet, srhd_jet_config
    c = NAMED[args.workload]
    n, ng = c["n"], c["ng"]
    K = min(args.steps, c["steps"]) if args.steps else c["steps"]
    d = 1.0 / n
    res = {}
    for prec in c["precisions"]:
        learned = prec == "mixed+learned"
        if c["physics"] == "srhd":
            core, noz = srhd_jet_config(n, ng, boundaries=args.boundaries, **c["scheme"])
            mod, host = srhd_core, srhd_jet(n, ng)
            src = None
        else:
            core, noz, src = rmhd_jet_config(n, ng, vjet=0.99, boundaries=args.boundaries)
            core = dict(core, RESISTIVE_ENABLED=False, N_PASSIVE=0)
            mod, host = rmhd_core, np.ascontiguousarray(rmhd_jet(n, ng)[:9])
        mod.configure(dict(core, PRECISION=prec.split("+")[0], FLUX_MODE=args.flux_mode,
                           C2P_GUESS="learned" if learned else "reference",
                           STAGE_KERNEL=args.stage_kernel))
        if learned:
            mod.set_c2p_network(learned_c2p.load(args.c2p_net or learned_c2p.DATA))
        yz = boundary.apply_outflow_yz if noz.get("YZ_BOUNDARY") == "outflow" else \
            boundary.apply_periodic_yz
        rng = np.random.default_rng(1234)
        a = torch.from_numpy(host).cuda()
        b = torch.empty_like(a)
        N = a.shape[1]
        step = mod.step_ssprk3 if core["RK_ORDER"] == 3 else mod.step_ssprk2

        def one(a, b):
            amax = srhd_core.max_char_speed(a, N, N, N) if c["physics"] == "srhd" else 1.0
            dt = core["CFL"] * d / max(amax, 1e-12)
            yz(a, ng)
            boundary.apply_outflow_right_x(a, ng)
            nozzle.apply_nozzle_left_x(a, d, d, d, n, n, 0.5, 0.5, rng, noz)
            step(a, d, d, d, dt, out=b)
            return b, a

        for _ in range(args.warmup):
            a, b = one(a, b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(K):
            a, b = one(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[prec] = {"zone_updates_per_s": n ** 3 * K / (ms / 1e3), "ms_per_step": ms / K,
                     "finite": bool(torch.isfinite(a).all().item())}
        del a, b
        torch.cuda.empty_cache()
    line = {"metric": f"zone-updates/s {args.workload.upper()} ({c['desc']})",
            "value": res[c["precisions"][-1]]["zone_updates_per_s"], "unit": UNIT,
            "n_gpus": 1, "steps": K, "warmup": args.warmup, "higher_is_better": True,
            "data": "synthetic (seeded jet)", "arms": res,
            "config": {"workload": args.workload, "grid": [n, n, n], "ng": ng,
                       "flux_mode": args.flux_mode, "boundaries": args.boundaries}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload != "c5" and args.impl == "ours":
        named_config(args)
        return
    if args.validate_steps:
        (validate_srhd if args.validate_srhd else validate)(args)
        return
    if args.c2p_batch:
        c2p_batch(args)
        return
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        r = cpu_sample(args, args.steps, args.warmup)
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "impl": "reference", "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"rmhd-jet-{args.n}^3 weno5/hlld ssprk3 + resistive + "
                                       "two-temperature + cooling", "sample_x_cells":
                               args.cpu_x_cells, "flux_mode": "reference",
                               "boundaries": args.boundaries},
                "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"],
                                 "kind": r["kind"], "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "vs_baseline": None}
        print(json.dumps(line), flush=True)
        return

    import torch
    from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config
    rank, world, local = dist_init(args)
    n = args.n
    cfgs = rmhd_jet_config(n, 3, boundaries=args.boundaries)
    pr_host = rmhd_jet(n, 3, seed=2024 + rank)
    zones = n ** 3 * args.steps * world

    learned = not args.no_learned
    mixed = time_arm(args, world, "mixed", pr_host, cfgs, profile=True, learned=learned)
    fp64 = None if args.no_fp64 else time_arm(args, world, "fp64", pr_host, cfgs, profile=False)
    e2e = None if args.no_e2e else time_e2e(args, world, "mixed", pr_host, cfgs, learned=learned)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(args, steps=1, warmup=0)
    rho_after = None
    if fp64 is not None:
        a, b = mixed["state"], fp64["state"]
        rho_after = float(((a[0] - b[0]).abs().mean() / b[0].abs().mean()).item())
    accuracy = None
    if world == 1 and not args.no_accuracy:
        del mixed["state"]
        if fp64 is not None:
            del fp64["state"]
        torch.cuda.empty_cache()
        # untimed: density L1 against plain float64 of the headline path, the
        # float64 floor and the path's two halves, (1) on this workload over
        # the steps a timed step can reach (warm-up + one segment), (2) on its
        # stable member over 100 steps, where the bar L1 < 1e-4 is measurable
        k = args.warmup + (args.segment if 0 < args.segment < args.steps else args.steps)
        spec = rho_l1_arms(n, k, 0.995, 0.5, 0.01, args.boundaries, args.flux_mode,
                           args.c2p_net, every=k, stage_kernel=args.stage_kernel)
        stab = rho_l1_arms(n, 100, boundaries=args.boundaries, flux_mode=args.flux_mode,
                           net=args.c2p_net, every=25, stage_kernel=args.stage_kernel, **STABLE)
        accuracy = {
            "this_workload": {"steps": k, "rho_l1_vs_fp64": spec["rho_l1"],
                              "c2p_mixed_learned": spec["c2p_counts"]["mixed_learned"]},
            "stable_member": {"steps": 100, "jet": "unmagnetised, v 0.99 (W 7.09)",
                              "rho_l1_vs_fp64": stab["rho_l1"],
                              "rho_l1_history": stab["rho_l1_history"],
                              "meets_l1_1e-4": stab["rho_l1"]["mixed_learned"] < 1e-4},
        }

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    value = zones / (mixed["ms"] / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mixed["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 state/con2prim, f32 flux",
        "data": "synthetic (seeded magnetised jet)",
        "config": {"workload": f"rmhd-jet-{n}^3 weno5/hlld ssprk3 + resistive 1e-4 + "
                               "two-temperature + cooling (driver-loop iteration)",
                   "grid": [n, n, n], "ng": 3, "nv": 11, "precision": "mixed",
                   "c2p_guess": "learned" if learned else "reference",
                   "flux_mode": args.flux_mode, "boundaries": args.boundaries,
                   "l2": "inputs larger than L2 (1.6 GB arrays)",
                   "timed_segments": f"{mixed['segments']} x <= {mixed['segment']} steps, each "
                                     "from the state after the warm-up (restored untimed)",
                   "stage_kernel": args.stage_kernel,
                   "parallelism": ("single GPU" if world == 1 else
                                   f"x-slabs x{world}, 3 ghost layers exchanged per "
                                   f"{args.halo} (NCCL send/recv)" if args.decomp == "slab" else
                                   f"replicas x{world}")},
        "gpu_launches": mixed["launches"],
        "launch_mode": mixed["launch_mode"],
        "clocks": mixed["clocks"],
        "roofline": roofline(args, mixed["prof_ms"], mixed["prof_n"], "mixed", learned,
                             (mixed["clocks"] or {}).get("sm_mhz")),
        # the whole step against the minimum unique HBM bytes of an SSPRK3
        # step with 11 float64 variables: 1056 B per zone update (read the
        # step input and the stage states, write U and the primitives)
        "step_roofline": {"bytes_per_zone_update": 1056,
                          "achieved": round(n ** 3 * 1056 / (mixed["ms"] / args.steps / 1e3) / 1e9, 1),
                          "unit": "GB/s", "frac": round(n ** 3 * 1056 / (mixed["ms"] / args.steps / 1e3)
                                                        / 1e9 / _hbm_peak(), 4)},
        "kernel_ms_per_step": {k: round(mixed["prof_ms"][c] / mixed["prof_steps"], 3)
                               for k, c in (("face", 0), ("update", 1), ("c2p_learned", 3),
                                            ("c2p_fallback", 4), ("other", 2))},
        "kernel_times_from": mixed["times_from"],
        "finite": mixed["finite"],
        "c2p": mixed["c2p"],
    }
    if fp64 is not None:
        v64 = zones / (fp64["ms"] / 1e3)
        line["fp64_value"] = v64
        line["speedup_vs_fp64"] = value / v64
        line["rho_l1_vs_fp64_after_steps"] = rho_after
    if accuracy is not None:
        line["accuracy"] = accuracy
    if e2e is not None:
        line["e2e"] = {"value": n ** 3 * e2e["steps"] * world / (e2e["ms"] / 1e3), "unit": UNIT,
                       "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                       "copies": "pinned host blocks, double-buffered: upload k+1 and read-back "
                                 "k-1 overlap step k",
                       "steps": e2e["steps"],
                       "link_floor_ms_per_step": round(e2e["link_ms"], 3),
                       "link_frac": round(e2e["link_ms"] / (e2e["ms"] / e2e["steps"]), 3)}
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"],
                                "kind": cpu["kind"], "sample": cpu["sample"]}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
