#!/usr/bin/env python
"""PBD particle-steps/s on the 2,097,152-particle dam-break (one B200 per rank).

One step = one dam-break frame through the C ABI (pk_pbf_step): box boundary,
neighbour query (cap 64, radius 2.5 spacing), integration and 5 DensityPBD
Jacobi iterations, on synthetic seeded inputs of the configuration's shape.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pk|reference]

--impl reference times the CPU restatement of the same step (the reference is
CUDA only; its kernel bodies restated in C with OpenMP) on the host cores, on
a bounded sample of the workload per step.  With N > 1 (torchrun) the scene
does not shard: every rank steps its own replica ("replicas only").
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "physika-old_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import scenes  # noqa: E402

METRIC = "PBD particle-steps/s at 2M (HBM %roofline); batched+adjoint vs plain, same GPU"
UNIT = "particle-steps/s"


def pbd_bytes_per_particle_step(kbar, iters):
    """Algorithmic HBM bytes of one PBD particle-step: neighbour build (read x,
    write list + count), integration, per iteration pass A (x, list, lambda) and
    pass B (x, lambda, list, x'), velocity update, density out, boundary pass."""
    return 176.0 + 4.0 * kbar + iters * (44.0 + 8.0 * kbar)


WORKLOAD = ("dam_break_2m: 128^3 jittered lattice, spacing 0.0025, radius 0.00625, cap 64, "
            "5 Jacobi iterations, dt 5e-4, box 2x1x1")


def stage_bytes(kind, kbar, kunion):
    """Algorithmic bytes per particle of one launch of a stage of the frame;
    the stages add up to pbd_bytes_per_particle_step."""
    if kind == "sort":  # boundary (read x, v; write x, v) + integrate (read x, v; write x, v, x_old)
        return 48.0 + 60.0
    if kind == "build":  # neighbour build: read x, write the list and its count
        return 12.0 + 4.0 * kbar + 4.0
    if kind == "density":  # pass A: read x_i, the N(i) row, write lambda
        return 12.0 + 4.0 * kbar + 4.0
    if kind == "disp":  # pass B: read x_i, lambda_i, the row, write x_i'
        return 12.0 + 4.0 + 4.0 * kunion + 12.0
    if kind == "finish":  # velocity update (read x, x_old, v; write v) + density out
        return 48.0 + 4.0
    raise ValueError(kind)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        self.bus_id = (bus_id or "").lower()
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [s.strip() for s in line.split(",")]
            if len(f) < 10:
                continue
            if self.bus_id and self.bus_id not in f[1].lower():
                continue
            rows.append(f)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].lower() == "active"})
        out.update(sm_mhz=statistics.median(sm) if sm else None,
                   sm_max_mhz=float(rows[0][3]) if rows[0][3].replace(".", "").isdigit() else None,
                   reasons=reasons, samples=len(rows))
        return out


class NvmlClocks:
    """In-process NVML sampling (read-only queries) of the SM clock, its maximum
    and the clock-event reasons every 5 ms during a region, so that a region of
    ~0.1 s still gets samples; falls back to nvidia-smi sampling when NVML is
    not importable or the device is not found."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown", 0x8),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap", 0x4))

    def __init__(self, bus_id=None):
        self.bus_id = bus_id
        self.fallback = None
        self.samples = []
        self.thread = None
        self.running = False
        self.nv = None
        self.h = None

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByPciBusId((self.bus_id + ".0").encode()) if self.bus_id \
                else nv.nvmlDeviceGetHandleByIndex(0)
            get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.sm_max = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        except Exception:
            self.nv = None
            self.fallback = Clocks(self.bus_id)
            self.fallback.start()
            return

        def run():
            while self.running:
                try:
                    self.samples.append((float(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)),
                                         int(get(self.h))))
                except Exception:
                    pass
                time.sleep(0.005)

        self.running = True
        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.fallback is not None:
            return self.fallback.stop()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": "nvml"}
        if self.nv is None:
            return out
        self.running = False
        self.thread.join(1.0)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        if not self.samples:
            return out
        reasons = sorted({name for _, bits in self.samples for name, attr, dflt in self.REASONS
                          if bits & getattr(self.nv, attr, dflt)})
        out.update(sm_mhz=statistics.median(c for c, _ in self.samples), sm_max_mhz=self.sm_max,
                   reasons=reasons, samples=len(self.samples))
        return out


def bus_id_of(dev):
    try:
        import torch
        p = torch.cuda.get_device_properties(dev)
        return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}"
    except Exception:
        return None


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# --------------------------------------------------------------- CPU arm

def cpu_step_sample(sc_params, x, v, sdf, rnd):
    import pk_oracle as po
    x, v = po.sdf_constrain(x, v, sdf, rnd, 0.95, 0.0, sc_params.dt)
    ri, re = po.neighbor_query(x, sc_params.radius, sc_params.lo, sc_params.hi, sc_params.cap)
    x, v = po.integrate(x, v, sc_params.gravity, sc_params.dt)
    f, m = po.density_scaling(sc_params.spacing, sc_params.radius, sc_params.rest_density)
    x, v, _ = po.pbd_constrain(x, v, ri, re, sc_params.cap, sc_params.radius, f * m,
                               sc_params.iterations, sc_params.dt)
    return x, v


def cpu_sample_scene():
    # 64^3 = 262,144 particles with the 2M scene's spacing, radius, cap, dt
    return scenes.dam_break_2m(seed=0, n_side=64)


def time_cpu(steps, warmup, threads=0):
    import pk_oracle as po
    po.set_threads(threads)
    sc = cpu_sample_scene()
    sdf = po.sdf_box(sc.lo, sc.hi, sc.sdf_spacing, True)
    rnd = np.random.default_rng(0).uniform(0, 1, sc.x.shape[0]).astype(np.float32)
    x, v = sc.x.copy(), sc.v.copy()
    for _ in range(warmup):
        x, v = cpu_step_sample(sc, x, v, sdf, rnd)
    t0 = time.perf_counter()
    for _ in range(steps):
        x, v = cpu_step_sample(sc, x, v, sdf, rnd)
    dt = time.perf_counter() - t0
    return sc.x.shape[0] * steps / dt, po.max_threads(), sc.x.shape[0]


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    v, cores, n = time_cpu(args.steps, args.warmup)
    sample = (f"{n} particles (64^3 block, 2M-scene spacing/radius/cap 64/dt/5 iterations) "
              f"per step, CPU restatement with OpenMP")
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": n / v * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "particles": 2097152, "sample_particles": n, "cap": 64,
                   "iterations": 5},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- GPU arm

def load_traffic():
    """ncu DRAM bytes per launch of the dominant kernel, from the committed
    profile summary (None when no capture has been summarised yet)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


BATCHED_WORKLOAD = ("256 independent dam-break scenes, particle counts log-uniform in [1024, 65536] "
                    "(PCG64 seed 0), each a jittered lattice block in its own unit box with the 32k "
                    "dam break's parameters (spacing 0.005, radius 0.0125, cap 60, dt 1e-3, 5 iterations)")


def measure_batched(local, steps, warmup, barrier, max_over_ranks, rank, world):
    """The batched frame (one pk_pbf_step_batched for all scenes, eager and
    replayed as a graph recorded by pk_graph_capture) against per-scene plain
    frames (one pk_pbf_step per scene per frame, issued from the C++ host loop
    pkf_pbf_frames_per_scene), same scenes, same GPU, device time with CUDA
    events.  With several ranks the scenes are partitioned (largest first to
    the least-loaded rank) and each rank steps its share; times are the max
    over ranks, values the whole job."""
    import ctypes
    import torch
    import pkhot
    from sharding import partition_scenes, subset

    dev = torch.device("cuda", local)
    b_all = scenes.batched_mix(seed=0)
    sc0 = b_all.scenes[0]
    n_all = int(b_all.offsets[-1])
    mine = partition_scenes(np.diff(b_all.offsets), world)[rank]
    bx, bv, boff = subset(b_all.x, b_all.v, b_all.offsets, mine)
    b = scenes.BatchedScenes(b_all.name, [b_all.scenes[s] for s in mine], bx, bv, boff)
    n = int(b.offsets[-1])
    ctx = pkhot.Context(local)
    ctx.boundary_set_box(sc0.lo, sc0.hi, sc0.sdf_spacing, True)
    prm = pkhot.pbf_params(pkhot.nq_params(sc0.radius, sc0.lo, sc0.hi, sc0.cap),
                           pkhot.pbd_params(sc0.radius, sc0.spacing, sc0.rest_density, sc0.iterations,
                                            sc0.dt), sc0.gravity, boundary=True)
    x = torch.from_numpy(b.x.copy()).to(dev)
    v = torch.zeros_like(x)
    off = torch.from_numpy(b.offsets.astype(np.int32)).to(dev)

    def timed(fn, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(torch.cuda.current_stream())
        for _ in range(k):
            fn()
        e1.record(torch.cuda.current_stream())
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / k)

    for _ in range(warmup):
        ctx.pbf_step_batched(x, v, off, prm)
    ctx.check_status()
    launches = ctx.launch_count()
    kbar, kunion, _ = ctx.row_stats()
    ms_eager = timed(lambda: ctx.pbf_step_batched(x, v, off, prm), steps)
    ctx.graph_capture(x, v, prm, off)
    ms_graph = timed(ctx.graph_launch, steps)
    ctx.graph_release()
    ctx.check_status()
    # per-scene plain frames, issued from C++
    fw = ctypes.CDLL(os.path.join(os.path.dirname(pkhot.LIB_PATH), "libpkframework.so"))
    fw.pkf_pbf_frames_per_scene.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int, ctypes.POINTER(pkhot.PbfParams), ctypes.c_int,
                                            ctypes.c_void_p]
    offs_host = (ctypes.c_int * len(b.offsets))(*[int(q) for q in b.offsets])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def plain_frame():
        rc = fw.pkf_pbf_frames_per_scene(ctx.h, x.data_ptr(), v.data_ptr(), offs_host, len(b.scenes),
                                         ctypes.byref(prm), 1, stream)
        if rc != 0:
            raise RuntimeError(f"pkf_pbf_frames_per_scene: {rc}")

    plain_frame()
    ctx.check_status()
    ms_plain = timed(plain_frame, max(2, min(steps, 5)))
    ctx.check_status()
    ctx.close()

    def entry(ms):
        return {"value": n_all / (ms / 1e3), "unit": UNIT, "ms_per_step": ms}

    peak, peak_kind = peaks()
    best = min(ms_eager, ms_graph)
    # sum over scenes of B_PBD(N_s, K_s) plus the scene-offset table; the
    # bytes are linear in K, so the whole job's mean K gives the sum
    frame_bytes = world * (n * pbd_bytes_per_particle_step(kbar, sc0.iterations) + 16.0 * len(b.scenes))
    return {"workload": BATCHED_WORKLOAD, "scenes": len(b_all.scenes), "particles": n_all,
            "scenes_per_rank": "largest-first greedy partition" if world > 1 else "all",
            "batched_eager": entry(ms_eager), "batched_graph": entry(ms_graph),
            "plain_per_scene": entry(ms_plain),
            "plain_per_scene_issue": "pkf_pbf_frames_per_scene: C++ host loop, one pk_pbf_step per scene",
            "launches_per_frame": {"batched": launches, "plain": launches * len(b.scenes)},
            "speedup_vs_plain": ms_plain / best,
            "roofline": {"bound": "hbm", "bytes_per_frame": frame_bytes, "kbar": kbar,
                         "achieved": frame_bytes / (best / 1e3) / 1e9 / world, "peak": peak, "unit": "GB/s",
                         "frac": frame_bytes / (best / 1e3) / 1e9 / world / peak, "peak_source": peak_kind}}


ADJOINT_WORKLOAD = ("differentiable rollout: 64x32x32 = 65,536-particle peridynamics block, spacing 0.004, "
                    "horizon 3 spacing, cap 80, 10 projection iterations, dt 1e-3, 200 steps, checkpoint "
                    "every 20; loss = mean |x_T - x_target|^2, target from hidden stiffness U[0.5, 2]e4 and "
                    "v0 ~ N(0, 0.05^2) (PCG64 seeds 0, 1); guess: stiffness 1e4, v0 ~ N(0, 0.05^2) (seed 3)")
PD_WORKLOAD = ("peridynamics bar 256x64x32 = 524,288 particles, spacing 0.004, horizon 3 spacing, cap 80, "
               "stiffness U[0.8, 1.2]e4, 10 projection iterations, bonds break at 2% stretch, x-index 0 "
               "clamped, last x layer pulled at 0.5 m/s, dt 1e-3")


def pd_bytes_per_particle_step(kb, iters):
    """Algorithmic HBM bytes of one peridynamics particle-step (bond indices read
    per iteration, K^-1/bulk/x per particle; breaks: alive bits)."""
    return 108.0 + iters * (108.0 + 4.0 * kb + kb / 8.0) + 4.0 * kb + kb / 8.0


def measure_pd(local, steps, warmup, barrier):
    """The elastic bar with fracture: integrate, pins, projection with stretch
    break, pins; particle-steps/s over `steps` steps, device time."""
    import torch
    import pkhot

    dev = torch.device("cuda", local)
    sc = scenes.elastic_bar(seed=0)
    n = sc.x.shape[0]
    ctx = pkhot.Context(local)
    x = torch.from_numpy(sc.x.copy()).to(dev)
    v = torch.zeros_like(x)
    idx, el, tot = ctx.nq_build(x, sc.horizon, sc.lo, sc.hi, sc.cap)
    kb = float(idx.double().mean())
    ctx.pd_init(x, idx, el, sc.cap, tot, sc.horizon)
    ctx.pd_set_bulk(torch.from_numpy(sc.bulk).to(dev))
    dims = sc.dims
    ix = np.arange(n) // (dims[1] * dims[2])
    left, right = np.nonzero(ix == 0)[0], np.nonzero(ix == dims[0] - 1)[0]
    ids = torch.from_numpy(np.concatenate([left, right]).astype(np.int32)).to(dev)
    base = x[ids.long()].clone()
    vel = torch.zeros_like(base)
    vel[left.shape[0]:, 0] = 0.5
    step_no = [0]

    def step():
        step_no[0] += 1
        tgt = base + vel * (step_no[0] * sc.dt)
        ctx.integrate(x, v, (0.0, -9.8, 0.0), sc.dt)
        ctx.fixed_points(x, v, ids, tgt, vel)
        ctx.pd_solve(x, v, sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt, sc.break_stretch)
        ctx.fixed_points(x, v, ids, tgt, vel)

    for _ in range(warmup):
        step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.current_stream())
    for _ in range(steps):
        step()
    e1.record(torch.cuda.current_stream())
    barrier()
    ctx.check_status()
    ms = e0.elapsed_time(e1) / steps
    ctx.close()
    peak, kind = peaks()
    val = n / (ms / 1e3)
    b = pd_bytes_per_particle_step(kb, sc.iterations)
    return {"workload": PD_WORKLOAD, "particles": n, "value": val, "unit": UNIT, "ms_per_step": ms,
            "steps": steps, "kbar_bonds": kb,
            "step_roofline": {"bytes_per_particle_step": b, "frac": val * b / (peak * 1e9), "peak_source": kind}}


EP_WORKLOAD = ("elastoplastic block 64x32x32 = 65,536 particles, spacing 0.004, horizon 3 spacing, dynamic "
               "lists, cohesion 1e-4, friction angle 60, shear flow 0.5 m/s; ParticleElastoplasticBody frame: "
               "integrate, query, 10 x (projection + 1-iteration DensityPBD), query, rest-shape rotation, "
               "yielding, reconstruction, 5 viscosity sweeps, dt 1e-3")


def measure_elastoplastic(local, steps, warmup, barrier):
    """ParticleElastoplasticBody::advance (ParticleElastoplasticBody.cpp:73-91)
    composed from C-ABI calls; device time per frame (the dynamic lists and the
    reconstruction's bond count synchronise the host every frame, as the
    reference's thrust::reduce does)."""
    import torch
    import pkhot

    dev = torch.device("cuda", local)
    sc = scenes.elastic_bar(seed=0, dims=(64, 32, 32), cap=0)
    n, h, dt = sc.x.shape[0], sc.horizon, sc.dt
    rng = np.random.default_rng(0)
    x0 = (sc.x + rng.uniform(-0.02, 0.02, sc.x.shape) * sc.spacing).astype(np.float32)
    v0 = np.zeros_like(x0)
    v0[:, 0] = 0.5 * (x0[:, 1] - x0[:, 1].mean()) / (x0[:, 1].max() - x0[:, 1].mean())
    ctx = pkhot.Context(local)
    x, v = torch.from_numpy(x0).to(dev), torch.from_numpy(v0).to(dev)
    prm = pkhot.pbd_params(h, 0.005, 1000.0, 1, dt)
    A = float(np.float32(6.0 * 1e-4 * np.cos(60 / 180) / (3.0 + np.sin(60 / 180)) / np.sqrt(3.0)))
    B = float(np.float32(2.0 * np.sin(60 / 180) / (3.0 + np.sin(60 / 180)) / np.sqrt(3.0)))
    idx, el, tot = ctx.nq_build(x, h, sc.lo, sc.hi, 0)
    ctx.pd_init(x, idx, el, 0, tot, h)
    ones = torch.ones(n, device=dev)

    def frame():
        ctx.integrate(x, v, (0.0, -9.8, 0.0), dt)
        i1, e1, t1 = ctx.nq_build(x, h, sc.lo, sc.hi, 0)
        ctx.pd_begin(x, h, 0.05, 0.1, dt)
        ctx.pd_compute_inverse_k(h)
        for _ in range(10):
            ctx.pd_enforce(x, h, 0.05, 0.1, dt)
            ctx.pbd_solve(x, v, i1, e1, 0, t1, prm)
        ctx.pd_update_velocity(x, v, dt)
        i2, e2, t2 = ctx.nq_build(x, h, sc.lo, sc.hi, 0)
        ctx.pd_rotate_rest_shape(x, h)
        ctx.pd_set_bulk(ones)
        ctx.pd_apply_yielding(x, h, A, B, 0.05, 0.1)
        ctx.pd_reconstruct_rest_shape(x, i2, e2, 0, t2, h, False)
        ctx.viscosity(x, v, i2, e2, 0, t2, 1.0, h, 5, dt)

    for _ in range(warmup):
        frame()
    barrier()
    e0, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.current_stream())
    for _ in range(steps):
        frame()
    e1_.record(torch.cuda.current_stream())
    barrier()
    ctx.check_status()
    ms = e0.elapsed_time(e1_) / steps
    y1, y2, _ = ctx.pd_get_yield(n)
    yielding = int((y2 > 0).sum())
    ctx.close()
    return {"workload": EP_WORKLOAD, "particles": n, "value": n / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "steps": steps, "yielding_particles_last_frame": yielding}


def measure_adjoint(local, fd_coords=64):
    """cfg4: float rollout with checkpoints, its reverse pass, and a check of
    the double-precision adjoint against central differences of double rollouts."""
    import torch
    import pkhot

    dev = torch.device("cuda", local)
    sc = scenes.elastic_bar(seed=0, dims=(64, 32, 32), cap=80, stiffness=(0.5e4, 2.0e4))
    n = sc.x.shape[0]
    ctx = pkhot.Context(local)
    x0 = torch.from_numpy(sc.x.copy()).to(dev)
    idx, el, tot = ctx.nq_build(x0, sc.horizon, sc.lo, sc.hi, sc.cap)
    ctx.pd_init(x0, idx, el, sc.cap, tot, sc.horizon)
    steps, every = 200, 20
    rng = np.random.Generator(np.random.PCG64(0))
    bulk_true = rng.uniform(0.5e4, 2.0e4, n)
    v_true = np.random.Generator(np.random.PCG64(1)).normal(0, 0.05, (n, 3))
    args = (sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt)

    def roll32(v, bulk, ck):
        x = x0.clone()
        vv = v.clone()
        ctx.pd_set_bulk(bulk)
        ctx.pd_rollout(x, vv, *args, steps, ck)
        return x

    target = roll32(torch.from_numpy(v_true.astype(np.float32)).to(dev),
                    torch.from_numpy(bulk_true.astype(np.float32)).to(dev), 0)
    # the initial guess: uniform stiffness, initial velocities from another draw
    bulk = torch.full((n,), 1.0e4, dtype=torch.float32, device=dev)
    v0 = torch.from_numpy(np.random.Generator(np.random.PCG64(3)).normal(0, 0.05, (n, 3))
                          .astype(np.float32)).to(dev)
    roll32(v0, bulk, every)  # warm-up (workspace allocation)
    ctx.pd_rollout_backward(torch.ones_like(x0))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record()
    xT = roll32(v0, bulk, every)
    ev[1].record()
    seed = 2.0 * (xT - target) / n
    gx, gv, gb = ctx.pd_rollout_backward(seed)
    ev[2].record()
    torch.cuda.synchronize()
    fwd, bwd = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    loss32 = float(((xT - target) ** 2).sum(1).mean())

    # double: adjoint gradient and central differences
    x064, t64 = x0.double(), target.double()

    def roll64(v, b, ck):
        x = x064.clone()
        vv = v.clone()
        ctx.pd_rollout(x, vv, *args, steps, ck, bulk64=b)
        return x

    b64, v64 = bulk.double(), v0.double()
    xT64 = roll64(v64, b64, every)
    gx64, gv64, gb64 = ctx.pd_rollout_backward(2.0 * (xT64 - t64) / n)

    def dL(vp, bp, vm, bm):
        # L(+) - L(-) from the two trajectories, without subtracting two losses
        xp, xm = roll64(vp, bp, 0), roll64(vm, bm, 0)
        return float(((xp - xm) * (xp + xm - 2.0 * t64)).sum(1).mean())

    pick = np.random.Generator(np.random.PCG64(2))
    # a coordinate is compared when its central difference is resolved: the
    # differences at eps and 2 eps agree to 1e-3 (far below 1e-3 of the
    # largest gradient entry they scatter: a stiffness entry 1/1900 of the
    # largest moved by 4e-3 between eps 1e-4, 2e-4 and 1e-5); the error is
    # relative with a floor of 1e-3 of the largest entry
    floor = {"bulk": 1e-3 * float(gb64.abs().max()), "v0": 1e-3 * float(gv64.abs().max())}

    def fd_bulk(k, rel_eps):
        eps = rel_eps * float(b64[k])
        bp, bm = b64.clone(), b64.clone()
        bp[k] += eps
        bm[k] -= eps
        return dL(v64, bp, v64, bm) / (2 * eps)

    def fd_v0(k, eps):
        vp, vm = v64.clone(), v64.clone()
        vp.view(-1)[k] += eps
        vm.view(-1)[k] -= eps
        return dL(vp, b64, vm, b64) / (2 * eps)

    errs = {"bulk": [], "v0": []}
    tried = {"bulk": 0, "v0": 0}
    plan = {"bulk": (pick.choice(n, 3 * fd_coords // 4, replace=False), fd_bulk, gb64.view(-1)),
            "v0": (pick.choice(3 * n, 3 * fd_coords // 4, replace=False), fd_v0, gv64.view(-1))}
    for key, (coords, fd_fn, grad) in plan.items():
        for k in coords:
            if len(errs[key]) == fd_coords // 2:
                break
            tried[key] += 1
            f1, f2 = fd_fn(int(k), 1e-4), fd_fn(int(k), 2e-4)
            scale = max(abs(f1), floor[key])
            if abs(f1 - f2) > 1e-3 * scale:
                continue
            errs[key].append(abs(f1 - float(grad[int(k)])) / scale)
    ctx.check_status()
    rel32 = {"bulk": float((gb - gb64).norm() / gb64.norm()),
             "v0": float((gv.double() - gv64).norm() / gv64.norm())}
    ctx.close()
    return {"workload": ADJOINT_WORKLOAD, "particles": n, "steps": steps, "checkpoint_every": every,
            "forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
            "forward_particle_steps_per_s": n * steps / (fwd / 1e3), "loss": loss32,
            "fd_check": {"coords": {k: len(v) for k, v in errs.items()}, "tried": tried, "eps": 1e-4,
                         "eps_note": "relative for stiffness, absolute for velocity",
                         "precision": "fp64, central differences from trajectory differences",
                         "error": "|fd - adjoint| / max(|fd|, 1e-3 max|gradient|), over coordinates whose "
                                  "differences at eps and 2 eps agree to 1e-3",
                         "max_rel_err": {k: max(v) for k, v in errs.items()},
                         "median_rel_err": {k: float(np.median(v)) for k, v in errs.items()}},
            "fp32_vs_fp64_gradient_rel": rel32}


PBD_ADJOINT_WORKLOAD = ("differentiable dam-break rollout: 64x32x32 = 65,536-particle fluid block with the 32k "
                        "dam break's parameters (spacing 0.005, +-0.1 spacing jitter, radius 0.0125, cap 60, "
                        "5 DensityPBD iterations, dt 1e-3, gravity), off the walls (no boundary), initial "
                        "velocities N(0, 0.05^2) (PCG64 seed 1), 200 frames, checkpoint every 20; loss = mean "
                        "|x_T - x_target|^2 against a run from half the initial velocities")


def measure_pbd_adjoint(local):
    """The DensityPBD rollout with checkpoints and its reverse pass
    (pk_pbd_rollout / pk_pbd_rollout_backward), device time; the gradient
    checks against central differences are the tests'."""
    import torch
    import pkhot

    dev = torch.device("cuda", local)
    base = scenes.dam_break_small(seed=0, n_side=1)
    x0 = torch.from_numpy(scenes.lattice(64, 32, 32, base.spacing, 0.1, 0, origin=(0.3, 0.3, 0.3))).to(dev)
    v0 = torch.from_numpy(np.random.Generator(np.random.PCG64(1)).normal(0.0, 0.05, tuple(x0.shape))
                          .astype(np.float32)).to(dev)
    n = x0.shape[0]
    prm = pkhot.pbf_params(pkhot.nq_params(base.radius, base.lo, base.hi, base.cap),
                           pkhot.pbd_params(base.radius, base.spacing, base.rest_density, base.iterations,
                                            base.dt), base.gravity, boundary=False)
    steps, every = 200, 20
    ctx = pkhot.Context(local)
    xt, vt = x0.clone(), v0 * 0.5
    ctx.pbd_rollout(xt, vt, prm, steps, 0)
    x, v = x0.clone(), v0.clone()
    ctx.pbd_rollout(x, v, prm, steps, every)  # warm-up: workspaces
    ctx.pbd_rollout_backward(2.0 * (x - xt) / n)
    x, v = x0.clone(), v0.clone()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record()
    ctx.pbd_rollout(x, v, prm, steps, every)
    ev[1].record()
    gx, gv = ctx.pbd_rollout_backward(2.0 * (x - xt) / n)
    ev[2].record()
    torch.cuda.synchronize()
    ctx.check_status()
    fwd, bwd = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    loss = float(((x - xt) ** 2).sum(1).mean())
    ctx.close()
    return {"workload": PBD_ADJOINT_WORKLOAD, "particles": n, "steps": steps, "checkpoint_every": every,
            "forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
            "forward_particle_steps_per_s": n * steps / (fwd / 1e3), "loss": loss,
            "gradient_norm": {"x0": float(gx.norm()), "v0": float(gv.norm())}}


def measure_fp64(local, frames=10):
    """The headline lattice (2,097,152 particles, cap 64) moved off the walls,
    at rest: `frames` fused float frames against the same frames run in double
    on the GPU (pk_pbd_rollout_f64: the same method with double positions,
    velocities, integration and Jacobi passes; lists from the double positions
    rounded to float)."""
    import torch
    import pkhot

    dev = torch.device("cuda", local)
    sc = scenes.dam_break_2m(seed=0)
    x0 = torch.from_numpy((sc.x + np.array([0.5, 0.3, 0.3], np.float32)).astype(np.float32)).to(dev)
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                           sc.gravity, boundary=False)
    ctx = pkhot.Context(local)
    x32, v32 = x0.clone(), torch.zeros_like(x0)
    for _ in range(frames):
        ctx.pbf_step(x32, v32, prm)
    x64, v64 = x0.double(), torch.zeros_like(x0, dtype=torch.float64)
    ctx.pbd_rollout(x64, v64, prm, frames, 0)
    ctx.check_status()
    ctx.close()
    rel = lambda a, b: float((a.double() - b).norm() / b.norm())
    return {"workload": f"{WORKLOAD}, moved off the walls, at rest, {frames} frames", "frames": frames,
            "x_rel_error": rel(x32, x64), "v_rel_error": rel(v32, v64),
            "reference": "the same frames in double on the GPU (pk_pbd_rollout_f64)"}


def run_pk(args):
    import torch
    import torch.distributed as dist
    import pkhot

    world, rank, local = dist_setup()
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    sc = scenes.dam_break_2m(seed=0, n_side=args.side)
    n = sc.x.shape[0]
    ctx = pkhot.Context(local)
    ctx.boundary_set_box(sc.lo, sc.hi, sc.sdf_spacing, True)
    x = torch.from_numpy(sc.x.copy()).to(dev)
    v = torch.from_numpy(sc.v.copy()).to(dev)
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                           sc.gravity, boundary=True)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(val):
        if world == 1:
            return val
        t = torch.tensor([val], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # K-bar (list counts incl. self) and the solver-row length of the start state
    ctx.nq_build(x, sc.radius, sc.lo, sc.hi, sc.cap, want_list=False)
    kbar, kunion, kmax = ctx.row_stats()

    # the context's autotuner picks the pass block size and the sweep's
    # particles per pass in its first four frames (untimed); warm-up runs on
    # until it has settled
    ctx.autotune(not args.no_autotune)
    w = 0
    while w < args.warmup or ctx.tuning()[2]:
        ctx.pbf_step(x, v, prm)
        w += 1
    ctx.check_status()
    tuned_pass, tuned_build, _ = ctx.tuning()
    tuned_resident = ctx.tuning_resident()
    launches_per_step = ctx.launch_count()
    barrier()

    # Timed: K eager frames (pk_pbf_step), then K replays of the frame recorded
    # as a CUDA graph through the C ABI (pk_graph_capture runs one frame to
    # size every buffer and records the next, untimed; pk_graph_launch replays
    # the same kernels on the same buffers without the launch gaps between
    # them).  `value` is the graph replay, the fixed-frame loop's fastest form
    # in this library; the eager figure is reported beside it.
    clocks = NvmlClocks(bus_id_of(local))
    clocks.start()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        ctx.pbf_step(x, v, prm)
    e1.record(stream)
    barrier()
    eager_ms = max_over_ranks(e0.elapsed_time(e1))
    ctx.check_status()
    ctx.graph_capture(x, v, prm)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    g0.record(stream)
    for _ in range(args.steps):
        ctx.graph_launch()
    g1.record(stream)
    barrier()
    ms_max = max_over_ranks(g0.elapsed_time(g1))
    clk = clocks.stop()
    ctx.graph_release()
    ctx.check_status()
    value = world * n * args.steps / (ms_max / 1e3)

    # ---- the per-kernel split: as many frames again with the context's
    # per-kernel-class CUDA events on (they sit between the kernels, so these
    # frames are not the ones timed above)
    ctx.profile(True)
    for _ in range(args.steps):
        ctx.pbf_step(x, v, prm)
    prof = ctx.profile_read()
    ctx.profile(False)
    ctx.check_status()


    # ---- end to end through the C-ABI call on host buffers (pk_pbf_step_host:
    # every frame copies x, v in from page-locked memory and the results back)
    e2e_steps = max(3, min(args.steps, 20))
    xh = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    vh = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    xh.copy_(x.cpu())
    vh.copy_(v.cpu())
    ctx.pbf_step_host(xh, vh, prm)  # untimed: sizes the context's device copies
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        ctx.pbf_step_host(xh, vh, prm)
    f1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1))
    e2e_val = world * n * e2e_steps / (e2e_ms / 1e3)
    ctx.check_status()

    peak, peak_kind = peaks()
    # stages of the frame: the neighbour build is the sweep + selection
    # ("select") and the row emission ("emit")
    stages = {"sort": prof["sort"], "build": (prof["select"][0] + prof["emit"][0], prof["select"][1]),
              "density": prof["density"], "disp": prof["disp"], "finish": prof["finish"]}
    total_ms = sum(t for t, _ in stages.values())
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms, dom_launches = stages[dom]
    traffic = load_traffic().get(dom)
    per_launch_bytes = n * stage_bytes(dom, kbar, kunion)
    achieved = per_launch_bytes / (dom_ms / dom_launches / 1e3) / 1e9
    step_bytes = pbd_bytes_per_particle_step(kbar, sc.iterations)
    step_frac = value / world * step_bytes / (peak * 1e9)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "particles": n, "kbar": kbar, "solver_row_mean": kunion,
                   "solver_row_max": kmax, "iterations": sc.iterations,
                   "parallelism": "replicas" if world > 1 else "single",
                   "tuned": {"pass_threads_per_block": tuned_pass, "build_particles_per_pass": tuned_build,
                             "passes_as_resident_grid": tuned_resident},
                   "l2": "working set > L2 (neighbour rows alone are > 1 GB); no flush"},
        "roofline": {"bound": "hbm", "kernel": dom, "share": dom_ms / total_ms, "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": per_launch_bytes,
                     "frame": {"bytes_per_particle_step": step_bytes,
                               "achieved": value / world * step_bytes / 1e9, "frac": step_frac}},
        "stage_roofline": {k: {"share": t / total_ms,
                               "frac": n * stage_bytes(k, kbar, kunion) / (t / nl / 1e3) / 1e9 / peak}
                           for k, (t, nl) in stages.items()},
        "step_roofline": {"bytes_per_particle_step": step_bytes, "frac": step_frac,
                          "peak_source": peak_kind},
        "kernel_ms": {k: {"total_ms": prof[k][0], "launches": prof[k][1]} for k in prof},
        "api": "pk_graph_capture / pk_graph_launch (the frame replayed as a CUDA graph)",
        "eager": {"value": world * n * args.steps / (eager_ms / 1e3), "unit": UNIT,
                  "ms_per_step": eager_ms / args.steps, "api": "pk_pbf_step"},
        "e2e": {"value": e2e_val, "unit": UNIT, "api": "pk_pbf_step_host", "h2d_bytes_per_step": 2 * n * 12,
                "d2h_bytes_per_step": 2 * n * 12, "steps": e2e_steps},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    # ---- the stock model's frame: the same frame plus ImplicitViscosity (viscosity 1, 5 sweeps)
    prm_vis = pkhot.pbf_params(prm.nq, prm.pbd, sc.gravity, boundary=True, viscosity=1.0, viscosity_iterations=5)
    vis_steps = max(3, min(args.steps, 20))
    for _ in range(max(3, args.warmup)):
        ctx.pbf_step(x, v, prm_vis)
    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(vis_steps):
        ctx.pbf_step(x, v, prm_vis)
    g1.record(stream)
    barrier()
    vis_ms = max_over_ranks(g0.elapsed_time(g1)) / vis_steps
    ctx.check_status()
    line["viscosity"] = {"ms_per_step": vis_ms, "value": world * n / (vis_ms / 1e3), "unit": UNIT,
                         "stage_ms": vis_ms - eager_ms / args.steps, "iterations": 5,
                         "note": "PositionBasedFluidModel frame with ImplicitViscosity (viscosity 1) "
                                 "on the solver rows, eager pk_pbf_step frames (stage_ms against the "
                                 "eager plain frame)"}
    ctx.close()
    if not args.no_batched:
        line["batched"] = measure_batched(local, max(3, min(args.steps, 20)), max(3, args.warmup), barrier,
                                          max_over_ranks, rank, world)
    if not args.no_pd:
        line["peridynamics"] = measure_pd(local, max(3, min(args.steps, 20)), max(3, args.warmup), barrier)
    if not args.no_pd:
        line["elastoplastic"] = measure_elastoplastic(local, max(3, min(args.steps, 10)), 3, barrier)
    if not args.no_adjoint:
        line["adjoint"] = measure_adjoint(local)
        line["adjoint_pbd"] = measure_pbd_adjoint(local)
    if args.side == 128:
        line["fp64_check"] = measure_fp64(local)
    if rank == 0 and world == 1 and not args.no_cpu:
        cv, cores, cn = time_cpu(steps=2, warmup=1)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"2 steps of a {cn}-particle block with the 2M scene's "
                                          "parameters, CPU restatement, OpenMP"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="pk", choices=["pk", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-scenes comparison")
    ap.add_argument("--no-pd", action="store_true", help="skip the peridynamics bar")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable rollout")
    ap.add_argument("--pd-only", action="store_true",
                    help="run only the elastic bar (524,288 particles) and print its dict; for profiler "
                         "captures of the peridynamics step")
    ap.add_argument("--elastoplastic-only", action="store_true",
                    help="run only the elastoplastic frame (65,536 particles) and print its dict; for "
                         "profiler captures of that frame")
    ap.add_argument("--pbd-adjoint-only", action="store_true",
                    help="run only the DensityPBD rollout and its reverse pass (65,536 particles, 200 frames) and "
                         "print its dict; for profiler captures of the adjoint kernels")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default shapes (256 threads per pass block, 8 particles per sweep pass) "
                         "instead of tuning during warm-up; for profiler captures, whose serialised "
                         "launches would mislead the tuner")
    ap.add_argument("--side", type=int, default=128,
                    help="lattice side of the scene (128 = the 2,097,152-particle workload; "
                         "smaller sides are for profiling captures only)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.pd_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(measure_pd(0, args.steps, args.warmup, torch.cuda.synchronize)), flush=True)
        return 0
    if args.pbd_adjoint_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(measure_pbd_adjoint(0)), flush=True)
        return 0
    if args.elastoplastic_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(measure_elastoplastic(0, args.steps, args.warmup, torch.cuda.synchronize)), flush=True)
        return 0
    return run_pk(args)


if __name__ == "__main__":
    sys.exit(main())
