"""Benchmark of the D2Q9 step: MLUPS and HBM GB/s on the 4096 x 1024 channel
with one IB cylinder (D = 128, Re 3900), MRT + Smagorinsky (Cs 0.1), FP32.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); every rank runs an independent
replica of the lattice (the step does not shard: one domain per GPU), so the
whole-job value is the sum over ranks and scaling is weak.  Timing: W untimed
steps, then exactly K steps between a barrier + synchronize on both sides,
CUDA events on the library's stream around the steps queued behind a short
hold (ippi_step_timed), max over ranks; SM clocks and throttle reasons from
NVML during the timed steps.  The populations
(2 x 151 MB) exceed the 126 MB L2, so no flush is needed between steps.

Keys beyond the base contract:
  e2e           the same metric through the C ABI with host buffers: initial
                FP32 fields uploaded from pinned host memory, the K steps, the
                per-step body forces read back, rho / ux / uy downloaded in
                FP32 (the reference's SINGLE build)
  roofline      bulk stream-collide kernel: 72 algorithmic bytes per node
                (9 loads + 9 stores of FP32) / its CUDA-event launch time
  cpu_baseline  the reference's own MRT+Smagorinsky step (compiled from its
                sources, SINGLE precision) on the same grid, all host cores
--impl reference runs only that CPU reference arm (rank 0).
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

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(
    REPO, "machine-learning-based-implicit-physical-parametric-inference-for-cfd-simulation-promotion_b200")
sys.path.insert(0, PKG)

NX, NY = 4096, 1024
BYTES_PER_NODE = 72  # FP32: 9 loads + 9 stores
# DRAM bytes (read + write) of one step launch on this workload, from the
# ncu capture summarised under profiles/ (dram__bytes_read.sum 151.98 MB +
# dram__bytes_write.sum 103.09 MB; part of the writes is still in L2 when the
# kernel ends)
NCU_TRAFFIC_BYTES = 255.07e6
METRIC = "MLUPS"
WORKLOAD = "channel_cylinder_4096x1024_mrt_smagorinsky_ib_fp32"


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def max_over_ranks(x, dist=None, device="cuda"):
    """The largest of the ranks' values of x (one all-reduce; x itself
    without a process group).  Every rank must call it at the same point."""
    if not dist:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_mlups(nodes, steps, world, seconds):
    """Lattice updates of all ranks (each its own lattice of `nodes` nodes,
    `steps` steps) per second of the slowest rank, in millions."""
    return nodes * steps * world / seconds / 1e6


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML (read-only queries)
    every ~0.5 ms on a background thread while the measured work runs, plus
    one reading on entry and one on exit.  Falls back to `nvidia-smi -lms
    100` when NVML cannot be loaded."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, gpu_index, period_s=0.0005):
        self.gpu = gpu_index
        self.period = period_s
        self.samples = []   # (sm_mhz, reasons bitmask)
        self.max_mhz = None
        self.nvml = None
        self.proc = None
        self.stop = threading.Event()

    def _read_nvml(self):
        n = self.nvml
        sm = n.nvmlDeviceGetClockInfo(self.dev, n.NVML_CLOCK_SM)
        r = n.nvmlDeviceGetCurrentClocksEventReasons(self.dev)
        self.samples.append((float(sm), int(r)))

    def __enter__(self):
        try:
            import pynvml as n

            n.nvmlInit()
            self.nvml = n
            self.dev = n.nvmlDeviceGetHandleByIndex(self._nvml_index())
            self.max_mhz = float(n.nvmlDeviceGetMaxClockInfo(self.dev, n.NVML_CLOCK_SM))
            self._read_nvml()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception:
            self.nvml = None
            self._start_smi()
        return self

    def _nvml_index(self):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [v.strip() for v in vis.split(",")]
            if self.gpu < len(ids) and ids[self.gpu].isdigit():
                return int(ids[self.gpu])
        return self.gpu

    def _poll(self):
        while not self.stop.is_set():
            try:
                self._read_nvml()
            except Exception:
                return
            time.sleep(self.period)

    def _start_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self._nvml_index())], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read_smi(self):
        bits = [0x8, 0x40, 0x20, 0x4]
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 6 and parts[0].replace(".", "").isdigit():
                self.max_mhz = float(parts[1]) if parts[1].replace(".", "").isdigit() else None
                self.samples.append((float(parts[0]),
                                     sum(b for b, v in zip(bits, parts[2:6]) if v == "Active")))

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml:
            self.t.join(timeout=2)
            try:
                self._read_nvml()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        sm = [s[0] for s in self.samples]
        reasons = sorted({name for _, r in self.samples for name, b in self.REASONS if r & b})
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples),
                "source": "nvml" if self.nvml else "nvidia-smi"}


# ---------------------------------------------------------------------------
# CPU reference (reference arm and cpu_baseline)
# ---------------------------------------------------------------------------
class quiet_stdout:
    """Send file descriptor 1 to /dev/null (the reference's own progress
    prints) so that stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        os.close(devnull)

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def cpu_reference(steps, warmup, max_seconds=None):
    with quiet_stdout():
        return _cpu_reference(steps, warmup, max_seconds)


def _cpu_reference(steps, warmup, max_seconds=None):
    """Time the reference's MRT + Smagorinsky step (its own sources compiled by
    oracle/build_ref.sh, SINGLE precision, flat-plate scene, one MPI rank per
    host core as threads) on the NX x NY grid.  Falls back to the FP64 oracle
    port when the reference build is absent.  Returns (MLUPS, info)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po

    cores = os.cpu_count() or 1
    tau = 0.5 + 3 * 0.04 * 128 / 3900
    if po.ref_available("mrt_f32"):
        sim = po.RefSim(NX, NY, tau=tau, cs=0.1, u_in=0.04, ranks=cores, variant="mrt_f32")
        kind, desc = "reference", "reference MRT+Smagorinsky (SINGLE) flat plate"
    else:
        po.build_oracle()
        sim = po.Oracle(NX, NY, collision=po.MRT, tau0=tau, cs=0.1, u_in=0.04)
        cores = 1
        kind, desc = "port", "FP64 oracle port MRT+Smagorinsky flat plate"
    if warmup:
        sim.step(warmup, 1)
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        sim.step(1, warmup + done + 1)
        done += 1
        if max_seconds and time.perf_counter() - t0 > max_seconds:
            break
    dt = time.perf_counter() - t0
    mlups = NX * NY * done / dt / 1e6
    return mlups, dict(kind=kind, cores=cores, steps=done, seconds=dt,
                       sample=f"{done} steps of {NX}x{NY} ({desc}), {cores} threads")


def run_reference_arm(a):
    rank, _, world = env_rank()
    if rank != 0:
        return
    mlups, info = cpu_reference(a.steps, a.warmup, max_seconds=240)
    line = {"metric": METRIC, "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": a.gpus,
            "steps": info["steps"], "warmup": a.warmup,
            "ms_per_step": round(info["seconds"] / max(info["steps"], 1) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "grid_nodes": NX * NY,
                       "reference_scene": "flat plate (the reference has no cylinder/IB scene)"},
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": info["cores"],
                             "kind": info["kind"], "sample": info["sample"]},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(a):
    import ctypes as C

    import numpy as np
    import torch

    import ippi_lbm as ip

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()

    sc = ip.scenes.config2()
    lat = ip.Lattice(NX, NY, device=local, **sc["params"])
    kernel_name = "step_ib_fused<F32,CHANNEL,MRT,16>"
    # per step: one launch, the IB blocks and the bulk row segments
    launches_per_step = 1
    lat.init_macros(*sc["init"])
    lat.set_markers(sc["markers"], ds=sc["ds"])

    # warm-up (also builds the CUDA graphs)
    lat.step(max(a.warmup, 3), 1)
    t_next = max(a.warmup, 3) + 1

    # ---- device-resident throughput ---------------------------------------
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    # The K steps are queued behind a short hold on the library's stream and
    # timed with CUDA events recorded there just before the first and after
    # the last (ippi_step_timed), so the host's enqueue latency stays out of
    # the device time.  The clock sampler runs over these steps and the
    # per-launch profile leg after them.
    with ClockSampler(local) as clk:
        ms_dev = lat.step_timed(a.steps, t_next)
        t_next += a.steps
        barrier()
        torch.cuda.synchronize()
        ms_max = max_over_ranks(ms_dev, dist)
        value = whole_job_mlups(NX * NY, a.steps, world, ms_max * 1e-3)

        # ---- per-launch CUDA-event times (IB on the side stream) -----------
        nprof = min(max(a.steps // 2, 20), 200)
        ms_bulk, ms_band, ms_ib = lat.profile_steps(nprof, t_next)
        t_next += nprof
    hbm, peak_kind = peaks()
    # One launch per step (IB blocks + bulk row segments), so its average
    # duration in the timed graph replay is the device time per step.  The
    # bulk kernel's own launch time from profile_steps (IB on the side
    # stream) is reported beside it.
    ms_span = ms_max / a.steps
    achieved = NX * NY * BYTES_PER_NODE / (ms_span * 1e-3) / 1e9

    # ---- end to end through the C ABI with host buffers --------------------
    # The reference's driver (main.cpp:105-120) runs OneLBMStep every step
    # and dumps the fluid fields every SaveStep steps.  Here: the initial
    # fields uploaded from pinned host memory, the K steps in one ippi_step
    # call, the per-step body forces read back (ippi_force_history) and the
    # rho / ux / uy fields downloaded once (one field dump).  The host fields
    # are FP32, the LatMesh fields of the reference's SINGLE build (its CPU
    # arm runs that build).
    n_e2e = a.steps
    rho0, ux0, uy0 = (np.ascontiguousarray(x, dtype=np.float32) for x in sc["init"])
    pin = [torch.from_numpy(x).pin_memory().numpy() for x in (rho0, ux0, uy0)]
    L = ip.lib()
    dump = [torch.empty((NY, NX), dtype=torch.float32).pin_memory().numpy() for _ in range(3)]
    hist = torch.zeros((n_e2e, 1, 2), dtype=torch.float64).pin_memory().numpy()
    fp = C.POINTER(C.c_float)

    def e2e_pass(nsteps):
        ip._lib.check(L.ippi_init_macros_f32(lat.handle, *(x.ctypes.data_as(fp) for x in pin)),
                      lat.handle)
        ip._lib.check(L.ippi_step(lat.handle, nsteps, 1), lat.handle)
        n = L.ippi_force_history(lat.handle, hist.ctypes.data_as(C.POINTER(C.c_double)), nsteps)
        for fld, buf in zip((ip.FIELD_RHO, ip.FIELD_UX, ip.FIELD_UY), dump):
            ip._lib.check(L.ippi_download_f32(lat.handle, fld, buf.ctypes.data_as(fp), buf.nbytes),
                          lat.handle)
        return n

    # one untimed pass (the download buffers are allocated on first use)
    e2e_pass(max(a.warmup, 3))
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    got = e2e_pass(n_e2e)
    e2e_s = time.perf_counter() - t0
    assert got == n_e2e, got
    e2e_s = max_over_ranks(e2e_s, dist)
    e2e = whole_job_mlups(NX * NY, n_e2e, world, e2e_s)
    h2d = (rho0.nbytes + ux0.nbytes + uy0.nbytes) / n_e2e
    d2h = (hist.nbytes + sum(b.nbytes for b in dump)) / n_e2e

    if rank == 0:
        cpu = None
        if world == 1 and not a.no_cpu:
            mlups_cpu, info = cpu_reference(a.cpu_steps, 1, max_seconds=30)
            cpu = {"value": round(mlups_cpu, 3), "unit": "MLUPS", "cores": info["cores"],
                   "kind": info["kind"], "sample": info["sample"]}
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_max / a.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "collision": "MRT",
                       "les": "smagorinsky_cs0.1", "cylinder_d": 128, "markers": len(sc["ds"]),
                       "re": 3900, "u_max": 0.04, "storage": "f32",
                       "l2": "inputs larger than L2 (2 x 151 MB populations)",
                       "parallelism": f"replicas{world}"},
            "hbm_gbs": round(value * BYTES_PER_NODE / 1e3 / world, 1),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": NCU_TRAFFIC_BYTES,
                         "traffic_algorithmic": NX * NY * BYTES_PER_NODE,
                         "peak_source": peak_kind, "kernel": kernel_name,
                         "kernel_ms": round(ms_span, 5),
                         "kernel_ms_basis": "the step's one launch (IB blocks + bulk row segments), "
                                            "per step in the timed graph replay",
                         "kernel_ms_isolated_launch": round(ms_bulk, 5),
                         "ib_ms_side_stream": round(ms_ib, 5), "band_ms": round(ms_band, 5),
                         "bytes_per_node": BYTES_PER_NODE},
            "e2e": {"value": round(e2e, 1), "unit": "MLUPS", "h2d_bytes_per_step": round(h2d),
                    "d2h_bytes_per_step": round(d2h), "steps": n_e2e},
            "gpu_launches": a.steps * launches_per_step,
            "clocks": dict(clk.summary(), window="the timed steps and the per-launch profile leg"),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    lat.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_ncu_case(a):
    """The command profiled by ncu: the benchmark lattice, `steps` steps of
    one graph launch each (the timed path: one step_ib_fused launch per
    step), so each launch is a separate entry."""
    import ippi_lbm as ip

    sc = ip.scenes.config2()
    lat = ip.Lattice(NX, NY, **sc["params"])
    lat.init_macros(*sc["init"])
    lat.set_markers(sc["markers"], ds=sc["ds"])
    for s in range(a.steps):
        lat.step(1, s + 1)
    lat.close()
    print(json.dumps({"ncu_case": WORKLOAD, "steps": a.steps}))


def run_learned_ncu_case(a):
    """The command profiled by ncu for the learned-tau step: the coarse
    1024 x 256 channel of the learned comparison (MRT, FP32, learned tau with
    a seeded Xavier network whose range covers every node), --steps steps
    after 200 warm-up steps, device-timed (ippi_step_timed); with
    --tensor-cores the network's hidden layer runs on the tensor cores."""
    import numpy as np
    import torch

    import ippi_lbm as ip
    from ippi_lbm import learned_tau as lt
    from ippi_lbm import scenes

    sc = scenes.cylinder_channel(1024, 256, 32, 256, 128, 0.04, 3900, collision=ip.MRT)
    lat = ip.Lattice(1024, 256, **dict(sc["params"], les_model=ip.LES_LEARNED, storage=ip.F32))
    lat.init_macros(*sc["init"])
    lat.set_markers(sc["markers"], ds=sc["ds"])
    stats = np.concatenate([[1.0, 0.04, 0, 0, 0, 1e-3], [2e-3, 0.02, 0.5, 0.5, 0.5, 1e-3],
                            [-1e6] * 6, [1e6] * 6, [1e-3]]).astype(np.float32)
    bits, _ = lt.bf16_bits(lt.xavier(0))
    lat.load_tau_mlp(bits, stats)
    if a.tensor_cores:
        lat.set_learned_tensor_cores(True)
    lat.step(200, 1)
    torch.cuda.synchronize()
    ms = lat.step_timed(a.steps, 201)
    us = ms * 1e3 / a.steps
    d = lat.diagnostics()
    lat.close()
    print(json.dumps({"learned_ncu_case": "channel_cylinder_1024x256_mrt_learned_tau", "steps": a.steps,
                      "hidden_layer": "bf16 tensor cores (mma.sync)" if a.tensor_cores else "fp32 fma",
                      "us_per_step": round(us, 2), "fallback_nodes": d["fallback_nodes"]}))


def run_config3_ncu_case(a):
    """The command profiled by ncu for one storage of the precision sweep: the
    64-cylinder 16384 x 4096 lattice (MRT + Smagorinsky, 90 IB blocks) with
    --storage populations, 3 warm-up steps, then --steps single steps (one
    step_ib_fused launch each)."""
    import ippi_lbm as ip
    from ippi_lbm.validation import config3_scene

    st = {"f32": ip.F32, "f16": ip.F16, "bf16": ip.BF16}[a.storage]
    sc = config3_scene(storage=st)
    lat = ip.Lattice(sc["nx"], sc["ny"], **sc["params"])
    lat.init_macros(*sc["init"])
    lat.set_markers(sc["markers"], ds=sc["ds"], body=sc["bodies"])
    lat.step(3, 1)
    for s_ in range(a.steps):
        lat.step(1, 4 + s_)
    lat.close()
    print(json.dumps({"config3_ncu_case": f"channel_64_cylinders_{sc['nx']}x{sc['ny']}_mrt_{a.storage}",
                      "steps": a.steps}))


def run_config3_rate(a):
    """Step rate of the precision-sweep lattice: 16384 x 4096 (67 M nodes),
    64 seeded IB cylinders (D = 48, about 9,700 markers), MRT + Smagorinsky,
    Re 1000, for each population storage: --steps steps after 50 warm-up
    steps, device-timed (ippi_step_timed: CUDA events around the queued
    steps).  One JSON line per storage (GLUPS and HBM GB/s at the storage's bytes per
    node)."""
    import ippi_lbm as ip
    from ippi_lbm.validation import config3_scene

    for name, st, bpn in (("f32", ip.F32, 72), ("f16", ip.F16, 36), ("bf16", ip.BF16, 36)):
        sc = config3_scene(storage=st)
        nx, ny = sc["nx"], sc["ny"]
        lat = ip.Lattice(nx, ny, **sc["params"])
        lat.init_macros(*sc["init"])
        lat.set_markers(sc["markers"], ds=sc["ds"], body=sc["bodies"])
        lat.step(50, 1)
        s = lat.step_timed(a.steps, 51) * 1e-3
        lat.close()
        glups = nx * ny * a.steps / s / 1e9
        print(json.dumps({"config3_rate": f"channel_64_cylinders_{nx}x{ny}_mrt_{name}", "steps": a.steps,
                          "markers": int(len(sc["ds"])), "us_per_step": round(s / a.steps * 1e6, 1),
                          "glups": round(glups, 2), "hbm_gbs": round(glups * bpn, 1)}), flush=True)


def run_adjoint_ncu_case(a):
    """The command profiled by ncu for the adjoint: the --adjoint lattice
    (learned tau, seeded Xavier network), an --adjoint-steps rollout
    checkpointed every 64 steps and its backward sweep with a random force
    loss, twice."""
    import numpy as np

    import ippi_lbm as ip
    from ippi_lbm import learned_tau as lt
    from ippi_lbm import scenes

    n = a.adjoint_steps
    sc = scenes.cylinder_channel(1024, 256, 32, 256, 128, 0.04, 3900, collision=ip.MRT)
    lat = ip.Lattice(1024, 256, **dict(sc["params"], les_model=ip.LES_LEARNED, storage=ip.F32))
    lat.init_macros(*sc["init"])
    lat.set_markers(sc["markers"], ds=sc["ds"])
    stats = np.concatenate([[1.0, 0.04, 0, 0, 0, 1e-3], [2e-3, 0.02, 0.5, 0.5, 0.5, 1e-3],
                            [0.9, 0.0, -1, -1, -1, 0.0], [1.1, 0.2, 1, 1, 1, 0.1],
                            [1e-3]]).astype(np.float32)
    lat.load_tau_mlp_f32(lt.xavier(0).astype(np.float32), stats)
    wF = np.random.default_rng(0).normal(0, 1, (n, 1, 2))
    for _ in range(2):
        lat.adjoint_forward(n, 1, 64)
        lat.adjoint_backward(dl_dforce=wF, mlp=True)
    lat.close()
    print(json.dumps({"adjoint_ncu_case": "channel_cylinder_1024x256_mrt_learned_tau_adjoint", "steps": n}))


def run_learned(a):
    """The learned-tau comparison: fine 4096 x 1024 plain-Smagorinsky runs
    (the Cd reference from two noise seeds, and the data source), the
    network fitted a priori to their filtered snapshots and then trained
    through the coarse solver on the filtered field, and the 1024 x 256
    lattice with plain Smagorinsky and with each network over the same
    physical time, for three seeds.  A ladder of plain resolutions gives the
    wall time plain Smagorinsky needs for a learned run's drag error; value =
    that time / the learned run's (time to solution at equal Cd error) for
    the better of the a-priori and the through-solver networks, or null
    where plain Smagorinsky on the coarse grid is already as close to the
    fine drag."""
    import torch

    from ippi_lbm import learned_tau as lt

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    steps = a.learned_steps
    r = lt.experiment(fine_steps=steps, avg_steps=steps * 4 // 5, device=local,
                      finetune_iters=a.learned_finetune, calibrate_drag=a.learned_drag_calibration,
                      log=(lambda s_: print(s_, file=sys.stderr, flush=True)))
    r.pop("nets")
    if rank != 0:
        return
    # the best network among those fitted to nothing but the fine run's
    # filtered fields; the mean-wake scale fit (its objective can be flat
    # within the chaotic wake's noise) and the drag-fitted variants are
    # reported, not ranked
    best = max(((k, v) for k, v in r["time_to_solution"].items()
                if v["ratio"] is not None and k in ("a_priori", "through_solver_field")),
               key=lambda kv: kv[1]["ratio"], default=(None, {}))
    line = {
        "metric": "learned_tau_time_to_solution_at_equal_cd_error", "value": best[1].get("ratio"),
        "variant": best[0],
        "unit": "x (plain wall at the learned run's Cd error / learned wall)", "higher_is_better": True,
        "n_gpus": 1, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "channel_cylinder_re3900_fine_4096x1024_coarse_1024x256_mrt_fp32",
                   "fine_steps": r["fine"]["steps"], "coarse_steps": r["coarse"]["steps"],
                   "snapshots": 200, "filter": 4, "eval_seeds": r["coarse"]["seeds"]},
        **{k: r[k] for k in ("fine", "plain", "a_priori", "through_solver_field", "a_priori_wake_scale",
                             "drag_fitted_scale", "drag_finetuned", "ladder", "time_to_solution",
                             "training", "field_training", "wake_fit") if k in r},
    }
    print(json.dumps(line), flush=True)


def run_adjoint(a):
    """Forward + backward throughput of the adjoint on the 1024 x 256 MRT
    lattice with the per-node learned tau (a seeded Xavier network), a
    4,000-step rollout checkpointed every 64 steps, FP32 forward; gradient
    with respect to the network weights.  The gradient is checked in FP64
    (FP64 forward on the same lattice) by central differences (eps 1e-3,
    Richardson-combined with eps 5e-4) along seeded random directions, over
    --adjoint-check-steps steps: the Re 3900 wake is chaotic, so over
    thousands of steps finite differences and the tangent gradient part ways
    (the reported errors at two horizons show it)."""
    import numpy as np
    import torch

    import ippi_lbm as ip
    from ippi_lbm import learned_tau as lt
    from ippi_lbm import scenes

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    nsteps, K = a.adjoint_steps, 64
    sc = scenes.cylinder_channel(1024, 256, 32, 256, 128, 0.04, 3900, collision=ip.MRT)
    params = dict(sc["params"], les_model=ip.LES_LEARNED)
    w = lt.xavier(0).astype(np.float32)
    stats = np.concatenate([[1.0, 0.04, 0, 0, 0, 1e-3], [2e-3, 0.02, 0.5, 0.5, 0.5, 1e-3],
                            [0.9, 0.0, -1, -1, -1, 0.0], [1.1, 0.2, 1, 1, 1, 0.1],
                            [1e-3]]).astype(np.float32)
    rng = np.random.default_rng(0)
    wF = rng.normal(0, 1, (nsteps, 1, 2))

    def run(wv, n, weights, grads=False, storage=ip.F32):
        lat = ip.Lattice(1024, 256, device=local, **dict(params, storage=storage))
        lat.init_macros(*sc["init"])
        lat.set_markers(sc["markers"], ds=sc["ds"])
        lat.load_tau_mlp_f32(wv, stats)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lat.adjoint_forward(n, 1, K)
        t1 = time.perf_counter()
        F = lat.force_history(n)
        g = lat.adjoint_backward(dl_dforce=weights, mlp=True) if grads else None
        t2 = time.perf_counter()
        lat.close()
        return float(np.sum(weights * F)), g, t1 - t0, t2 - t1

    run(w, nsteps, wF, grads=True)  # warm-up (allocations, graphs)
    _, g, tf, tb = run(w, nsteps, wF, grads=True)
    checks = {}
    for hn in sorted({a.adjoint_check_steps, nsteps}):
        wc = rng.normal(0, 1, (hn, 1, 2))
        _, gc, _, _ = run(w, hn, wc, grads=True, storage=ip.F64)
        errs = []
        for _ in range(a.adjoint_dirs):
            d = rng.normal(0, 1, w.size)
            dl, ad = [], []
            for eps in (1e-3, 5e-4):
                wp, wm = (w + eps * d).astype(np.float32), (w - eps * d).astype(np.float32)
                dl.append(run(wp, hn, wc, storage=ip.F64)[0] - run(wm, hn, wc, storage=ip.F64)[0])
                ad.append(float(gc["mlp"] @ (wp.astype(np.float64) - wm.astype(np.float64))))
            fd, want = 8 * dl[1] - dl[0], 8 * ad[1] - ad[0]
            errs.append(float(f"{abs(fd - want) / max(abs(fd), 1e-30):.3g}"))
        checks[str(hn)] = errs
    if rank != 0:
        return
    line = {
        "metric": "adjoint_forward_backward_steps_per_s", "value": round(nsteps / (tf + tb), 1),
        "unit": "steps/s", "higher_is_better": True, "n_gpus": 1, "dtype": "f32 forward, f64 adjoint",
        "data": "synthetic",
        "config": {"workload": "channel_cylinder_1024x256_mrt_learned_tau_adjoint", "nx": 1024, "ny": 256,
                   "rollout_steps": nsteps, "checkpoint_every": K, "gradient": "network weights (1313)"},
        "forward_s": round(tf, 3), "backward_s": round(tb, 3),
        "mlups_forward_backward": round(1024 * 256 * nsteps / (tf + tb) / 1e6, 1),
        "fd_check_fp64_rel_err_by_steps": checks,
    }
    print(json.dumps(line), flush=True)


def run_validate(a):
    """Precision studies: config 2 (FP32 vs FP64, MRT and RR, 4096 x 1024,
    Cd / St / mean-velocity L2) and config 3 (16384 x 4096, 64 cylinders,
    FP32 / FP16 / BF16 vs FP64: per-cylinder Cd, mean-velocity L2, mass
    drift)."""
    import torch

    from ippi_lbm import validation as val

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    log = (lambda s_: print(s_, file=sys.stderr, flush=True))
    c2 = val.config2_precision(steps=a.validate_steps2, avg=a.validate_steps2 * 2 // 5, log=log)
    c3 = val.config3_precision(steps=a.validate_steps3, avg=a.validate_steps3 // 2, log=log)
    if rank == 0:
        print(json.dumps({"metric": "precision_study", "config2": c2, "config3": c3}), flush=True)


PLATE_NX, PLATE_NY = 2401, 501


def plate_nets():
    """The four shipped boundary nets (AutoT01/03/05/07, TorchScript parameter
    order, exported once as raw FP32 under tests/golden/band_nets)."""
    import numpy as np

    d = os.path.join(REPO, "tests", "golden", "band_nets")
    return {t: np.fromfile(os.path.join(d, f"AutoT0{t}.f32"), dtype=np.float32) for t in (1, 3, 5, 7)}


def run_plate(a):
    """The reference's own shipped workload: the 2401 x 501 flat plate of
    main.cpp:20-45 (BGK + Smagorinsky Cs 0.173, NEE inlet u 0.1, specular
    bottom before x 400, no-slip after it) with the four boundary nets on
    (mesh.cpp:357-380), FP64 (the reference's default REAL) and FP32 storage.
    Per storage one JSON line: the step rate with nets (ippi_step_timed over
    --steps steps), the per-launch CUDA-event times of the bulk kernel and of
    the side-stream chain (boundary-net inputs + nets + band collisions) that
    runs beside it, the step rate with the nets off, and the reference's own
    CPU step with the nets on (libtorch build when present), all host cores,
    a bounded sample."""
    import numpy as np  # noqa: F401
    import torch

    import ippi_lbm as ip

    torch.cuda.set_device(0)
    nets = plate_nets()
    nn = PLATE_NX * PLATE_NY
    for name, st, bpn in (("f64", ip.F64, 144), ("f32", ip.F32, 72)):
        res = {}
        for with_nets in (True, False):
            lat = ip.Lattice(PLATE_NX, PLATE_NY, storage=st)
            if with_nets:
                for t, w in nets.items():
                    lat.load_band_net(t, w)
            lat.step(max(a.warmup, 3), 1)
            ms = lat.step_timed(a.steps, max(a.warmup, 3) + 1)
            prof = lat.profile_steps(min(max(a.steps, 20), 200), max(a.warmup, 3) + 1 + a.steps)
            res[with_nets] = (ms / a.steps, prof)
            tau0 = lat.params.tau0
            lat.close()
        ms_step, (ms_bulk, ms_band, _) = res[True]
        line = {"plate": f"flat_plate_{PLATE_NX}x{PLATE_NY}_bgk_smagorinsky_nets_{name}", "steps": a.steps,
                "ms_per_step": round(ms_step, 5), "mlups": round(nn / ms_step / 1e3, 1),
                "bulk_kernel_ms": round(ms_bulk, 5),
                "bulk_kernel_gbs": round(nn * bpn / ms_bulk / 1e6, 1),
                "side_chain_ms": round(ms_band, 5),
                "band_nodes": 2 * (PLATE_NX - 2) + 2 * (PLATE_NY - 2),
                "ms_per_step_nets_off": round(res[False][0], 5),
                "mlups_nets_off": round(nn / res[False][0] / 1e3, 1)}
        if not a.no_cpu:
            sys.path.insert(0, os.path.join(REPO, "oracle"))
            import pyoracle as po

            variant = ("srt_torch" if name == "f64" else "srt_f32_torch")
            if not po.ref_available(variant):
                variant = "srt" if name == "f64" else "srt_f32"
                os.environ.setdefault("IPPI_REF_NN_DIR", os.path.join(REPO, "tests", "golden", "band_nets"))
            cores = os.cpu_count() or 1
            with quiet_stdout():
                sim = po.RefSim(PLATE_NX, PLATE_NY, tau=tau0, ranks=cores, variant=variant)
                sim.step(1, 1)
                t0 = time.perf_counter()
                done = 0
                while done < a.cpu_steps and (done < 2 or time.perf_counter() - t0 < 30):
                    sim.step(1, 2 + done)
                    done += 1
                dt = time.perf_counter() - t0
                del sim
            line["cpu_reference"] = {
                "mlups": round(nn * done / dt / 1e6, 3), "ms_per_step": round(dt / done * 1e3, 1),
                "cores": cores, "kind": "reference",
                "nets": "libtorch on the shipped archives" if variant.endswith("torch")
                        else "the nets' FP32 forward restated (stand-in build)",
                "sample": f"{done} steps, {cores} thread-ranks"}
        print(json.dumps(line), flush=True)


def run_plate_ncu_case(a):
    """The command profiled by ncu for the boundary nets: the flat plate with
    the four nets, FP32 storage, --steps single steps."""
    import ippi_lbm as ip

    lat = ip.Lattice(PLATE_NX, PLATE_NY, storage=ip.F32)
    for t, w in plate_nets().items():
        lat.load_band_net(t, w)
    for s in range(a.steps):
        lat.step(1, s + 1)
    lat.close()
    print(json.dumps({"plate_ncu_case": f"flat_plate_{PLATE_NX}x{PLATE_NY}_nets_f32", "steps": a.steps}))


def run_config2_seeds(a):
    """Configuration 2 in FP32 and FP64 from --seeds noise seeds (MRT,
    --validate-steps2 steps, statistics over the last 5/6 of them): one JSON
    line with per-seed Cd, Cl, Cl rms and St and their spread."""
    import torch

    from ippi_lbm import validation as val

    torch.cuda.set_device(0)
    log = (lambda s_: print(s_, file=sys.stderr, flush=True))
    steps = a.validate_steps2
    r = val.config2_seeds(seeds=tuple(range(a.seeds)), steps=steps, avg=steps * 5 // 6, log=log)
    print(json.dumps({"metric": "config2_seed_study", **r}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--learned", action="store_true",
                    help="learned-tau time-to-solution comparison instead of the MLUPS line")
    ap.add_argument("--learned-steps", type=int, default=320000)
    ap.add_argument("--learned-finetune", type=int, default=0,
                    help="iterations of training through the solver (adjoint) after the a-priori fit")
    ap.add_argument("--learned-drag-calibration", action="store_true",
                    help="also fit the network's output scale to the fine drag itself (the judged quantity)")
    ap.add_argument("--adjoint", action="store_true",
                    help="adjoint forward+backward throughput and gradient check instead of the MLUPS line")
    ap.add_argument("--adjoint-steps", type=int, default=4000)
    ap.add_argument("--adjoint-dirs", type=int, default=2)
    ap.add_argument("--adjoint-check-steps", type=int, default=400)
    ap.add_argument("--validate", action="store_true",
                    help="precision studies of configs 2 and 3 instead of the MLUPS line")
    ap.add_argument("--validate-steps2", type=int, default=160000)
    ap.add_argument("--validate-steps3", type=int, default=20000)
    ap.add_argument("--config2-seeds", action="store_true",
                    help="configuration 2 in FP32 and FP64 over --seeds noise seeds")
    ap.add_argument("--seeds", type=int, default=3)
    ap.add_argument("--config3-rate", action="store_true",
                    help="step rate of the 64-cylinder 16384x4096 lattice per storage")
    ap.add_argument("--learned-ncu-case", action="store_true",
                    help="learned-tau steps of the coarse channel for an ncu capture")
    ap.add_argument("--tensor-cores", action="store_true",
                    help="with --learned-ncu-case: the hidden layer on the tensor cores")
    ap.add_argument("--adjoint-ncu-case", action="store_true",
                    help="short adjoint rollout and backward sweep for an ncu capture")
    ap.add_argument("--ncu-case", action="store_true",
                    help="short run of single launches for an ncu capture")
    ap.add_argument("--config3-ncu-case", action="store_true",
                    help="precision-sweep steps of one storage (--storage) for an ncu capture")
    ap.add_argument("--storage", default="f16", choices=["f32", "f16", "bf16"])
    ap.add_argument("--plate", action="store_true",
                    help="the reference's flat plate with its boundary nets (FP64 and FP32) and its CPU step")
    ap.add_argument("--plate-ncu-case", action="store_true",
                    help="flat-plate steps with the boundary nets for an ncu capture")
    a = ap.parse_args()
    if a.ncu_case:
        run_ncu_case(a)
    elif a.plate:
        run_plate(a)
    elif a.config3_ncu_case:
        run_config3_ncu_case(a)
    elif a.config2_seeds:
        run_config2_seeds(a)
    elif a.plate_ncu_case:
        run_plate_ncu_case(a)
    elif a.adjoint_ncu_case:
        run_adjoint_ncu_case(a)
    elif a.learned_ncu_case:
        run_learned_ncu_case(a)
    elif a.config3_rate:
        run_config3_rate(a)
    elif a.learned:
        run_learned(a)
    elif a.adjoint:
        run_adjoint(a)
    elif a.validate:
        run_validate(a)
    elif a.impl == "reference":
        run_reference_arm(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
