"""Benchmark: MPM particle-substeps per second of the explicit MLS/APIC substep on one B200.

Workload (default): the Drucker-Prager two-box scene -- boxes [0.1,0.45]x[0.1,0.6]x[0.1,0.9]
and [0.55,0.9]x[0.1,0.4]x[0.1,0.9] at dx=1/256 with 8 jittered particles per cell
(30,089,900 particles from the geometry), E=3.5e5, nu=0.3, rho=2200, friction 30 deg,
second box moving at (-1,0,0) m/s, slip walls, dt=5e-5.  A step is one full substep
(activation, binning, P2G, grid update, G2P with SVD + return map).  Inputs (4.4 GB of
particle state) are larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--scene dp|dp128|fc|snow16m|batch256]

--scene batch256 runs the batched workload: 256 independent scenes (15,386,080 particles,
per-scene counts log-uniform in [4k, 200k], half fixed corotated, half Drucker-Prager) advanced
together, one launch per stage.  Launch shapes are picked by the library's autotuner first.

Under torchrun every rank runs an independent replica (the path has no exchange step) and
rank 0 prints one JSON line; time is the max over ranks of CUDA-event time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MPM particle-substeps/sec on 1 B200, learned vs plain closure at stated error"
UNIT = "particle-substeps/s"
PEAKS = ROOT / "MEASURED_PEAKS.json"
# the closure's training: (epochs, batch, learning rate) stages of Adam over the projected states
TRAIN_SCHEDULE = ((20, 4096, 2e-3), (20, 4096, 5e-4), (16, 8192, 1e-4), (12, 16384, 3e-5), (8, 32768, 1e-5))


def hbm_peak():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def scene_for(name: str):
    from zsmpm_b200 import scenes
    if name == "dp":
        return scenes.config2(), "dp_two_boxes_dx256_8ppc"
    if name == "dp128":
        return scenes.config2(dx=1 / 128), "dp_two_boxes_dx128_8ppc"
    if name == "fc":
        return scenes.config1(), "fc_cube_dx128_8ppc"
    if name in ("fc_boxes", "fc_boxes128"):
        # the two-box geometry in fixed corotated (the cell-centric transfers have no plasticity)
        import dataclasses
        from zsmpm_b200 import _abi
        dx = 1 / 256 if name == "fc_boxes" else 1 / 128
        spec = dataclasses.replace(scenes.config2(dx=dx), name=f"fc_two_boxes_dx{round(1 / dx)}",
                                   material=scenes.MaterialSpec(model=_abi.FIXED_COROTATED, E=3.5e5, nu=0.3,
                                                                rho=2200.0))
        return spec, f"fc_two_boxes_dx{round(1 / dx)}_8ppc"
    if name == "snow16m":
        return scenes.config5_16m(), "snow_sphere_slab_dx295_4ppc"
    if name == "batch256":
        from zsmpm_b200 import batch
        return batch.config4(), "batch_256_scenes_dx128_8ppc"
    raise SystemExit(f"unknown scene {name}")


def generate_workload(spec):
    """(concatenated particles, per-scene Particles list or None)."""
    from zsmpm_b200 import batch, scenes
    if isinstance(spec, list):
        parts = batch.generate_all(spec)
        return batch._concat(parts), parts
    return scenes.generate(spec), None


class ClockSampler:
    """SM clock and throttle reasons sampled every few milliseconds during the timed region.

    NVML is read in a thread of this process (read-only queries; nothing is set), and only the
    samples taken between mark_start() and mark_end() count.  Without NVML it falls back to an
    nvidia-smi subprocess sampling every 100 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device_index: int, period_s: float = 0.004):
        self.idx = device_index
        self.period = period_s
        self.proc = None
        self.file = None
        self.thread = None
        self.stop = None
        self.samples = []  # (time, sm MHz, max sm MHz, reason bits)
        self.t0 = self.t1 = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.idx)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.stop = threading.Event()

            def run():
                while not self.stop.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((time.perf_counter(), sm, mx, bits))
                    except Exception:
                        pass
                    time.sleep(self.period)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def __exit__(self, *exc):
        if self.thread:
            time.sleep(2 * self.period)
            self.stop.set()
            self.thread.join(1.0)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if self.thread is not None:
            t0 = self.t0 if self.t0 is not None else -1e30
            t1 = self.t1 if self.t1 is not None else 1e30
            rows = [r for r in self.samples if t0 <= r[0] <= t1]
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            reasons = sorted({name for r in rows for name, bit in self.REASONS if r[3] & bit})
            return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": max(r[2] for r in rows),
                    "reasons": reasons, "samples": len(rows), "source": "nvml, every 4 ms in the timed region"}
        if not self.file:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = [n for n, _ in self.REASONS]
        for r in rows:
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "source": "nvidia-smi"}


def max_over_ranks(x: float, ws: int) -> float:
    from zsmpm_b200 import replicas
    return replicas.max_over_ranks(x) if ws > 1 else x


def barrier(ws: int):
    from zsmpm_b200 import replicas
    if ws > 1:
        replicas.barrier()


# DRAM bytes (read + write) per particle of one k_g2p launch, from ncu captures of the same
# kernel (dram__bytes_read.sum + dram__bytes_write.sum over the particles of the launch):
#   two-box sand scene: captured at dx = 1/128 (3.7 M particles; the 30 M workload is scaled by
#   the particle count, traffic grows in proportion): 756.4 MB / 3,703,824
#   256-scene batch: captured at full size: 3.569 GB / 15,386,080
#   16 M snow scene: captured at full size: 3.522 GB / 15,988,466
G2P_TRAFFIC_PER_PARTICLE = {"dp_two_boxes_dx256_8ppc": 756.44e6 / 3703824,
                            "dp_two_boxes_dx128_8ppc": 756.44e6 / 3703824,
                            "batch_256_scenes_dx128_8ppc": 3.5687e9 / 15386080,
                            "snow_sphere_slab_dx295_4ppc": 3.5218e9 / 15988466}


def g2p_algorithmic_bytes(n: int, nb: int, plastic: bool) -> int:
    """G2P per launch, the survey's accounting: per particle reads x 12 and F 36 and writes
    x 12, v 12, C 36, F 36 and the stress term 36 (180 B; +8 B for the plastic state read and
    written); per active block reads the 3-channel velocity halo, 12 B per cell of the block
    (halo reads beyond the block come from neighbours that are counted as their own blocks)."""
    return n * (180 + (8 if plastic else 0)) + nb * 512 * 12


def g2p_implementation_bytes(n: int, nb: int, plastic: bool) -> int:
    """What this k_g2p actually moves per launch: per particle reads slot index 4, x|m 16,
    F 36, id 4 (+ plastic 4) and writes x|m 16, v 16 (float4), C 36, A 36, F 36, id 4
    (+ plastic 4), plus the same 12 B per block cell."""
    per_particle = 4 + 16 + 36 + 4 + 16 + 16 + 36 + 36 + 36 + 4 + (8 if plastic else 0)
    return n * per_particle + nb * 512 * 12


def substep_algorithmic_bytes(n: int, nb: int, plastic: bool) -> int:
    """Whole substep, the survey's accounting (unfused P2G / grid / G2P): P2G reads x, v, C,
    m, tau (100 B), G2P reads x, F and writes x, v, C, F, tau (180 B, +8 for plastic state),
    binning 16 B, grid 72 B per active cell."""
    return n * (100 + 180 + (8 if plastic else 0) + 16) + nb * 512 * 72


def learned_leg(args, zs, sc, spec, n, upload_pinned, stream, sptr, ws, plain_ms, mlp=True):
    """The same workload with the learned closure in G2P.  The closure is trained on the GPU
    (this library's forward/backward/Adam kernels) on random trial states plus trial states
    logged from a few plain substeps of this scene, then the scene is re-uploaded, warmed up and
    timed like the plain leg with one particle in 100 audited per substep."""
    import torch

    from zsmpm_b200 import closure as cl
    # trial states from the plain path
    upload_pinned()
    period = max(1, -(-n * 4 // args.train_logged))
    buf = torch.empty((args.train_logged, 6), dtype=torch.float32, device="cuda")
    cl.set_state_log(sc, buf, period)
    sc.run(4, stream=sptr)
    n_log = cl.state_log_count(sc)
    cl.set_state_log(sc, None, 0)
    torch.cuda.synchronize()
    c = cl.Closure(spec.material, spec.volume, device=torch.cuda.current_device())
    t0 = time.perf_counter()
    c.build_dataset(args.train_random, seed=7, logged=buf[:n_log].contiguous())
    schedule = TRAIN_SCHEDULE
    losses = c.fit(schedule)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    # timed leg from the initial state
    upload_pinned()
    cl.attach(sc, c, audit_period=100)
    sc.run(args.warmup, stream=sptr)
    sc.run(0, stream=sptr)  # captures the substep graph the timed run replays, if not yet captured
    sc.status()
    cl.audit(sc, reset=True)
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sc.run(args.steps, stream=sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    sc.status()
    lms = max_over_ranks(e0.elapsed_time(e1), ws)
    a = cl.audit(sc)
    sc.set_stage_timing(True)
    g2p = 0.0
    reps = min(args.steps, 8)
    for _ in range(reps):
        sc.substep(stream=sptr)
        g2p += sc.stage_times()[4]
    sc.set_stage_timing(False)
    sc.status()
    cl.attach(sc, None)
    mlp = mlp_inference_leg(c, n_rows=min(n, 16_777_216)) if mlp else None
    kept = c.dataset_size()[1]
    c.close()
    value = n * args.steps * ws / (lms * 1e-3)
    return {"value": value, "unit": UNIT, "ms_per_step": lms / args.steps,
            "vs_plain": (plain_ms * args.steps) / lms, "g2p_ms": g2p / reps,
            "audit": {"period": 100, **a,
                      "what": "principal Kirchhoff stress of audited particles vs the plain return map; "
                              "rel = |dtau| / (|tau| + 1e-4 (3 lambda + 2 mu)); agg = sqrt(sum|dtau|^2/sum|tau|^2)"},
            "training": {"random_states": args.train_random, "logged_states": n_log,
                         "projected_states_kept": kept,
                         "cohesion": "Pa mapped to the log-strain shift c / (3 lambda + 2 mu)",
                         "epochs": sum(e for e, _, _ in schedule), "seconds": train_s,
                         "first_loss": float(losses[0]), "final_loss": float(losses[-1])},
            "inference": ("exact branch test in G2P; projections inside the training hull queued and run "
                          "through the network by tcgen05.mma (split-BF16 operands: hi + lo pairs, three MMAs "
                          "per step; FP32 accumulators in tensor memory, 128-row tiles), completed by a finish "
                          "kernel"),
            "mlp_inference": mlp}


def batch_learned_leg(args, zs, sc, specs, parts, upload_pinned, stream, sptr, ws, plain_ms):
    """The batch with one Drucker-Prager closure serving its sand scenes (the fixed-corotated
    scenes keep the plain path).  The closure is trained on random states plus trial states
    logged from the first sand scene run alone, then the batch is re-uploaded, warmed up and
    timed like the plain leg with one particle in 100 audited per substep."""
    import torch

    from zsmpm_b200 import closure as cl
    k = next(i for i, sp in enumerate(specs) if sp.material.model == zs.DRUCKER_PRAGER)
    one = zs.Scene(specs[k], parts[k])
    buf = torch.empty((args.train_logged, 6), dtype=torch.float32, device="cuda")
    cl.set_state_log(one, buf, max(1, -(-parts[k].n * 8 // args.train_logged)))
    one.run(8)
    n_log = min(cl.state_log_count(one), args.train_logged)
    cl.set_state_log(one, None, 0)
    one.close()
    c = cl.Closure(specs[k].material, specs[k].volume, device=torch.cuda.current_device())
    t0 = time.perf_counter()
    c.build_dataset(args.train_random, seed=7, logged=buf[:n_log].contiguous())
    schedule = TRAIN_SCHEDULE
    losses = c.fit(schedule)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    upload_pinned()
    cl.attach(sc, c, audit_period=100)
    sc.run(args.warmup, stream=sptr)
    sc.run(0, stream=sptr)  # captures the substep graph the timed run replays, if not yet captured
    sc.status()
    cl.audit(sc, reset=True)
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sc.run(args.steps, stream=sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    sc.status()
    lms = max_over_ranks(e0.elapsed_time(e1), ws)
    a = cl.audit(sc)
    cl.attach(sc, None)
    kept = c.dataset_size()[1]
    c.close()
    n = sum(q.n for q in parts)
    return {"value": n * args.steps * ws / (lms * 1e-3), "unit": UNIT, "ms_per_step": lms / args.steps,
            "vs_plain": (plain_ms * args.steps) / lms,
            "scenes_served": sum(1 for sp in specs if sp.material.model == zs.DRUCKER_PRAGER),
            "audit": {"period": 100, **a},
            "training": {"random_states": args.train_random, "logged_states": n_log,
                         "projected_states_kept": kept,
                         "logged_from": f"scene {k} alone", "seconds": train_s,
                         "first_loss": float(losses[0]), "final_loss": float(losses[-1])}}


def mlp_inference_leg(c, n_rows: int, reps: int = 5) -> dict:
    """The closure's network alone over n_rows feature rows, on the tensor-core paths: the
    mma.sync forward, the tcgen05 forward (tensor-memory accumulators) with BF16 operands, and
    the tcgen05 forward with split-BF16 operands that the substep runs (three MMAs per step).
    17,920 useful FLOP per row (6-64-64-64-6); peak = measured dense BF16 (burst)."""
    import torch
    try:
        peak = float(json.loads(PEAKS.read_text())["bf16_tflops"])
        peak_kind = "measured"
    except Exception:
        peak, peak_kind = 1590.0, "fallback"
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.zeros((n_rows, 6), dtype=torch.float32, device="cuda")
    x[:, :3] = (torch.rand((n_rows, 3), generator=g, device="cuda") - 0.5) * 0.02
    x[:, :3] = torch.sort(x[:, :3], dim=1, descending=True).values
    x[:, 3] = 30.0
    out = {"rows": n_rows, "flop_per_row": 17920, "peak_tflops": peak, "peak_kind": peak_kind}
    for path in ("mma_sync", "tcgen05", "tcgen05_split"):
        c.infer(x, path=path)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            c.infer(x, path=path)
        e1.record()
        torch.cuda.synchronize()
        c.status()
        ms = e0.elapsed_time(e1) / reps
        tf = n_rows * 17920 / (ms * 1e-3) / 1e12
        out[path] = {"ms": ms, "rows_per_s": n_rows / (ms * 1e-3), "tflops": tf, "frac_of_peak": tf / peak}
    return out


def g2p2g_algorithmic_bytes(n: int, nb: int, plastic: bool) -> int:
    """G2P2G per launch: per particle reads slot index 4, x|m 16, F 36 (+ plastic 4); per
    active block reads the 3-component velocity of its 512 nodes (12 B each) and adds the
    3-component force into them (read + write, 24 B each)."""
    return n * (4 + 16 + 36 + (4 if plastic else 0)) + nb * 512 * 36


def implicit_leg(args, zs, sc, spec, upload_pinned, stream, sptr, cpu_sample) -> dict:
    """The implicit system on the same workload: G2P2GTransfer launches over the grid velocity
    of a P2G + grid update (timed with CUDA events on the launching stream), and a conjugate-
    gradient solve of ImplicitMPMSystem for b = m v from x = 0.  cpu_sample: (particles, keys,
    velocity field) for the reference's own G2P2GTransfer under omp_exec, or None."""
    import torch

    from zsmpm_b200.implicit import ConjugateGradient, ImplicitMPMSystem
    upload_pinned()
    sc.run(2, stream=sptr)
    sc.activate_blocks(stream=sptr)
    sc.bin_particles(stream=sptr)
    sc.p2g(stream=sptr)
    sc.grid_update(stream=sptr)
    torch.cuda.synchronize()
    keys, grid = sc.download_grid()
    nb = len(keys)
    n = sc.n
    plastic = spec.material.model != zs.FIXED_COROTATED
    # an implicit step is taken 40x longer than the explicit one, so that the stress term
    # f dt^2 of the system matrix is not lost against the node mass in FP32
    dt_implicit = 40.0 * spec.dt
    system = ImplicitMPMSystem(sc, dt_implicit)
    v = torch.from_numpy(np.ascontiguousarray(grid[:, 1:4, :].transpose(0, 2, 1).reshape(-1))).to("cuda")
    f = system.zeros()
    for _ in range(3):
        system.g2p2g(v, f, stream=stream)
    reps = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        system.g2p2g(v, f, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    sc.status()
    ms = e0.elapsed_time(e1) / reps
    nbytes = g2p2g_algorithmic_bytes(n, nb, plastic)
    peak, peak_kind = hbm_peak()
    m = torch.from_numpy(np.repeat(grid[:, 0, :].reshape(-1), 3)).to("cuda")
    b = m * v
    x = system.zeros()
    converged = ConjugateGradient(max_iters=20).solve(system, x, b, stream=stream)  # also sizes the scratch
    # a fixed iteration count for the per-iteration time (tol 0 never stops early)
    fixed = ConjugateGradient(max_iters=10, tol=0.0)
    x.zero_()
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    iters = fixed.solve(system, x, b, stream=stream)
    c1.record(stream)
    torch.cuda.synchronize()
    cg_ms = c0.elapsed_time(c1)
    out = {"particles": n, "active_blocks": nb, "dt": dt_implicit, "g2p2g_ms": ms, "particles_per_s": n / (ms * 1e-3),
           "g2p2g_roofline": {"bound": "issue (SVD and return map per particle)", "algorithmic_bytes": nbytes,
                              "achieved_gbs": nbytes / (ms * 1e-3) / 1e9, "hbm_peak": peak,
                              "hbm_frac": nbytes / (ms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind},
           "cg": {"b": "m v of the updated grid", "x0": "0", "iterations_to_converge": converged,
                  "timed_iterations": iters, "ms": cg_ms, "ms_per_iteration": cg_ms / max(iters, 1),
                  "what": "CUDA events around zsmpm_implicit_cg with tol 0 and max_iters 10 (the host reads "
                          "the stopping flag every 8 iterations)"}}
    if cpu_sample is not None:
        try:
            from oracle import reference
            q, qkeys, qv, desc = cpu_sample
            threads = os.cpu_count() or 1
            _, secs = reference.g2p2g(spec, q.x, q.F, q.plastic, qkeys, qv, policy=reference.POLICY_OMP,
                                      threads=threads, timeout=900)
            out["cpu_baseline"] = {"value": q.n / secs, "unit": "particles/s", "cores": threads, "kind": "reference",
                                   "sample": f"{desc}; G2P2GTransfer under zs::omp_exec"}
        except Exception as exc:
            out["cpu_baseline"] = {"value": None, "sample": f"failed: {exc}"}
    return out


def implicit_cpu_sample(spec, p, max_particles: int):
    """A z-slab of the workload, its canonical block keys and a smooth velocity field on them."""
    from oracle import reference
    q, desc = cpu_baseline_sample(spec, p, max_particles)
    keys, _slots, _npb, _ts = reference.activate(q.x, spec.dx, max(q.n // 512, 64), cap=1 << 20)
    keys = keys[np.lexsort((keys[:, 2], keys[:, 1], keys[:, 0]))]
    cell = np.arange(512)
    loc = np.stack([cell >> 6, (cell >> 3) & 7, cell & 7], 1)
    pos = (keys[:, None, :].astype(np.int64) * 8 + loc[None]) * spec.dx
    vel = np.stack([np.sin(7 * pos[..., 1]), np.cos(5 * pos[..., 2]), np.sin(3 * pos[..., 0])], -1)
    return q, keys, vel.astype(np.float32).reshape(-1), desc


def cpu_baseline_sample(spec, p, max_particles: int):
    """A spatial slab of the workload (all particles with z below a cut), keeping density."""
    from zsmpm_b200.scenes import Particles
    z = p.x[:, 2]
    if p.n <= max_particles:
        return p, "full scene"
    cut = float(np.quantile(z, max_particles / p.n))
    idx = np.nonzero(z < cut)[0]
    return p.subset(idx), f"slab z < {cut:.4f} of the workload ({len(idx)} particles)"


def reference_cpu_rate(spec, p, parts, steps, warmup, max_particles, threads, timeout, cell=False):
    """Particle-substeps/s of the reference's omp_exec path (oracle/_ref) on a bounded sample:
    a z-slab of a single scene, or the first scenes of a batch (each its own system, as the
    reference advances them one after another) up to max_particles."""
    from oracle import reference
    if parts is None:
        sample, desc = cpu_baseline_sample(spec, p, max_particles)
        jobs = [(spec, sample)]
    else:
        jobs, total = [], 0
        for sp, q in zip(spec, parts):
            if total and total + q.n > max_particles:
                break
            jobs.append((sp, q))
            total += q.n
        desc = f"the first {len(jobs)} of {len(spec)} scenes ({total} particles), run one after another"
    if warmup:
        sp0, q0 = jobs[0]
        reference.run(sp0, q0, warmup, policy=reference.POLICY_OMP, threads=threads, cap_blocks=0, timeout=timeout,
                      cell=cell)
    seconds, work = 0.0, 0
    for sp, q in jobs:
        r = reference.run(sp, q, steps, policy=reference.POLICY_OMP, threads=threads, cap_blocks=0, timeout=timeout,
                          cell=cell)
        seconds += r.seconds
        work += q.n * steps
    return work / seconds, desc, sum(q.n for _, q in jobs)


def run_reference_arm(args, spec, workload, n_full):
    from oracle import reference
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/zsref_cli not built "
                          "(the reference sources were not present when build() ran)"}))
        return 0
    p, parts = generate_workload(spec)
    threads = os.cpu_count() or 1
    # the sample shrinks with the step count so that the run stays within a few minutes
    # (about 1.5e8 particle-substeps at ~3e6 particle-substeps/s on 16 cores)
    sample_particles = max(100_000, min(args.ref_particles, int(1.5e8 // max(args.steps, 1))))
    value, desc, sampled = reference_cpu_rate(spec, p, parts, args.steps, max(args.warmup, 1),
                                              sample_particles, threads, 3600, cell=args.transfer == "cell")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * n_full / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload, "particles": n_full, "parallelism": "omp",
                       "policy": "zs::omp_exec"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": desc},
            "extrapolated_from": sampled,
            "extrapolation": (f"particle-substeps/s measured on {sampled} of the workload's {n_full} particles; "
                              "ms_per_step is the whole workload at that rate") if sampled < n_full else None,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


class Workload:
    """One scene (or batch) resident on the GPU, with pinned host copies of its inputs for the
    end-to-end leg."""

    def __init__(self, zs, spec, p, parts, local, stream, transfer: str = "apic"):
        import torch
        self.zs, self.spec, self.p, self.parts = zs, spec, p, parts
        self.n = p.n
        self.stream, self.sptr = stream, stream.cuda_stream
        self.specs = spec if isinstance(spec, list) else [spec]
        self.plastic = any(sp.material.model != zs.FIXED_COROTATED for sp in self.specs)
        self.pinned = {k: torch.from_numpy(getattr(p, k)).pin_memory() for k in ("m", "x", "v", "C", "F", "plastic")}
        self.out_x = torch.empty((self.n, 3), dtype=torch.float32).pin_memory()
        self.out_v = torch.empty((self.n, 3), dtype=torch.float32).pin_memory()
        self.h2d_bytes = sum(t.numel() * 4 for t in self.pinned.values())
        self.d2h_bytes = (self.out_x.numel() + self.out_v.numel()) * 4 + 4
        self.lib = zs._abi.lib()
        if parts is None:
            self.sc = zs.Scene(spec, device=local, transfer=transfer)
        else:
            from zsmpm_b200 import batch
            self.sc = batch.Batch(spec, device=local)
            self.counts = (C.c_int64 * len(parts))(*[q.n for q in parts])

    def upload_pinned(self):
        zs = self.zs
        arrs = zs._abi.ParticleArrays(**{k: C.c_void_p(t.data_ptr()) for k, t in self.pinned.items()})
        if self.parts is None:
            zs._abi.check(self.lib.zsmpm_scene_upload(self.sc.handle, C.byref(arrs), self.n, 0,
                                                      C.c_void_p(self.sptr)), "upload")
        else:
            zs._abi.check(self.lib.zsmpm_batch_upload(self.sc.handle, C.byref(arrs), self.counts, 0,
                                                      C.c_void_p(self.sptr)), "upload")
        self.sc.n = self.n

    def download_xv(self):
        zs = self.zs
        arrs = zs._abi.ParticleArrays(x=C.c_void_p(self.out_x.data_ptr()), v=C.c_void_p(self.out_v.data_ptr()))
        zs._abi.check(self.lib.zsmpm_scene_download(self.sc.handle, C.byref(arrs), 0, C.c_void_p(self.sptr)),
                      "download")

    def close(self):
        self.sc.close()


def plain_leg(args, w, ws, local, with_e2e=True):
    """Device-resident throughput over args.steps substeps (CUDA events on the launching stream,
    clocks sampled inside the timed region), then a per-stage timing pass, then (optionally)
    the end-to-end leg: pinned upload, args.steps substeps, download of x and v, status read."""
    import torch
    sc, stream, sptr, n = w.sc, w.stream, w.sptr, w.n
    tuning = None
    if not args.no_autotune:
        w.upload_pinned()
        tuning = sc.autotune(trials=2, stream=sptr)
    w.upload_pinned()
    torch.cuda.synchronize()
    sc.run(args.warmup, stream=sptr)
    sc.run(0, stream=sptr)  # captures the substep graph the timed run replays, if not yet captured
    sc.status()
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        clk.mark_start()
        e0.record(stream)
        sc.run(args.steps, stream=sptr)
        e1.record(stream)
        torch.cuda.synchronize()
        clk.mark_end()
    sc.status()
    ms = max_over_ranks(e0.elapsed_time(e1), ws)
    barrier(ws)
    nb = sc.num_blocks()
    # per-stage timing pass (events between the stages of single substeps)
    sc.set_stage_timing(True)
    stage = np.zeros(5)
    reps = min(args.steps, 8)
    for _ in range(reps):
        sc.substep(stream=sptr)
        stage += np.array(sc.stage_times())
    sc.set_stage_timing(False)
    stage /= reps
    sc.status()
    peak, peak_kind = hbm_peak()
    g2p_bytes = g2p_algorithmic_bytes(n, nb, w.plastic)
    g2p_gbs = g2p_bytes / (stage[4] * 1e-3) / 1e9
    total_bytes = substep_algorithmic_bytes(n, nb, w.plastic)
    out = {
        "value": n * args.steps * ws / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / args.steps,
        "particles": n, "active_blocks": nb, "launch_shapes": tuning, "clocks": clk.summary(),
        "stage_ms": {"activate": stage[0], "bin": stage[1], "p2g": stage[2], "grid_update": stage[3],
                     "g2p": stage[4]},
        "g2p_roofline": {"bound": "hbm", "kernel": "k_g2p", "achieved": g2p_gbs, "peak": peak, "unit": "GB/s",
                         "frac": g2p_gbs / peak, "peak_kind": f"{peak_kind} copy bandwidth",
                         "algorithmic_bytes_per_launch": g2p_bytes,
                         "implementation_bytes_per_launch": g2p_implementation_bytes(n, nb, w.plastic),
                         "launch_ms": stage[4]},
        "substep_roofline": {"algorithmic_bytes_per_substep": total_bytes,
                             "achieved_gbs": total_bytes / (ms / args.steps * 1e-3) / 1e9,
                             "frac": total_bytes / (ms / args.steps * 1e-3) / 1e9 / peak,
                             "peak": peak, "peak_kind": f"{peak_kind} copy bandwidth"},
        "gpu_launches": sc.kernels_per_substep() * args.steps,
    }
    if with_e2e:
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        w.upload_pinned()
        sc.run(args.steps, stream=sptr)
        w.download_xv()
        f1.record(stream)
        sc.status()  # device -> host status word
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(f0.elapsed_time(f1), ws)
        out["e2e"] = {"value": n * args.steps * ws / (e2e_ms * 1e-3), "unit": UNIT,
                      "h2d_bytes_per_step": w.h2d_bytes / args.steps, "d2h_bytes_per_step": w.d2h_bytes / args.steps,
                      "wall_s": time.perf_counter() - t0,
                      "what": "upload from pinned host, K substeps, download x and v, status read"}
    return out


def cpu_baselines(args, spec, p, parts):
    """The compiled reference's zs::omp_exec path on a bounded sample, on all host cores and at
    zpc's default thread count (hardware_concurrency - 1, omp/execution/ExecutionPolicy.hpp:1242)."""
    from oracle import reference
    if not reference.available():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/zsref_cli not built"}
    try:
        threads = os.cpu_count() or 1
        cell = args.transfer == "cell"
        rate, desc, sampled = reference_cpu_rate(spec, p, parts, args.ref_steps, 0, args.ref_particles, threads, 900,
                                                 cell=cell)
        out = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": f"{desc}, {args.ref_steps} substeps, zs::omp_exec", "extrapolated_from": sampled}
        # zpc's own default: omp_exec() with hardware_concurrency - 1 threads (threads <= 0 in the driver)
        rate_d, _, _ = reference_cpu_rate(spec, p, parts, args.ref_steps, 0, args.ref_particles, 0, 900, cell=cell)
        out["zpc_default_threads"] = {"value": rate_d, "unit": UNIT, "cores": max(threads - 1, 1),
                                      "what": "zs::omp_exec() default, hardware_concurrency - 1 threads"}
        return out
    except Exception as exc:  # report, never fail the GPU line
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {exc}"}


def extra_leg(args, name, ws, local, stream, learned: bool):
    """Another workload of the survey's configurations, measured the same way as the main one
    (plain device-resident throughput, stage times and rooflines; learned closure if asked)."""
    import zsmpm_b200 as zs
    spec, workload = scene_for(name)
    p, parts = generate_workload(spec)
    w = Workload(zs, spec, p, parts, local, stream)
    try:
        out = {"workload": workload, **plain_leg(args, w, ws, local, with_e2e=False)}
        if workload in G2P_TRAFFIC_PER_PARTICLE and "g2p_roofline" in out:
            out["g2p_roofline"]["traffic"] = G2P_TRAFFIC_PER_PARTICLE[workload] * w.n
        if learned:
            if parts is None:
                out["learned"] = learned_leg(args, zs, w.sc, spec, w.n, w.upload_pinned, stream, w.sptr, ws,
                                             out["ms_per_step"], mlp=False)
            else:
                out["learned"] = batch_learned_leg(args, zs, w.sc, spec, parts, w.upload_pinned, stream, w.sptr,
                                                   ws, out["ms_per_step"])
    finally:
        w.close()
    return out


def cell_leg(args, ws, local, stream, cpu: bool) -> dict:
    """The cell-centric transfer pair (P2C2GTransfer / G2C2PTransfer) against the APIC pair on
    the benchmark's two-box geometry in fixed corotated (the pair has no plasticity branch):
    30,089,900 particles, each pair measured like the main leg, and the reference's own cell
    path under zs::omp_exec on a bounded slab."""
    import zsmpm_b200 as zs
    from zsmpm_b200 import scenes
    spec, _ = scene_for("fc_boxes")
    p = scenes.generate(spec)
    w = Workload(zs, spec, p, None, local, stream)
    try:
        apic = plain_leg(args, w, ws, local, with_e2e=False)
        w.sc.set_transfer("cell")
        cell = plain_leg(args, w, ws, local, with_e2e=False)
    finally:
        w.close()
    peak, peak_kind = hbm_peak()
    n, nb = cell["particles"], cell["active_blocks"]
    # P2C2G's algorithmic bytes: x|m 16, v 12 and the affine term 36 per particle read once, and
    # the block's 512 nodes x 4 channels written
    p2c2g_bytes = n * 64 + nb * 512 * 16
    p2c2g_ms = cell["stage_ms"]["p2g"]
    out = {"workload": "fc_two_boxes_dx256_8ppc", "particles": n, "material": "fixed_corotated",
           "apic": {k: apic[k] for k in ("value", "ms_per_step", "stage_ms", "launch_shapes", "clocks")},
           "cell": {k: cell[k] for k in ("value", "ms_per_step", "stage_ms", "launch_shapes", "clocks",
                                         "gpu_launches")},
           "cell_vs_apic": cell["value"] / apic["value"],
           "p2c2g_roofline": {"kernel": "k_p2g (cell variant: P2C2G)", "bound": "hbm",
                              "algorithmic_bytes_per_launch": p2c2g_bytes,
                              "achieved": p2c2g_bytes / (p2c2g_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                              "frac": p2c2g_bytes / (p2c2g_ms * 1e-3) / 1e9 / peak,
                              "peak_kind": f"{peak_kind} copy bandwidth", "launch_ms": p2c2g_ms},
           "g2c2p_roofline": {**cell["g2p_roofline"], "kernel": "k_g2p (cell variant: G2C2P)"}}
    if cpu:
        try:
            from oracle import reference
            if reference.available():
                threads = os.cpu_count() or 1
                q, desc = cpu_baseline_sample(spec, p, min(args.ref_particles, 500_000))
                r = reference.run(spec, q, args.ref_steps, policy=reference.POLICY_OMP, threads=threads,
                                  cap_blocks=0, cell=True, timeout=900)
                out["cpu_baseline"] = {"value": q.n * args.ref_steps / r.seconds, "unit": UNIT, "cores": threads,
                                       "kind": "reference",
                                       "sample": f"{desc}, {args.ref_steps} substeps of the cell pair, zs::omp_exec"}
        except Exception as exc:
            out["cpu_baseline"] = {"value": None, "sample": f"failed: {exc}"}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scene", default="dp", choices=["dp", "dp128", "fc", "fc_boxes", "fc_boxes128", "snow16m",
                                                      "batch256"])
    ap.add_argument("--transfer", default="apic", choices=["apic", "cell"],
                    help="the transfer pair of the main leg: P2G / G2P, or the cell-centric P2C2G / G2C2P "
                         "(fixed-corotated scenes)")
    ap.add_argument("--ref-particles", type=int, default=1_500_000)
    ap.add_argument("--ref-steps", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-closure legs")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes")
    ap.add_argument("--no-implicit", action="store_true", help="skip the implicit-system leg")
    ap.add_argument("--no-extra", action="store_true",
                    help="measure only --scene (by default the sand scene run also measures the 16 M snow "
                         "scene, plain and learned, the 256-scene batch and the cell-centric transfer pair)")
    # 20 M training states in all, as the learned-closure configuration states: random trial
    # states plus states logged from the plain path
    ap.add_argument("--train-random", type=int, default=16_000_000)
    ap.add_argument("--train-logged", type=int, default=4_000_000)
    args = ap.parse_args(argv)

    spec, workload = scene_for(args.scene)
    from zsmpm_b200 import scenes
    if args.impl == "reference":
        n_full = (sum(scenes.count_particles(sp) for sp in spec) if isinstance(spec, list)
                  else scenes.count_particles(spec))
        return run_reference_arm(args, spec, workload, n_full)

    from zsmpm_b200 import replicas
    ws, rank, local = replicas.init("nccl")
    import torch

    import zsmpm_b200 as zs
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    p, parts = generate_workload(spec)
    w = Workload(zs, spec, p, parts, local, stream, transfer=args.transfer)
    n = w.n
    specs = w.specs
    main_leg = plain_leg(args, w, ws, local, with_e2e=True)
    ms = main_leg["ms_per_step"] * args.steps

    # ---------------------------------------------------------------- learned-closure leg
    learned = None
    if args.transfer != "apic":
        pass  # the learned closure and the implicit system work with the APIC pair
    elif w.plastic and parts is None and not args.no_learned:
        learned = learned_leg(args, zs, w.sc, spec, n, w.upload_pinned, stream, w.sptr, ws, ms / args.steps)
    elif w.plastic and not args.no_learned:
        learned = batch_learned_leg(args, zs, w.sc, specs, parts, w.upload_pinned, stream, w.sptr, ws,
                                    ms / args.steps)

    # ---------------------------------------------------------------- implicit-system leg
    implicit = None
    if parts is None and not args.no_implicit and args.transfer == "apic":
        sample = None
        if rank == 0 and ws == 1 and not args.no_cpu_baseline:
            try:
                from oracle import reference
                if reference.available():
                    sample = implicit_cpu_sample(spec, p, args.ref_particles)
            except Exception:
                sample = None
        implicit = implicit_leg(args, zs, w.sc, spec, w.upload_pinned, stream, w.sptr, sample)
    w.close()
    del w

    # ---------------------------------------------------------------- the other stated workloads
    legs = {}
    if args.scene == "dp" and not args.no_extra:
        legs["snow16m"] = extra_leg(args, "snow16m", ws, local, stream, learned=not args.no_learned)
        legs["batch256"] = extra_leg(args, "batch256", ws, local, stream, learned=False)
        legs["cell_transfer"] = cell_leg(args, ws, local, stream,
                                         cpu=rank == 0 and ws == 1 and not args.no_cpu_baseline)

    # ---------------------------------------------------------------- CPU baseline (rank 0, N=1)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baselines(args, spec, p, parts)

    if rank == 0:
        g2p = main_leg["g2p_roofline"]
        line = {
            "metric": METRIC, "value": main_leg["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main_leg["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload, "particles": n, "active_blocks": main_leg["active_blocks"],
                       "scenes": len(specs), "dx": specs[0].dx, "ppc": specs[0].ppc, "dt": specs[0].dt,
                       "material": "mixed fixed_corotated / drucker_prager" if len(specs) > 1 else
                       ("drucker_prager" if specs[0].material.model == zs.DRUCKER_PRAGER else
                        ("snow" if specs[0].material.model == zs.SNOW else "fixed_corotated")),
                       "closure": "plain", "transfer": args.transfer, "parallelism": f"replicas{ws}",
                       "launch_shapes": main_leg["launch_shapes"],
                       "l2": "inputs larger than L2 (particle state 2+ GB per workload)",
                       "substep_graph": "CUDA graph of 4 substeps"},
            "roofline": {**g2p,
                         "traffic": (G2P_TRAFFIC_PER_PARTICLE[workload] * n if workload in G2P_TRAFFIC_PER_PARTICLE
                                     else None),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per particle of a "
                                           "k_g2p launch (profiles/), times this launch's particles"},
            "stage_ms": main_leg["stage_ms"],
            "substep_roofline": main_leg["substep_roofline"],
            "e2e": main_leg["e2e"],
            "gpu_launches": main_leg["gpu_launches"],
            "clocks": main_leg["clocks"],
            "cpu_baseline": cpu,
            "learned": learned,
            "implicit": implicit,
            "legs": legs,
        }
        print(json.dumps(line))
    replicas.finish()
    return 0


if __name__ == "__main__":
    sys.exit(main())
