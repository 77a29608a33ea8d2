"""Parity of the CUDA path at the stated workload configurations, against the reference's own
CPU path (oracle/_ref/zsref_cli, compiled from the zpc sources) with every error also stated
against the FP64 restatement.

- The fixed-corotated cube (140,608 particles, dx = 1/128, sticky walls, dt = 1e-4) for its
  full 100 substeps, against the reference under seq_exec.
- The two-box Drucker-Prager sand scene at dx = 1/128 (3.76 M particles, slip walls,
  dt = 5e-5) for 5 substeps, against the reference under omp_exec on all host cores.
- A snow column of the 16 M-particle snow scene with the sphere started in contact with the
  slab, so that the Stomakhin clamp projects a share of the particles: the plain GPU path and
  the learned closure against the FP64 restatement (the reference has no snow pipeline).

Both reference comparisons use the reference's own ordering (the return map on a copy of F
inside P2G, F not projected); the GPU keeps logJp one projection ahead, as the header states,
so the reference's logJp is advanced by one projection before it is compared.  The tolerance
of the survey's target, 1e-5 relative L2, applies to x, v, F and the grid's mass and
momentum.
"""
import os
import threading

import numpy as np
import pytest

from helpers import aligned_grids, grid_mass_momentum, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2 against the reference's CPU path


class _Bg(threading.Thread):
    """Runs a CPU oracle call beside the GPU work (ctypes and subprocess release the GIL)."""

    def __init__(self, fn, *a, **k):
        super().__init__(daemon=True)
        self.fn, self.a, self.k, self.out, self.err = fn, a, k, None, None
        self.start()

    def run(self):
        try:
            self.out = self.fn(*self.a, **self.k)
        except BaseException as e:  # noqa: BLE001 -- re-raised in the test thread
            self.err = e

    def result(self):
        self.join()
        if self.err is not None:
            raise self.err
        return self.out


def _gpu_run(zs, spec, p, steps):
    with zs.Scene(spec, p) as sc:
        sc.run(steps)
        sc.status()
        out = sc.download()
        keys, grid = sc.download_grid()
    return out, keys, grid


def _errors(g, gk, gg, base, x0):
    """Relative L2 errors of a GPU result against another result (reference or oracle)."""
    eye = np.eye(3).reshape(9)
    mg, pg = grid_mass_momentum(gk, gg)
    mb, pb = grid_mass_momentum(base.keys, base.grid)
    _, _, diff = aligned_grids(gk, gg, base.keys, base.grid)
    return {
        "x": rel_l2(g.x, base.x), "disp": rel_l2(g.x - x0, base.x - x0), "v": rel_l2(g.v, base.v),
        "F": rel_l2(g.F, base.F), "F-I": rel_l2(g.F - eye, base.F - eye), "C": rel_l2(g.C, base.C),
        "mass": abs(mg - mb) / mb, "momentum": float(np.linalg.norm(pg - pb) / np.linalg.norm(pb)),
        "blocks_differ": len(diff),
    }


def _fmt(e):
    return " ".join(f"{k} {v:.2e}" if isinstance(v, float) else f"{k} {v}" for k, v in e.items())


def test_fc_cube_100_substeps_vs_reference(zs, gpu, reference_cli):
    """The fixed-corotated cube exactly as configured: 140,608 particles, 100 substeps."""
    from oracle import restated
    from zsmpm_b200 import scenes
    spec = scenes.config1()
    spec.material.plasticity_mode = zs.PLASTICITY_REFERENCE
    p = scenes.generate(spec)
    assert p.n == 140_608
    steps = spec.substeps
    assert steps == 100
    ref_job = _Bg(reference_cli.run, spec, p, steps, policy=reference_cli.POLICY_SEQ, timeout=1200.0)
    o64_job = _Bg(restated.run, spec, p, steps, "f64", mode=1)
    g, gk, gg = _gpu_run(zs, spec, p, steps)
    ref = ref_job.result()
    o64 = o64_job.result()
    assert ref.status == 0
    e_ref = _errors(g, gk, gg, ref, p.x)
    e_gpu64 = _errors(g, gk, gg, o64, p.x)
    e_cpu64 = {k: rel_l2(getattr(ref, k), getattr(o64, k)) for k in ("x", "v", "F")}
    print(f"\nfc cube {p.n} particles, {steps} substeps (seq_exec reference):\n"
          f"  GPU vs reference CPU: {_fmt(e_ref)}\n  GPU vs FP64: {_fmt(e_gpu64)}\n"
          f"  reference CPU vs FP64: {_fmt(e_cpu64)}")
    dx_count = int(np.count_nonzero(g.x != ref.x))
    print(f"  x values that differ from the reference: {dx_count} of {g.x.size}, "
          f"max |dx| {float(np.abs(g.x - ref.x).max()):.2e}")
    assert e_ref["blocks_differ"] == 0
    for k in ("x", "v", "F", "mass", "momentum"):
        assert e_ref[k] < TOL, (k, e_ref[k])
    # The cube falls freely (it meets no wall in 0.01 s), so F stays I up to FP32 rounding and
    # the velocity's deviation from the uniform fall is the rounding noise of the stress of a
    # near-identity F, summed over 100 substeps.  Both FP32 paths stay within the same bound
    # of the FP64 run (the GPU's noise measured 5.2e-6 against the CPU's 1.3e-6).
    assert e_gpu64["v"] < TOL and e_cpu64["v"] < TOL
    assert e_gpu64["x"] < max(2 * e_cpu64["x"], 1e-7)


def test_sand_two_boxes_dx128_vs_reference_omp(zs, gpu, reference_cli):
    """The two-box sand scene at dx = 1/128 (3.76 M particles), 5 substeps, against the
    reference under omp_exec on all host cores."""
    from oracle import restated
    from zsmpm_b200 import scenes
    spec = scenes.config2(dx=1 / 128)
    spec.material.plasticity_mode = zs.PLASTICITY_REFERENCE
    p = scenes.generate(spec)
    assert 3_700_000 < p.n < 3_800_000
    steps = 5
    threads = os.cpu_count() or 1
    ref_job = _Bg(reference_cli.run, spec, p, steps, policy=reference_cli.POLICY_OMP, threads=threads,
                  cap_blocks=1 << 16, timeout=1800.0)
    o64_job = _Bg(restated.run, spec, p, steps, "f64", mode=1)
    g, gk, gg = _gpu_run(zs, spec, p, steps)
    ref = ref_job.result()
    o64 = o64_job.result()
    assert ref.status == 0
    e_ref = _errors(g, gk, gg, ref, p.x)
    e_gpu64 = _errors(g, gk, gg, o64, p.x)
    e_cpu64 = {k: rel_l2(getattr(ref, k), getattr(o64, k)) for k in ("x", "v", "F")}
    e_cpu64["disp"] = rel_l2(ref.x - p.x, o64.x - p.x)
    # the GPU keeps logJp one projection ahead: advance the reference's by one projection
    _, _, lj = restated.stress(spec, ref.F, ref.logJp, mode=1)
    e_lj = float(np.max(np.abs(g.plastic - lj)))
    print(f"\nsand two boxes {p.n} particles, {steps} substeps (omp_exec reference, {threads} threads):\n"
          f"  GPU vs reference CPU: {_fmt(e_ref)} logJp max abs {e_lj:.2e}\n"
          f"  GPU vs FP64: {_fmt(e_gpu64)}\n  reference CPU vs FP64: {_fmt(e_cpu64)}")
    dx_count = int(np.count_nonzero(g.x != ref.x))
    print(f"  x values that differ from the reference: {dx_count} of {g.x.size}, "
          f"max |dx| {float(np.abs(g.x - ref.x).max()):.2e}")
    assert e_ref["blocks_differ"] == 0
    for k in ("x", "v", "F", "mass", "momentum"):
        assert e_ref[k] < TOL, (k, e_ref[k])
    assert e_lj < 1e-4
    assert e_gpu64["v"] < max(2 * e_cpu64["v"], 1e-6)
    assert e_gpu64["disp"] < max(2 * e_cpu64["disp"], 1e-6)


def _snow_contact_column():
    """A column (x in [0.42, 0.58), z in [0.44, 0.56)) of the 16 M-particle snow scene with the
    sphere lowered to touch the slab: the sphere's lowest particles sit half a cell above the
    slab's top face, falling at 3 m/s."""
    from zsmpm_b200 import scenes
    spec = scenes.config5_16m()
    slab, sphere = spec.shapes
    r = sphere.hi[0]
    sphere.lo = (sphere.lo[0], slab.hi[1] + r + 0.5 * spec.dx, sphere.lo[2])
    p = scenes.generate(spec)
    x = p.x
    idx = np.nonzero((x[:, 0] >= 0.42) & (x[:, 0] < 0.58) & (x[:, 2] >= 0.44) & (x[:, 2] < 0.56))[0]
    return spec, p.subset(idx)


def test_snow_with_active_plasticity_plain_and_learned_vs_fp64(zs, gpu):
    import torch

    from oracle import restated
    from zsmpm_b200 import closure as cl
    spec, q = _snow_contact_column()
    assert 800_000 < q.n < 1_300_000
    # 24 substeps: the sphere has sunk 0.4 cells into the slab and the compression front has
    # run about 2.5 cells into both; in 12 substeps the clamp had engaged on 0.3% of the column
    steps = 24
    o64_job = _Bg(restated.run, spec, q, steps, "f64")
    o32_job = _Bg(restated.run, spec, q, steps, "f32")
    with zs.Scene(spec, q) as sc:
        sc.run(steps)
        sc.status()
        g = sc.download()
        # learned closure: random snow states plus states logged from plain substeps of this column
        sc.upload(q)
        buf = torch.empty((400_000, 6), dtype=torch.float32, device=gpu)
        cl.set_state_log(sc, buf, max(1, q.n * steps // 400_000))
        sc.run(steps)
        n_log = cl.state_log_count(sc)
        cl.set_state_log(sc, None, 0)
        c = cl.Closure(spec.material, spec.volume)
        c.build_dataset(1_000_000, seed=5, logged=buf[:min(n_log, 400_000)].contiguous())
        c.fit(cl.SCHEDULE_LONG)
        sc.upload(q)
        cl.attach(sc, c, audit_period=20)
        sc.run(steps)
        sc.status()
        a = cl.audit(sc)
        lrn = sc.download()
        cl.attach(sc, None)
        c.close()
    o64 = o64_job.result()
    o32 = o32_job.result()
    # the clamp engaged: Jp moved off 1 for a share of the particles, in every path
    projected = float(np.mean(np.abs(g.plastic - 1.0) > 1e-6))
    projected64 = float(np.mean(np.abs(o64.plastic - 1.0) > 1e-6))
    err = {"gpu_disp": rel_l2(g.x - q.x, o64.x - q.x), "gpu_v": rel_l2(g.v, o64.v),
           "gpu_F": rel_l2(g.F, o64.F), "gpu_Jp": rel_l2(g.plastic, o64.plastic),
           "cpu32_disp": rel_l2(o32.x - q.x, o64.x - q.x), "cpu32_v": rel_l2(o32.v, o64.v),
           "cpu32_F": rel_l2(o32.F, o64.F), "cpu32_Jp": rel_l2(o32.plastic, o64.plastic),
           "learned_disp": rel_l2(lrn.x - q.x, o64.x - q.x), "learned_v": rel_l2(lrn.v, o64.v),
           "learned_Jp": rel_l2(lrn.plastic, o64.plastic)}
    print(f"\nsnow column in contact, {q.n} particles, {steps} substeps: projected share GPU {projected:.3f} "
          f"FP64 {projected64:.3f}; relative L2 against FP64: " + _fmt(err)
          + f"; learned audit mean {a['mean_rel_error']:.2e} max {a['max_rel_error']:.2e} "
            f"agg {a['agg_rel_error']:.2e} fallbacks {a['fallbacks']}")
    assert projected > 0.003 and projected64 > 0.003
    # the plain GPU path is as close to FP64 as the FP32 CPU restatement (within 2x)
    for k in ("disp", "v", "F", "Jp"):
        assert err["gpu_" + k] <= max(2 * err["cpu32_" + k], 1e-6), k
    # the network projected the states outside the clamp box, and the learned run stays near
    # the plain path
    assert a["network_updates"] > 0 and a["audited"] > 0
    assert err["learned_v"] < 1e-2
    # the snow stress is steep in the projected strain (a log-strain error d moves it by about
    # d / theta_c, and the hardening exp(xi (1 - Jp)) multiplies the Jp error by xi = 10):
    # measured aggregate 2.9e-2 with the long schedule
    assert a["agg_rel_error"] < 0.1
