"""The 16 M snow scene (a sphere of radius 0.2 falling onto a slab, dx = 1/295, 4 particles per
cell, fixed corotated with Stomakhin snow plasticity): the plain GPU path and the learned
closure, retrained on snow states, both against the FP64 oracle on a subset of about one
million particles (a column through the sphere and the slab)."""
import numpy as np
import pytest

from helpers import rel_l2

STEPS = 10


def _subset():
    from zsmpm_b200 import scenes
    spec = scenes.config5_16m()
    p = scenes.generate(spec)
    x = p.x
    idx = np.nonzero((x[:, 0] >= 0.42) & (x[:, 0] < 0.58) & (x[:, 2] >= 0.44) & (x[:, 2] < 0.56))[0]
    return spec, p.subset(idx), p.n


@pytest.mark.gpu
def test_snow_subset_plain_and_learned_against_fp64(zs, gpu):
    import torch

    from oracle import restated
    from zsmpm_b200 import closure as cl
    spec, q, n_full = _subset()
    assert n_full > 15_900_000 and 900_000 < q.n < 1_200_000
    o64 = restated.run(spec, q, STEPS, "f64")
    o32 = restated.run(spec, q, STEPS, "f32")
    with zs.Scene(spec, q) as sc:
        sc.run(STEPS)
        sc.status()
        g = sc.download()
        # learned closure: random snow states plus states logged from plain substeps of this subset
        sc.upload(q)
        buf = torch.empty((200_000, 6), dtype=torch.float32, device=gpu)
        cl.set_state_log(sc, buf, max(1, q.n * 4 // 200_000))
        sc.run(4)
        n_log = cl.state_log_count(sc)
        cl.set_state_log(sc, None, 0)
        c = cl.Closure(spec.material, spec.volume)
        c.build_dataset(500_000, seed=3, logged=buf[:min(n_log, 200_000)].contiguous())
        c.fit()
        sc.upload(q)
        cl.attach(sc, c, audit_period=100)
        sc.run(STEPS)
        sc.status()
        a = cl.audit(sc)
        lrn = sc.download()
        cl.attach(sc, None)
        c.close()
    err = {"gpu_x": rel_l2(g.x - q.x, o64.x - q.x), "gpu_v": rel_l2(g.v, o64.v),
           "cpu32_x": rel_l2(o32.x - q.x, o64.x - q.x), "cpu32_v": rel_l2(o32.v, o64.v),
           "learned_x": rel_l2(lrn.x - q.x, o64.x - q.x), "learned_v": rel_l2(lrn.v, o64.v)}
    print(f"\nsnow subset {q.n} of {n_full} particles, {STEPS} substeps, relative L2 against FP64: "
          + ", ".join(f"{k} {v:.2e}" for k, v in err.items())
          + f"; learned audit {a}")
    # the plain GPU path is as close to FP64 as the FP32 CPU restatement (within 2x)
    assert err["gpu_v"] <= max(2 * err["cpu32_v"], 1e-6)
    assert err["gpu_x"] <= max(2 * err["cpu32_x"], 1e-6)
    assert rel_l2(g.v, o32.v) < 5e-5
    # In these 10 substeps the sphere has not reached the slab: every trial state stays inside
    # the clamp box, the exact branch test keeps the strain, and the network never runs (the
    # snow column started in contact, tests/test_config_parity.py, exercises it).
    assert a["network_updates"] == 0 and a["updates"] == q.n * STEPS
    assert err["learned_v"] <= max(2 * err["cpu32_v"], 1e-6)
