"""The learned return-mapping closure: its CUDA forward/backward kernels against the float64
NumPy oracle (oracle/mlp.py), its training targets against the restated return map, training,
BF16 tensor-core inference, the hull fallback and the per-substep audit inside G2P, and what the
trained network gains over leaving the return map out."""
import dataclasses

import numpy as np
import pytest

from oracle import mlp

DP, SNOW = 1, 2


# ---------------------------------------------------------------- CPU: the oracle itself
def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(scale=0.3, size=mlp.N_PARAMS)
    x = rng.normal(size=(16, 6))
    y = rng.normal(size=(16, 6))
    loss, g = mlp.loss_and_grad(p, x, y)
    assert g.shape == (mlp.N_PARAMS,)
    idx = np.concatenate([rng.choice(mlp.N_PARAMS, 60, replace=False),
                          [0, 383, 384, 447, 448, 4543, 4544, 8767, 8768, 9151, 9152, 9157]])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (mlp.loss_and_grad(p + e, x, y)[0] - mlp.loss_and_grad(p - e, x, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])
    assert np.isclose(loss, np.mean((mlp.forward(p, x) - y) ** 2))


def random_rows(model, n, seed, E, nu):
    """Trial states drawn like the library's training set (log singular values sorted
    descending, in [log 0.5, log 2] for Drucker-Prager and [-0.1, 0.05] for snow, plus the
    model's three features)."""
    rng = np.random.default_rng(seed)
    l = -np.sort(-rng.uniform(np.log(0.5), np.log(2.0), size=(n, 3)), axis=1)
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    if model == DP:
        f = np.stack([rng.uniform(20, 45, n),
                      np.where(rng.uniform(size=n) < 0.25, 0.0, rng.uniform(0, 100, n) / (3 * lam + 2 * mu)),
                      np.where(rng.uniform(size=n) < 0.5, 0.0, rng.uniform(0, 0.2, n))], 1)
    else:
        l = -np.sort(-rng.uniform(-0.1, 0.05, size=(n, 3)), axis=1)
        f = np.stack([rng.uniform(0.015, 0.035, n), rng.uniform(0.005, 0.01, n), rng.uniform(-0.15, 0.15, n)], 1)
    return np.ascontiguousarray(np.concatenate([l, f], 1), dtype=np.float32)


def projected(model, rows, E, nu):
    """Rows whose trial state the plain return map projects: Drucker-Prager onto the cone
    (tr < 0 and dgamma > 0, compute_stress_sand), snow when a singular value leaves
    [1 - theta_c, 1 + theta_s].  The closure's network replaces that branch only."""
    r = rows.astype(np.float64)
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    if model == DP:
        eps = r[:, :3] - r[:, 4:5]
        tr = eps.sum(1) + r[:, 5]
        eh = eps - tr[:, None] / 3
        s = np.sin(np.radians(r[:, 3]))
        ys = np.sqrt(2 / 3) * 2 * s / (3 - s)
        dg = np.linalg.norm(eh, axis=1) + (3 * lam + 2 * mu) / (2 * mu) * tr * ys
        return (tr < 0) & (dg > 0)
    S = np.exp(r[:, :3])
    return np.any((S < 1 - r[:, 3:4]) | (S > 1 + r[:, 4:5]), axis=1)


def oracle_targets(spec, rows):
    """(D, tau) of the restated return map (float64) on F = diag(exp(l))."""
    from oracle import restated
    model = spec.material.model
    out = np.zeros((len(rows), 6))
    for i, r in enumerate(rows.astype(np.float64)):
        if model == DP:
            mat = dataclasses.replace(spec.material, friction_deg=float(r[3]), cohesion=float(r[4]))
            pl = np.array([r[5]])
        else:
            mat = dataclasses.replace(spec.material, theta_c=float(r[3]), theta_s=float(r[4]))
            pl = np.array([np.exp(r[5])])
        s = dataclasses.replace(spec, material=mat)
        F = np.diag(np.exp(r[:3])).T.reshape(1, 9)
        tau, Fp, _ = restated.stress(s, F, pl, precision="f64")
        Fp = Fp.reshape(3, 3).T
        tau = tau.reshape(3, 3).T / spec.volume
        out[i, :3] = np.log(np.abs(np.diag(Fp))) - r[:3]
        out[i, 3:] = np.diag(tau)
    return out


def _spec(model):
    from zsmpm_b200 import scenes
    return scenes.small_scene(model=model)


def _closure(zs, model, n_random=20000, seed=1):
    from zsmpm_b200.closure import Closure
    spec = _spec(model)
    c = Closure(spec.material, spec.volume)
    c.build_dataset(n_random, seed=seed)
    return spec, c


def _mu_lam(mat):
    return mat.E / (2 * (1 + mat.nu)), mat.E * mat.nu / ((1 + mat.nu) * (1 - 2 * mat.nu))


def _kappa(mat):
    mu, lam = _mu_lam(mat)
    return 3 * lam + 2 * mu


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("model", [DP, SNOW])
def test_targets_match_restated_return_map(zs, gpu, model):
    import torch
    spec, c = _closure(zs, model, n_random=1000)
    rows = random_rows(model, 300, 5, spec.material.E, spec.material.nu)
    y = c.targets(torch.from_numpy(rows).to(gpu)).cpu().numpy().astype(np.float64)
    ref = oracle_targets(spec, rows)
    mu, lam = _mu_lam(spec.material)
    # FP32 return map on the GPU against the float64 restatement: log strains to 2e-6 absolute,
    # principal stresses to 1e-5 relative plus 2e-6 of the stress scale 3 lambda + 2 mu
    assert np.max(np.abs(y[:, :3] - ref[:, :3])) < 2e-6
    assert np.all(np.abs(y[:, 3:] - ref[:, 3:]) <= 1e-5 * np.abs(ref[:, 3:]) + 2e-6 * (3 * lam + 2 * mu))
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("model", [DP, SNOW])
def test_loss_and_gradient_match_cpu_oracle(zs, gpu, model):
    import torch
    spec, c = _closure(zs, model)
    st = c.state_arrays()
    rows = random_rows(model, 777, 3, spec.material.E, spec.material.nu)  # a ragged last tile
    x = torch.from_numpy(rows).to(gpu)
    y = c.targets(x)
    loss, grad = c.loss_grad(x, y)
    torch.cuda.synchronize()
    k, xi = _kappa(spec.material), spec.material.hardening
    xin = mlp.inputs(model, rows, k, xi)[0]
    xn = (xin - st["in_mean"]) * st["in_inv_std"]
    yn = mlp.net_targets(model, rows, y.cpu().numpy(), k, xi) / st["out_scale"]
    ref_loss, ref_grad = mlp.loss_and_grad(st["params"], xn, yn)
    # FP32 kernels (atomic accumulation over 25 tiles) against float64
    assert abs(loss.item() - ref_loss) <= 1e-5 * ref_loss
    g = grad.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - ref_grad) <= 1e-4 * np.linalg.norm(ref_grad)
    for lo, hi in ((0, 384), (384, 448), (448, 4544), (4608, 8704), (8768, 9152), (9152, 9158)):
        assert np.linalg.norm(g[lo:hi] - ref_grad[lo:hi]) <= 1e-4 * np.linalg.norm(ref_grad[lo:hi]) + 1e-9
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("model", [DP, SNOW])
def test_inference_fp32_and_bf16_match_cpu_oracle(zs, gpu, model):
    import torch
    spec, c = _closure(zs, model)
    c.train(2, batch=2048, lr=1e-3)
    st = c.state_arrays()
    rows = random_rows(model, 1000, 11, spec.material.E, spec.material.nu)
    x = torch.from_numpy(rows).to(gpu)
    y32 = c.infer(x, bf16=False).cpu().numpy().astype(np.float64)
    y16 = c.infer(x, bf16=True).cpu().numpy().astype(np.float64)
    k, xi = _kappa(spec.material), spec.material.hardening
    xin = mlp.inputs(model, rows, k, xi)[0]
    xn = (xin - st["in_mean"]) * st["in_inv_std"]
    ref = mlp.from_net(model, rows, mlp.forward(st["params"], xn) * st["out_scale"], k, xi)
    # per output group against its rms size: FP32 forward, rounding only; BF16 operands and
    # activations with FP32 accumulation, about 1e-2
    for lo in (0, 3):
        scale = np.linalg.norm(ref[:, lo:lo + 3]) / np.sqrt(3)
        for k in range(lo, lo + 3):
            assert np.linalg.norm(y32[:, k] - ref[:, k]) <= 1e-5 * scale
            assert np.linalg.norm(y16[:, k] - ref[:, k]) <= 3e-2 * scale
    print("bf16 relative error per output:",
          [float(np.linalg.norm(y16[:, k] - ref[:, k]) / np.linalg.norm(ref[:, k])) for k in range(6)])
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("model", [DP, SNOW])
def test_tcgen05_inference_matches_mma_sync_and_oracle(zs, gpu, model):
    """The tcgen05 forward (BF16 operands in shared memory, FP32 accumulators in tensor memory)
    against the mma.sync forward and the float64 oracle, on ragged row counts."""
    import torch
    spec, c = _closure(zs, model)
    c.train(2, batch=2048, lr=1e-3)
    st = c.state_arrays()
    k, xi = _kappa(spec.material), spec.material.hardening
    for n in (1, 128, 1000, 70001):
        rows = random_rows(model, n, 21 + n, spec.material.E, spec.material.nu)
        x = torch.from_numpy(rows).to(gpu)
        ytc = c.infer(x, path="tcgen05").cpu().numpy().astype(np.float64)
        c.status()
        ysplit = c.infer(x, path="tcgen05_split").cpu().numpy().astype(np.float64)
        c.status()
        ymma = c.infer(x, path="mma_sync").cpu().numpy().astype(np.float64)
        xin = mlp.inputs(model, rows, k, xi)[0]
        ref = mlp.from_net(model, rows, mlp.forward(st["params"], (xin - st["in_mean"]) * st["in_inv_std"])
                           * st["out_scale"], k, xi)
        assert np.all(np.isfinite(ytc))
        for lo in (0, 3):
            scale = np.linalg.norm(ref[:, lo:lo + 3]) / np.sqrt(3) + 1e-30
            for col in range(lo, lo + 3):
                # BF16 operands and activations, FP32 accumulation: as the mma.sync path
                assert np.linalg.norm(ytc[:, col] - ref[:, col]) <= 3e-2 * scale
                # the two tensor-core paths round the same values; they differ by accumulation order
                assert np.linalg.norm(ytc[:, col] - ymma[:, col]) <= 5e-3 * scale
                # split-BF16 operands (hi + lo pairs, three MMAs per step) and FP32 SiLU: products
                # to about 16 significant bits
                assert np.linalg.norm(ysplit[:, col] - ref[:, col]) <= 3e-4 * scale
    c.close()


def stress_errors(y, ref, mat):
    """Relative principal-stress error per row, floored at 1e-4 of the stress scale, and the
    aggregate sqrt(sum |dtau|^2 / sum |tau|^2)."""
    mu, lam = _mu_lam(mat)
    d = np.linalg.norm(y[:, 3:] - ref[:, 3:], axis=1)
    t = np.linalg.norm(ref[:, 3:], axis=1)
    return d / (t + 1e-4 * (3 * lam + 2 * mu)), np.sqrt(np.sum(d * d) / np.sum(t * t))


@pytest.mark.gpu
@pytest.mark.parametrize("model", [DP, SNOW])
def test_training_reduces_loss_and_beats_no_return_map(zs, gpu, model):
    """What the trained network gains over the method without it: on held-out trial states that
    the return map projects (the branch the network replaces), its stress error against the
    plain return map is compared with the error of dropping the return map (the elastic trial
    stress)."""
    import torch
    spec, c = _closure(zs, model, n_random=400000)
    losses = c.fit()
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.02 * losses[0]
    rows = random_rows(model, 100000, 99, spec.material.E, spec.material.nu)
    rows = rows[projected(model, rows, spec.material.E, spec.material.nu)][:50000]
    x = torch.from_numpy(rows).to(gpu)
    ref = c.targets(x).cpu().numpy().astype(np.float64)
    y16 = c.infer(x, bf16=True).cpu().numpy().astype(np.float64)
    mu, lam = _mu_lam(spec.material)
    l = rows[:, :3].astype(np.float64)
    elastic = np.zeros_like(ref)
    if model == DP:
        elastic[:, 3:] = 2 * mu * l + lam * l.sum(1, keepdims=True)
    else:
        # fixed corotated with the state's hardened Lame parameters and no projection
        Jp = np.exp(rows[:, 5].astype(np.float64))
        h = np.exp(spec.material.hardening * (1 - Jp))[:, None]
        S = np.exp(l)
        J = S.prod(1, keepdims=True)
        elastic[:, 3:] = 2 * mu * h * (S - 1) * S + lam * h * (J - 1) * J
    rel_net, agg_net = stress_errors(y16, ref, spec.material)
    rel_el, agg_el = stress_errors(elastic, ref, spec.material)
    print(f"model {model}: net agg {agg_net:.3e} mean {rel_net.mean():.3e} | "
          f"no return map agg {agg_el:.3e} mean {rel_el.mean():.3e} | loss {losses[0]:.3e} -> {losses[-1]:.3e}")
    assert agg_net < 0.1 * agg_el
    assert np.mean(rel_net) < 0.1 * np.mean(rel_el)
    c.close()


def _run_scene(zs, spec, steps, closure=None, audit_period=100):
    from zsmpm_b200 import closure as cl
    sc = zs.Scene(spec, zs.generate(spec))
    if closure is not None:
        cl.attach(sc, closure, audit_period)
    sc.run(steps)
    sc.status()
    out = sc.download()
    a = cl.audit(sc) if closure is not None else None
    sc.close()
    return out, a


def _sand_scene():
    from zsmpm_b200 import scenes
    # the box's bottom starts 0.7 cm above the sticky floor and lands after ~35 substeps
    return scenes.small_scene(model=DP, n_side=0.08, velocity=(0.0, -2.0, 0.0), center=(0.5, 0.07, 0.5))


@pytest.mark.gpu
def test_learned_scene_follows_plain_and_audits(zs, gpu):
    """A sand box thrown onto the floor: the learned closure (trained on random states plus the
    trial states logged from the plain run) against the plain return map, with the 1% audit."""
    import torch
    from zsmpm_b200 import closure as cl
    spec = _sand_scene()
    steps = 200
    parts = zs.generate(spec)
    sc = zs.Scene(spec, parts)
    buf = torch.empty((400000, 6), dtype=torch.float32, device=gpu)
    cl.set_state_log(sc, buf, 7)
    sc.run(steps)
    n_log = cl.state_log_count(sc)
    assert n_log > 0.9 * min(parts.n * steps / 7, 400000)
    logged = buf[:n_log].contiguous()
    assert torch.isfinite(logged).all()
    cl.set_state_log(sc, None, 0)
    plain = sc.download()
    sc.close()
    c = cl.Closure(spec.material, spec.volume)
    c.build_dataset(200000, seed=4, logged=logged)
    c.fit(cl.SCHEDULE_LONG)
    learned, a = _run_scene(zs, spec, steps, closure=c, audit_period=100)
    # the method without the return map: the same box in fixed corotated
    el_spec = dataclasses.replace(spec, material=dataclasses.replace(spec.material, model=0))
    elastic, _ = _run_scene(zs, el_spec, steps)
    x0 = parts.x.astype(np.float64)
    disp = np.linalg.norm(plain.x - x0)
    err_learned = np.linalg.norm(learned.x.astype(np.float64) - plain.x) / disp
    err_elastic = np.linalg.norm(elastic.x.astype(np.float64) - plain.x) / disp
    print(f"audit {a}; displacement error learned {err_learned:.3e} elastic {err_elastic:.3e}")
    # every particle update is counted; one in 100 of those the network projected is audited
    assert a["updates"] == parts.n * steps
    assert a["network_updates"] > 0
    expect = a["network_updates"] / 100
    assert 0.7 * expect < a["audited"] < 1.3 * expect + 5
    assert np.isfinite(a["mean_rel_error"]) and a["max_rel_error"] >= a["mean_rel_error"]
    # the long schedule gives mean 1.9e-3 and aggregate 1.5e-3 on this scene
    assert a["mean_rel_error"] < 5e-3 and a["agg_rel_error"] < 5e-3
    assert err_learned < 0.2 * err_elastic
    c.close()


@pytest.mark.gpu
def test_outside_hull_falls_back_to_plain(zs, gpu):
    """A hull that excludes every state: each projection takes the plain return map."""
    spec = _sand_scene()
    steps = 60  # the box lands after ~35 substeps, and its particles start to project
    _, c = _closure(zs, DP, n_random=5000)
    st = c.get_state()
    st.in_max[0] = -10.0  # no trial state has a largest log singular value below -10
    c.set_state(st)
    learned, a = _run_scene(zs, spec, steps, closure=c, audit_period=0)
    plain, _ = _run_scene(zs, spec, steps)
    # the box lands: projections happen, each by the plain map, none by the network
    assert a["fallbacks"] > 0 and a["network_updates"] == 0
    assert a["audited"] == 0
    # the same arithmetic as the plain path; two runs differ by the order of P2G's float sums,
    # which the landing's plastic flow amplifies in F over 60 substeps
    assert np.max(np.abs(learned.x - plain.x)) <= 1e-6
    assert np.max(np.abs(learned.F - plain.F)) <= 1e-4
    c.close()
