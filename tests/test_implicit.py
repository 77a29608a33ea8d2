"""The implicit system: G2P2GTransfer (simulation/transfer/G2P2G.hpp), ImplicitMPMSystem's
multiply / project / precondition (simulation/mpm/ImplicitMPM.hpp) and ConjugateGradient::solve
(math/linear/ConjugateGradient.hpp).

CPU: the restated oracle (oracle_g2p2g + oracle/implicit.py) against the reference's own outputs
(tests/golden/ref_implicit_*.npz, made by tests/golden/make_golden.py from the compiled
reference).  GPU: the CUDA path through the C ABI against the pinned restatement on the state the
scene holds, and size-independent properties at a larger size."""
from pathlib import Path

import numpy as np
import pytest

from helpers import rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"
MODELS = ("fc", "dp")


def _spec(model: int):
    from zsmpm_b200 import scenes
    return scenes.small_scene(model=model, mode=1, n_side=0.04)


def _golden(name):
    return np.load(GOLDEN / f"ref_implicit_{name}.npz")


# ------------------------------------------------------------------ CPU: oracle pin
@pytest.mark.parametrize("name", MODELS)
def test_restated_g2p2g_bit_exact_with_reference(name):
    from oracle import restated
    g = _golden(name)
    spec = _spec(int(g["model"]))
    f = restated.g2p2g(spec, g["x"], g["F"], g["plastic"], g["keys"], g["vel"], dt=float(g["dt"]))
    assert np.array_equal(f, g["f"])
    assert np.abs(g["f"]).max() > 0


@pytest.mark.parametrize("name", MODELS)
def test_restated_implicit_operators_bit_exact_with_reference(name):
    from oracle import implicit
    g = _golden(name)
    spec = _spec(int(g["model"]))
    state = (g["x"], g["F"], g["plastic"])
    dt = float(g["dt"])
    assert np.array_equal(implicit.multiply(spec, state, g["keys"], g["mass"], g["vel"], dt), g["mult"])
    assert np.array_equal(implicit.project(spec, g["keys"], g["mass"], g["vel"]), g["proj"])
    assert np.array_equal(implicit.precondition(g["mass"], g["vel"], g["prec_base"]), g["prec"])
    # project zeroes the massless nodes, precondition leaves them as they were
    massless = np.repeat(g["mass"].reshape(-1) <= 0, 3)
    assert massless.any() and np.all(g["proj"][massless] == 0)
    assert np.all(g["prec"][massless] == g["prec_base"][massless])


@pytest.mark.parametrize("name", MODELS)
def test_restated_cg_matches_reference(name):
    from oracle import implicit
    g = _golden(name)
    spec = _spec(int(g["model"]))
    x, it = implicit.cg_solve(spec, (g["x"], g["F"], g["plastic"]), g["keys"], g["mass"], np.zeros_like(g["b"]),
                              g["b"], float(g["dt"]), max_iters=int(g["cg_max_iters"]))
    assert it == int(g["cg_iters"])
    # the dot products sum in another order (float64 here, the reference's float reduce)
    assert np.abs(x - g["cg_x"]).max() <= 1e-5 * np.abs(g["cg_x"]).max()


@pytest.mark.parametrize("name", MODELS)
def test_restated_g2p2g_f64_close(name):
    """The reference's FP32 forces against the FP64 restatement: the FP32 SVD (four Jacobi
    sweeps) bounds the agreement near 3e-5."""
    from oracle import restated
    g = _golden(name)
    spec = _spec(int(g["model"]))
    f64 = restated.g2p2g(spec, g["x"], g["F"], g["plastic"], g["keys"], g["vel"], dt=float(g["dt"]), precision="f64")
    assert rel_l2(g["f"], f64) < 1e-4


# ------------------------------------------------------------------ GPU
def _scene_from_golden(zs, name):
    from zsmpm_b200.scenes import Particles
    g = _golden(name)
    spec = _spec(int(g["model"]))
    p = Particles(m=g["m"], x=g["x"], v=g["v"], C=g["C"], F=g["F"], plastic=g["plastic"])
    scene = zs.Scene(spec, p)
    scene.activate_blocks()
    scene.bin_particles()
    return g, spec, scene


def _t(a, gpu):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("name", MODELS)
def test_g2p2g_matches_oracle(zs, gpu, name):
    import torch
    from oracle import restated
    from zsmpm_b200.implicit import ImplicitMPMSystem
    g, spec, scene = _scene_from_golden(zs, name)
    keys, _ = scene.download_grid()
    assert np.array_equal(keys, g["keys"])
    st = scene.download()  # the state the scene holds (the upload's stress pass may move logJp)
    dt = float(g["dt"])
    sys_ = ImplicitMPMSystem(scene, dt)
    assert sys_.ndofs == g["vel"].size
    v = _t(g["vel"], gpu)
    f = torch.zeros_like(v)
    sys_.g2p2g(v, f)
    torch.cuda.synchronize()
    scene.status()
    fg = f.cpu().numpy()
    fo = restated.g2p2g(spec, st.x, st.F, st.plastic, keys, g["vel"], dt=dt)
    scale = np.abs(fo).max()
    # FP32 on both sides; atomics sum in another order and the GPU contracts to FMA
    assert np.abs(fg - fo).max() <= 2e-4 * scale, np.abs(fg - fo).max() / scale
    assert rel_l2(fg, fo) < 2e-5
    if np.array_equal(st.F, g["F"]) and np.array_equal(st.plastic, g["plastic"]):
        assert np.abs(fg - g["f"]).max() <= 2e-4 * scale
    # G2P2G adds: a second call doubles
    sys_.g2p2g(v, f)
    torch.cuda.synchronize()
    assert np.abs(f.cpu().numpy() - 2 * fg).max() <= 1e-6 * scale
    scene.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", MODELS)
def test_implicit_operators_match_oracle(zs, gpu, name):
    import torch
    from oracle import implicit
    from zsmpm_b200.implicit import ImplicitMPMSystem
    g, spec, scene = _scene_from_golden(zs, name)
    st = scene.download()
    scene.p2g()
    keys, grid = scene.download_grid()
    mass = grid[:, 0, :]
    # the grid mass of the scene's P2G against the reference's P2GTransfer
    assert np.abs(mass - g["mass"]).max() <= 1e-5 * g["mass"].max()
    dt = float(g["dt"])
    sys_ = ImplicitMPMSystem(scene, dt)
    state = (st.x, st.F, st.plastic)
    v = _t(g["vel"], gpu)
    out = torch.empty_like(v)
    sys_.multiply(v, out)
    ref = implicit.multiply(spec, state, keys, mass, g["vel"], dt)
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()
    w = v.clone()
    sys_.project(w)
    ref = implicit.project(spec, keys, mass, g["vel"])
    assert np.array_equal(w.cpu().numpy(), ref)  # elementwise, no rounding differences
    o = _t(g["prec_base"], gpu)
    sys_.precondition(v, o)
    ref = implicit.precondition(mass, g["vel"], g["prec_base"])
    assert np.abs(o.cpu().numpy() - ref).max() <= 1e-6 * np.abs(ref).max()
    scene.status()
    scene.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", MODELS)
def test_cg_matches_oracle(zs, gpu, name):
    from oracle import implicit
    from zsmpm_b200.implicit import ConjugateGradient, ImplicitMPMSystem
    g, spec, scene = _scene_from_golden(zs, name)
    st = scene.download()
    scene.p2g()
    keys, grid = scene.download_grid()
    mass = grid[:, 0, :]
    dt = float(g["dt"])
    b = (np.repeat(mass.reshape(-1), 3) * g["vel"]).astype(np.float32)
    sys_ = ImplicitMPMSystem(scene, dt)
    for iters in (1, 3, int(g["cg_max_iters"])):
        x = sys_.zeros()
        n = ConjugateGradient(max_iters=iters).solve(sys_, x, _t(b, gpu))
        xo, no = implicit.cg_solve(spec, (st.x, st.F, st.plastic), keys, mass, np.zeros_like(b), b, dt,
                                   max_iters=iters)
        assert n == no
        assert np.abs(x.cpu().numpy() - xo).max() <= 1e-4 * np.abs(xo).max()
    # converged: the solution approximately recovers the field on massive nodes
    has = np.repeat(mass.reshape(-1) > 0, 3)
    xs = x.cpu().numpy()
    assert rel_l2(xs[has], implicit.project(spec, keys, mass, g["vel"])[has]) < 0.05
    scene.close()


@pytest.mark.gpu
def test_implicit_rejects_short_vectors_and_unbinned_scene(zs, gpu):
    import torch
    from zsmpm_b200.implicit import ImplicitMPMSystem
    g, spec, scene = _scene_from_golden(zs, "fc")
    sys_ = ImplicitMPMSystem(scene, 1e-3)
    short = torch.full((sys_.ndofs - 1536,), 5.0, device=gpu)
    other = torch.full_like(short, 5.0)
    sys_.g2p2g(short, other)
    torch.cuda.synchronize()
    with pytest.raises(zs._abi.ZsmpmError):
        scene.status()  # capacity: the vectors hold fewer blocks than the grid
    assert torch.all(other == 5.0)
    with pytest.raises(ValueError):
        sys_.multiply(short, torch.zeros(7, device=gpu))
    scene.substep()  # positions moved: the binning no longer matches them
    with pytest.raises(zs._abi.ZsmpmError):
        sys_.g2p2g(sys_.zeros(), sys_.zeros())
    scene.close()


@pytest.mark.gpu
def test_g2p2g_conserves_momentum_at_scale(zs, gpu):
    """Sum_i W_ip (x_i - x_p) = 0 for the quadratic B-spline, so the forces of every particle sum
    to zero: a size-independent check on 2.3 M particles (sand two-box scene at dx = 1/128)."""
    import torch
    from zsmpm_b200 import scenes
    from zsmpm_b200.implicit import ImplicitMPMSystem
    spec = scenes.config2(dx=1 / 128)
    p = scenes.generate(spec)
    rng = np.random.default_rng(1)
    p.F = (np.tile(np.eye(3, dtype=np.float32).reshape(1, 9), (p.n, 1))
           + rng.normal(0, 0.02, (p.n, 9)).astype(np.float32))
    scene = zs.Scene(spec, p)
    scene.activate_blocks()
    scene.bin_particles()
    sys_ = ImplicitMPMSystem(scene, spec.dt)
    keys, _ = scene.download_grid()
    cell = np.arange(512)
    loc = np.stack([cell >> 6, (cell >> 3) & 7, cell & 7], 1)
    pos = (keys[:, None, :].astype(np.int64) * 8 + loc[None]) * spec.dx
    vel = np.stack([np.sin(7 * pos[..., 1]), np.cos(5 * pos[..., 2]), np.sin(3 * pos[..., 0])], -1)
    v = _t(vel.reshape(-1), gpu)
    f = sys_.zeros()
    sys_.g2p2g(v, f)
    torch.cuda.synchronize()
    scene.status()
    fd = f.double().view(-1, 3)
    total = fd.sum(0).abs().max().item()
    assert total <= 1e-5 * fd.abs().sum().item()
    scene.close()
