"""CPU: the restated oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the compiled reference), and against the compiled
reference directly when oracle/_ref/zsref_cli is present.  FP32 agreement is bit-exact."""
from pathlib import Path

import numpy as np
import pytest

from helpers import rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"


def _particles(z):
    from zsmpm_b200.scenes import Particles
    return Particles(m=z["m"], x=z["x0"], v=z["v0"], C=z["C0"], F=z["F0"], plastic=z["plastic0"])


@pytest.mark.parametrize("name", ["fc", "dp"])
def test_restatement_bit_exact_with_reference_substeps(name):
    from oracle import restated
    from zsmpm_b200 import scenes
    z = np.load(GOLDEN / f"ref_substep_{name}.npz")
    spec = scenes.small_scene(model=int(z["model"]), mode=1, velocity=(0.4, -0.3, 0.2))
    p = _particles(z)
    assert np.array_equal(p.x, scenes.generate(spec).x), "scene generator changed"
    o = restated.run(spec, p, int(z["steps"]), "f32", mode=1)
    for f in ("x", "v", "C", "F"):
        assert np.array_equal(getattr(o, f), z[f]), f
    assert np.array_equal(o.plastic, z["logJp"])
    assert np.array_equal(o.keys, z["keys"])
    assert np.array_equal(o.grid, z["grid"])


def test_restatement_fp64_close_to_reference():
    """The FP64 run of the same algorithm differs from the FP32 reference only by rounding."""
    from oracle import restated
    from zsmpm_b200 import scenes
    z = np.load(GOLDEN / "ref_substep_dp.npz")
    spec = scenes.small_scene(model=1, mode=1, velocity=(0.4, -0.3, 0.2))
    o = restated.run(spec, _particles(z), int(z["steps"]), "f64", mode=1)
    assert rel_l2(o.v, z["v"]) < 1e-5
    assert rel_l2(o.x, z["x"]) < 1e-6
    # FP32 rounding of x += v dt (x ~ 0.5, v dt ~ 4e-5) dominates the displacement error
    assert rel_l2(o.x - z["x0"], z["x"] - z["x0"]) < 2e-3


def test_svd_bit_exact_with_reference():
    from oracle import restated
    z = np.load(GOLDEN / "ref_svd.npz")
    U, S, V = restated.svd(z["A"])
    assert np.array_equal(U, z["U"]) and np.array_equal(S, z["S"]) and np.array_equal(V, z["V"])


def test_svd_fp64_reconstructs():
    from oracle import restated
    z = np.load(GOLDEN / "ref_svd.npz")
    A = z["A"].astype(np.float64)
    U, S, V = restated.svd(A, "f64")
    Um = U.reshape(-1, 3, 3).transpose(0, 2, 1)
    Vm = V.reshape(-1, 3, 3).transpose(0, 2, 1)
    R = Um @ (S[:, :, None] * np.eye(3)) @ Vm.transpose(0, 2, 1)
    assert np.max(np.abs(R - A.reshape(-1, 3, 3).transpose(0, 2, 1))) < 1e-12
    assert np.allclose(np.abs(S), np.abs(z["S"]), rtol=2e-6)


def test_stress_bit_exact_with_reference():
    from oracle import restated
    from zsmpm_b200 import scenes
    z = np.load(GOLDEN / "ref_stress.npz")
    tau, _, _ = restated.stress(scenes.small_scene(model=0), z["F"], np.zeros(len(z["F"])), mode=1)
    assert np.array_equal(tau, z["PF_fc"])
    tau, F, lj = restated.stress(scenes.small_scene(model=1, mode=1), z["F"], z["logJp"], mode=1)
    assert np.array_equal(tau, z["PF_dp"])
    assert np.array_equal(F, z["F_dp"])
    assert np.array_equal(lj, z["logJp_dp"])


def test_activation_keys_and_slots_bit_exact():
    from oracle import restated
    z = np.load(GOLDEN / "ref_activation.npz")
    keys, slots, npb, ts = restated.activate(z["x"], float(z["dx"]), int(z["expected"]))
    assert ts == int(z["table_size"]) and npb == int(z["nparblocks"])
    assert np.array_equal(keys, z["keys"])
    assert np.array_equal(slots, z["slots"])


def test_hash_slot_formula():
    """(do_hash(k) % T + T) % T with the 64-bit hash_combine, checked on hand-computed keys."""
    from oracle import restated
    M = (1 << 64) - 1

    def do_hash(k):
        seed = k[0] & M
        for v in k[1:]:
            seed ^= ((v & M) + 0x9E3779B97F4A7C15 + ((seed << 12) & M) + (seed >> 4)) & M
        h = seed & 0xFFFFFFFF
        return h - (1 << 32) if h >= 1 << 31 else h

    for k in [(0, 0, 0), (1, 2, 3), (-1, 5, -7), (63, -64, 1000), (-100000, 7, 9)]:
        T = 1 << 12
        h = do_hash(k)
        expected = (int(np.fmod(h, T)) + T) % T
        assert restated.hash_slot(k, T) == expected


def test_bin_order_definition():
    """A stable sort by (block, cell): cells ascending inside a block, indices ascending in a cell."""
    from oracle import restated
    rng = np.random.default_rng(3)
    n = 5000
    block = rng.integers(0, 4, n).astype(np.int32)
    cell = rng.integers(0, 512, n).astype(np.int32)
    order, bstart = restated.bin_order(block, cell, 4)
    expected = np.lexsort((np.arange(n), cell, block))
    assert np.array_equal(order, expected)
    assert np.array_equal(bstart, np.searchsorted(block[expected], np.arange(5)))


@pytest.mark.slow
def test_restatement_matches_reference_live_omp():
    """Against the compiled reference run live (OpenMP, 4 threads): equal up to the float
    atomic summation order of the parallel P2G."""
    from oracle import reference, restated
    from zsmpm_b200 import scenes
    if not reference.available():
        pytest.skip("oracle/_ref/zsref_cli not built (needs the reference sources)")
    spec = scenes.small_scene(model=1, mode=1, velocity=(0.4, -0.3, 0.2), n_side=0.1)
    p = scenes.generate(spec)
    r = reference.run(spec, p, 5, policy=reference.POLICY_OMP, threads=4)
    o = restated.run(spec, p, 5, "f32", mode=1)
    assert rel_l2(o.v, r.v) < 1e-5
    assert rel_l2(o.x, r.x) < 1e-6


def _cell_particles(z):
    from zsmpm_b200.scenes import Particles
    n = len(z["m"])
    return Particles(m=z["m"], x=z["x0"], v=z["v0"], C=z["C0"], F=z["F0"], plastic=np.zeros(n, np.float32))


def test_cell_transfer_restatement_bit_exact_with_reference():
    """P2C2GTransfer / G2C2PTransfer (fixed corotated) restated: 5 substeps equal the compiled
    reference's sequential run bit for bit (particles, keys and grid)."""
    from oracle import restated
    from zsmpm_b200 import scenes
    z = np.load(GOLDEN / "ref_cell_fc.npz")
    spec = scenes.small_scene(model=0, mode=0, velocity=(0.4, -0.3, 0.2))
    p = _cell_particles(z)
    assert np.array_equal(p.x, scenes.generate(spec).x), "scene generator changed"
    o = restated.run_cell(spec, p, int(z["steps"]), "f32")
    for f in ("x", "v", "C", "F"):
        assert np.array_equal(getattr(o, f), z[f]), f
    assert np.array_equal(o.keys, z["keys"])
    assert np.array_equal(o.grid, z["grid"])


def test_cell_transfer_fp64_against_reference():
    """The FP64 restatement against the FP32 reference: x and v differ by rounding.  B (the C
    attribute) and F - I differ by about 1%: G2C2P forms B as W (sum_i v_i x_i / 8 - v_c x_p)
    from absolute positions (x ~ 0.5) for a term of size v dx, so FP32 keeps only about
    eps * 0.5 / dx of it."""
    from oracle import restated
    from zsmpm_b200 import scenes
    z = np.load(GOLDEN / "ref_cell_fc.npz")
    spec = scenes.small_scene(model=0, mode=0, velocity=(0.4, -0.3, 0.2))
    o = restated.run_cell(spec, _cell_particles(z), int(z["steps"]), "f64")
    assert rel_l2(o.v, z["v"]) < 1e-5
    assert rel_l2(o.x - z["x0"], z["x"] - z["x0"]) < 2e-3
    assert rel_l2(o.C, z["C"]) < 5e-2
    assert rel_l2(o.F - z["F0"], z["F"] - z["F0"]) < 5e-2
    # mass: the pair's node weights sum to one per particle
    assert abs(float(o.grid[:, 0].sum()) / float(z["m"].sum()) - 1) < 1e-12
