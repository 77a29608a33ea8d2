"""GPU: the allocation-free activation entry point (zsmpm_activate_blocks_noalloc) against the
scene path's zsmpm_activate_blocks.

That entry point exists for callers that cannot allocate device memory when they need block
activation (a host whose pool already holds the GPU, plug-in loops that forbid allocation
after start-up); its scratch is a fixed device array
shared by all calls.  The keys are integers, so the comparison is exact.  Two calls in a row
check that the shared scratch left by one call does not leak into the next.  This file is
named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(zs, x_dev, n, dx, keys_dev, cap, count_dev):
    return zs._abi.lib().zsmpm_activate_blocks_noalloc(
        C.c_void_p(x_dev.data_ptr()), n, dx, C.c_void_p(keys_dev.data_ptr()), cap,
        C.c_void_p(count_dev.data_ptr()), None)


def _scene_keys(zs, spec, p):
    with zs.Scene(spec, p) as sc:
        sc.activate_blocks()
        keys, _ = sc.download_grid()
    return keys


def test_noalloc_activation_matches_scene_path_twice(zs, gpu):
    import torch
    from zsmpm_b200 import scenes
    spec_a = scenes.small_scene(model=0, n_side=0.2, velocity=(0, 0, 0))
    spec_b = scenes.small_scene(model=0, n_side=0.12, center=(0.3, 0.6, 0.45), seed=11)
    pa, pb = scenes.generate(spec_a), scenes.generate(spec_b)
    ka, kb = _scene_keys(zs, spec_a, pa), _scene_keys(zs, spec_b, pb)
    cap = 4096
    keys = torch.empty((cap, 3), dtype=torch.int32, device=gpu)
    count = torch.empty(1, dtype=torch.int32, device=gpu)
    for p, spec, expected in ((pa, spec_a, ka), (pa, spec_a, ka), (pb, spec_b, kb)):
        x = torch.from_numpy(p.x).to(gpu)
        keys.fill_(-7)
        count.fill_(-99)
        zs._abi.check(_noalloc(zs, x, p.n, spec.dx, keys, cap, count), "activate_blocks_noalloc")
        torch.cuda.synchronize()
        nb = int(count.item())
        assert nb == len(expected)
        assert np.array_equal(keys[:nb].cpu().numpy(), expected)


def test_noalloc_rejects_sizes_beyond_its_limits(zs, gpu):
    import torch
    keys = torch.empty((16, 3), dtype=torch.int32, device=gpu)
    count = torch.empty(1, dtype=torch.int32, device=gpu)
    x = torch.full((8, 3), 0.5, dtype=torch.float32, device=gpu)
    st = _noalloc(zs, x, 1_048_577, 1 / 128, keys, 16, count)
    assert st == zs._abi.ERR_CAPACITY
    assert b"1048576" in zs._abi.lib().zsmpm_last_error_string()
    # more blocks than the caller's capacity: reported on the device as -2
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=0, n_side=0.2, velocity=(0, 0, 0))
    p = scenes.generate(spec)
    xd = torch.from_numpy(p.x).to(gpu)
    zs._abi.check(_noalloc(zs, xd, p.n, spec.dx, keys, 16, count), "activate_blocks_noalloc")
    torch.cuda.synchronize()
    assert int(count.item()) == -2


def _run_codes(zs, gpu, x_np, dx, cap=40000):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(x_np, np.float32)).to(gpu)
    keys = torch.empty((cap, 3), dtype=torch.int32, device=gpu)
    count = torch.full((1,), -99, dtype=torch.int32, device=gpu)
    zs._abi.check(_noalloc(zs, x, x.shape[0], dx, keys, cap, count), "activate_blocks_noalloc")
    torch.cuda.synchronize()
    return int(count.item()), keys


def test_noalloc_device_codes(zs, gpu):
    # -1: 4,096 particles two blocks apart on every axis; each particle block and its seven
    # +{0,1}^3 neighbours are distinct, 32,768 blocks against the 32,748 the table takes
    # (a few particles, so this also checks that the whole table serves a small n)
    g = np.arange(16, dtype=np.float32)
    lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    dx = 1.0 / 128
    x = (lattice * 16 + 4.0) * dx  # cells 4 + 16 i: block 2 i after the -2 stencil shift
    code, _ = _run_codes(zs, gpu, x, dx)
    assert code == -1
    # the same lattice minus a 3 x 3 x 3 corner of particles fits: 4,069 x 8 = 32,552 blocks
    keep = ~np.all(lattice < 3, axis=1)
    code, keys = _run_codes(zs, gpu, x[keep], dx)
    assert code == 8 * int(keep.sum())
    k = keys[:code].cpu().numpy().astype(np.int64)
    assert np.all(np.diff((k[:, 0] << 42) + (k[:, 1] << 21) + k[:, 2]) > 0)
    # -1: two particles 2^22 cells apart, a block bounding box beyond 2^21 positions
    code, _ = _run_codes(zs, gpu, np.array([[0.0, 0.0, 0.0], [float(1 << 22), 0.0, 0.0]]), 1.0)
    assert code == -1
    # -3: a NaN position
    x = np.full((64, 3), 0.5, np.float32)
    x[17, 1] = np.nan
    code, _ = _run_codes(zs, gpu, x, dx)
    assert code == -3


def test_noalloc_rejects_empty_input(zs, gpu):
    import torch
    keys = torch.empty((16, 3), dtype=torch.int32, device=gpu)
    count = torch.empty(1, dtype=torch.int32, device=gpu)
    x = torch.full((8, 3), 0.5, dtype=torch.float32, device=gpu)
    assert _noalloc(zs, x, 0, 1 / 128, keys, 16, count) == zs._abi.ERR_CAPACITY


_RESET_CHILD = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from zsmpm_b200 import _abi, scenes
lib = _abi.lib()
rt = C.CDLL("libcudart.so.12")
rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
rt.cudaFree.argtypes = [C.c_void_p]
spec = scenes.small_scene(model=0, n_side=0.2, velocity=(0, 0, 0))
p = scenes.generate(spec)
x = np.ascontiguousarray(p.x, np.float32)
cap = 4096

def once():
    bufs = [C.c_void_p() for _ in range(3)]
    for b, size in zip(bufs, (x.nbytes, cap * 12, 4)):
        assert rt.cudaMalloc(C.byref(b), size) == 0
    assert rt.cudaMemcpy(bufs[0], x.ctypes.data, x.nbytes, 1) == 0
    st = lib.zsmpm_activate_blocks_noalloc(bufs[0], p.n, spec.dx, bufs[1], cap, bufs[2], None)
    assert st == 0, lib.zsmpm_last_error_string()
    assert rt.cudaDeviceSynchronize() == 0
    n = np.zeros(1, np.int32)
    assert rt.cudaMemcpy(n.ctypes.data, bufs[2], 4, 2) == 0
    assert n[0] > 0, n[0]
    keys = np.zeros((n[0], 3), np.int32)
    assert rt.cudaMemcpy(keys.ctypes.data, bufs[1], keys.nbytes, 2) == 0
    for b in bufs:
        assert rt.cudaFree(b) == 0
    return keys

a = once()
assert rt.cudaDeviceReset() == 0  # ends this process's own context only
b = once()
assert np.array_equal(a, b)
print("reset ok", len(a))
"""


def test_noalloc_after_device_reset(zs, gpu):
    # The array's device address belongs to a CUDA context.  In a child process (so that the
    # reset does not touch this process's tensors): a call, cudaDeviceReset, which rebuilds
    # the primary context, and a second call that must look the address up again.
    import subprocess
    import sys
    from pathlib import Path
    root = str(Path(__file__).resolve().parents[1])
    r = subprocess.run([sys.executable, "-c", _RESET_CHILD, root], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "reset ok" in r.stdout
