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
