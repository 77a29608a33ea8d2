"""CPU: the C-ABI library builds, loads without a GPU, exports every symbol the public headers
declare, and the ctypes mirror matches the header; host-side argument checks."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"ZSMPM_API\s+[^;{]*?\b(zsmpm_\w+)\s*\(", text, flags=re.S))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("zsmpm_scene_create", "zsmpm_activate_blocks", "zsmpm_bin_particles", "zsmpm_p2g",
                     "zsmpm_grid_update", "zsmpm_g2p", "zsmpm_substep", "zsmpm_run"):
        assert required in names


def test_library_exports_every_declared_symbol(zs):
    out = subprocess.run(["nm", "-D", "--defined-only", str(zs._abi.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT\s+(zsmpm_\w+)", out))
    missing = declared_symbols() - exported
    assert not missing, missing


def test_ctypes_mirror_covers_header(zs):
    assert declared_symbols() <= set(zs._abi.SIGNATURES)


def test_struct_layouts_match_header(zs, tmp_path):
    """Compiles a C probe against include/zsmpm.h and compares sizeof/offsetof with ctypes."""
    probe = tmp_path / "probe.c"
    probe.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "zsmpm.h"\n'
                     "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu\\n\","
                     "sizeof(zsmpm_material), sizeof(zsmpm_scene_desc), offsetof(zsmpm_scene_desc, material),"
                     "offsetof(zsmpm_scene_desc, max_particles), sizeof(zsmpm_particle_arrays),"
                     "sizeof(zsmpm_tilevector_view), sizeof(zsmpm_table_view));"
                     "printf(\"%zu %zu %zu %zu\\n\", sizeof(zsmpm_closure_state),"
                     "offsetof(zsmpm_closure_state, in_mean), sizeof(zsmpm_closure_audit),"
                     "offsetof(zsmpm_closure_audit, fallbacks));"
                     "printf(\"%zu %zu %zu\\n\", sizeof(zsmpm_bht_view), offsetof(zsmpm_bht_view, table_size),"
                     "sizeof(zsmpm_tuning));"
                     "printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(zsmpm_collider), offsetof(zsmpm_collider, R),"
                     "sizeof(zsmpm_levelset_desc), offsetof(zsmpm_levelset_desc, background),"
                     "offsetof(zsmpm_levelset_desc, t), sizeof(zsmpm_cg_options));return 0;}\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(probe), "-o", str(exe)], check=True)
    vals = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()))
    a = zs._abi
    assert vals == [C.sizeof(a.Material), C.sizeof(a.SceneDesc), a.SceneDesc.material.offset,
                    a.SceneDesc.max_particles.offset, C.sizeof(a.ParticleArrays),
                    C.sizeof(a.TileVectorView), C.sizeof(a.TableView),
                    C.sizeof(a.ClosureState), a.ClosureState.in_mean.offset, C.sizeof(a.ClosureAudit),
                    a.ClosureAudit.fallbacks.offset, C.sizeof(a.BhtView), a.BhtView.table_size.offset,
                    C.sizeof(a.Tuning),
                    C.sizeof(a.Collider), a.Collider.R.offset, C.sizeof(a.LevelSetDesc),
                    a.LevelSetDesc.background.offset, a.LevelSetDesc.t.offset, C.sizeof(a.CgOptions)]


def test_host_side_argument_checks_without_gpu(zs):
    lib = zs._abi.lib()
    assert lib.zsmpm_scene_create(None, None) == zs._abi.ERR_INVALID_ARG
    assert b"null" in lib.zsmpm_last_error_string()
    desc = zs._abi.SceneDesc()
    h = C.c_void_p()
    desc.dx = 0.0
    assert lib.zsmpm_scene_create(C.byref(desc), C.byref(h)) == zs._abi.ERR_INVALID_ARG
    desc.dx, desc.dt = 0.01, 1e-4
    desc.material.model = 7
    assert lib.zsmpm_scene_create(C.byref(desc), C.byref(h)) == zs._abi.ERR_INVALID_ARG
    assert lib.zsmpm_svd3(None, None, None, None, -1, None) == zs._abi.ERR_INVALID_ARG
    assert lib.zsmpm_scene_destroy(None) == zs._abi.OK
    mat = zs._abi.Material(model=zs.FIXED_COROTATED)
    c = C.c_void_p()
    # the closure replaces a return map, which the elastic model does not have
    assert lib.zsmpm_closure_create(C.byref(mat), 0, C.byref(c)) == zs._abi.ERR_INVALID_ARG
    assert lib.zsmpm_closure_train(None, 1, 32, C.c_float(1e-3), 0, None, None) == zs._abi.ERR_INVALID_ARG
    assert lib.zsmpm_closure_destroy(None) == zs._abi.OK
    assert lib.zsmpm_version().startswith(b"zsmpm")


def test_no_device_is_reported(zs):
    if zs.device_count() > 0:
        pytest.skip("a GPU is visible")
    from zsmpm_b200 import scenes
    with pytest.raises(zs.ZsmpmError) as e:
        zs.Scene(scenes.small_scene())
    assert e.value.status == zs._abi.ERR_NO_DEVICE
