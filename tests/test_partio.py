"""Particle output (.bgeo) of zsmpm_write_partio*, the counterparts of zs::write_partio,
write_partio_with_stress and write_partio_with_grid (io/ParticleIO.hpp:11-22).  The partio
library that the reference writes through is not in its tree, so the files are checked
against the published layout of Houdini's classic binary geometry by a reader written here
(big-endian "Bgeo" V5 header, point attribute dictionary, points with homogeneous positions,
one particle-system primitive, the 0x00 0xff trailer).  CPU only: the writer needs no device."""
import struct

import numpy as np
import pytest


def read_bgeo(path):
    b = open(path, "rb").read()
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from(">" + fmt, b, off)
        off += struct.calcsize(">" + fmt)
        return v

    def string():
        (n,) = take("H")
        nonlocal off
        s = b[off:off + n].decode()
        off += n
        return s

    assert b[:4] == b"Bgeo"
    off = 4
    (v,) = take("c")
    assert v == b"V"
    (version,) = take("i")
    npts, nprims, npg, nprg, npa, nva, nprima, nda = take("8i")
    attrs = []
    for _ in range(npa):
        name = string()
        (size,) = take("H")
        (typ,) = take("i")
        take(f"{size}i")  # defaults
        attrs.append((name, size, typ))
    P = np.zeros((npts, 4), np.float32)
    vals = {name: np.zeros((npts, size), np.float32) for name, size, _ in attrs}
    for i in range(npts):
        P[i] = take("4f")
        for name, size, _ in attrs:
            vals[name][i] = take(f"{size}f")
    prim_attrs = []
    for _ in range(nprima):
        name = string()
        (size,) = take("H")
        (typ,) = take("i")
        (nstr,) = take("i")
        strs = [string() for _ in range(nstr)]
        prim_attrs.append((name, size, typ, strs))
    (ptype,) = take("i")
    (count,) = take("i")
    idx = take(f"{count}H" if count < 65536 else f"{count}i")
    (gen,) = take("i")
    trailer = b[off:off + 2]
    return {"version": version, "counts": (npts, nprims, npg, nprg, npa, nva, nprima, nda), "attrs": attrs,
            "P": P, "vals": vals, "prim_attrs": prim_attrs, "prim_type": ptype, "indices": np.array(idx),
            "generator": gen, "trailer": trailer, "size": len(b), "end": off + 2}


@pytest.mark.parametrize("n", [0, 1, 1000, 70000])
def test_write_partio_positions(zs, tmp_path, n):
    from zsmpm_b200 import partio
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    path = tmp_path / "p.bgeo"
    partio.write_partio(path, x)
    f = read_bgeo(path)
    assert f["version"] == 5
    assert f["counts"] == (n, 1, 0, 0, 0, 0, 1, 0)
    assert np.array_equal(f["P"][:, :3], x) and np.all(f["P"][:, 3] == 1.0)
    assert f["prim_attrs"] == [("generator", 1, 4, ["papi"])]
    assert f["prim_type"] == 0x8000 and np.array_equal(f["indices"], np.arange(n)) and f["generator"] == 0
    assert f["trailer"] == b"\x00\xff" and f["end"] == f["size"]


def test_write_partio_with_stress_and_grid(zs, tmp_path):
    from zsmpm_b200 import partio
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, (257, 3)).astype(np.float32)
    s = rng.uniform(0, 1e3, 257).astype(np.float32)
    fo = rng.normal(size=(257, 3)).astype(np.float32)
    partio.write_partio_with_stress(tmp_path / "s.bgeo", x, s)
    f = read_bgeo(tmp_path / "s.bgeo")
    assert f["attrs"] == [("stress", 1, 0)]
    assert np.array_equal(f["P"][:, :3], x) and np.array_equal(f["vals"]["stress"][:, 0], s)
    partio.write_partio_with_grid(tmp_path / "g.bgeo", x, fo)
    f = read_bgeo(tmp_path / "g.bgeo")
    assert f["attrs"] == [("force", 3, 5)]
    assert np.array_equal(f["P"][:, :3], x) and np.array_equal(f["vals"]["force"], fo)
    # another tag: a vector attribute of that name, positions zero
    partio.write_partio(tmp_path / "v.bgeo", fo, tag="velocity")
    f = read_bgeo(tmp_path / "v.bgeo")
    assert f["attrs"] == [("velocity", 3, 5)]
    assert np.array_equal(f["vals"]["velocity"], fo) and np.all(f["P"][:, :3] == 0)


def test_write_partio_rejects_other_formats(zs, tmp_path):
    from zsmpm_b200 import partio
    x = np.zeros((4, 3), np.float32)
    for name in ("p.bgeo.gz", "p.geo", "p"):
        with pytest.raises(zs.ZsmpmError) as e:
            partio.write_partio(tmp_path / name, x)
        assert e.value.status == zs._abi.ERR_INVALID_ARG


@pytest.mark.gpu
def test_scene_write_partio(zs, gpu, tmp_path):
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=0)
    p = scenes.generate(spec)
    with zs.Scene(spec, p) as sc:
        sc.run(2)
        out = sc.download()
        zs._abi.check(zs._abi.lib().zsmpm_scene_write_partio(sc.handle, str(tmp_path / "scene.bgeo").encode()),
                      "scene_write_partio")
    f = read_bgeo(tmp_path / "scene.bgeo")
    assert np.array_equal(f["P"][:, :3], out.x)
