"""Particle output as Houdini classic binary geometry (.bgeo), mirroring zs::write_partio,
zs::write_partio_with_stress and zs::write_partio_with_grid (io/ParticleIO.hpp:11-22): the
arrays go to the library's writer (zsmpm_write_partio*, include/zsmpm.h), which needs no
device."""
from __future__ import annotations

import numpy as np

from . import _abi


def _arr(a, cols):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.reshape(-1, cols) if cols > 1 else a.reshape(-1)


def write_partio(filename: str, data, tag: str = "position") -> None:
    """Points with `data` [n, 3] as positions (tag "position") or as a vector attribute `tag`."""
    d = _arr(data, 3)
    _abi.check(_abi.lib().zsmpm_write_partio(str(filename).encode(), d.ctypes.data, len(d), tag.encode()),
               "write_partio")


def write_partio_with_stress(filename: str, data, stress) -> None:
    """Positions [n, 3] and one float per point, the attribute "stress"."""
    d, s = _arr(data, 3), _arr(stress, 1)
    if len(s) != len(d):
        raise ValueError("one stress value per point")
    _abi.check(_abi.lib().zsmpm_write_partio_with_stress(str(filename).encode(), d.ctypes.data, s.ctypes.data,
                                                         len(d)), "write_partio_with_stress")


def write_partio_with_grid(filename: str, pos, force) -> None:
    """Positions [n, 3] and a vector per point, the attribute "force"."""
    p, f = _arr(pos, 3), _arr(force, 3)
    if len(p) != len(f):
        raise ValueError("one force per point")
    _abi.check(_abi.lib().zsmpm_write_partio_with_grid(str(filename).encode(), p.ctypes.data, f.ctypes.data,
                                                       len(p)), "write_partio_with_grid")
