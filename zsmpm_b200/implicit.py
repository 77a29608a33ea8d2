"""The implicit MPM system on a scene's grid: ImplicitMPMSystem (simulation/mpm/ImplicitMPM.hpp)
with the G2P2GTransfer force operator (simulation/transfer/G2P2G.hpp) and the conjugate-gradient
solve over it (math/linear/ConjugateGradient.hpp), each a launch sequence of libzsmpm.so.

Dof vectors are contiguous float32 CUDA tensors of `system.ndofs` entries, node-major over the
scene's active blocks in canonical order: entry (block*512 + cell)*3 + d, cell = x*64 + y*8 + z.
The scene must be binned for its current positions (activate_blocks + bin_particles), and every
operator but g2p2g reads the grid mass of a p2g of that activation.
"""
from __future__ import annotations

import ctypes as C

from . import _abi


def _stream(stream) -> C.c_void_p:
    if stream is None or stream == 0:
        return C.c_void_p(0)
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


class ImplicitMPMSystem:
    """ImplicitMPMSystem(simulator, dt, partI) (ImplicitMPM.hpp:13-15) for one scene."""

    def __init__(self, scene, dt: float):
        self.scene = scene
        self.dt = float(dt)
        self._lib = scene._lib

    @property
    def ndofs(self) -> int:
        return 1536 * self.scene.num_blocks()

    def zeros(self):
        import torch
        return torch.zeros(self.ndofs, dtype=torch.float32, device=f"cuda:{self.scene.device}")

    def _vec(self, t, name):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
        return C.c_void_p(t.data_ptr()), t.numel()

    def _n(self, *vecs):
        sizes = {v[1] for v in vecs}
        if len(sizes) != 1:
            raise ValueError("dof vectors differ in length")
        return sizes.pop()

    def g2p2g(self, v, f, stream=None) -> None:
        """G2P2GTransfer: adds the stress forces of the trial state of velocity field v to f."""
        pv, pf = self._vec(v, "v"), self._vec(f, "f")
        _abi.check(self._lib.zsmpm_g2p2g(self.scene.handle, pv[0], pf[0], self._n(pv, pf), self.dt,
                                         _stream(stream)), "g2p2g")

    def multiply(self, inp, out, stream=None) -> None:
        pi, po = self._vec(inp, "in"), self._vec(out, "out")
        _abi.check(self._lib.zsmpm_implicit_multiply(self.scene.handle, pi[0], po[0], self._n(pi, po), self.dt,
                                                     _stream(stream)), "implicit_multiply")

    def project(self, inout, stream=None) -> None:
        p = self._vec(inout, "inout")
        _abi.check(self._lib.zsmpm_implicit_project(self.scene.handle, p[0], p[1], _stream(stream)),
                   "implicit_project")

    def precondition(self, inp, out, stream=None) -> None:
        pi, po = self._vec(inp, "in"), self._vec(out, "out")
        _abi.check(self._lib.zsmpm_implicit_precondition(self.scene.handle, pi[0], po[0], self._n(pi, po),
                                                         _stream(stream)), "implicit_precondition")


class ConjugateGradient:
    """ConjugateGradient<float, 3> (ConjugateGradient.hpp:10-38): maxIters, tol, relTol."""

    def __init__(self, max_iters: int = 1000, tol: float = 1e-6, rel_tol: float = 0.5):
        self.max_iters = int(max_iters)
        self.tol = float(tol)
        self.rel_tol = float(rel_tol)

    def solve(self, system: ImplicitMPMSystem, x, b, stream=None) -> int:
        """x (in: guess, out: result) and b are dof vectors; returns the iteration count."""
        px, pb = system._vec(x, "x"), system._vec(b, "b")
        opts = _abi.CgOptions(self.max_iters, self.tol, self.rel_tol)
        iters = C.c_int32()
        _abi.check(system._lib.zsmpm_implicit_cg(system.scene.handle, px[0], pb[0], system._n(px, pb), system.dt,
                                                 C.byref(opts), C.byref(iters), _stream(stream)), "implicit_cg")
        return iters.value
