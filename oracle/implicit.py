"""Test infrastructure: NumPy restatement of the implicit MPM system
(simulation/mpm/ImplicitMPM.hpp:13-159) and of ConjugateGradient::solve
(math/linear/ConjugateGradient.hpp:69-172), over the C restatement of G2P2GTransfer
(oracle_g2p2g_f32 / _f64).  It checks the CUDA path; the product never imports it.

Dof vectors hold 1536 values per block, node-major: entry (block*512 + cell)*3 + d.  `mass`
is the grid mass per node [nb, 512] (from a P2G of the same activation).  The float32 version
evaluates every expression in float32 in the reference's order.
"""
from __future__ import annotations

import numpy as np

from . import restated


def _node_mass(mass, dtype):
    return np.repeat(np.asarray(mass, dtype).reshape(-1), 3)


def multiply(spec, state, keys, mass, a, dt, precision: str = "f32"):
    """ImplicitMPMSystem::multiply (:34-61): out = G2P2G(a), then where m > 0,
    out = (out dt dt + m) a (ForceDtSqrPlusMass, :17-33)."""
    t = np.float32 if precision == "f32" else np.float64
    x, F, pl = state
    f = restated.g2p2g(spec, x, F, pl, keys, a, dt=dt, precision=precision).astype(t)
    m = _node_mass(mass, t)
    a = np.asarray(a, t).reshape(-1)
    dt_ = t(dt)
    out = f.copy()
    pos = m > 0
    out[pos] = (f[pos] * dt_ * dt_ + m[pos]) * a[pos]
    return out


def project(spec, keys, mass, a, precision: str = "f32"):
    """ImplicitMPMSystem::project (:99-124) with the six walls (Projector, :63-97;
    Collider::resolveCollision, geometry/Collider.h:80-110)."""
    t = np.float32 if precision == "f32" else np.float64
    out = np.asarray(a, t).reshape(-1, 512, 3).copy()
    mass = np.asarray(mass).reshape(-1, 512)
    keys = np.asarray(keys, np.int64).reshape(-1, 3)
    cell = np.arange(512)
    coord = np.stack([cell >> 6, (cell >> 3) & 7, cell & 7], 1)
    dx = t(spec.dx)
    pos = (keys[:, None, :] * 8 + coord[None]).astype(t) * dx
    has = mass > 0
    out[~has] = 0
    if spec.wall_type != 3:
        lo = t(spec.wall_cells) * dx
        hi = t(1) - t(spec.wall_cells) * dx
        for w in range(6):
            axis, upper = w >> 1, w & 1
            sgn = t(-1) if upper else t(1)
            sd = sgn * (pos[..., axis] - (hi if upper else lo))
            hit = has & (sd < 0)
            if spec.wall_type == 0:
                out[hit] = 0
            else:
                proj = sgn * out[..., axis]
                sel = hit if spec.wall_type == 1 else hit & (proj < 0)
                out[..., axis] = np.where(sel, out[..., axis] - proj * sgn, out[..., axis])
    return out.reshape(-1)


def precondition(mass, a, out, precision: str = "f32"):
    """ImplicitMPMSystem::precondition (:139-153; DivPernodeMass, :126-137): out = a / m where
    m > 0, other entries of out kept."""
    t = np.float32 if precision == "f32" else np.float64
    m = _node_mass(mass, t)
    out = np.asarray(out, t).reshape(-1).copy()
    pos = m > 0
    out[pos] = np.asarray(a, t).reshape(-1)[pos] / m[pos]
    return out


def cg_solve(spec, state, keys, mass, x0, b, dt, max_iters=1000, tol=1e-6, rel_tol=0.5,
             precision: str = "f32"):
    """ConjugateGradient::solve (:69-172) on the implicit system; q starts at zero.  Returns
    (x, iterations)."""
    t = np.float32 if precision == "f32" else np.float64
    x = np.asarray(x0, t).reshape(-1).copy()
    b = np.asarray(b, t).reshape(-1)
    dot = (lambda u, v: t(np.dot(u.astype(np.float64), v.astype(np.float64))))
    temp = multiply(spec, state, keys, mass, x, dt, precision)
    r = (b - temp).astype(t)
    r = project(spec, keys, mass, r, precision)
    q = precondition(mass, r, np.zeros_like(r), precision)
    p = q.copy()
    ztrk = dot(r, q)
    norm = t(np.sqrt(ztrk))
    local_tol = min(t(rel_tol) * norm, t(tol))
    it = 0
    while it != max_iters:
        if norm <= local_tol:
            break
        temp = multiply(spec, state, keys, mass, p, dt, precision)
        temp = project(spec, keys, mass, temp, precision)
        alpha = ztrk / dot(temp, p)
        x = (alpha * p + x).astype(t)
        r = (-alpha * temp + r).astype(t)
        q = precondition(mass, r, q, precision)
        last = ztrk
        ztrk = dot(q, r)
        beta = ztrk / last
        p = (beta * p + q).astype(t)
        norm = t(np.sqrt(ztrk))
        it += 1
    return x, it
