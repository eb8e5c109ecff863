"""Learned Newton initial guess: trajectory collection, scaling and training.

The network itself (forward, backward, Adam) runs on the GPU in
csrc/mpnn.cu; this module drives it:

* ``collect_trajectory`` runs the plain solver (the library's own time step)
  from rest and keeps the nodal solution after every step;
* ``fit_scales`` picks per-component scales for u_n, u_n - u_{n-1} and the
  network's target, the correction over linear extrapolation
  u_{n+1} - 2 u_n + u_{n-1}, from that trajectory;
* ``train_guess`` adds the (u_{n-1}, u_n, u_{n+1}) samples and runs Adam.

``Mpnn.attach()`` then makes ``cfdgpu_step`` start Newton from
u_n + a1*(predicted increment) + a2*(u_n - u_{n-1}), the coefficients
minimising the iteration-0 residual exactly (the residual is affine in the
state), whenever that lowers it, and from the reference's constant
predictor otherwise.  The converged answer always comes from the unchanged
Newton-GMRES loop.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Tuple

import numpy as np

from ._lib import Handle, Mpnn


def collect_trajectory(mesh, ctrl, steps: int, **solver_kw) -> Tuple[List[np.ndarray], List[Dict]]:
    """Plain-solver states u_0 = 0, u_1, ..., u_steps and the step statistics."""
    h = Handle(mesh, ctrl, **solver_kw)
    traj = [np.zeros(mesh.nNode * mesh.ndof)]
    stats = []
    t = ctrl.dt
    for _ in range(steps):
        stats.append(h.step(t, t if t <= 1.0 else 1.0).as_dict())
        traj.append(h.get_solution())
        t = t + ctrl.dt
    h.close()
    return traj, stats


def fit_scales(traj: List[np.ndarray], ndof: int, floor: float = 1e-6) -> Tuple[np.ndarray, np.ndarray]:
    """Root-mean-square per component of u_n, u_n - u_{n-1} (features) and of
    u_{n+1} - 2 u_n + u_{n-1} (target)."""
    S = np.stack(traj)
    U = S[1:].reshape(len(traj) - 1, -1, ndof)
    D = np.diff(S, axis=0).reshape(len(traj) - 1, -1, ndof)
    su = np.maximum(np.sqrt(np.mean(U ** 2, axis=(0, 1))), floor)
    sd = np.maximum(np.sqrt(np.mean(D ** 2, axis=(0, 1))), floor)
    if len(traj) >= 3:
        D2 = np.diff(S, n=2, axis=0).reshape(len(traj) - 2, -1, ndof)
        s2 = np.maximum(np.sqrt(np.mean(D2 ** 2, axis=(0, 1))), floor * 1e-3)
    else:
        s2 = sd
    return np.concatenate([su, sd]).astype(np.float32), s2.astype(np.float32)


def train_guess(handle: Handle, traj: List[np.ndarray], iters: int = 2000, lr: float = 2e-3, seed: int = 0,
                first: int = 1, last: Optional[int] = None, net: Optional[Mpnn] = None) -> Tuple[Mpnn, List[float]]:
    """Train on samples n = first..last-1 of a trajectory (u_{n-1}, u_n -> u_{n+1})."""
    ndof = handle.ndof
    last = len(traj) - 1 if last is None else last
    m = net if net is not None else Mpnn(handle, seed=seed)
    in_s, out_s = fit_scales(traj[: last + 1], ndof)
    m.set_scales(in_s, out_s)
    for n in range(first, last):
        m.add_sample(traj[n - 1], traj[n], traj[n + 1])
    losses = []
    chunk = max(1, iters // 20)
    done = 0
    while done < iters:
        k = min(chunk, iters - done)
        losses.append(m.train(k, lr))
        done += k
    return m, losses
