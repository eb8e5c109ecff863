"""Learned Newton initial guess: trajectory collection, scaling and training.

The network itself (forward, backward, Adam) runs on the GPU in
csrc/mpnn.cu; this module drives it:

* ``collect_trajectory`` runs the plain solver (the library's own time step)
  from rest and keeps the nodal solution after every step;
* ``fit_scales`` picks per-component scales for u_n, u_n - u_{n-1} and the
  network's target, the correction over linear extrapolation
  u_{n+1} - 2 u_n + u_{n-1}, from that trajectory;
* ``train_guess`` adds the (u_{n-1}, u_n, u_{n+1}) samples and runs Adam;
* ``train_shared`` trains one network on samples of many instances (each on
  its own mesh graph, with a condition value such as a scaled Reynolds
  number) and ``attach_shared`` gives every instance a network with those
  weights and its own condition.

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


def fit_scales_pooled(trajs: List[List[np.ndarray]], ndof: int, floor: float = 1e-6) -> Tuple[np.ndarray, np.ndarray]:
    """fit_scales over several instances' trajectories (meshes of any size):
    root-mean-square per component over every node and step of all of them."""
    su2 = np.zeros(ndof); sd2 = np.zeros(ndof); s22 = np.zeros(ndof)
    cu = cd = c2 = 0
    for traj in trajs:
        S = np.stack(traj)
        U = S[1:].reshape(len(traj) - 1, -1, ndof)
        D = np.diff(S, axis=0).reshape(len(traj) - 1, -1, ndof)
        su2 += (U ** 2).sum(axis=(0, 1)); cu += U.shape[0] * U.shape[1]
        sd2 += (D ** 2).sum(axis=(0, 1)); cd += D.shape[0] * D.shape[1]
        if len(traj) >= 3:
            D2 = np.diff(S, n=2, axis=0).reshape(len(traj) - 2, -1, ndof)
            s22 += (D2 ** 2).sum(axis=(0, 1)); c2 += D2.shape[0] * D2.shape[1]
    su = np.maximum(np.sqrt(su2 / max(cu, 1)), floor)
    sd = np.maximum(np.sqrt(sd2 / max(cd, 1)), floor)
    s2 = np.maximum(np.sqrt(s22 / c2), floor * 1e-3) if c2 else sd
    return np.concatenate([su, sd]).astype(np.float32), s2.astype(np.float32)


def train_shared(handles: List[Handle], trajs: List[List[np.ndarray]], conds: List[float], iters: int = 2000,
                 lr: float = 2e-3, seed: int = 0, first: int = 1) -> Tuple[Mpnn, Tuple, List[float]]:
    """One network for many instances: samples n = first..len-1 of every
    instance's trajectory, each on its own mesh graph and with its own
    condition value (e.g. a scaled Reynolds number), train the same weights.
    The network lives on the instance with the most nodes; returns it, the
    (params, in_scale, out_scale) to copy into each instance's network
    (attach_shared), and the training losses."""
    ndof = handles[0].ndof
    owner = max(range(len(handles)), key=lambda k: handles[k].n)
    m = Mpnn(handles[owner], seed=seed)
    in_s, out_s = fit_scales_pooled(trajs, ndof)
    m.set_scales(in_s, out_s)
    for k, (h, traj) in enumerate(zip(handles, trajs)):
        for n in range(first, len(traj) - 1):
            if k == owner:
                m.add_sample(traj[n - 1], traj[n], traj[n + 1], cond=conds[k])
            else:
                m.add_sample(traj[n - 1], traj[n], traj[n + 1], handle=h, cond=conds[k])
    losses = []
    chunk = max(1, iters // 20)
    done = 0
    while done < iters:
        k = min(chunk, iters - done)
        losses.append(m.train(k, lr))
        done += k
    return m, (m.get_params(), in_s, out_s), losses


def attach_shared(handle: Handle, shared: Tuple, cond: float, mode=("network", "extrapolation"), seed: int = 0) -> Mpnn:
    """A network on `handle` with the shared trained weights and this
    instance's condition value, attached as its Newton initial guess."""
    params, in_s, out_s = shared
    m = Mpnn(handle, seed=seed)
    m.set_scales(in_s, out_s)
    m.set_params(params)
    m.set_condition(cond)
    m.attach(mode)
    return m
