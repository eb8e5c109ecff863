"""Synthetic cases in the reference's input formats.

The reference ships only the two 2D cavity meshes; the 3D graded-cube cavity
and the other workloads are generated here with the shapes, boundary
conditions and physics of the named configurations:

* 2D cavity: unit square, n x n bilinear quads, node (i, j) = i + (n+1) j,
  counter-clockwise element nodes (the ordering of the reference's
  testdata/ldc2dquad10/LDC2Dquad10.dat).  Lid (1, 0) on y = 1 including both top
  corners, no-slip elsewhere, pressure pinned at a chosen node.
* 3D graded cube: n^3 trilinear hexes, x_i = 0.5 (1 + tanh(1.5 (2i/n - 1)) /
  tanh(1.5)) in each axis, node (i, j, k) = i + (n+1)(j + (n+1) k), element
  nodes in VTK hexahedron order (the order the reference hands to
  vtkHexahedron, src/base/StabFEM3.cpp:128-133).  Lid (1, 0, 0) on z = 1
  (including its edges), no-slip elsewhere, pressure pinned at the origin.
"""
from __future__ import annotations

import os
from typing import Optional, Tuple

import numpy as np

from .io import Control, Mesh, write_control, write_mesh, write_options


def graded(n: int, beta: float = 1.5) -> np.ndarray:
    i = np.arange(n + 1, dtype=np.float64)
    return 0.5 * (1.0 + np.tanh(beta * (2.0 * i / n - 1.0)) / np.tanh(beta))


def cavity2d(n: int, pin_node: int = 0, graded_beta: Optional[float] = None,
             lid: float = 1.0) -> Mesh:
    x = graded(n, graded_beta) if graded_beta else np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(x, x, indexing="xy")
    coords = np.stack([X.ravel(), Y.ravel()], axis=1)
    nid = lambda i, j: i + (n + 1) * j
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    ii = ii.ravel(); jj = jj.ravel()
    conn = np.stack([nid(ii, jj), nid(ii + 1, jj), nid(ii + 1, jj + 1), nid(ii, jj + 1)], axis=1).astype(np.int32)
    rows = []
    for node in range(coords.shape[0]):
        i, j = node % (n + 1), node // (n + 1)
        if j == n:
            rows += [(node, 0, lid), (node, 1, 0.0)]
        elif i == 0 or i == n or j == 0:
            rows += [(node, 0, 0.0), (node, 1, 0.0)]
    rows.append((pin_node, 2, 0.0))
    dbc = np.array(rows, dtype=np.float64)
    return Mesh(ndim=2, npElem=4, coords=coords, conn=conn, dbc=dbc,
                output_nodes=np.zeros(0, np.int32))


def cavity3d(n: int, beta: float = 1.5, lid: float = 1.0) -> Mesh:
    x = graded(n, beta)
    m = n + 1
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    coords = np.stack([x[i.ravel()], x[j.ravel()], x[k.ravel()]], axis=1)
    nid = lambda i, j, k: i + m * (j + m * k)
    ek, ej, ei = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ei = ei.ravel(); ej = ej.ravel(); ek = ek.ravel()
    conn = np.stack([nid(ei, ej, ek), nid(ei + 1, ej, ek), nid(ei + 1, ej + 1, ek), nid(ei, ej + 1, ek),
                     nid(ei, ej, ek + 1), nid(ei + 1, ej, ek + 1), nid(ei + 1, ej + 1, ek + 1),
                     nid(ei, ej + 1, ek + 1)], axis=1).astype(np.int32)
    I, J, K = i.ravel(), j.ravel(), k.ravel()
    nodes = np.arange(m ** 3)
    top = K == n
    wall = (I == 0) | (I == n) | (J == 0) | (J == n) | (K == 0)
    bnd = nodes[top | wall]
    is_top = top[bnd]
    dbc = np.zeros((3 * len(bnd) + 1, 3))
    dbc[0:-1:3, 0] = bnd; dbc[0:-1:3, 1] = 0; dbc[0:-1:3, 2] = np.where(is_top, lid, 0.0)
    dbc[1:-1:3, 0] = bnd; dbc[1:-1:3, 1] = 1
    dbc[2:-1:3, 0] = bnd; dbc[2:-1:3, 1] = 2
    dbc[-1] = (0, 3, 0.0)
    return Mesh(ndim=3, npElem=8, coords=coords, conn=conn, dbc=dbc,
                output_nodes=np.zeros(0, np.int32))


def control_for(steps: int, dt: float, mu: float, tis: int = 2, rhoInf: float = 0.0,
                rho: float = 1.0) -> Control:
    """Control with FinalTime past the last step so MaximumSteps governs."""
    return Control(rho=rho, mu=mu, bodyforce=(0.0, 0.0, 0.0), stab=(1.0, 1.0, 0.0), tis=tis,
                   rhoInf=rhoInf, dt=dt, timeFinal=steps * dt + dt, stepsMax=steps,
                   output_freq=1, tolerance=1e-6)


GMRES_OPTIONS = {"-ksp_type": "gmres", "-ksp_gmres_restart": "50", "-pc_type": "jacobi",
                 "-ksp_rtol": "1.e-10"}

# name -> (builder, control, options) for the configurations named by the
# benchmark description.  The 2D and 3D cavities start from rest.
CASES = {
    "cylinder": lambda: (cylinder_ogrid(), control_for(3000, 0.1, 0.01), dict(GMRES_OPTIONS)),
    "ldc2d_10": lambda: (cavity2d(10), control_for(20, 0.1, 0.01), dict(GMRES_OPTIONS)),
    "ldc3d_32": lambda: (cavity3d(32), control_for(50, 0.1, 0.001), dict(GMRES_OPTIONS)),
    "ldc3d_115": lambda: (cavity3d(115), control_for(20, 0.1, 0.001), dict(GMRES_OPTIONS)),
}


def case_hex(n: int, steps: int, mu: float = 0.001, dt: float = 0.1):
    return cavity3d(n), control_for(steps, dt, mu), dict(GMRES_OPTIONS)


def _geometric_ratio(n: int, r0: float, r1: float, dr0: float) -> float:
    """q with r0 + dr0 (q^n - 1)/(q - 1) = r1 (bisection)."""
    lo, hi = 1.0 + 1e-12, 2.0
    f = lambda q: r0 + dr0 * (q ** n - 1.0) / (q - 1.0) - r1
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def cylinder_ogrid(nt: int = 256, nr: int = 128, r_in: float = 0.5, r_out: float = 20.0,
                   dr0: float = 0.005) -> Mesh:
    """O-grid around a cylinder of diameter 2 r_in at the origin inside a
    circle of radius r_out: nt quads around, nr quads outward with geometric
    radial spacing starting at dr0.  Boundary conditions: no-slip on the
    cylinder, inflow (1, 0) on the outer arc where x < 0, traction-free
    (nothing prescribed) where x >= 0; no pressure pin (the free outflow fixes
    the pressure level).  Nodes are numbered ray by ray (i counter-clockwise
    from the +x axis), k outward within a ray.  (Ring-by-ring numbering
    would chain every row of an incomplete-LU factorisation in natural order
    to the one before it through the ring's closure, a dependency depth of
    the node count; ray by ray the depth is about nr + 2 nt.)"""
    q = _geometric_ratio(nr, r_in, r_out, dr0)
    r = r_in + dr0 * (q ** np.arange(nr + 1) - 1.0) / (q - 1.0)
    r[-1] = r_out
    th = 2.0 * np.pi * np.arange(nt) / nt
    TH, R = np.meshgrid(th, r, indexing="ij")          # (nt, nr+1)
    coords = np.stack([(R * np.cos(TH)).ravel(), (R * np.sin(TH)).ravel()], axis=1)
    nid = lambda i, k: k + (nr + 1) * (i % nt)
    kk, ii = np.meshgrid(np.arange(nr), np.arange(nt), indexing="ij")
    kk = kk.ravel(); ii = ii.ravel()
    # (radial, then tangential) edge order: counter-clockwise in (x, y)
    conn = np.stack([nid(ii, kk), nid(ii, kk + 1), nid(ii + 1, kk + 1), nid(ii + 1, kk)], axis=1).astype(np.int32)
    rows = []
    for i in range(nt):
        rows += [(nid(i, 0), 0, 0.0), (nid(i, 0), 1, 0.0)]
    for i in range(nt):
        node = nid(i, nr)
        if coords[node, 0] < 0.0:
            rows += [(node, 0, 1.0), (node, 1, 0.0)]
    dbc = np.array(rows, dtype=np.float64)
    return Mesh(ndim=2, npElem=4, coords=coords, conn=conn, dbc=dbc, output_nodes=np.zeros(0, np.int32))


def cylinder_initial_state(mesh: Mesh, amplitude: float = 1e-3, seed: int = 12345) -> np.ndarray:
    """Rest state with the transverse velocity perturbed by seeded uniform
    noise of the given amplitude (triggers vortex shedding)."""
    rng = np.random.default_rng(seed)
    u = np.zeros((mesh.nNode, 3))
    u[:, 1] = rng.uniform(-amplitude, amplitude, mesh.nNode)
    return u.ravel()


def batch_cases(count: int = 64, n_lo: int = 24, n_hi: int = 160, re_lo: float = 100.0, re_hi: float = 5000.0,
                dt: float = 0.05, steps: int = 100, seed: int = 2024):
    """Independent 2D lid-driven cavities of uneven size and Reynolds number:
    n ~ U{n_lo..n_hi} elements per side, log Re ~ U[log re_lo, log re_hi]
    (unit lid speed and side, rho 1, so mu = 1/Re), all from rest.
    Returns [(mesh, control, n, Re)]."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, count)
    res = np.exp(rng.uniform(np.log(re_lo), np.log(re_hi), count))
    return [(cavity2d(int(n)), control_for(steps, dt, 1.0 / float(re)), int(n), float(re)) for n, re in zip(ns, res)]


def write_case(directory: str, name: str, mesh: Mesh, ctrl: Control, opts: dict) -> Tuple[str, str, str]:
    """Write mesh/control/options files; returns (mesh prefix, control path, options path)."""
    os.makedirs(directory, exist_ok=True)
    prefix = os.path.join(directory, name)
    write_mesh(prefix, mesh)
    cpath = os.path.join(directory, name + "-control.dat")
    write_control(cpath, ctrl)
    opath = os.path.join(directory, name + "-options.dat")
    write_options(opath, opts)
    return prefix, cpath, opath
