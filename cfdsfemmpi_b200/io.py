"""Readers and writers for the reference's file formats.

Mesh file ``<prefix>.dat`` (StabFEM::readInputData, src/base/StabFEM.cpp:80-264):
keyword/value header (ndim, npElem, nNode, nElem, nDBC, nFBC, nOutputFaceLoads),
then ``nodes`` with ``id x y [z]`` rows, ``elements`` with
``id a b c n1 .. nk`` rows (1-based node ids in the last npElem columns), a
three-word Dirichlet header followed by ``node dof value`` rows (1-based), and
an ``outputnodes`` keyword followed by nOutputFaceLoads node ids.

Control file (StabFEM::readControlParameters, src/base/StabFEM.cpp:268-322):
eleven keyword/value lines read by position only.

Solver-options file: PETSc options, one ``-key [value]`` per line, as passed to
PetscInitialize (src/cfdsfemmpi.cpp:40).

Result file (StabFEM::writeResult / checkResult, src/base/StabFEM.cpp:457-554):
``nNode`` then one row of nodal values per node, ``%.8f``, tab separated.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional

import numpy as np


class InputError(RuntimeError):
    """Raised where the reference prints an error and calls exit()."""


@dataclasses.dataclass
class Mesh:
    ndim: int
    npElem: int
    coords: np.ndarray            # (nNode, ndim) float64
    conn: np.ndarray              # (nElem, npElem) int32, 0-based
    dbc: np.ndarray               # (nDBC, 3) float64: node (0-based), dof (0-based), value
    output_nodes: np.ndarray      # (nOutputFaceLoads,) int32, 0-based
    nFBC: int = 0
    prefix: str = ""

    @property
    def nNode(self) -> int:
        return int(self.coords.shape[0])

    @property
    def nElem(self) -> int:
        return int(self.conn.shape[0])

    @property
    def ndof(self) -> int:
        return self.ndim + 1

    @property
    def nDBC(self) -> int:
        return int(self.dbc.shape[0])

    @property
    def elem_type(self) -> int:
        """0 tri3, 1 quad4, 2 tet4, 3 hex8 (StabFEM::prepareInputData, StabFEM.cpp:351-366)."""
        if self.ndim == 2:
            if self.npElem == 3:
                return 0
            if self.npElem == 4:
                return 1
        else:
            if self.npElem == 4:
                return 2
            if self.npElem == 8:
                return 3
        raise InputError(f" Invalid npElem {self.npElem}")


@dataclasses.dataclass
class Control:
    """Control parameters in the reference's positional order.

    elemData layout as the reference fills it: [0] rho, [1] mu, [2..4] body
    force, [8..10] SUPG/PSPG/LSIC factors.  ``tolerance``, ``output_freq`` are
    read and kept but, as in the reference, not used by the time loop.
    """
    rho: float = 1.0
    mu: float = 0.01
    bodyforce: tuple = (0.0, 0.0, 0.0)
    stab: tuple = (1.0, 1.0, 0.0)
    tis: int = 2
    rhoInf: float = 0.0
    dt: float = 0.1
    timeFinal: float = 1.0
    stepsMax: int = 10
    output_freq: int = 1
    tolerance: float = 1e-6

    def elem_data(self) -> np.ndarray:
        ed = np.zeros(50)
        ed[0] = self.rho
        ed[1] = self.mu
        ed[2:5] = self.bodyforce
        ed[8:11] = self.stab
        return ed


def _exists(path: str) -> bool:
    return os.path.exists(path) or os.path.exists(path + ".gz")


def _tokens(path: str) -> List[str]:
    """Whitespace tokens of a text file; ``path.gz`` is read if ``path`` is absent."""
    if not os.path.exists(path) and os.path.exists(path + ".gz"):
        import gzip
        with gzip.open(path + ".gz", "rt") as f:
            return f.read().split()
    with open(path, "r") as f:
        return f.read().split()


def read_mesh(prefix: str) -> Mesh:
    """Parse ``prefix + '.dat'`` exactly as StabFEM::readInputData does."""
    fname = prefix + ".dat"
    if not _exists(fname):
        raise InputError("\n\n Could not open the input nodes file \n\n")
    tok = _tokens(fname)
    p = 0

    def kv():
        nonlocal p
        v = tok[p + 1]
        p += 2
        return v

    ndim = int(kv())
    npElem = int(kv())
    nNode = int(kv())
    nElem = int(kv())
    nDBC = int(kv())
    nFBC = int(kv())
    nOut = int(kv())
    p += 1  # "nodes"
    w = ndim + 1
    arr = np.array(tok[p:p + nNode * w], dtype=np.float64).reshape(nNode, w)
    p += nNode * w
    coords = np.ascontiguousarray(arr[:, 1:])
    p += 1  # "elements"
    if npElem not in (3, 4, 8):
        raise InputError(f" Invalid npElem {npElem}")
    w = 4 + npElem
    earr = np.array(tok[p:p + nElem * w], dtype=np.int64).reshape(nElem, w)
    p += nElem * w
    conn = np.ascontiguousarray(earr[:, 4:] - 1, dtype=np.int32)
    p += 3  # three-word Dirichlet header
    dbc = np.zeros((nDBC, 3))
    if nDBC:
        d = tok[p:p + 3 * nDBC]
        p += 3 * nDBC
        dbc[:, 0] = np.array(d[0::3], dtype=np.int64) - 1
        dbc[:, 1] = np.array(d[1::3], dtype=np.int64) - 1
        dbc[:, 2] = np.array(d[2::3], dtype=np.float64)
    p += 1  # "outputnodes"
    outn = np.array(tok[p:p + nOut], dtype=np.int64) - 1 if nOut else np.zeros(0, np.int64)
    return Mesh(ndim=ndim, npElem=npElem, coords=coords, conn=conn, dbc=dbc,
                output_nodes=outn.astype(np.int32), nFBC=nFBC, prefix=prefix)


def write_mesh(prefix: str, mesh: Mesh) -> None:
    """Write a mesh in the reference's input format."""
    lines = [f"ndim       {mesh.ndim}", f"npElem     {mesh.npElem}", f"nNode      {mesh.nNode}",
             f"nElem      {mesh.nElem}", f"nDBC       {mesh.nDBC}", f"nFBC       {mesh.nFBC}",
             f"nOutNodes  {len(mesh.output_nodes)}", "nodes"]
    ids = np.arange(1, mesh.nNode + 1)
    if mesh.ndim == 2:
        body = "\n".join(f"{i}\t{x:.17g}\t{y:.17g}" for i, (x, y) in zip(ids, mesh.coords))
    else:
        body = "\n".join(f"{i}\t{x:.17g}\t{y:.17g}\t{z:.17g}" for i, (x, y, z) in zip(ids, mesh.coords))
    lines.append(body)
    lines.append("elements")
    c1 = mesh.conn + 1
    lines.append("\n".join(f"{e + 1}\t1\t1\t1\t" + "\t".join(str(v) for v in row) for e, row in enumerate(c1)))
    lines.append("prescribed boundary conditions")
    lines.append("\n".join(f"{int(n) + 1}\t{int(d) + 1}\t{v:.17g}" for n, d, v in mesh.dbc))
    lines.append("outputnodes")
    if len(mesh.output_nodes):
        lines.append("\n".join(str(int(n) + 1) for n in mesh.output_nodes))
    with open(prefix + ".dat", "w") as f:
        f.write("\n".join(l for l in lines if l != "") + "\n")


def read_control(path: str) -> Control:
    """Positional read, StabFEM.cpp:285-315 (keywords are skipped)."""
    if not _exists(path):
        raise InputError(" Could not open 'control-parameters.dat' file ")
    t = _tokens(path)
    c = Control()
    c.rho = float(t[1])
    c.mu = float(t[3])
    c.bodyforce = (float(t[5]), float(t[6]), float(t[7]))
    c.stab = (float(t[9]), float(t[10]), float(t[11]))
    c.tis = int(t[13])
    c.rhoInf = float(t[15])
    c.dt = float(t[17])
    c.timeFinal = float(t[19])
    c.stepsMax = int(t[21])
    c.output_freq = int(t[23])
    c.tolerance = float(t[25])
    return c


def write_control(path: str, c: Control) -> None:
    rows = [("density", f"{c.rho!r}"), ("viscosity", f"{c.mu!r}"),
            ("bodyforce", " ".join(repr(float(v)) for v in c.bodyforce)),
            ("stabilisation", " ".join(repr(float(v)) for v in c.stab)),
            ("tis", str(c.tis)), ("rhoInf", repr(float(c.rhoInf))), ("dt", repr(float(c.dt))),
            ("FinalTime", repr(float(c.timeFinal))), ("MaximumSteps", str(c.stepsMax)),
            ("OutputFrequency", str(c.output_freq)), ("tolerance", repr(float(c.tolerance)))]
    with open(path, "w") as f:
        for k, v in rows:
            f.write(f"{k:<18}{v}\n")


def read_options(path: Optional[str]) -> Dict[str, str]:
    """PETSc options file -> {'-ksp_type': 'gmres', ...} (flags map to '')."""
    opts: Dict[str, str] = {}
    if path is None:
        return opts
    if not os.path.exists(path) and os.path.exists(path + ".gz"):
        import gzip
        with gzip.open(path + ".gz", "rt") as f:
            text = f.read()
    else:
        with open(path) as f:
            text = f.read()
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        parts = line.split()
        if not parts[0].startswith("-"):
            continue
        opts[parts[0]] = " ".join(parts[1:]) if len(parts) > 1 else ""
    return opts


def write_options(path: str, opts: Dict[str, str]) -> None:
    with open(path, "w") as f:
        for k, v in opts.items():
            f.write(f"{k} {v}\n" if v != "" else f"{k}\n")


def write_result(path: str, soln: np.ndarray, nNode: int, ndof: int) -> int:
    """StabFEM::writeResult (StabFEM.cpp:457-494): fixed, 8 decimals."""
    s = np.asarray(soln).reshape(nNode, ndof)
    with open(path, "w") as f:
        f.write(f"{nNode}\n")
        for row in s:
            f.write("\t".join(f"{v:.8f}" for v in row) + "\n")
    return 0


def read_result(path: str) -> np.ndarray:
    t = _tokens(path)
    n = int(t[0])
    vals = np.array(t[1:], dtype=np.float64)
    return vals.reshape(n, -1)


def check_result(path: str, soln: np.ndarray, nNode: int, ndim: int) -> int:
    """StabFEM::checkResult (StabFEM.cpp:501-554).

    Returns -1 on a node-count mismatch, -2 when some node's Euclidean (u,v,p)
    difference exceeds 1e-4 (2D), 0 otherwise.  As in the reference, 3D files
    are read but not compared.
    """
    if not _exists(path):
        raise InputError(" Could not open the file in 'StabFEM::checkResult' ... ")
    t = _tokens(path)
    if int(t[0]) != nNode:
        return -1
    ndof = ndim + 1
    if ndim != 2:
        return 0
    ref = np.array(t[1:1 + 3 * nNode], dtype=np.float64).reshape(nNode, 3)
    s = np.asarray(soln).reshape(nNode, ndof)
    d = ref - s[:, :3]
    for row in d:
        if math.sqrt(row[0] * row[0] + row[1] * row[1] + row[2] * row[2]) > 1.0e-4:
            return -2
    return 0
