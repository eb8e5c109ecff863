"""CPU oracle driver: the reference's time loop over the C restatement.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg, never by the product package.

Restates, file:line within the reference project:
  * StabFEM::prepareMatrixPattern free-dof numbering and assyForSoln
    (src/base/StabFEM2.cpp:57-81, 172-183)
  * StabFEM::solveFullyImplicit (src/base/StabFEM2.cpp:593-832): ramp
    (:636-644), assignBoundaryConditions (src/base/StabFEM.cpp:391-410),
    Newton loop (:654-799) with the absolute 1e-8 test and the 10-iteration
    cap, iteration-0 lifting and Dirichlet update (:678-730), solution update
    (:785-788), and the time update / break (:819-822)
  * SolutionData::timeUpdate / updateIterStep (src/base/SolutionData.cpp:64-91)
  * SetTimeParametersFluid (src/base/UtilitiesGeneral.cpp:5-205)

Linear solvers: ``lu`` (scipy SuperLU; stands in for the tests' MUMPS LU,
testdata/*/petsc_options.dat), ``gmres``, ``bcgs`` and ``preonly`` (oracle.c's
restatements of PETSc 3.10 KSPGMRES, KSPBCGS and KSPPREONLY) with the jacobi,
point-block jacobi or block-Jacobi ILU(k) preconditioner
(input/petsc_options_gmres.dat, input/petsc_options_bcgs.dat).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import time
from typing import Dict, List, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return path


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(build())
        L.orc_element.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                  ctypes.c_void_p]
        L.orc_element.restype = ctypes.c_int
        L.orc_element_fi.argtypes = L.orc_element.argtypes
        L.orc_element_fi.restype = ctypes.c_int
        L.orc_set_formulation.argtypes = [ctypes.c_int]
        L.orc_set_formulation.restype = None
        L.orc_pattern.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, _i32p,
                                  ctypes.c_int, _i32p, ctypes.c_void_p]
        L.orc_pattern.restype = ctypes.c_long
        L.orc_assemble.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, _f64p, _i32p, _f64p, _f64p,
                                   _f64p, _f64p, _f64p, _f64p, ctypes.c_int, ctypes.c_int, _i32p, _i32p,
                                   ctypes.c_long, _f64p, ctypes.c_int, _f64p, ctypes.c_int, _i32p, _i32p,
                                   ctypes.c_int]
        L.orc_assemble.restype = ctypes.c_int
        L.orc_gmres.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, ctypes.c_int, _f64p, _f64p, ctypes.c_int,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.orc_gmres.restype = ctypes.c_int
        L.orc_set_blocks.argtypes = [ctypes.c_int, _i32p]
        L.orc_set_blocks.restype = None
        L.orc_bcgs.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, ctypes.c_int, _f64p, _f64p,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.orc_bcgs.restype = ctypes.c_int
        L.orc_ilu_symbolic.argtypes = [ctypes.c_int, _i32p, _i32p, ctypes.c_int, _i32p, ctypes.c_int]
        L.orc_ilu_symbolic.restype = ctypes.c_long
        L.orc_ilu_numeric.argtypes = [_i32p, _i32p, _f64p, ctypes.c_int]
        L.orc_ilu_numeric.restype = ctypes.c_int
        L.orc_ilu_zero_pivot_row.argtypes = []
        L.orc_ilu_zero_pivot_row.restype = ctypes.c_int
        L.orc_ilu_apply.argtypes = [_f64p, _f64p, ctypes.c_int]
        L.orc_ilu_apply.restype = None
        L.orc_ilu_pattern.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_ilu_pattern.restype = None
        L.orc_ilu_values.argtypes = [_f64p]
        L.orc_ilu_values.restype = None
        L.orc_color.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, _i32p]
        L.orc_color.restype = ctypes.c_int
        L.orc_norm2.argtypes = [ctypes.c_int, _f64p]
        L.orc_norm2.restype = ctypes.c_double
        L.orc_spmv.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, ctypes.c_int]
        L.orc_spmv.restype = None
        _LIB = L
    return _LIB


ELEM_INFO = {0: (2, 3, 1), 1: (2, 4, 4), 2: (3, 4, 1), 3: (3, 8, 8)}  # ndim, npe, ngp


FORMULATIONS = {"semi_implicit": 0, "fully_implicit": 1}


def element(et: int, X, prev, cur, dotcur, elem_data, td, form: str = "semi_implicit"):
    """K (nsize x nsize) and F of one element; also (elemVol, charlen).
    form: "semi_implicit" (the reference's active type-B routine) or
    "fully_implicit" (its commented-out fully-implicit routine)."""
    ndim, npe, _ = ELEM_INFO[et]
    ndof = ndim + 1
    nsize = npe * ndof
    K = np.zeros(nsize * nsize)
    F = np.zeros(nsize)
    info = np.zeros(2)
    fn = lib().orc_element_fi if FORMULATIONS[form] else lib().orc_element
    rc = fn(et, np.ascontiguousarray(X, dtype=np.float64).ravel(),
                           np.ascontiguousarray(prev, dtype=np.float64).ravel(),
                           np.ascontiguousarray(cur, dtype=np.float64).ravel(),
                           np.ascontiguousarray(dotcur, dtype=np.float64).ravel(),
                           np.ascontiguousarray(elem_data, dtype=np.float64), np.ascontiguousarray(td, dtype=np.float64),
                           K, F, info.ctypes.data)
    return K.reshape(nsize, nsize), F, info, rc


def time_params(tis: int, rho: float, dt: float) -> np.ndarray:
    """SetTimeParametersFluid (src/base/UtilitiesGeneral.cpp:5-205)."""
    td = np.zeros(100)
    td[0] = dt
    if tis == 0:
        td[1] = 1.0; td[2] = 1.0; td[3] = 1.0; td[4] = 1.0
    elif tis == 1:
        alpf = 1.0 / (1.0 + rho); alpm = 1.0; gamm = 1.0
        td[1] = alpm; td[2] = alpf; td[3] = alpm; td[4] = gamm
        td[5] = alpf * dt; td[6] = alpm / gamm; td[7] = 1.0 - alpm / gamm; td[8] = 0.0
        td[9] = 1.0 / dt; td[10] = -td[9]; td[11] = 0.0; td[12] = 0.0; td[15] = 0.0
    elif tis in (2, 4):
        alpf = 1.0 / (1.0 + rho); alpm = 0.5 * (3.0 - rho) / (1.0 + rho); gamm = 0.5 + alpm - alpf
        td[1] = alpm; td[2] = alpf; td[3] = alpm; td[4] = gamm
        td[5] = alpf * dt; td[6] = alpm / gamm; td[7] = 1.0 - alpm / gamm; td[8] = alpm / gamm / dt
        td[9] = 1.0 / gamm / dt; td[10] = -td[9]; td[11] = 0.0; td[12] = 0.0; td[13] = 0.0
        td[15] = 1.0 - 1.0 / gamm
    elif tis in (3, 5, 6, 7):
        td[1] = 1.0; td[2] = 1.0; td[3] = 1.0; td[4] = 1.0
        td[5] = dt; td[6] = 1.0; td[7] = 0.0; td[8] = 1.0 / dt
        coef = {3: (1.0 / dt, -1.0 / dt, 0.0, 0.0, 0.0),
                5: (1.5 / dt, -2.0 / dt, 0.5 / dt, 0.0, 0.0),
                6: ((11.0 / 6.0) / dt, -3.0 / dt, 1.5 / dt, -(1.0 / 3.0) / dt, 0.0),
                7: ((25.0 / 12.0) / dt, -4.0 / dt, 3.0 / dt, -(4.0 / 3.0) / dt, (1.0 / 4.0) / dt)}[tis]
        td[9:14] = coef
        td[15] = 0.0
    return td


def bjacobi_rows(nNode: int, ndof: int, dofmap: np.ndarray, nblocks: int) -> np.ndarray:
    """Free-dof row offsets of the block-Jacobi blocks: nblocks contiguous node
    ranges (nNode // nblocks nodes each, the first nNode % nblocks ranges one
    more), each block starting at the first free row of its first node (the
    free numbering is node-major).  The CUDA library cuts its blocks by the
    same rule."""
    nb = max(1, min(int(nblocks), nNode))
    q, r = divmod(nNode, nb)
    node_start = np.array([b * q + min(b, r) for b in range(nb + 1)], dtype=np.int64)
    free = (dofmap.reshape(nNode, ndof) >= 0).sum(axis=1)
    first_row = np.r_[0, np.cumsum(free)]
    return np.ascontiguousarray(first_row[node_start].astype(np.int32))


class OracleFEM:
    """CPU restatement of StabFEM's serial hot path.

    solver: 'lu' or 'gmres'; gmres options follow PETSc names.
    threads: 1 runs the element loop in the reference's element order;
    >1 runs it colour by colour with OpenMP (same sums, fixed order).
    """

    def __init__(self, mesh, ctrl, solver: str = "gmres", restart: int = 50, rtol: float = 1e-10,
                 atol: float = 1e-50, dtol: float = 1e4, max_it: int = 10000, pc: str = "jacobi",
                 threads: int = 1, newton_tol: float = 1e-8, newton_max: int = 10, verbose: bool = False,
                 form: str = "semi_implicit", ilu_levels: int = 0, bjacobi_blocks: int = 1):
        self.mesh = mesh
        self.form = FORMULATIONS[form]
        self.ctrl = ctrl
        self.solver = solver
        self.restart, self.rtol, self.atol, self.dtol, self.max_it = restart, rtol, atol, dtol, max_it
        self.pc = {"none": 0, "jacobi": 1, "pbjacobi": 2, "bjacobi": 3}[pc]
        self.ilu_levels, self.bjacobi_blocks = ilu_levels, bjacobi_blocks
        self._ilu_ready = False
        self.threads = threads
        self.newton_tol, self.newton_max = newton_tol, newton_max
        self.verbose = verbose
        self.et = mesh.elem_type
        self.ndim, self.npe, _ = ELEM_INFO[self.et]
        self.ndof = self.ndim + 1
        nN = mesh.nNode
        self.conn = np.ascontiguousarray(mesh.conn, dtype=np.int32)
        self.coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
        self.elem_data = np.ascontiguousarray(ctrl.elem_data())
        # free-dof numbering, node-major (StabFEM2.cpp:57-81)
        fixed = np.zeros(nN * self.ndof, dtype=bool)
        dbcn = mesh.dbc[:, 0].astype(np.int64); dbcd = mesh.dbc[:, 1].astype(np.int64)
        self.dbc_index = dbcn * self.ndof + dbcd
        self.dbc_value = mesh.dbc[:, 2].copy()
        fixed[self.dbc_index] = True
        self.dofmap = np.full(nN * self.ndof, -1, dtype=np.int32)
        free = np.nonzero(~fixed)[0]
        self.dofmap[free] = np.arange(len(free), dtype=np.int32)
        self.assyForSoln = free.astype(np.int64)       # StabFEM2.cpp:172-183
        self.ntot = len(free)
        # point blocks: each node's free dofs (contiguous in node-major order)
        owner = free // self.ndof
        starts = np.nonzero(np.r_[True, owner[1:] != owner[:-1]])[0] if len(free) else np.zeros(0, np.int64)
        self.blk_ptr = np.ascontiguousarray(np.r_[starts, len(free)].astype(np.int32))
        # block-Jacobi blocks: contiguous node ranges cut at free-row offsets
        self.bj_rows = bjacobi_rows(nN, self.ndof, self.dofmap, bjacobi_blocks)
        L = lib()
        self.rowptr = np.zeros(self.ntot + 1, dtype=np.int32)
        nnz = L.orc_pattern(nN, self.ndof, mesh.nElem, self.npe, self.conn, self.dofmap, self.ntot,
                            self.rowptr, None)
        self.colidx = np.zeros(nnz, dtype=np.int32)
        L.orc_pattern(nN, self.ndof, mesh.nElem, self.npe, self.conn, self.dofmap, self.ntot, self.rowptr,
                      self.colidx.ctypes.data)
        self.nnz = int(nnz)
        self.vals = np.zeros(self.nnz)
        self.rhs = np.zeros(self.ntot)
        if threads > 1:
            color = np.zeros(mesh.nElem, dtype=np.int32)
            self.ncolors = L.orc_color(nN, mesh.nElem, self.npe, self.conn, color)
            order = np.argsort(color, kind="stable").astype(np.int32)
            self.color_elems = np.ascontiguousarray(order)
            self.color_ptr = np.zeros(self.ncolors + 1, dtype=np.int32)
            self.color_ptr[1:] = np.cumsum(np.bincount(color, minlength=self.ncolors))
        else:
            self.ncolors = 0
            self.color_elems = np.zeros(1, dtype=np.int32)
            self.color_ptr = np.zeros(1, dtype=np.int32)
        # SolutionData::initialise (SolutionData.cpp:16-35)
        n = nN * self.ndof
        z = lambda: np.zeros(n)
        self.soln, self.solnPrev, self.solnPrev2, self.solnPrev3, self.solnPrev4 = z(), z(), z(), z(), z()
        self.solnCur, self.solnDot, self.solnDotPrev, self.solnDotCur, self.solnApplied = z(), z(), z(), z(), z()
        self.td = np.zeros(100)
        self.timeNow = ctrl.dt
        self.stats: List[Dict] = []
        self.timers = {"assembly": 0.0, "solver": 0.0}
        self.steps_done = 0

    # ---- SolutionData ----
    def time_update(self):
        self.solnPrev4 = self.solnPrev3.copy()
        self.solnPrev3 = self.solnPrev2.copy()
        self.solnPrev2 = self.solnPrev.copy()
        self.solnPrev = self.soln.copy()
        self.solnDotPrev = self.solnDot.copy()

    def update_iter_step(self):
        td = self.td
        self.solnDot = (td[9] * self.soln + td[10] * self.solnPrev + td[11] * self.solnPrev2
                        + td[12] * self.solnPrev3 + td[13] * self.solnPrev4 + td[15] * self.solnDotPrev)
        self.solnCur = td[2] * self.soln + (1.0 - td[2]) * self.solnPrev
        self.solnDotCur = td[1] * self.solnDot + (1.0 - td[1]) * self.solnDotPrev

    def assemble(self, it: int, want_K: bool = True) -> int:
        lib().orc_set_formulation(self.form)
        return lib().orc_assemble(self.et, self.mesh.nNode, self.mesh.nElem, self.conn, self.coords, self.dofmap,
                                  self.solnPrev, self.solnCur, self.solnDotCur, self.solnApplied, self.elem_data,
                                  self.td, it, 1 if want_K else 0, self.rowptr, self.colidx, self.nnz, self.vals,
                                  self.ntot, self.rhs, self.ncolors, self.color_ptr, self.color_elems,
                                  self.threads)

    def csr(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.vals, self.colidx, self.rowptr), shape=(self.ntot, self.ntot))

    def factor_ilu(self):
        """Block-Jacobi ILU(k) factors of the current matrix (symbolic once)."""
        L = lib()
        if not self._ilu_ready:
            L.orc_ilu_symbolic(self.ntot, self.rowptr, self.colidx, len(self.bj_rows) - 1, self.bj_rows,
                               self.ilu_levels)
            self._ilu_ready = True
        if L.orc_ilu_numeric(self.rowptr, self.colidx, self.vals, self.threads) != 0:
            raise RuntimeError(f"zero pivot in ILU at row {L.orc_ilu_zero_pivot_row()}")

    def linear_solve(self):
        if self.solver == "lu":
            import scipy.sparse.linalg as spla
            x = spla.spsolve(self.csr().tocsc(), self.rhs)
            return x, {"its": 1, "reason": 0, "rnorm": 0.0}
        x = np.zeros(self.ntot)
        if self.pc == 2:
            lib().orc_set_blocks(len(self.blk_ptr) - 1, self.blk_ptr)
        if self.pc == 3:
            self.factor_ilu()
        its = ctypes.c_int(0)
        rn = ctypes.c_double(0.0)
        if self.solver == "preonly":
            # KSPSolve_PREONLY: one preconditioner application
            if self.pc != 3:
                raise ValueError("preonly is used with the bjacobi ILU/LU preconditioner")
            lib().orc_ilu_apply(np.ascontiguousarray(self.rhs), x, self.threads)
            return x, {"its": 1, "reason": 4, "rnorm": 0.0}
        if self.solver == "bcgs":
            reason = lib().orc_bcgs(self.ntot, self.rowptr, self.colidx, self.vals, self.pc, self.rhs, x,
                                    self.rtol, self.atol, self.dtol, self.max_it, ctypes.byref(its),
                                    ctypes.byref(rn), self.threads)
        else:
            reason = lib().orc_gmres(self.ntot, self.rowptr, self.colidx, self.vals, self.pc, self.rhs, x,
                                     self.restart, self.rtol, self.atol, self.dtol, self.max_it,
                                     ctypes.byref(its), ctypes.byref(rn), self.threads)
        return x, {"its": its.value, "reason": reason, "rnorm": rn.value}

    def step(self) -> Dict:
        """One pass of the time-loop body (StabFEM2.cpp:628-822)."""
        c = self.ctrl
        self.td = time_params(c.tis, c.rhoInf, c.dt)
        self.time_update()
        timeFact = self.timeNow if self.timeNow <= 1.0 else 1.0
        # assignBoundaryConditions
        self.solnApplied[self.dbc_index] = self.dbc_value * timeFact - self.soln[self.dbc_index]
        st = {"time": self.timeNow, "norms": [], "gmres_its": [], "reasons": [], "converged": False}
        for it in range(self.newton_max):
            self.update_iter_step()
            t0 = time.perf_counter()
            nneg = self.assemble(it)
            self.timers["assembly"] += time.perf_counter() - t0
            if nneg:
                raise RuntimeError("Negative Jacobian")
            if it == 0:
                # soln[d] += solnApplied[d] in DBC list order (StabFEM2.cpp:719-730)
                for k in range(len(self.dbc_index)):
                    j = self.dbc_index[k]
                    self.soln[j] += self.solnApplied[j]
            norm = lib().orc_norm2(self.ntot, self.rhs)
            st["norms"].append(norm)
            if self.verbose:
                print(f" Iteration = {it + 1}  \t RHS norm = {norm:E}")
            if norm < self.newton_tol:
                st["converged"] = True
                break
            t0 = time.perf_counter()
            x, info = self.linear_solve()
            self.timers["solver"] += time.perf_counter() - t0
            st["gmres_its"].append(info["its"])
            st["reasons"].append(info["reason"])
            if info["reason"] < 0:
                raise RuntimeError(f"KSP diverged, reason {info['reason']} after {info['its']} its")
            self.soln[self.assyForSoln] += x
        self.stats.append(st)
        self.steps_done += 1
        return st

    def solve(self, steps: Optional[int] = None) -> List[Dict]:
        """StabFEM::solveFullyImplicit's time loop."""
        c = self.ctrl
        n = c.stepsMax if steps is None else steps
        out = []
        for tstep in range(n):
            out.append(self.step())
            self.timeNow = self.timeNow + c.dt
            if self.timeNow > c.timeFinal:
                break
        return out

    def solution(self) -> np.ndarray:
        return self.soln.copy()
