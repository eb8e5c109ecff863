"""``StabFEM`` host driver over the CUDA library.

Mirrors the public methods of the reference's driver class
(src/base/StabFEM.h:89-153) so a caller of the reference switches by changing
the import.  Input formats are the reference's (see io.py); the solver-options
file carries PETSc option names, with PETSc's defaults for a serial run:

  -ksp_type gmres|bcgs|preonly          -ksp_gmres_restart m (30)
  -ksp_rtol r (1e-5)  -ksp_atol a (1e-50)  -ksp_divtol d (1e4)  -ksp_max_it k (10000)
  -pc_type none|jacobi|pbjacobi|ilu|lu|bjacobi   (default ilu, PETSc's serial default)
  -pc_factor_levels k                   (-pc_type ilu, default 0)
  -sub_pc_type ilu|lu                   (-pc_type bjacobi, default ilu)
  -sub_pc_factor_levels k               (-pc_type bjacobi with ILU blocks, default 0)
  -pc_bjacobi_blocks B                  (default 1: one block per process, one process)

``-pc_type lu`` and ``-sub_pc_type lu`` are the library's complete block LU in
natural ordering (the ILU machinery without a level limit), so the reference's
tests (``-ksp_type preonly -pc_type lu``) run as direct solves; the
``-pc_factor_mat_solver_type`` package name (MUMPS in the reference) is
recorded but has no other effect.  An option value the library does not
implement raises ``io.InputError`` instead of being replaced by another method.

Library keys:

  -gpu_precision fp64|mixed   -gpu_inner_restart m    -gpu_inner_rtol r
  -gpu_reuse_tangent 0|1      -gpu_refine_rtol r      -gpu_refine_atol a
  -gpu_newton_rtol r
  -gpu_formulation semi_implicit|fully_implicit   (element routine; the
        reference's active one, or its commented-out fully-implicit one)
  -gpu_guess constant|extrapolation   (Newton initial guess; constant = the
                                       reference's, extrapolation = u_n plus
                                       the min-residual multiple of u_n - u_{n-1})
"""
from __future__ import annotations

import math
import os
import time
from typing import Dict, List, Optional

import numpy as np

from . import io
from ._lib import CfdGpuError, Handle


def solver_options_from_petsc(opts: Dict[str, str]) -> Dict:
    """PETSc option dictionary -> keyword arguments of Handle (with PETSc's
    defaults for a serial run).  Raises io.InputError for a method the library
    does not implement."""
    ksp = opts.get("-ksp_type", "gmres").lower()
    pc = opts.get("-pc_type", "ilu").lower()
    kw = {"restart": 30, "rtol": 1e-5, "atol": 1e-50, "dtol": 1e4, "max_it": 10000, "ksp": "gmres"}
    notes: List[str] = []
    if ksp not in ("gmres", "bcgs", "preonly"):
        raise io.InputError(f"-ksp_type {ksp} is not implemented (gmres, bcgs, preonly)")
    kw["ksp"] = ksp
    if pc in ("none", "jacobi", "pbjacobi"):
        kw["pc"] = pc
    elif pc in ("ilu", "lu"):
        kw.update(pc="bjacobi", bjacobi_blocks=1,
                  ilu_levels=-1 if pc == "lu" else int(opts.get("-pc_factor_levels", "0")))
    elif pc == "bjacobi":
        sub = opts.get("-sub_pc_type", "ilu").lower()
        if sub not in ("ilu", "lu"):
            raise io.InputError(f"-sub_pc_type {sub} is not implemented (ilu, lu)")
        sub_ksp = opts.get("-sub_ksp_type", "preonly").lower()
        if sub_ksp != "preonly":
            raise io.InputError(f"-sub_ksp_type {sub_ksp} is not implemented (preonly)")
        kw.update(pc="bjacobi", bjacobi_blocks=int(opts.get("-pc_bjacobi_blocks", "1")),
                  ilu_levels=-1 if sub == "lu" else int(opts.get("-sub_pc_factor_levels", "0")))
    else:
        raise io.InputError(f"-pc_type {pc} is not implemented (none, jacobi, pbjacobi, ilu, lu, bjacobi)")
    if "-pc_factor_mat_solver_type" in opts:
        notes.append(f"factorisation package {opts['-pc_factor_mat_solver_type']}: the library's block LU/ILU")
    if "-ksp_gmres_restart" in opts:
        kw["restart"] = int(opts["-ksp_gmres_restart"])
    for key, name, conv in (("-ksp_rtol", "rtol", float), ("-ksp_atol", "atol", float),
                            ("-ksp_divtol", "dtol", float), ("-ksp_max_it", "max_it", int)):
        if key in opts:
            kw[name] = conv(opts[key])
    kw["precision"] = opts.get("-gpu_precision", "fp64")
    if "-gpu_inner_restart" in opts:
        kw["inner_restart"] = int(opts["-gpu_inner_restart"])
    if "-gpu_inner_rtol" in opts:
        kw["inner_rtol"] = float(opts["-gpu_inner_rtol"])
    if "-gpu_reuse_tangent" in opts:
        kw["reuse_tangent"] = bool(int(opts["-gpu_reuse_tangent"]))
    if "-gpu_refine_rtol" in opts:
        kw["refine_rtol"] = float(opts["-gpu_refine_rtol"])
    if "-gpu_refine_atol" in opts:
        kw["refine_atol"] = float(opts["-gpu_refine_atol"])
    if "-gpu_newton_rtol" in opts:
        kw["newton_rtol"] = float(opts["-gpu_newton_rtol"])
    if "-gpu_guess" in opts:
        kw["guess"] = opts["-gpu_guess"].lower()
    if "-gpu_formulation" in opts:
        kw["formulation"] = opts["-gpu_formulation"].lower()
    kw["_notes"] = notes
    return kw


class StabFEM:
    """Driver with the reference's method names (src/base/StabFEM.h:89-153)."""

    def __init__(self, verbose: bool = False):
        self.verbose = verbose
        self.mesh: Optional[io.Mesh] = None
        self.ctrl: Optional[io.Control] = None
        self.handle: Optional[Handle] = None
        self.options: Dict[str, str] = {}
        self.solver_kw: Dict = {}
        self.infilename = ""
        self.fileCount = 0
        self.step_stats: List[Dict] = []
        self.computerTimePattern = 0.0
        self.computerTimeAssembly = 0.0
        self.computerTimeSolver = 0.0
        self.computerTimePostprocess = 0.0
        self.computerTimeTimeLoop = 0.0
        self.timeNow = 0.0
        self._soln_cache: Optional[np.ndarray] = None
        self.write_vtu = False
        self.write_forces = True
        self.last_error = ""

    def _print(self, *a):
        if self.verbose:
            print(*a)

    # -- pre-processor (StabFEM.cpp:80-386) --
    def readInputData(self, fname: str) -> None:
        self.infilename = fname
        self.mesh = io.read_mesh(fname)
        self._print(f" ndim = {self.mesh.ndim}\n nNode_global = {self.mesh.nNode}\n nElem_global = {self.mesh.nElem}")

    def readControlParameters(self, fname: str) -> None:
        self.ctrl = io.read_control(fname)

    def prepareInputData(self) -> None:
        if self.mesh is None:
            raise io.InputError("readInputData first")
        _ = self.mesh.elem_type   # validates (ndim, npElem) like the element factory

    def setSolver(self, slv: int = 1, parm=None, cIO: bool = False, options=None) -> int:
        """Build the device structures (StabFEM::setSolver, StabFEM2.cpp:10-29).

        ``options``: a PETSc options file path or an option dictionary (the
        reference reads the file through PetscInitialize)."""
        if isinstance(options, str):
            self.options = io.read_options(options)
        elif isinstance(options, dict):
            self.options = dict(options)
        kw = solver_options_from_petsc(self.options)
        self.solver_kw = kw
        args = {k: v for k, v in kw.items() if not k.startswith("_")}
        t0 = time.perf_counter()
        if self.handle is not None:
            self.handle.close()
        self.handle = Handle(self.mesh, self.ctrl, **args)
        self.computerTimePattern = time.perf_counter() - t0
        return 0

    def solver_description(self) -> str:
        k = self.solver_kw
        ksp = {"gmres": f"GMRES({k['restart']})", "bcgs": "BCGS", "preonly": "preonly"}[k["ksp"]]
        pc = k["pc"]
        if pc == "bjacobi":
            lev = k["ilu_levels"]
            sub = "LU" if lev < 0 else f"ILU({lev})"
            pc = f"bjacobi[{k['bjacobi_blocks']} x {sub}]"
        s = f"{ksp} pc={pc} rtol={k['rtol']:g} max_it={k['max_it']} precision={k['precision']}"
        if k.get("guess", "constant") != "constant":
            s += f" guess={k['guess']}"
        if k.get("formulation", "semi_implicit") != "semi_implicit":
            s += f" formulation={k['formulation']}"
        if k.get("_notes"):
            s += " [" + "; ".join(k["_notes"]) + "]"
        return s

    # -- solution phase (StabFEM2.cpp:593-832) --
    def solveFullyImplicit(self, max_steps: Optional[int] = None) -> int:
        c = self.ctrl
        h = self.handle
        timeNow = c.dt
        forces = None
        if self.write_forces and self.infilename:
            forces = open(self.infilename + "-forces.dat", "w")
        t_loop = time.perf_counter()
        nsteps = c.stepsMax if max_steps is None else min(max_steps, c.stepsMax)
        rc = 0
        for tstep in range(nsteps):
            self._print(" " + "=" * 68 + f"\n Time = {timeNow:f} \n " + "=" * 68)
            timeFact = timeNow if timeNow <= 1.0 else 1.0
            try:
                st = h.step(timeNow, timeFact).as_dict()
            except CfdGpuError as e:
                self.last_error = str(e)
                self._print(" PETSc solver not converged. \n\n" if e.code == -4 else str(e))
                rc = -1
                break
            st["time"] = timeNow
            self.step_stats.append(st)
            self.computerTimeAssembly += st["ms_assembly"] * 1e-3
            self.computerTimeSolver += st["ms_solver"] * 1e-3
            if self.verbose:
                for i, nrm in enumerate(st["norms"]):
                    print(f" Iteration = {i + 1}  \t RHS norm = {nrm:E} ")
            self._soln_cache = None
            if self.write_vtu:
                t0 = time.perf_counter()
                self.postProcess()
                self.computerTimePostprocess += time.perf_counter() - t0
            if forces is not None:
                # reaction forces are never filled in the reference (StabFEM2.cpp:808-815)
                forces.write(f"{timeNow:.14f}\t{0.0:.14f}\t{0.0:.14f}\n")
            timeNow = timeNow + c.dt
            self.timeNow = timeNow
            if timeNow > c.timeFinal:
                break
        if forces is not None:
            forces.close()
        self.computerTimeTimeLoop = time.perf_counter() - t_loop
        return rc

    # -- post-processing --
    def solution(self) -> np.ndarray:
        if self._soln_cache is None:
            self._soln_cache = self.handle.get_solution()
        return self._soln_cache

    def writeResult(self, fname: str) -> int:
        return io.write_result(fname, self.solution(), self.mesh.nNode, self.mesh.ndof)

    def checkResult(self, fname: str) -> int:
        return io.check_result(fname, self.solution(), self.mesh.nNode, self.mesh.ndim)

    def postProcess(self) -> None:
        from .vtu import write_vtu
        fname = f"{self.infilename}-{self.fileCount:06d}.vtu"
        write_vtu(fname, self.mesh, self.solution())
        self.fileCount += 1

    def printComputerTimes(self) -> int:
        lines = [
            "\n====================================================================\n",
            "\n       Computer time in seconds \n",
            "\n====================================================================\n",
            f"\n\n     (1) Matrix Pattern                  = {self.computerTimePattern:12.6f} \n",
            f"\n\n     (2) Matrix Assembly                 = {self.computerTimeAssembly:12.6f} \n",
            f"\n\n     (3) Matrix Solver                   = {self.computerTimeSolver:12.6f} \n",
            f"\n\n     (4) Post process                    = {self.computerTimePostprocess:12.6f} \n",
            f"\n\n     (5) Total time in time loop         = {self.computerTimeTimeLoop:12.6f} \n",
            f"\n\n     (6) Difference (5-2-3-4)            = "
            f"{self.computerTimeTimeLoop - self.computerTimeAssembly - self.computerTimeSolver - self.computerTimePostprocess:12.6f} \n",
            "\n\n====================================================================\n\n",
        ]
        print("".join(lines))
        return 0

    def deallocatePetscObjects(self) -> int:
        if self.handle is not None:
            self.handle.close()
            self.handle = None
        return 0
