"""ctypes binding of the C ABI in include/cfdgpu.h (libcfdgpu.so, in-tree).

There is no CPU fallback: if the library is missing or cannot be loaded the
import of the GPU path raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcfdgpu.so")

# the symbols declared in include/cfdgpu.h, in declaration order
EXPORTS = [
    "cfdgpu_create", "cfdgpu_destroy", "cfdgpu_last_error", "cfdgpu_step", "cfdgpu_get_solution",
    "cfdgpu_set_solution", "cfdgpu_device_solution", "cfdgpu_stream", "cfdgpu_set_history", "cfdgpu_get_history",
    "cfdgpu_element_matrices", "cfdgpu_set_element_state", "cfdgpu_pattern_info_get", "cfdgpu_export_pattern",
    "cfdgpu_pattern_build", "cfdgpu_ilu_pattern_build", "cfdgpu_assemble_export", "cfdgpu_solve_export", "cfdgpu_timers", "cfdgpu_launch_count",
    "cfdgpu_set_profiling", "cfdgpu_kernel_stats", "cfdgpu_true_residual", "cfdgpu_residual_norm_noalloc",
    "cfdgpu_ilu_export", "cfdgpu_pc_apply_export",
    "cfdgpu_mpnn_create", "cfdgpu_mpnn_destroy", "cfdgpu_mpnn_num_params", "cfdgpu_mpnn_get_params",
    "cfdgpu_mpnn_set_params", "cfdgpu_mpnn_set_scales", "cfdgpu_mpnn_add_sample", "cfdgpu_mpnn_num_samples",
    "cfdgpu_mpnn_set_condition", "cfdgpu_mpnn_add_sample_on",
    "cfdgpu_mpnn_loss_grad", "cfdgpu_mpnn_train", "cfdgpu_mpnn_predict", "cfdgpu_set_guess_mode", "cfdgpu_set_guess",
    "cfdgpu_batch_create", "cfdgpu_batch_destroy", "cfdgpu_batch_last_error", "cfdgpu_batch_size",
    "cfdgpu_batch_handle", "cfdgpu_batch_set_schedule", "cfdgpu_batch_get_schedule", "cfdgpu_batch_step",
]
GUESS = {"network": 1, "network_velocity": 2, "extrapolation": 4}
FORM = {"semi_implicit": 0, "fully_implicit": 1}
KIND = {"spmv": 0, "elem_k": 1, "elem_f": 2, "ortho": 3, "trsv": 4, "ilu": 5, "bcgs": 6}

OK, EINVAL, ECUDA, ENEGJAC, EKSP, ENOMEM, ENODEV, ETOOBIG = 0, -1, -2, -3, -4, -5, -6, -7
PC = {"none": 0, "jacobi": 1, "pbjacobi": 2, "bjacobi": 3}
KSP = {"gmres": 0, "bcgs": 1, "preonly": 2}
PREC = {"fp64": 0, "mixed": 1}
MAX_NEWTON = 32


class Mesh(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("npElem", ctypes.c_int), ("nNode", ctypes.c_int), ("nElem", ctypes.c_int),
                ("coords", ctypes.c_void_p), ("conn", ctypes.c_void_p), ("nDBC", ctypes.c_int),
                ("dbc_node", ctypes.c_void_p), ("dbc_dof", ctypes.c_void_p), ("dbc_value", ctypes.c_void_p)]


class Control(ctypes.Structure):
    _fields_ = [("rho", ctypes.c_double), ("mu", ctypes.c_double), ("bodyforce", ctypes.c_double * 3),
                ("stab", ctypes.c_double * 3), ("tis", ctypes.c_int), ("rhoInf", ctypes.c_double),
                ("dt", ctypes.c_double), ("newton_tol", ctypes.c_double), ("newton_max_iter", ctypes.c_int)]


class SolverOpts(ctypes.Structure):
    _fields_ = [("restart", ctypes.c_int), ("rtol", ctypes.c_double), ("atol", ctypes.c_double),
                ("dtol", ctypes.c_double), ("max_it", ctypes.c_int), ("pc_type", ctypes.c_int),
                ("precision", ctypes.c_int), ("inner_restart", ctypes.c_int), ("inner_rtol", ctypes.c_double),
                ("reuse_tangent", ctypes.c_int), ("refine_rtol", ctypes.c_double), ("newton_rtol", ctypes.c_double),
                ("formulation", ctypes.c_int), ("ksp_type", ctypes.c_int), ("ilu_levels", ctypes.c_int),
                ("bjacobi_blocks", ctypes.c_int), ("refine_atol", ctypes.c_double)]


class StepStats(ctypes.Structure):
    _fields_ = [("newton_iters", ctypes.c_int), ("converged", ctypes.c_int),
                ("norms", ctypes.c_double * MAX_NEWTON), ("ksp_its", ctypes.c_int * MAX_NEWTON),
                ("ksp_reason", ctypes.c_int * MAX_NEWTON), ("refinements", ctypes.c_int * MAX_NEWTON),
                ("ms_assembly", ctypes.c_double), ("ms_solver", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("guess_used", ctypes.c_int), ("guess_norm", ctypes.c_double), ("plain_norm", ctypes.c_double),
                ("guess_alpha", ctypes.c_double), ("guess_alpha2", ctypes.c_double)]

    def as_dict(self) -> dict:
        n = self.newton_iters
        nsolve = n if not self.converged else n - 1
        return {"newton_iters": n, "converged": bool(self.converged), "norms": list(self.norms[:n]),
                "ksp_its": list(self.ksp_its[:nsolve]), "ksp_reason": list(self.ksp_reason[:nsolve]),
                "refinements": list(self.refinements[:nsolve]), "ms_assembly": self.ms_assembly,
                "ms_solver": self.ms_solver, "ms_total": self.ms_total, "guess_used": bool(self.guess_used),
                "guess_norm": self.guess_norm, "plain_norm": self.plain_norm, "guess_alpha": self.guess_alpha,
                "guess_alpha2": self.guess_alpha2}


class PatternInfo(ctypes.Structure):
    _fields_ = [("nNode", ctypes.c_int), ("nElem", ctypes.c_int), ("npElem", ctypes.c_int), ("ndof", ctypes.c_int),
                ("nnzb", ctypes.c_int64), ("ncolors", ctypes.c_int), ("nfixed", ctypes.c_int), ("nfree", ctypes.c_int)]


class IluInfo(ctypes.Structure):
    _fields_ = [("nNode", ctypes.c_int), ("nnzb", ctypes.c_int64), ("nchains_l", ctypes.c_int),
                ("nchains_u", ctypes.c_int), ("nlev_l", ctypes.c_int), ("nlev_u", ctypes.c_int),
                ("chain_levels_l", ctypes.c_int), ("chain_levels_u", ctypes.c_int)]


_LIB: Optional[ctypes.CDLL] = None


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Load libcfdgpu.so (building it with nvcc when absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH) and build_if_missing:
        from . import build as _build
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH}")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.cfdgpu_create.argtypes = [ctypes.POINTER(Mesh), ctypes.POINTER(Control), ctypes.POINTER(SolverOpts),
                                ctypes.POINTER(vp)]
    L.cfdgpu_destroy.argtypes = [vp]
    L.cfdgpu_last_error.argtypes = [vp]
    L.cfdgpu_last_error.restype = ctypes.c_char_p
    L.cfdgpu_step.argtypes = [vp, dp, dp, ctypes.POINTER(StepStats)]
    L.cfdgpu_get_solution.argtypes = [vp, vp]
    L.cfdgpu_set_solution.argtypes = [vp, vp]
    L.cfdgpu_device_solution.argtypes = [vp, ctypes.POINTER(vp)]
    L.cfdgpu_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.cfdgpu_set_history.argtypes = [vp, vp, vp]
    L.cfdgpu_get_history.argtypes = [vp, vp, vp]
    L.cfdgpu_element_matrices.argtypes = [vp, vp, ip, vp, vp]
    L.cfdgpu_set_element_state.argtypes = [vp, vp, vp, vp]
    L.cfdgpu_pattern_info_get.argtypes = [vp, ctypes.POINTER(PatternInfo)]
    L.cfdgpu_export_pattern.argtypes = [vp] + [vp] * 8
    L.cfdgpu_pattern_build.argtypes = [ctypes.POINTER(Mesh), ctypes.POINTER(PatternInfo)] + [vp] * 8
    L.cfdgpu_ilu_pattern_build.argtypes = [ctypes.POINTER(Mesh), ip, ip, ctypes.POINTER(IluInfo)] + [vp] * 9
    L.cfdgpu_assemble_export.argtypes = [vp, ip, vp, vp]
    L.cfdgpu_solve_export.argtypes = [vp, vp, vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.cfdgpu_timers.argtypes = [vp, vp]
    L.cfdgpu_true_residual.argtypes = [vp, vp, vp, ctypes.POINTER(ctypes.c_double)]
    L.cfdgpu_ilu_export.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), vp, vp, vp, vp, vp]
    L.cfdgpu_pc_apply_export.argtypes = [vp, vp, vp]
    L.cfdgpu_residual_norm_noalloc.argtypes = [ip, ip, vp, vp, vp, vp, vp, vp, vp]
    L.cfdgpu_mpnn_create.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.cfdgpu_mpnn_destroy.argtypes = [vp]
    L.cfdgpu_mpnn_num_params.argtypes = [vp]
    L.cfdgpu_mpnn_get_params.argtypes = [vp, vp]
    L.cfdgpu_mpnn_set_params.argtypes = [vp, vp]
    L.cfdgpu_mpnn_set_scales.argtypes = [vp, vp, vp]
    L.cfdgpu_mpnn_add_sample.argtypes = [vp, vp, vp, vp]
    L.cfdgpu_mpnn_set_condition.argtypes = [vp, dp]
    L.cfdgpu_mpnn_add_sample_on.argtypes = [vp, vp, dp, vp, vp, vp]
    L.cfdgpu_mpnn_num_samples.argtypes = [vp]
    L.cfdgpu_mpnn_loss_grad.argtypes = [vp, ip, vp, vp]
    L.cfdgpu_mpnn_train.argtypes = [vp, ip, ctypes.c_float, vp]
    L.cfdgpu_mpnn_predict.argtypes = [vp, vp, vp, vp]
    L.cfdgpu_set_guess.argtypes = [vp, vp]
    L.cfdgpu_set_guess_mode.argtypes = [vp, vp, ip]
    L.cfdgpu_batch_create.argtypes = [ip, ctypes.POINTER(Mesh), ctypes.POINTER(Control), ctypes.POINTER(SolverOpts),
                                      ctypes.POINTER(vp)]
    L.cfdgpu_batch_destroy.argtypes = [vp]
    L.cfdgpu_batch_last_error.argtypes = [vp]
    L.cfdgpu_batch_last_error.restype = ctypes.c_char_p
    L.cfdgpu_batch_size.argtypes = [vp]
    L.cfdgpu_batch_handle.argtypes = [vp, ip]
    L.cfdgpu_batch_handle.restype = vp
    L.cfdgpu_batch_set_schedule.argtypes = [vp, ip, ip, ip]
    L.cfdgpu_batch_get_schedule.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 4
    L.cfdgpu_batch_step.argtypes = [vp, vp, vp, ctypes.POINTER(StepStats), vp]
    L.cfdgpu_launch_count.argtypes = [vp]
    L.cfdgpu_launch_count.restype = ctypes.c_int64
    L.cfdgpu_set_profiling.argtypes = [vp, ip]
    L.cfdgpu_kernel_stats.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double)]
    for name in EXPORTS:
        if name not in ("cfdgpu_last_error", "cfdgpu_launch_count", "cfdgpu_batch_last_error", "cfdgpu_batch_handle"):
            getattr(L, name).restype = ctypes.c_int
    _LIB = L
    return L


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


_PATTERN_KEYS = ("rowptr", "colidx", "slot", "color", "color_ptr", "color_elems", "fixed_dofs", "dofmap")


def _pattern_arrays(pi) -> dict:
    return {"rowptr": np.zeros(pi.nNode + 1, np.int32), "colidx": np.zeros(max(pi.nnzb, 1), np.int32),
            "slot": np.zeros(pi.nElem * pi.npElem * pi.npElem, np.int32), "color": np.zeros(pi.nElem, np.int32),
            "color_ptr": np.zeros(pi.ncolors + 1, np.int32), "color_elems": np.zeros(pi.nElem, np.int32),
            "fixed_dofs": np.zeros(max(pi.nfixed, 1), np.int32), "dofmap": np.zeros(pi.nNode * pi.ndof, np.int32)}


def _mesh_struct(mesh):
    """(Mesh struct, keep-alive arrays) for a io.Mesh."""
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    conn = np.ascontiguousarray(mesh.conn, dtype=np.int32)
    dn = np.ascontiguousarray(mesh.dbc[:, 0], dtype=np.int32) if mesh.nDBC else np.zeros(1, np.int32)
    dd = np.ascontiguousarray(mesh.dbc[:, 1], dtype=np.int32) if mesh.nDBC else np.zeros(1, np.int32)
    dv = np.ascontiguousarray(mesh.dbc[:, 2], dtype=np.float64) if mesh.nDBC else np.zeros(1)
    m = Mesh(mesh.ndim, mesh.npElem, mesh.nNode, mesh.nElem, _ptr(coords), _ptr(conn), mesh.nDBC, _ptr(dn), _ptr(dd),
             _ptr(dv))
    return m, (coords, conn, dn, dd, dv)


def _control_opts(ctrl, restart=50, rtol=1e-10, atol=1e-50, dtol=1e4, max_it=10000, pc="jacobi", precision="fp64",
                  inner_restart=0, inner_rtol=1e-4, reuse_tangent=True, newton_tol=1e-8, newton_max_iter=10,
                  refine_rtol=1e-10, newton_rtol=0.0, formulation="semi_implicit", ksp="gmres", ilu_levels=0,
                  bjacobi_blocks=1, refine_atol=0.0):
    """(Control, SolverOpts) structs from an io.Control and solver keywords."""
    c = Control(ctrl.rho, ctrl.mu, (ctypes.c_double * 3)(*ctrl.bodyforce), (ctypes.c_double * 3)(*ctrl.stab),
                ctrl.tis, ctrl.rhoInf, ctrl.dt, newton_tol, newton_max_iter)
    o = SolverOpts(restart, rtol, atol, dtol, max_it, PC[pc], PREC[precision], inner_restart, inner_rtol,
                   1 if reuse_tangent else 0, refine_rtol, newton_rtol, FORM[formulation], KSP[ksp], ilu_levels,
                   bjacobi_blocks, refine_atol)
    return c, o


def pattern_build(mesh) -> dict:
    """Host-only pattern/colouring/slot-map build (cfdgpu_pattern_build); needs no GPU."""
    L = load()
    m, keep = _mesh_struct(mesh)
    pi = PatternInfo()
    rc = L.cfdgpu_pattern_build(ctypes.byref(m), ctypes.byref(pi), *([None] * 8))
    if rc != 0:
        raise CfdGpuError(rc, "pattern build failed")
    d = _pattern_arrays(pi)
    rc = L.cfdgpu_pattern_build(ctypes.byref(m), ctypes.byref(pi), *[_ptr(d[k]) for k in _PATTERN_KEYS])
    if rc != 0:
        raise CfdGpuError(rc, "pattern build failed")
    d["colidx"] = d["colidx"][:pi.nnzb]
    d["fixed_dofs"] = d["fixed_dofs"][:pi.nfixed]
    d["info"] = pi
    return d


def ilu_pattern_build(mesh, levels: int = 0, nblocks: int = 1) -> dict:
    """Host-only block ILU(k) symbolic phase and its schedules
    (cfdgpu_ilu_pattern_build); needs no GPU."""
    L = load()
    m, keep = _mesh_struct(mesh)
    info = IluInfo()
    rc = L.cfdgpu_ilu_pattern_build(ctypes.byref(m), levels, nblocks, ctypes.byref(info), *([None] * 9))
    if rc != 0:
        raise CfdGpuError(rc, "ILU pattern build failed")
    n = info.nNode
    d = {"rowptr": np.zeros(n + 1, np.int32), "colidx": np.zeros(max(info.nnzb, 1), np.int32),
         "perm": np.zeros(n, np.int32), "lorder": np.zeros(n, np.int32), "uorder": np.zeros(n, np.int32),
         "lchain": np.zeros(2 * max(info.nchains_l, 1), np.int32), "uchain": np.zeros(2 * max(info.nchains_u, 1), np.int32),
         "lchain_order": np.zeros(max(info.nchains_l, 1), np.int32),
         "uchain_order": np.zeros(max(info.nchains_u, 1), np.int32)}
    keys = ("rowptr", "colidx", "perm", "lorder", "uorder", "lchain", "uchain", "lchain_order", "uchain_order")
    rc = L.cfdgpu_ilu_pattern_build(ctypes.byref(m), levels, nblocks, ctypes.byref(info), *[_ptr(d[k]) for k in keys])
    if rc != 0:
        raise CfdGpuError(rc, "ILU pattern build failed")
    d["colidx"] = d["colidx"][:info.nnzb]
    d["lchain"] = d["lchain"][:2 * info.nchains_l].reshape(-1, 2)
    d["uchain"] = d["uchain"][:2 * info.nchains_u].reshape(-1, 2)
    d["lchain_order"] = d["lchain_order"][:info.nchains_l]
    d["uchain_order"] = d["uchain_order"][:info.nchains_u]
    d["info"] = info
    return d


class CfdGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cfdgpu error {code}: {msg}")
        self.code = code


class Handle:
    """Owning wrapper of a cfdgpu_handle."""

    def __init__(self, mesh, ctrl, restart: int = 50, rtol: float = 1e-10, atol: float = 1e-50, dtol: float = 1e4,
                 max_it: int = 10000, pc: str = "jacobi", precision: str = "fp64", inner_restart: int = 0,
                 inner_rtol: float = 1e-4, reuse_tangent: bool = True, newton_tol: float = 1e-8,
                 newton_max_iter: int = 10, refine_rtol: float = 1e-10, newton_rtol: float = 0.0,
                 guess: str = "constant", formulation: str = "semi_implicit", ksp: str = "gmres",
                 ilu_levels: int = 0, bjacobi_blocks: int = 1, refine_atol: float = 0.0):
        L = load()
        self._L = L
        self.h = ctypes.c_void_p()
        self._owned = True
        self._set_sizes(mesh)
        m, self._keep = _mesh_struct(mesh)
        c, o = _control_opts(ctrl, restart=restart, rtol=rtol, atol=atol, dtol=dtol, max_it=max_it, pc=pc,
                             precision=precision, inner_restart=inner_restart, inner_rtol=inner_rtol,
                             reuse_tangent=reuse_tangent, newton_tol=newton_tol, newton_max_iter=newton_max_iter,
                             refine_rtol=refine_rtol, newton_rtol=newton_rtol, formulation=formulation, ksp=ksp,
                             ilu_levels=ilu_levels, bjacobi_blocks=bjacobi_blocks, refine_atol=refine_atol)
        rc = L.cfdgpu_create(ctypes.byref(m), ctypes.byref(c), ctypes.byref(o), ctypes.byref(self.h))
        if rc != 0:
            msg = L.cfdgpu_last_error(self.h).decode() if self.h else "create failed"
            L.cfdgpu_destroy(self.h)
            self.h = ctypes.c_void_p()
            raise CfdGpuError(rc, msg)
        if guess == "extrapolation":
            self.set_guess_mode(("extrapolation",))
        elif guess != "constant":
            raise ValueError(f"guess must be 'constant' or 'extrapolation', not {guess!r}")

    def _set_sizes(self, mesh):
        self.ndim, self.npe = mesh.ndim, mesh.npElem
        self.ndof = mesh.ndim + 1
        self.nNode, self.nElem = mesh.nNode, mesh.nElem

    @classmethod
    def _borrow(cls, hptr, mesh, owner):
        """Non-owning view of a handle that another object (a Batch) owns."""
        self = cls.__new__(cls)
        self._L = load()
        self.h = ctypes.c_void_p(hptr)
        self._owned = False
        self._owner = owner
        self._set_sizes(mesh)
        return self

    def _check(self, rc: int):
        if rc != 0:
            raise CfdGpuError(rc, self._L.cfdgpu_last_error(self.h).decode())

    def close(self):
        if self.h and self._owned:
            self._L.cfdgpu_destroy(self.h)
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n(self) -> int:
        return self.nNode * self.ndof

    def step(self, timeNow: float, timeFact: float) -> StepStats:
        st = StepStats()
        rc = self._L.cfdgpu_step(self.h, timeNow, timeFact, ctypes.byref(st))
        if rc != 0:
            raise CfdGpuError(rc, self._L.cfdgpu_last_error(self.h).decode())
        return st

    def get_solution(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        out = np.empty(self.n) if out is None else out
        self._check(self._L.cfdgpu_get_solution(self.h, _ptr(out)))
        return out

    def set_solution(self, soln: np.ndarray):
        s = np.ascontiguousarray(soln, dtype=np.float64)
        self._check(self._L.cfdgpu_set_solution(self.h, _ptr(s)))

    def set_history(self, solnPrev=None, solnDot=None):
        a = None if solnPrev is None else np.ascontiguousarray(solnPrev, dtype=np.float64)
        b = None if solnDot is None else np.ascontiguousarray(solnDot, dtype=np.float64)
        self._check(self._L.cfdgpu_set_history(self.h, _ptr(a), _ptr(b)))

    def get_history(self):
        a, b = np.empty(self.n), np.empty(self.n)
        self._check(self._L.cfdgpu_get_history(self.h, _ptr(a), _ptr(b)))
        return a, b

    def set_solution_ptr(self, host_ptr: int):
        """H2D copy of soln from a raw host pointer (e.g. pinned memory)."""
        self._check(self._L.cfdgpu_set_solution(self.h, host_ptr))

    def get_solution_ptr(self, host_ptr: int):
        self._check(self._L.cfdgpu_get_solution(self.h, host_ptr))

    def stream_ptr(self) -> int:
        p = ctypes.c_void_p()
        self._check(self._L.cfdgpu_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def device_solution_ptr(self) -> int:
        p = ctypes.c_void_p()
        self._check(self._L.cfdgpu_device_solution(self.h, ctypes.byref(p)))
        return p.value or 0

    def set_element_state(self, prev, cur, dotcur):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (prev, cur, dotcur)]
        self._check(self._L.cfdgpu_set_element_state(self.h, *[_ptr(a) for a in arrs]))

    def element_matrices(self, elem_ids):
        ids = np.ascontiguousarray(elem_ids, dtype=np.int32)
        nsize = self.npe * self.ndof
        K = np.zeros((len(ids), nsize, nsize))
        F = np.zeros((len(ids), nsize))
        self._check(self._L.cfdgpu_element_matrices(self.h, _ptr(ids), len(ids), _ptr(K), _ptr(F)))
        return K, F

    def pattern_info(self) -> PatternInfo:
        pi = PatternInfo()
        self._check(self._L.cfdgpu_pattern_info_get(self.h, ctypes.byref(pi)))
        return pi

    def export_pattern(self) -> dict:
        pi = self.pattern_info()
        d = _pattern_arrays(pi)
        self._check(self._L.cfdgpu_export_pattern(self.h, *[_ptr(d[k]) for k in _PATTERN_KEYS]))
        d["colidx"] = d["colidx"][:pi.nnzb]
        d["fixed_dofs"] = d["fixed_dofs"][:pi.nfixed]
        d["info"] = pi
        return d

    def assemble_export(self, it: int = 0, want_values: bool = True):
        """Assemble the tangent and RHS of the current state; with
        want_values=False nothing is copied back (both returned as None)."""
        pi = self.pattern_info()
        if not want_values:
            self._check(self._L.cfdgpu_assemble_export(self.h, it, None, None))
            return None, None
        vals = np.zeros(pi.nnzb * pi.ndof * pi.ndof)
        rhs = np.zeros(self.n)
        self._check(self._L.cfdgpu_assemble_export(self.h, it, _ptr(vals), _ptr(rhs)))
        return vals.reshape(pi.nnzb, pi.ndof, pi.ndof), rhs

    def solve_export(self, b: np.ndarray):
        bb = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        its, reason = ctypes.c_int(), ctypes.c_int()
        self._check(self._L.cfdgpu_solve_export(self.h, _ptr(bb), _ptr(x), ctypes.byref(its), ctypes.byref(reason)))
        return x, its.value, reason.value

    def ilu_factors(self, values: bool = True) -> dict:
        """Block ILU factors of the last assembled matrix (pc='bjacobi'):
        rowptr, colidx, diag and, with values=True, the L/U blocks (nnzb x
        ndof x ndof) and the inverted diagonal blocks (nNode x ndof x ndof)."""
        nnzb = ctypes.c_int64()
        self._check(self._L.cfdgpu_ilu_export(self.h, ctypes.byref(nnzb), None, None, None, None, None))
        nb = self.ndof
        d = {"rowptr": np.zeros(self.nNode + 1, np.int32), "colidx": np.zeros(nnzb.value, np.int32),
             "diag": np.zeros(self.nNode, np.int32)}
        vals = np.zeros(nnzb.value * nb * nb) if values else None
        dinv = np.zeros(self.nNode * nb * nb) if values else None
        self._check(self._L.cfdgpu_ilu_export(self.h, None, _ptr(d["rowptr"]), _ptr(d["colidx"]), _ptr(d["diag"]),
                                              _ptr(vals), _ptr(dinv)))
        if values:
            d["vals"] = vals.reshape(-1, nb, nb)
            d["dinv"] = dinv.reshape(-1, nb, nb)
        return d

    def pc_apply(self, r: np.ndarray) -> np.ndarray:
        """z = M^-1 r with the preconditioner of the last assembled matrix."""
        rr = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros(self.n)
        self._check(self._L.cfdgpu_pc_apply_export(self.h, _ptr(rr), _ptr(z)))
        return z

    def true_residual(self, x: np.ndarray, b: np.ndarray) -> float:
        xx = np.ascontiguousarray(x, dtype=np.float64)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        out = ctypes.c_double()
        self._check(self._L.cfdgpu_true_residual(self.h, _ptr(xx), _ptr(bb), ctypes.byref(out)))
        return float(out.value)

    def timers(self) -> np.ndarray:
        t = np.zeros(5)
        self._check(self._L.cfdgpu_timers(self.h, _ptr(t)))
        return t

    def launch_count(self) -> int:
        return int(self._L.cfdgpu_launch_count(self.h))

    def set_guess_mode(self, mode=()):
        """Guess directions without a network (e.g. ("extrapolation",)); () = constant predictor."""
        flags = 0
        for k in mode:
            flags |= GUESS[k]
        self._check(self._L.cfdgpu_set_guess_mode(self.h, None, flags))

    def set_profiling(self, on: bool):
        self._check(self._L.cfdgpu_set_profiling(self.h, 1 if on else 0))

    def kernel_stats(self, kind: str):
        """(launches, total device ms, total algorithmic bytes) for a kernel kind
        since profiling was switched on."""
        n = ctypes.c_int64()
        ms = ctypes.c_double()
        by = ctypes.c_double()
        self._check(self._L.cfdgpu_kernel_stats(self.h, KIND[kind], ctypes.byref(n), ctypes.byref(ms),
                                                ctypes.byref(by)))
        return int(n.value), float(ms.value), float(by.value)


class Mpnn:
    """Learned Newton initial guess on a handle's mesh graph (cfdgpu_mpnn_*)."""

    def __init__(self, handle: Handle, seed: int = 0):
        self._L = handle._L
        self.handle = handle
        self.m = ctypes.c_void_p()
        rc = self._L.cfdgpu_mpnn_create(handle.h, seed, ctypes.byref(self.m))
        if rc != 0:
            self._L.cfdgpu_mpnn_destroy(self.m)
            self.m = ctypes.c_void_p()
            raise CfdGpuError(rc, "cfdgpu_mpnn_create failed")
        self.n = handle.n
        self.ndof = handle.ndof

    def _check(self, rc):
        if rc != 0:
            raise CfdGpuError(rc, "mpnn call failed")

    def close(self):
        if self.m:
            self._L.cfdgpu_mpnn_destroy(self.m)
            self.m = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_params(self) -> int:
        return int(self._L.cfdgpu_mpnn_num_params(self.m))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        self._check(self._L.cfdgpu_mpnn_get_params(self.m, _ptr(p)))
        return p

    def set_params(self, p):
        q = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self._L.cfdgpu_mpnn_set_params(self.m, _ptr(q)))

    def set_scales(self, in_scale, out_scale):
        a = np.ascontiguousarray(in_scale, dtype=np.float32)
        b = np.ascontiguousarray(out_scale, dtype=np.float32)
        self._check(self._L.cfdgpu_mpnn_set_scales(self.m, _ptr(a), _ptr(b)))

    def add_sample(self, u_nm1, u_n, u_np1, handle=None, cond=None):
        """A training sample (u_{n-1}, u_n -> u_{n+1}) on the network's own
        mesh, or on `handle`'s mesh (at most as many nodes) with condition
        value `cond`."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u_nm1, u_n, u_np1)]
        if handle is None:
            if cond is not None:
                self.set_condition(cond)
            self._check(self._L.cfdgpu_mpnn_add_sample(self.m, *[_ptr(a) for a in arrs]))
        else:
            self._check(self._L.cfdgpu_mpnn_add_sample_on(self.m, handle.h, float(cond or 0.0),
                                                          *[_ptr(a) for a in arrs]))

    def set_condition(self, cond: float):
        """Condition input channel for the own graph's samples and predictions."""
        self._check(self._L.cfdgpu_mpnn_set_condition(self.m, float(cond)))

    @property
    def num_samples(self) -> int:
        return int(self._L.cfdgpu_mpnn_num_samples(self.m))

    def loss_grad(self, sample: int):
        loss = np.zeros(1, np.float32)
        g = np.zeros(self.num_params, np.float32)
        self._check(self._L.cfdgpu_mpnn_loss_grad(self.m, sample, _ptr(loss), _ptr(g)))
        return float(loss[0]), g

    def train(self, iters: int, lr: float = 1e-3) -> float:
        loss = np.zeros(1, np.float32)
        self._check(self._L.cfdgpu_mpnn_train(self.m, iters, ctypes.c_float(lr), _ptr(loss)))
        return float(loss[0])

    def predict(self, u_nm1, u_n) -> np.ndarray:
        a = np.ascontiguousarray(u_nm1, dtype=np.float64)
        b = np.ascontiguousarray(u_n, dtype=np.float64)
        d = np.zeros(self.n)
        self._check(self._L.cfdgpu_mpnn_predict(self.m, _ptr(a), _ptr(b), _ptr(d)))
        return d

    def attach(self, mode=("network", "extrapolation")):
        """Use this network (and optionally the extrapolated increment) as the
        handle's Newton initial guess."""
        flags = 0
        for k in mode:
            flags |= GUESS[k]
        self._check(self._L.cfdgpu_set_guess_mode(self.handle.h, self.m, flags))

    def detach(self):
        self._check(self._L.cfdgpu_set_guess(self.handle.h, None))


class Batch:
    """Owning wrapper of a cfdgpu_batch: many independent instances (each an
    (io.Mesh, io.Control) pair with the same solver keywords) stepped
    concurrently on the current device."""

    def __init__(self, cases, guess: str = "constant", **solver_kw):
        L = load()
        self._L = L
        self.b = ctypes.c_void_p()
        self.cases = list(cases)
        n = len(self.cases)
        ms = (Mesh * n)()
        cs = (Control * n)()
        os_ = (SolverOpts * n)()
        self._keep = []
        for i, (mesh, ctrl) in enumerate(self.cases):
            m, keep = _mesh_struct(mesh)
            c, o = _control_opts(ctrl, **solver_kw)
            ms[i], cs[i], os_[i] = m, c, o
            self._keep.append(keep)
        rc = L.cfdgpu_batch_create(n, ms, cs, os_, ctypes.byref(self.b))
        if rc != 0:
            msg = L.cfdgpu_batch_last_error(self.b).decode() if self.b else "batch create failed"
            if self.b:
                L.cfdgpu_batch_destroy(self.b)
            self.b = ctypes.c_void_p()
            raise CfdGpuError(rc, msg)
        self.handles = [Handle._borrow(L.cfdgpu_batch_handle(self.b, i), mesh, self)
                        for i, (mesh, _) in enumerate(self.cases)]
        if guess == "extrapolation":
            for h in self.handles:
                h.set_guess_mode(("extrapolation",))
        elif guess != "constant":
            raise ValueError(f"guess must be 'constant' or 'extrapolation', not {guess!r}")

    def __len__(self):
        return len(self.cases)

    def _check(self, rc):
        if rc != 0:
            raise CfdGpuError(rc, self._L.cfdgpu_batch_last_error(self.b).decode())

    def set_schedule(self, concurrency: int = 0, chunk: int = 0, depth: int = 0):
        """(0, 0, 0): autotune over the next batch steps."""
        self._check(self._L.cfdgpu_batch_set_schedule(self.b, concurrency, chunk, depth))

    def schedule(self):
        v = [ctypes.c_int() for _ in range(4)]
        self._check(self._L.cfdgpu_batch_get_schedule(self.b, *[ctypes.byref(x) for x in v]))
        return {"concurrency": v[0].value, "chunk": v[1].value, "depth": v[2].value, "tuned": bool(v[3].value)}

    def step(self, times):
        """One step of every instance at times[i] (ramp factor min(t, 1)).
        Returns (list of StepStats, per-instance host latency in ms)."""
        n = len(self.cases)
        tn = np.ascontiguousarray(times, dtype=np.float64)
        tf = np.minimum(tn, 1.0)
        st = (StepStats * n)()
        lat = np.zeros(n)
        self._check(self._L.cfdgpu_batch_step(self.b, _ptr(tn), _ptr(tf), st, _ptr(lat)))
        return list(st), lat

    def close(self):
        if self.b:
            for h in self.handles:
                h.h = ctypes.c_void_p()
            self._L.cfdgpu_batch_destroy(self.b)
            self.b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
