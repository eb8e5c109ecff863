"""GPU parity of the reference's iterative and direct option families.

The reference reads its Krylov method and preconditioner from a PETSc options
file (SolverPetsc.cpp:101,111): GMRES(20) or BiCGStab with block Jacobi and
ILU(3) sub-solves (input/petsc_options_gmres.dat, input/petsc_options_bcgs.dat)
and, in its tests, preonly + LU (testdata/*/petsc_options.dat).  The library
runs these as block ILU(k) on the nodal-block matrix, BiCGStab with PETSc
KSPBCGS semantics, and the complete block factorisation with preonly.  The
oracle runs the scalar restatements on the free-dof CSR.

Tolerances:
  * preconditioner application z = M^-1 r: relative L2 1e-10 (block and
    scalar factorisations are equal in exact arithmetic; the difference is
    rounding amplified by cond(M));
  * fields after N steps with the same solver options: relative L2 1e-8;
  * BiCGStab / GMRES iteration counts: within 2 of the oracle's on every solve;
  * shipped known-answer tests: the reference's own check (1e-4 per node) and
    1e-7 max difference to the shipped values.
"""
import os

import numpy as np
import pytest

import oracle
from cfdsfemmpi_b200 import Handle, StabFEM, io, meshgen

pytestmark = pytest.mark.gpu


def _distorted(mesh, amp, seed):
    rng = np.random.default_rng(seed)
    m = io.Mesh(ndim=mesh.ndim, npElem=mesh.npElem, coords=mesh.coords.copy(), conn=mesh.conn, dbc=mesh.dbc,
                output_nodes=mesh.output_nodes)
    m.coords += amp / 40 * rng.uniform(-1, 1, m.coords.shape)
    return m


MESHES = {
    "quad4": lambda: _distorted(meshgen.cavity2d(9), 0.3, 1),
    "hex8": lambda: _distorted(meshgen.cavity3d(5), 0.1, 2),
}


def _same_state(mesh, ctrl, seed, **okw):
    """Oracle assembled from a random state (the GPU handle is given the same)."""
    ref = oracle.OracleFEM(mesh, ctrl, **okw)
    ref.td = oracle.time_params(ctrl.tis, ctrl.rhoInf, ctrl.dt)
    rng = np.random.default_rng(seed)
    ref.soln = rng.uniform(-0.5, 0.5, ref.soln.shape)
    ref.solnDot = rng.uniform(-0.5, 0.5, ref.soln.shape)
    ref.time_update()
    ref.update_iter_step()
    ref.assemble(1)
    return ref


@pytest.mark.parametrize("kind", list(MESHES))
@pytest.mark.parametrize("levels,blocks", [(0, 1), (1, 1), (2, 1), (1, 3), (-1, 1)])
def test_preconditioner_matches_oracle(kind, levels, blocks):
    """M^-1 r of the GPU block ILU(k) / block LU against the oracle's scalar
    ILU(k) on the free-dof matrix (same block partition)."""
    mesh = MESHES[kind]()
    ctrl = meshgen.control_for(5, 0.1, 0.01)
    olev = levels if levels >= 0 else 10 ** 6
    ref = _same_state(mesh, ctrl, 3, solver="gmres", pc="bjacobi", ilu_levels=olev, bjacobi_blocks=blocks)
    ref.factor_ilu()
    h = Handle(mesh, ctrl, pc="bjacobi", ilu_levels=levels, bjacobi_blocks=blocks)
    h.set_element_state(ref.solnPrev, ref.solnCur, ref.solnDotCur)
    h.assemble_export(1, want_values=False)
    rng = np.random.default_rng(9)
    free = ref.assyForSoln
    fixed = np.setdiff1d(np.arange(h.n), free)
    for _ in range(2):
        r = np.zeros(h.n)
        r[free] = rng.standard_normal(len(free))
        z = h.pc_apply(r)
        z_ref = np.zeros(ref.ntot)
        oracle.lib().orc_ilu_apply(np.ascontiguousarray(r[free]), z_ref, 1)
        rel = np.linalg.norm(z[free] - z_ref) / np.linalg.norm(z_ref)
        assert rel < 1e-10, (kind, levels, blocks, rel)
        assert np.all(z[fixed] == 0.0)
    f = h.ilu_factors(values=False)
    assert np.all(np.diff(f["rowptr"]) >= 1) and np.all(f["colidx"][f["diag"]] == np.arange(mesh.nNode))
    h.close()


def test_factorisation_is_deterministic():
    mesh = MESHES["hex8"]()
    ctrl = meshgen.control_for(5, 0.1, 0.001)
    ref = _same_state(mesh, ctrl, 4, solver="lu")
    out = []
    for _ in range(2):
        h = Handle(mesh, ctrl, pc="bjacobi", ilu_levels=1)
        h.set_element_state(ref.solnPrev, ref.solnCur, ref.solnDotCur)
        h.assemble_export(1, want_values=False)
        for _ in range(2):
            f = h.ilu_factors()
            out.append((f["vals"].copy(), f["dinv"].copy()))
        h.close()
    for v, d in out[1:]:
        assert np.array_equal(v, out[0][0]) and np.array_equal(d, out[0][1])


def _run_gpu(mesh, ctrl, steps=None, **kw):
    h = Handle(mesh, ctrl, **kw)
    timeNow = ctrl.dt
    stats = []
    n = ctrl.stepsMax if steps is None else steps
    for _ in range(n):
        tf = timeNow if timeNow <= 1.0 else 1.0
        stats.append(h.step(timeNow, tf).as_dict())
        timeNow = timeNow + ctrl.dt
    s = h.get_solution()
    h.close()
    return s, stats


@pytest.mark.parametrize("ksp,levels", [("bcgs", 0), ("bcgs", 1), ("gmres", 1)])
def test_ldc2d_ilu_krylov_matches_oracle(ksp, levels):
    """2D cavity configuration (20 steps, rtol 1e-10) with the reference's
    iterative option family, GPU against the oracle."""
    mesh, ctrl, _ = meshgen.CASES["ldc2d_10"]()
    ref = oracle.OracleFEM(mesh, ctrl, solver=ksp, restart=20, rtol=1e-10, pc="bjacobi", ilu_levels=levels)
    ref.solve()
    s, stats = _run_gpu(mesh, ctrl, ksp=ksp, restart=20, rtol=1e-10, pc="bjacobi", ilu_levels=levels)
    rel = np.linalg.norm(s - ref.soln) / np.linalg.norm(ref.soln)
    assert rel < 1e-8, rel
    assert all(st["converged"] for st in stats)
    its_gpu = [x for st in stats for x in st["ksp_its"]]
    its_ref = [x for st in ref.stats for x in st["gmres_its"]]
    assert len(its_gpu) == len(its_ref)
    assert max(abs(a - b) for a, b in zip(its_gpu, its_ref)) <= 2, (its_gpu, its_ref)


def test_ldc3d_bcgs_ilu_matches_oracle():
    """hex8 cavity 8^3, 4 steps, BiCGStab + ILU(0) at rtol 1e-10 on both sides."""
    mesh, ctrl, _ = meshgen.case_hex(8, 4)
    ref = oracle.OracleFEM(mesh, ctrl, solver="bcgs", rtol=1e-10, pc="bjacobi", ilu_levels=0, threads=4)
    ref.solve()
    s, stats = _run_gpu(mesh, ctrl, ksp="bcgs", rtol=1e-10, pc="bjacobi", ilu_levels=0)
    rel = np.linalg.norm(s - ref.soln) / np.linalg.norm(ref.soln)
    assert rel < 1e-8, rel
    its_gpu = [x for st in stats for x in st["ksp_its"]]
    its_ref = [x for st in ref.stats for x in st["gmres_its"]]
    assert len(its_gpu) == len(its_ref)
    assert max(abs(a - b) for a, b in zip(its_gpu, its_ref)) <= 2, (its_gpu, its_ref)


def test_preonly_lu_matches_oracle_lu_3d():
    """-ksp_type preonly -pc_type lu on the hex8 cavity 4^3: the complete
    block factorisation is a direct solve (against SuperLU in the oracle)."""
    mesh, ctrl, _ = meshgen.case_hex(4, 3)
    ref = oracle.OracleFEM(mesh, ctrl, solver="lu")
    ref.solve()
    s, stats = _run_gpu(mesh, ctrl, ksp="preonly", pc="bjacobi", ilu_levels=-1)
    rel = np.linalg.norm(s - ref.soln) / np.linalg.norm(ref.soln)
    assert rel < 1e-10, rel
    assert all(st["converged"] and st["newton_iters"] == 2 for st in stats)


def test_reference_option_files_through_driver(golden_dir, tmp_path):
    """The reference's input/petsc_options_bcgs.dat and _gmres.dat keys
    through the StabFEM driver on the 10x10 golden case (ILU(3) blocks),
    checked with the reference's own result check."""
    import shutil
    src = os.path.join(golden_dir, "ldc2dquad10")
    for f in os.listdir(src):
        shutil.copy(os.path.join(src, f), tmp_path / f)
    base = {"-pc_type": "bjacobi", "-sub_ksp_type": "preonly", "-sub_pc_type": "ilu",
            "-sub_pc_factor_levels": "3", "-sub_pc_factor_fill": "3", "-ksp_rtol": "1.e-10", "-ksp_max_it": "1000"}
    for opts in (dict(base, **{"-ksp_type": "bcgs"}), dict(base, **{"-ksp_type": "gmres", "-ksp_gmres_restart": "20"})):
        fem = StabFEM()
        fem.readInputData(str(tmp_path / "LDC2Dquad10"))
        fem.readControlParameters(str(tmp_path / "control-parameters-ldc-Re100.dat"))
        fem.setSolver(1, None, False, options=opts)
        assert "ILU(3)" in fem.solver_description()
        assert fem.solveFullyImplicit() == 0, fem.last_error
        assert fem.checkResult(str(tmp_path / "test-ldc-stru-nelem10-ref.dat")) == 0
        fem.deallocatePetscObjects()


def test_kat_ldc2dquad_mesh2_gpu(golden_dir, tmp_path):
    """The reference's 128x128 known-answer test (src/test-ldc-stru-mesh2.cpp:
    Re 1000, 10 passes of the time loop, preonly + LU) through the GPU StabFEM
    driver with the shipped options file."""
    import gzip
    import shutil
    src = os.path.join(golden_dir, "ldc2dquad-mesh2")
    for f in os.listdir(src):
        if f.endswith(".gz"):
            with gzip.open(os.path.join(src, f), "rb") as fi, open(tmp_path / f[:-3], "wb") as fo:
                shutil.copyfileobj(fi, fo)
        else:
            shutil.copy(os.path.join(src, f), tmp_path / f)
    fem = StabFEM()
    fem.readInputData(str(tmp_path / "LDC2Dquad-mesh2"))
    fem.readControlParameters(str(tmp_path / "control-parameters-Re1000.dat"))
    fem.setSolver(1, None, False, options=str(tmp_path / "petsc_options.dat"))
    assert "preonly" in fem.solver_description() and "LU" in fem.solver_description()
    assert fem.solveFullyImplicit() == 0, fem.last_error
    ref = str(tmp_path / "test-ldc-stru-mesh2-ref.dat")
    assert fem.checkResult(ref) == 0
    diff = np.abs(io.read_result(ref) - fem.solution().reshape(-1, 3)).max()
    assert diff < 1e-7, diff
    fem.deallocatePetscObjects()
