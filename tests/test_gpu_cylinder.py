"""The reference's cylinder-wake input through the GPU StabFEM driver.

input/cylinder2d-blockmesh-Re100-GA2-rho0p0-dt0p1-SI.dat (12,675 nodes,
12,400 quads, Re 100, dt 0.1, gen-alpha rho_inf 0) with the reference's own
iterative option files, input/petsc_options_bcgs.dat (BiCGStab) and
input/petsc_options_gmres.dat (GMRES(20)), both with block Jacobi and ILU(3)
sub-solves.  The reference ships no solution for this case, so the GPU run is
compared with the oracle running the same solver from rest on one host thread
(OpenMP reductions combine in no fixed order, and BiCGStab's first solve from
rest is chaotic: oracle runs on eight threads took 283 to 325 iterations or
broke down when (r, r0) summed to exactly zero at rounding level, one thread
503).  Fields after the
first steps agree to max(1e-8, 2 x the distance between the oracle's
BiCGStab and GMRES answers), which measures how far rtol 1e-10 determines the
solution.  GMRES counts agree within max(3, 5 %) on every solve; BiCGStab's
within a factor of two on the first solve and max(3, 10 %) after it.
"""
import gzip
import os
import shutil

import numpy as np
import pytest

import oracle
from cfdsfemmpi_b200 import StabFEM

pytestmark = pytest.mark.gpu

CASE = "cylinder2d-blockmesh-Re100-GA2-rho0p0-dt0p1-SI"
STEPS = 4


def _unpack(golden_dir, dst):
    src = os.path.join(golden_dir, "cylinder2d-blockmesh")
    for f in os.listdir(src):
        with gzip.open(os.path.join(src, f), "rb") as fi, open(dst / f[:-3], "wb") as fo:
            shutil.copyfileobj(fi, fo)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("options", ["petsc_options_bcgs.dat", "petsc_options_gmres.dat"])
def test_reference_cylinder_with_its_option_files(golden_dir, tmp_path, options):
    _unpack(golden_dir, tmp_path)
    fem = StabFEM()
    fem.readInputData(str(tmp_path / CASE))
    fem.readControlParameters(str(tmp_path / "control-parameters-Re100-dt0p1.dat"))
    fem.setSolver(1, None, False, options=str(tmp_path / options))
    assert "ILU(3)" in fem.solver_description()
    assert fem.solveFullyImplicit(max_steps=STEPS) == 0, fem.last_error
    s_gpu = fem.solution()
    its_gpu = [st["ksp_its"] for st in fem.step_stats]
    kw = fem.solver_kw
    fem.deallocatePetscObjects()

    def run_oracle(ksp):
        okw = dict(solver=ksp, rtol=kw["rtol"], max_it=kw["max_it"], pc="bjacobi", ilu_levels=kw["ilu_levels"],
                   bjacobi_blocks=kw["bjacobi_blocks"], restart=20, threads=1)
        ref = oracle.OracleFEM(fem.mesh, fem.ctrl, **okw)
        ref.solve(STEPS)
        return ref.solution(), [st["gmres_its"] for st in ref.stats]

    s_ref, its_ref = run_oracle(kw["ksp"])
    s_other, _ = run_oracle("gmres" if kw["ksp"] == "bcgs" else "bcgs")
    spread = _rel(s_other, s_ref)
    err = _rel(s_gpu, s_ref)
    assert err <= max(1e-8, 2.0 * spread), (err, spread)
    assert [len(a) for a in its_gpu] == [len(b) for b in its_ref]
    rec = (its_gpu, its_ref)
    if kw["ksp"] == "gmres":
        assert all(abs(x - y) <= max(3, 0.05 * y) for a, b in zip(its_gpu, its_ref) for x, y in zip(a, b)), rec
    else:
        assert all(0.5 * y <= x <= 2.0 * y for x, y in zip(its_gpu[0], its_ref[0])), rec
        assert all(abs(x - y) <= max(3, 0.1 * y) for a, b in zip(its_gpu[1:], its_ref[1:]) for x, y in zip(a, b)), rec


def test_learned_guess_on_the_cylinder_wake():
    """The learned-guess configuration's O-grid (256 x 128 quads, Re 100,
    dt 0.1, seeded perturbation) with the reference's BiCGStab + ILU(3):
    the network trained on steps 12..24 of the plain solve (after the inflow
    ramp) predicts steps 25..28, which it has not seen.  Every held-out step
    takes the guess, whose iteration-0 residual is below the constant
    predictor's, and the fields stay those of the plain run (velocity to
    1e-6: each solve stops at rtol 1e-10 relative to its own start)."""
    from cfdsfemmpi_b200 import Handle, meshgen
    from cfdsfemmpi_b200.surrogate import train_guess
    mesh = meshgen.cylinder_ogrid()
    ctrl = meshgen.control_for(40, 0.1, 0.01)
    kw = dict(ksp="bcgs", pc="bjacobi", ilu_levels=3, rtol=1e-10, max_it=10000)
    u0 = meshgen.cylinder_initial_state(mesh)
    h0 = Handle(mesh, ctrl, **kw)
    h0.set_solution(u0)
    traj = [u0]
    t = ctrl.dt
    for _ in range(24):
        assert h0.step(t, min(t, 1.0)).as_dict()["converged"]
        traj.append(h0.get_solution())
        t = t + ctrl.dt
    prev, dot = h0.get_history()
    h0.close()
    out = {}
    for mode in (None, ("network",)):
        h = Handle(mesh, ctrl, **kw)
        h.set_solution(traj[-1])
        h.set_history(prev, dot)
        net = None
        if mode:
            net, losses = train_guess(h, traj, iters=1500, lr=2e-3, seed=0, first=12)
            assert losses[-1] < losses[0]
            net.attach(mode)
        tt, st = t, []
        for _ in range(4):
            st.append(h.step(tt, min(tt, 1.0)).as_dict())
            tt = tt + ctrl.dt
        out[mode] = (h.get_solution().reshape(-1, 3), st)
        if net is not None:
            net.close()
        h.close()
    (base, base_st), (guess, guess_st) = out[None], out[("network",)]
    assert all(s["converged"] for s in guess_st)
    assert all(s["guess_used"] and s["guess_norm"] < s["plain_norm"] for s in guess_st), guess_st
    rel = np.linalg.norm(guess[:, :2] - base[:, :2]) / np.linalg.norm(base[:, :2])
    assert rel < 1e-6, rel
