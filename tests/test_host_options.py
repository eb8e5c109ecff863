"""PETSc-style option files -> solver options of the GPU library (host only)."""
import pytest

from cfdsfemmpi_b200.stabfem import LU_SUBSTITUTE, solver_options_from_petsc


def test_petsc_defaults_and_gmres_options():
    kw = solver_options_from_petsc({"-ksp_type": "gmres", "-ksp_gmres_restart": "50", "-pc_type": "jacobi",
                                    "-ksp_rtol": "1.e-10"})
    assert (kw["restart"], kw["pc"], kw["rtol"], kw["precision"]) == (50, "jacobi", 1e-10, "fp64")
    assert kw["atol"] == 1e-50 and kw["dtol"] == 1e4 and kw["max_it"] == 10000
    assert "guess" not in kw and kw["_notes"] == []


def test_direct_solver_is_substituted_and_reported():
    kw = solver_options_from_petsc({"-ksp_type": "preonly", "-pc_type": "lu", "-ksp_rtol": "1e-3"})
    for k, v in LU_SUBSTITUTE.items():
        assert kw[k] == v
    assert kw["_notes"]


def test_gpu_keys():
    kw = solver_options_from_petsc({"-gpu_precision": "mixed", "-gpu_inner_restart": "100", "-gpu_inner_rtol": "1e-3",
                                    "-gpu_reuse_tangent": "0", "-gpu_refine_rtol": "1e-9",
                                    "-gpu_newton_rtol": "1e-2", "-gpu_guess": "Extrapolation",
                                    "-gpu_formulation": "fully_implicit",
                                    "-pc_type": "bjacobi"})
    assert kw["precision"] == "mixed" and kw["inner_restart"] == 100 and kw["inner_rtol"] == 1e-3
    assert kw["reuse_tangent"] is False and kw["refine_rtol"] == 1e-9 and kw["newton_rtol"] == 1e-2
    assert kw["guess"] == "extrapolation" and kw["pc"] == "pbjacobi" and kw["_notes"]
    assert kw["formulation"] == "fully_implicit"


@pytest.mark.parametrize("pc", ["none", "jacobi", "pbjacobi"])
def test_preconditioners_pass_through(pc):
    assert solver_options_from_petsc({"-pc_type": pc})["pc"] == pc
