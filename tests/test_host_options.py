"""PETSc-style option files -> solver options of the GPU library (host only)."""
import pytest

from cfdsfemmpi_b200 import io
from cfdsfemmpi_b200.stabfem import solver_options_from_petsc


def test_petsc_defaults_and_gmres_options():
    kw = solver_options_from_petsc({"-ksp_type": "gmres", "-ksp_gmres_restart": "50", "-pc_type": "jacobi",
                                    "-ksp_rtol": "1.e-10"})
    assert (kw["restart"], kw["pc"], kw["rtol"], kw["precision"], kw["ksp"]) == (50, "jacobi", 1e-10, "fp64", "gmres")
    assert kw["atol"] == 1e-50 and kw["dtol"] == 1e4 and kw["max_it"] == 10000
    assert "guess" not in kw and kw["_notes"] == []


def test_petsc_serial_default_preconditioner_is_ilu0():
    kw = solver_options_from_petsc({})
    assert (kw["ksp"], kw["pc"], kw["ilu_levels"], kw["bjacobi_blocks"], kw["restart"], kw["rtol"]) == \
        ("gmres", "bjacobi", 0, 1, 30, 1e-5)


def test_reference_iterative_option_files():
    # input/petsc_options_gmres.dat and input/petsc_options_bcgs.dat
    gm = {"-ksp_type": "gmres", "-pc_type": "bjacobi", "-sub_ksp_type": "preonly", "-sub_pc_type": "ilu",
          "-sub_pc_factor_levels": "3", "-sub_pc_factor_fill": "3", "-ksp_gmres_restart": "20",
          "-ksp_rtol": "1.e-10", "-ksp_max_it": "1000"}
    kw = solver_options_from_petsc(gm)
    assert (kw["ksp"], kw["pc"], kw["ilu_levels"], kw["bjacobi_blocks"], kw["restart"], kw["rtol"], kw["max_it"]) == \
        ("gmres", "bjacobi", 3, 1, 20, 1e-10, 1000)
    bc = dict(gm, **{"-ksp_type": "bcgs"})
    del bc["-ksp_gmres_restart"]
    kw = solver_options_from_petsc(bc)
    assert (kw["ksp"], kw["ilu_levels"]) == ("bcgs", 3)
    kw = solver_options_from_petsc(dict(gm, **{"-pc_bjacobi_blocks": "4"}))
    assert kw["bjacobi_blocks"] == 4


def test_direct_solver_is_a_complete_factorisation():
    # testdata/*/petsc_options.dat
    kw = solver_options_from_petsc({"-ksp_type": "preonly", "-pc_type": "lu", "-pc_factor_mat_solver_type": "mumps"})
    assert (kw["ksp"], kw["pc"], kw["ilu_levels"], kw["bjacobi_blocks"]) == ("preonly", "bjacobi", -1, 1)
    assert kw["_notes"]
    kw = solver_options_from_petsc({"-pc_type": "bjacobi", "-sub_pc_type": "lu", "-pc_bjacobi_blocks": "2"})
    assert (kw["ilu_levels"], kw["bjacobi_blocks"]) == (-1, 2)


@pytest.mark.parametrize("opts", [{"-ksp_type": "cg"}, {"-pc_type": "asm"}, {"-pc_type": "bjacobi", "-sub_pc_type": "icc"},
                                  {"-pc_type": "bjacobi", "-sub_ksp_type": "gmres"}])
def test_unimplemented_methods_are_refused(opts):
    with pytest.raises(io.InputError):
        solver_options_from_petsc(opts)


def test_gpu_keys():
    kw = solver_options_from_petsc({"-gpu_precision": "mixed", "-gpu_inner_restart": "100", "-gpu_inner_rtol": "1e-3",
                                    "-gpu_reuse_tangent": "0", "-gpu_refine_rtol": "1e-9",
                                    "-gpu_newton_rtol": "1e-2", "-gpu_guess": "Extrapolation",
                                    "-gpu_formulation": "fully_implicit",
                                    "-pc_type": "pbjacobi"})
    assert kw["precision"] == "mixed" and kw["inner_restart"] == 100 and kw["inner_rtol"] == 1e-3
    assert kw["reuse_tangent"] is False and kw["refine_rtol"] == 1e-9 and kw["newton_rtol"] == 1e-2
    assert kw["guess"] == "extrapolation" and kw["pc"] == "pbjacobi"
    assert kw["formulation"] == "fully_implicit"


@pytest.mark.parametrize("pc", ["none", "jacobi", "pbjacobi"])
def test_preconditioners_pass_through(pc):
    assert solver_options_from_petsc({"-pc_type": pc})["pc"] == pc
