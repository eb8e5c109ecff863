"""The C++ host driver: the reference-shaped programs built on the C ABI.

bin/test-ldc-stru follows src/test-ldc-stru-nelem10.cpp (read the three input
files, run the time loop, StabFEM::checkResult against the shipped solution);
bin/cfdsfemmpi keeps the reference's three-argument command line
(src/cfdsfemmpi.cpp:35-37)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cfdsfemmpi_b200", "bin")


def _copy_case(golden_dir, tmp_path):
    src = os.path.join(golden_dir, "ldc2dquad10")
    for f in os.listdir(src):
        shutil.copy(os.path.join(src, f), tmp_path / f)
    return (str(tmp_path / "LDC2Dquad10"), str(tmp_path / "control-parameters-ldc-Re100.dat"),
            str(tmp_path / "petsc_options.dat"), str(tmp_path / "test-ldc-stru-nelem10-ref.dat"))


def _built():
    from cfdsfemmpi_b200 import build
    build.build()
    return os.path.exists(os.path.join(BIN, "test-ldc-stru"))


def test_programs_build_and_fail_loudly_without_device(golden_dir, tmp_path):
    assert _built()
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    mesh, ctrl, opts, ref = _copy_case(golden_dir, tmp_path)
    r = subprocess.run([os.path.join(BIN, "cfdsfemmpi"), mesh, ctrl, opts], capture_output=True, text=True)
    assert r.returncode != 0
    assert "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_kat_ldc2dquad10_cpp_driver(golden_dir, tmp_path):
    assert _built()
    mesh, ctrl, opts, ref = _copy_case(golden_dir, tmp_path)
    r = subprocess.run([os.path.join(BIN, "test-ldc-stru"), mesh, ctrl, opts, ref], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Result matches" in r.stdout
    # forces file written next to the mesh, one line per step, zero forces as in the reference
    lines = open(mesh + "-forces.dat").read().split("\n")
    assert len([l for l in lines if l.strip()]) == 10


@pytest.mark.gpu
def test_cli_runs_with_gmres_options(golden_dir, tmp_path):
    assert _built()
    mesh, ctrl, _, _ = _copy_case(golden_dir, tmp_path)
    opts = tmp_path / "gmres.dat"
    opts.write_text("-ksp_type gmres\n-ksp_gmres_restart 50\n-pc_type jacobi\n-ksp_rtol 1.e-10\n")
    r = subprocess.run([os.path.join(BIN, "cfdsfemmpi"), mesh, ctrl, str(opts)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Program is successful" in r.stdout
    assert "GMRES(50) pc=jacobi" in r.stdout
    assert "Convergence in" in r.stdout


@pytest.mark.gpu
def test_kat_with_extrapolation_guess_and_cli_options(golden_dir, tmp_path):
    """The library's own option keys through the C++ driver: the min-residual
    extrapolation guess still reproduces the shipped 10x10 solution (the guess
    only changes where Newton starts), and the fully-implicit formulation and
    bad option values are accepted or rejected as documented."""
    assert _built()
    mesh, ctrl, opts, ref = _copy_case(golden_dir, tmp_path)
    with open(opts, "a") as f:
        f.write("\n-gpu_guess extrapolation\n")
    r = subprocess.run([os.path.join(BIN, "test-ldc-stru"), mesh, ctrl, opts, ref], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Result matches" in r.stdout
    fi = tmp_path / "fi.dat"
    fi.write_text("-ksp_type gmres\n-ksp_gmres_restart 50\n-pc_type jacobi\n-ksp_rtol 1.e-10\n"
                  "-gpu_formulation fully_implicit\n")
    r = subprocess.run([os.path.join(BIN, "cfdsfemmpi"), mesh, ctrl, str(fi)], capture_output=True, text=True)
    assert r.returncode == 0 and "Program is successful" in r.stdout, r.stderr[-2000:]
    bad = tmp_path / "bad.dat"
    bad.write_text("-gpu_formulation sideways\n")
    r = subprocess.run([os.path.join(BIN, "cfdsfemmpi"), mesh, ctrl, str(bad)], capture_output=True, text=True)
    assert r.returncode != 0 and "-gpu_formulation must be" in r.stderr


def test_cli_reports_missing_input_files(tmp_path):
    """Input errors come back before any device work, with the file named."""
    assert _built()
    r = subprocess.run([os.path.join(BIN, "cfdsfemmpi"), str(tmp_path / "nomesh"), str(tmp_path / "noctrl"),
                        str(tmp_path / "noopts")], capture_output=True, text=True)
    assert r.returncode != 0
    assert "nomesh" in (r.stdout + r.stderr)
