"""Copy the reference's shipped known-answer fixtures into tests/golden/.

The reference keeps two usable 2D lid-driven-cavity goldens (the 3D one lacks
its mesh file): testdata/ldc2dquad10/ and testdata/ldc2dquad-mesh2/.  It also
ships a cylinder-wake input (input/cylinder2d-blockmesh-*, 12,400 quads) with
its control parameters and its iterative solver option files, which have no
reference solution.  They are data files (mesh, control parameters, solver
options, reference solution), so the tests can run where the reference tree
is absent.  The larger cases are stored gzip-compressed.  Run from the
repository root:

    python tests/golden/make_fixtures.py /path/to/reference
"""
import gzip
import os
import shutil
import sys

# fixture folder: (folder in the reference tree, files)
CASES = {
    "ldc2dquad10": ("testdata/ldc2dquad10", ["LDC2Dquad10.dat", "control-parameters-ldc-Re100.dat",
                                             "petsc_options.dat", "test-ldc-stru-nelem10-ref.dat"]),
    "ldc2dquad-mesh2": ("testdata/ldc2dquad-mesh2", ["LDC2Dquad-mesh2.dat", "control-parameters-Re1000.dat",
                                                     "petsc_options.dat", "test-ldc-stru-mesh2-ref.dat"]),
    "cylinder2d-blockmesh": ("input", ["cylinder2d-blockmesh-Re100-GA2-rho0p0-dt0p1-SI.dat",
                                       "control-parameters-Re100-dt0p1.dat", "petsc_options_bcgs.dat",
                                       "petsc_options_gmres.dat"]),
}
COMPRESS = {"ldc2dquad-mesh2", "cylinder2d-blockmesh"}


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for case, (folder, files) in CASES.items():
        dst = os.path.join(here, case)
        os.makedirs(dst, exist_ok=True)
        for f in files:
            src = os.path.join(ref_root, folder, f)
            if case in COMPRESS:
                with open(src, "rb") as fi, open(os.path.join(dst, f + ".gz"), "wb") as raw:
                    with gzip.GzipFile(filename="", mode="wb", fileobj=raw, mtime=0) as fo:
                        shutil.copyfileobj(fi, fo)
            else:
                shutil.copyfile(src, os.path.join(dst, f))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference project root>")
    main(sys.argv[1])
