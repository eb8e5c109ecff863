"""Copy the reference's shipped known-answer fixtures into tests/golden/.

The reference keeps two usable 2D lid-driven-cavity goldens (the 3D one lacks
its mesh file): testdata/ldc2dquad10/ and testdata/ldc2dquad-mesh2/.  They are
data files (mesh, control parameters, solver options, reference solution), so
the tests can run where the reference tree is absent.  The larger case is
stored gzip-compressed.  Run from the repository root:

    python tests/golden/make_fixtures.py /path/to/reference
"""
import gzip
import os
import shutil
import sys

CASES = {
    "ldc2dquad10": ["LDC2Dquad10.dat", "control-parameters-ldc-Re100.dat", "petsc_options.dat",
                    "test-ldc-stru-nelem10-ref.dat"],
    "ldc2dquad-mesh2": ["LDC2Dquad-mesh2.dat", "control-parameters-Re1000.dat", "petsc_options.dat",
                        "test-ldc-stru-mesh2-ref.dat"],
}
COMPRESS = {"ldc2dquad-mesh2"}


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for case, files in CASES.items():
        dst = os.path.join(here, case)
        os.makedirs(dst, exist_ok=True)
        for f in files:
            src = os.path.join(ref_root, "testdata", case, f)
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
