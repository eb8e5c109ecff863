"""A small, bounded case for profiling the hot kernels in isolation.

Assembles the graded-cube hex8 cavity tangent once (iteration-0 semantics at
the first time level) and runs a fixed number of GMRES iterations on it, so a
profiler sees the element kernels, the BSR SpMV and the Gram-Schmidt kernels
with realistic sizes, and the run ends by itself:

    python -m cfdsfemmpi_b200.kernel_case --n 64 --restart 40 --max-it 40
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import Handle, meshgen


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=64)
    p.add_argument("--restart", type=int, default=40)
    p.add_argument("--max-it", type=int, default=40)
    p.add_argument("--pc", default="pbjacobi")
    p.add_argument("--repeat", type=int, default=1)
    a = p.parse_args(argv)
    mesh, ctrl, _ = meshgen.case_hex(a.n, 2)
    h = Handle(mesh, ctrl, restart=a.restart, rtol=1e-30, pc=a.pc, max_it=a.max_it)
    rng = np.random.default_rng(0)
    n = mesh.nNode * mesh.ndof
    prev = 0.1 * rng.standard_normal(n)
    h.set_element_state(prev, prev, np.zeros(n))
    t0 = time.perf_counter()
    for _ in range(a.repeat):
        h._check(h._L.cfdgpu_assemble_export(h.h, 0, None, None))
    b = rng.standard_normal(n)
    d = h.export_pattern()
    b[d["fixed_dofs"]] = 0.0
    x, its, reason = h.solve_export(b)
    dt = time.perf_counter() - t0
    print(json.dumps({"n": a.n, "nodes": mesh.nNode, "its": its, "reason": reason, "seconds": dt,
                      "launches": h.launch_count()}))
    h.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
