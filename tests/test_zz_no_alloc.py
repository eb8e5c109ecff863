"""Allocation-free residual norm, checked against the allocating entry point.

Callers that may not allocate device memory -- a code running inside another
framework's memory pool, or one that is only handed a stream to enqueue on --
call cfdgpu_residual_norm_noalloc on BSR data they already hold on the device;
its scratch is a fixed array inside the library.  This test builds such data
with torch for a hex8 cavity (4x4 blocks) and a quad4 cavity (3x3 blocks),
calls the entry point through the C ABI twice in a row for each, and compares
each result with cfdgpu_true_residual, which computes the same norm with the
handle's own device memory, and with a host BSR product (scipy) on the
exported pattern, which shares no code with the GPU kernels.  It sorts last
so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_residual(d, vals, x, b, ndof):
    import scipy.sparse as sp
    nnode = len(d["rowptr"]) - 1
    A = sp.bsr_matrix((np.asarray(vals).reshape(-1, ndof, ndof), d["colidx"], d["rowptr"]),
                      shape=(nnode * ndof, nnode * ndof))
    return float(np.linalg.norm(b - A @ x))


@pytest.mark.parametrize("case", ["hex8", "quad4"])
def test_residual_norm_noalloc_matches_allocating_entry_point(case):
    import torch
    from cfdsfemmpi_b200 import Handle, _lib, meshgen

    if case == "hex8":
        mesh, ctrl, _ = meshgen.case_hex(6, 2)
    else:
        mesh, ctrl = meshgen.cavity2d(13), meshgen.control_for(2, 0.1, 0.01)
    h = Handle(mesh, ctrl)
    rng = np.random.default_rng(4)
    n = h.n
    h.set_element_state(0.1 * rng.standard_normal(n), 0.1 * rng.standard_normal(n), np.zeros(n))
    vals, rhs = h.assemble_export(0)
    d = h.export_pattern()
    dev = torch.device("cuda", 0)
    rowptr = torch.from_numpy(d["rowptr"]).to(dev)
    colidx = torch.from_numpy(d["colidx"]).to(dev)
    val = torch.from_numpy(np.ascontiguousarray(vals).ravel()).to(dev)
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    L = _lib.load()
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        x = rng.standard_normal(n)
        x[d["fixed_dofs"]] = 0.0
        b = rhs if call == 0 else rng.standard_normal(n)
        ref = h.true_residual(x, b)
        host = _host_residual(d, vals, x, b, mesh.ndof)
        xd = torch.from_numpy(x).to(dev)
        bd = torch.from_numpy(b).to(dev)
        rc = L.cfdgpu_residual_norm_noalloc(mesh.nNode, mesh.ndof, rowptr.data_ptr(), colidx.data_ptr(),
                                            val.data_ptr(), xd.data_ptr(), bd.data_ptr(), out.data_ptr(),
                                            ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = float(out.item())
        assert ref > 0.0
        assert abs(got - ref) <= 1e-12 * ref, (case, call, got, ref)
        assert abs(got - host) <= 1e-12 * host, (case, call, got, host)
    # a system larger than the fixed scratch is refused before any work is enqueued
    rc = L.cfdgpu_residual_norm_noalloc(600000, 4, rowptr.data_ptr(), colidx.data_ptr(), val.data_ptr(),
                                        xd.data_ptr(), bd.data_ptr(), out.data_ptr(),
                                        ctypes.c_void_p(stream.cuda_stream))
    assert rc == _lib.ETOOBIG
    # so is a vector that does not start on a 16-byte boundary
    rc = L.cfdgpu_residual_norm_noalloc(mesh.nNode, mesh.ndof, rowptr.data_ptr(), colidx.data_ptr(),
                                        val.data_ptr(), xd.data_ptr() + 8, bd.data_ptr(), out.data_ptr(),
                                        ctypes.c_void_p(stream.cuda_stream))
    assert rc == _lib.EINVAL
    torch.cuda.synchronize()
    assert float(out.item()) == got
    h.close()
