"""CPU reference of the learned-guess network (TEST INFRASTRUCTURE ONLY).

NumPy restatement of cfdsfemmpi_b200/csrc/mpnn.cu's forward pass, masked
MSE loss and backward pass, with BF16 rounding (round to nearest even)
applied exactly where the GPU kernels round: GEMM operands, the aggregated
messages and the upstream gradients fed to the backward GEMMs.  Used by the
tests to check the GPU gradients; the network has no counterpart in the
reference.
"""
from __future__ import annotations

import numpy as np

HID, LAYERS, FIN, FOUT = 64, 3, 16, 16


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (x >> 16) & 1
    x = (x + 0x7FFF + lsb) & 0xFFFF0000
    return x.astype(np.uint32).view(np.float32)


def layout():
    off = {}
    o = 0
    off["We"] = (o, FIN, HID); o += FIN * HID
    off["be"] = (o, HID); o += HID
    for l in range(LAYERS):
        off[f"W{l}"] = (o, 2 * HID, HID); o += 2 * HID * HID
        off[f"b{l}"] = (o, HID); o += HID
    off["Wd"] = (o, HID, FOUT); o += HID * FOUT
    off["bd"] = (o, FOUT); o += FOUT
    return off, o


def unpack(p):
    off, _ = layout()
    out = {}
    for k, v in off.items():
        if len(v) == 3:
            out[k] = p[v[0]:v[0] + v[1] * v[2]].reshape(v[1], v[2]).astype(np.float32)
        else:
            out[k] = p[v[0]:v[0] + v[1]].astype(np.float32)
    return out


def features(u_nm1, u_n, coords, ndof, ndim, in_scale, cond=0.0):
    N = coords.shape[0]
    f = np.zeros((N, FIN), np.float32)
    un = u_n.reshape(N, ndof)
    du = un - u_nm1.reshape(N, ndof)
    for c in range(ndof):
        f[:, c] = (un[:, c] / np.float64(np.float32(in_scale[c]))).astype(np.float32)
        f[:, ndof + c] = (du[:, c] / np.float64(np.float32(in_scale[ndof + c]))).astype(np.float32)
    for c in range(ndim):
        lo, hi = coords[:, c].min(), coords[:, c].max()
        inv = 1.0 / (hi - lo) if hi > lo else 1.0
        f[:, 2 * ndof + c] = (2.0 * ((coords[:, c] - lo) * inv) - 1.0).astype(np.float32)
    f[:, 2 * ndof + ndim] = np.float32(cond)
    return bf16(f)


def targets(u_nm1, u_n, u_np1, ndof, out_scale):
    """Scaled correction over linear extrapolation, u_{n+1} - 2 u_n + u_{n-1}."""
    N = u_n.size // ndof
    t = np.zeros((N, FOUT), np.float32)
    d = ((u_np1 - u_n) - (u_n - u_nm1)).reshape(N, ndof)
    for c in range(ndof):
        t[:, c] = (d[:, c] / np.float64(np.float32(out_scale[c]))).astype(np.float32)
    return t


def mean_agg(h, rowptr, colidx):
    N = len(rowptr) - 1
    out = np.zeros((N, h.shape[1]), np.float32)
    for i in range(N):
        nb = colidx[rowptr[i]:rowptr[i + 1]]
        acc = np.zeros(h.shape[1], np.float32)
        for j in nb:
            acc = (acc + h[j]).astype(np.float32)
        out[i] = acc * (np.float32(1.0) / np.float32(len(nb)))
    return out


def mean_agg_T(g, rowptr, colidx):
    N = len(rowptr) - 1
    deg = np.diff(rowptr).astype(np.float32)
    out = np.zeros_like(g)
    for i in range(N):
        acc = np.zeros(g.shape[1], np.float32)
        for j in colidx[rowptr[i]:rowptr[i + 1]]:
            acc = (acc + g[j] * (np.float32(1.0) / deg[j])).astype(np.float32)
        out[i] = acc
    return out


def loss_and_grad(p, X, T, mask, rowptr, colidx, nfree):
    """Returns (loss, flat gradient) in the GPU parameter layout."""
    w = unpack(p)
    off, total = layout()
    Wb = {k: bf16(v) for k, v in w.items() if k.startswith("W")}
    f64 = lambda a: a.astype(np.float64)
    Ze = (f64(X) @ f64(Wb["We"]) + w["be"]).astype(np.float32)
    Hf = [np.maximum(Ze, 0).astype(np.float32)]
    Cat, Z = [], []
    for l in range(LAYERS):
        hb = bf16(Hf[l])
        m = bf16(mean_agg(hb, rowptr, colidx))
        cat = np.concatenate([hb, m], axis=1)
        Cat.append(cat)
        z = (f64(cat) @ f64(Wb[f"W{l}"]) + w[f"b{l}"]).astype(np.float32)
        Z.append(z)
        Hf.append((np.maximum(z, 0) + Hf[l]).astype(np.float32))
    H3b = bf16(Hf[LAYERS])
    Y = (f64(H3b) @ f64(Wb["Wd"]) + w["bd"]).astype(np.float32)
    inv = 1.0 / max(1, nfree)
    d = (Y - T) * mask
    loss = float(np.sum(f64(d) ** 2) * inv)
    dY = (2.0 * d * np.float32(inv)).astype(np.float32)
    g = np.zeros(total)

    def put(name, val):
        o = off[name]
        g[o[0]:o[0] + val.size] = val.ravel()

    put("Wd", f64(H3b).T @ f64(dY))
    put("bd", dY.sum(0))
    dH = (f64(bf16(dY)) @ f64(Wb["Wd"]).T).astype(np.float32)
    for l in reversed(range(LAYERS)):
        dZ = np.where(Z[l] > 0, dH, 0).astype(np.float32)
        put(f"W{l}", f64(Cat[l]).T @ f64(dZ))
        put(f"b{l}", dZ.sum(0))
        dCat = (f64(bf16(dZ)) @ f64(Wb[f"W{l}"]).T).astype(np.float32)
        dH = (dH + dCat[:, :HID]).astype(np.float32)
        dM = bf16(dCat[:, HID:])
        dH = (dH + mean_agg_T(dM, rowptr, colidx)).astype(np.float32)
    dZe = np.where(Ze > 0, dH, 0).astype(np.float32)
    put("We", f64(X).T @ f64(dZe))
    put("be", dZe.sum(0))
    return loss, g
