"""Learned Newton initial guess: GPU network gradients against the CPU
reference, training, the fallback rule, and what the trained guess gains."""
import numpy as np
import pytest

import mpnn_ref
from cfdsfemmpi_b200 import Handle, meshgen
from cfdsfemmpi_b200._lib import Mpnn
from cfdsfemmpi_b200.surrogate import collect_trajectory, fit_scales, train_guess

pytestmark = pytest.mark.gpu


def _blocks():
    off, total = mpnn_ref.layout()
    return off, total


def test_network_gradient_matches_cpu_reference():
    mesh, ctrl, _ = meshgen.case_hex(3, 2)
    h = Handle(mesh, ctrl)
    m = Mpnn(h, seed=3)
    rng = np.random.default_rng(0)
    n = h.n
    u = [0.1 * rng.standard_normal(n) for _ in range(3)]
    in_s = np.array([0.1, 0.1, 0.1, 0.05, 0.02, 0.02, 0.02, 0.01], np.float32)
    out_s = np.array([0.02, 0.02, 0.02, 0.01], np.float32)
    m.set_scales(in_s, out_s)
    m.add_sample(u[0], u[1], u[2])
    p = m.get_params()
    # give the decoder a non-trivial scale so every block has gradient signal
    off, total = _blocks()
    o = off["Wd"]
    p[o[0]:o[0] + o[1] * o[2]] = 0.2 * rng.standard_normal(o[1] * o[2]).astype(np.float32)
    m.set_params(p)
    loss_gpu, g_gpu = m.loss_grad(0)
    d = h.export_pattern()
    X = mpnn_ref.features(u[0], u[1], mesh.coords, 4, 3, in_s)
    T = mpnn_ref.targets(u[0], u[1], u[2], 4, out_s)
    mask = np.zeros((mesh.nNode, mpnn_ref.FOUT), np.float32)
    free = (d["dofmap"].reshape(-1, 4) >= 0)
    mask[:, :4] = free
    loss_ref, g_ref = mpnn_ref.loss_and_grad(p, X, T, mask, d["rowptr"], d["colidx"], int(free.sum()))
    assert abs(loss_gpu - loss_ref) <= 1e-4 * abs(loss_ref)
    for name, o in off.items():
        size = o[1] * o[2] if len(o) == 3 else o[1]
        a = g_gpu[o[0]:o[0] + size]
        b = g_ref[o[0]:o[0] + size]
        if np.abs(b).max() == 0:
            assert np.abs(a).max() == 0, name
            continue
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err < 2e-2, (name, err)
    m.close()
    h.close()


def test_training_reduces_loss_and_is_deterministic():
    mesh, ctrl, _ = meshgen.case_hex(6, 8)
    traj, _ = collect_trajectory(mesh, ctrl, 8, restart=200, rtol=1e-10, pc="pbjacobi")
    out = []
    for _ in range(2):
        h = Handle(mesh, ctrl)
        m, _ = train_guess(h, traj, iters=0, seed=1)
        before = np.mean([m.loss_grad(s)[0] for s in range(m.num_samples)])
        losses = [m.train(100, 2e-3) for _ in range(6)]
        after = np.mean([m.loss_grad(s)[0] for s in range(m.num_samples)])
        out.append((before, after, losses, m.get_params()))
        m.close()
        h.close()
    before, after = out[0][0], out[0][1]
    assert after < 0.5 * before, (before, after)
    assert out[0][2] == out[1][2] and np.array_equal(out[0][3], out[1][3])


def _run(mesh, ctrl, steps, net_builder=None, mode=("network",), **kw):
    h = Handle(mesh, ctrl, **kw)
    net = net_builder(h) if net_builder else None
    if net is not None:
        net.attach(mode)
    t = ctrl.dt
    st = []
    for _ in range(steps):
        st.append(h.step(t, t if t <= 1.0 else 1.0).as_dict())
        t = t + ctrl.dt
    s = h.get_solution()
    if net is not None:
        net.close()
    h.close()
    return s, st


def test_fallback_keeps_the_plain_path_bitwise():
    """A guess that cannot lower the iteration-0 residual is rejected and the
    run is bitwise identical to a run without it: here a network whose
    decoder is NaN (every predicted increment NaN), and the extrapolation
    direction on the first step from rest (u_1 - u_0 = 0)."""
    mesh, ctrl, _ = meshgen.case_hex(6, 3)
    kw = dict(restart=200, rtol=1e-10, pc="pbjacobi")
    plain, plain_st = _run(mesh, ctrl, 3, **kw)

    def bad(h):
        m = Mpnn(h, seed=5)
        m.set_scales(np.ones(8, np.float32), np.ones(4, np.float32))
        p = m.get_params()
        off, _ = mpnn_ref.layout()
        for name in ("Wd", "bd"):
            o = off[name]
            size = o[1] * o[2] if len(o) == 3 else o[1]
            p[o[0]:o[0] + size] = np.nan
        m.set_params(p)
        return m

    guessed, st = _run(mesh, ctrl, 3, bad, **kw)
    assert not any(s["guess_used"] for s in st)
    assert all(s["guess_norm"] == s["plain_norm"] for s in st)
    assert np.array_equal(plain, guessed)

    h = Handle(mesh, ctrl, **kw)
    h.set_guess_mode(("extrapolation",))
    s1 = h.step(ctrl.dt, ctrl.dt).as_dict()
    assert not s1["guess_used"] and s1["guess_norm"] == s1["plain_norm"]
    assert s1["norms"] == plain_st[0]["norms"]
    h.close()


def _post_ramp_runs(variants, train_iters=1500):
    """Plain FP64 trajectory of the 8^3 cavity to step 20 (the lid ramp ends
    at step 10), then steps 21..28 in the mixed-precision path from that
    state, once per guess variant: None (constant predictor),
    "extrapolation", or a tuple of modes for a network trained on steps
    12..20 (post-ramp samples only)."""
    mesh, ctrl, _ = meshgen.case_hex(8, 40)
    h0 = Handle(mesh, ctrl, restart=400, rtol=1e-10, pc="pbjacobi")
    traj = [np.zeros(h0.n)]
    t = ctrl.dt
    for _ in range(20):
        h0.step(t, t if t <= 1.0 else 1.0)
        traj.append(h0.get_solution())
        t = t + ctrl.dt
    prev, dot = h0.get_history()
    h0.close()
    kw = dict(restart=30, pc="bjacobi", ilu_levels=0, precision="mixed", inner_restart=20, inner_rtol=1e-2,
              max_it=2000)
    out = {}
    for v in variants:
        h = Handle(mesh, ctrl, **kw)
        h.set_solution(traj[-1])
        h.set_history(prev, dot)
        net = None
        if v == "extrapolation":
            h.set_guess_mode(("extrapolation",))
        elif v is not None:
            net, _ = train_guess(h, traj, iters=train_iters, lr=2e-3, seed=2, first=12)
            net.attach(v)
        tt, st = t, []
        for _ in range(8):
            st.append(h.step(tt, tt if tt <= 1.0 else 1.0).as_dict())
            tt = tt + ctrl.dt
        out[v] = (h.get_solution().reshape(-1, 4), st)
        if net is not None:
            net.close()
        h.close()
    return out


def _its(st):
    return sum(sum(s["ksp_its"]) for s in st)


def _field_diff(a, b):
    return np.linalg.norm(a[:, :3] - b[:, :3]) / np.linalg.norm(b[:, :3])


def test_extrapolation_guess_reduces_work_and_keeps_the_answer():
    """u_n + a*(u_n - u_{n-1}) with the exact min-residual a: every step
    takes it, the iteration-0 residual drops, the outer flexible-GMRES
    iterations do not grow, and every step still meets the 1e-8 Newton
    tolerance with the same velocity field.  (On this 8^3 cavity every outer
    step of 20 FP32 BiCGStab iterations gains two to three decades, so the
    fourfold smaller start saves less than one outer step per solve.)"""
    res = _post_ramp_runs([None, "extrapolation"])
    base, ext = res[None], res["extrapolation"]
    assert all(s["converged"] for s in ext[1])
    assert all(s["guess_used"] and s["guess_norm"] < 0.5 * s["plain_norm"] for s in ext[1])
    assert _its(ext[1]) <= _its(base[1]), (_its(ext[1]), _its(base[1]))
    d = _field_diff(ext[0], base[0])
    assert d < 1e-3, d


def test_trained_guess_lowers_initial_residual_and_keeps_the_answer():
    """The network trained on post-ramp steps 12..20 predicts steps 21..28
    (held out): its guess is taken on every step and lowers the iteration-0
    residual against the constant predictor, the mixed-precision path then
    needs at most 10 % more outer iterations than from the constant predictor
    (its error is rough at the element scale, which the inner solves remove
    more slowly than the norm reduction saves), and the answer is
    unchanged."""
    res = _post_ramp_runs([None, ("network",)])
    base, net = res[None], res[("network",)]
    assert all(s["converged"] for s in net[1])
    assert all(s["guess_used"] and s["guess_norm"] < s["plain_norm"] for s in net[1])
    assert _its(net[1]) <= 1.1 * _its(base[1]), (_its(net[1]), _its(base[1]))
    d = _field_diff(net[0], base[0])
    assert d < 1e-3, d


def test_guess_directions_cover_systems_above_one_grid_of_threads():
    """The guess directions are built by elementwise kernels whose grid is
    capped (148 x 16 CTAs of 256 threads = 606,208 entries per pass): on a
    hex8 cavity of 56^3 elements (740,772 dofs) the extrapolated increment
    must still cover every dof, so the min-residual guess cuts the
    iteration-0 residual during the lid ramp as it does on small meshes."""
    mesh, ctrl, _ = meshgen.case_hex(56, 4)
    assert mesh.nNode * mesh.ndof > 148 * 16 * 256
    h = Handle(mesh, ctrl, guess="extrapolation", ksp="bcgs", pc="bjacobi", ilu_levels=0, rtol=1e-10)
    t = ctrl.dt
    stats = []
    for _ in range(4):
        stats.append(h.step(t, min(t, 1.0)).as_dict())
        t = t + ctrl.dt
    h.close()
    assert all(s["converged"] for s in stats)
    for s in stats[2:]:
        assert s["guess_used"] and s["guess_norm"] < 0.5 * s["plain_norm"], s


def _mesh_sample_ref(h, mesh, u, in_s, out_s, cond, p):
    d = h.export_pattern()
    X = mpnn_ref.features(u[0], u[1], mesh.coords, 3, 2, in_s, cond)
    T = mpnn_ref.targets(u[0], u[1], u[2], 3, out_s)
    mask = np.zeros((mesh.nNode, mpnn_ref.FOUT), np.float32)
    free = (d["dofmap"].reshape(-1, 3) >= 0)
    mask[:, :3] = free
    return mpnn_ref.loss_and_grad(p, X, T, mask, d["rowptr"], d["colidx"], int(free.sum()))


def test_shared_network_samples_on_other_meshes_and_conditions():
    """One network trained on instances of different meshes and Reynolds
    numbers (the batched sweep's shared, Re-conditioned guess): a sample on
    another handle's smaller mesh, with its own condition value, gives the
    loss and gradients of the CPU reference on that mesh (the network's
    padding rows contribute nothing), as does a sample on its own mesh with
    a condition."""
    meshes = [meshgen.cavity2d(10), meshgen.cavity2d(7)]
    ctrl = meshgen.control_for(3, 0.05, 0.01)
    hs = [Handle(m, ctrl) for m in meshes]
    net = Mpnn(hs[0], seed=5)
    rng = np.random.default_rng(3)
    in_s = np.array([0.1, 0.1, 0.05, 0.02, 0.02, 0.01], np.float32)   # u (u, v, p), then u_n - u_{n-1}
    out_s = np.array([0.02, 0.02, 0.01], np.float32)
    net.set_scales(in_s, out_s)
    conds = [0.6, 0.9]
    us = [[0.1 * rng.standard_normal(h.n) for _ in range(3)] for h in hs]
    net.add_sample(*us[0], cond=conds[0])
    net.add_sample(*us[1], handle=hs[1], cond=conds[1])
    p = net.get_params()
    off, _ = _blocks()
    o = off["Wd"]
    p[o[0]:o[0] + o[1] * o[2]] = 0.2 * rng.standard_normal(o[1] * o[2]).astype(np.float32)
    net.set_params(p)
    for k in range(2):
        loss_gpu, g_gpu = net.loss_grad(k)
        loss_ref, g_ref = _mesh_sample_ref(hs[k], meshes[k], us[k], in_s, out_s, conds[k], p)
        assert abs(loss_gpu - loss_ref) <= 1e-4 * abs(loss_ref), (k, loss_gpu, loss_ref)
        for name, ob in off.items():
            size = ob[1] * ob[2] if len(ob) == 3 else ob[1]
            a = g_gpu[ob[0]:ob[0] + size]
            b = g_ref[ob[0]:ob[0] + size]
            if np.abs(b).max() == 0:
                assert np.abs(a).max() == 0, (k, name)
                continue
            assert np.abs(a - b).max() / np.abs(b).max() < 2e-2, (k, name)
    # a mesh with more nodes than the network's own is refused
    big = Handle(meshgen.cavity2d(12), ctrl)
    with pytest.raises(Exception):
        net.add_sample(*[np.zeros(big.n)] * 3, handle=big, cond=0.5)
    big.close()
    net.close()
    for h in hs:
        h.close()


def test_shared_network_guides_every_instance_of_a_batch():
    """The shared, Re-conditioned network trained on the first steps of a
    batch of cavities of different sizes and Reynolds numbers is attached to
    every instance (its own condition value): every later step converges,
    and the answers stay those of the batch without it (velocity to 1e-6;
    every solve stops at rtol 1e-8 relative to its own start)."""
    from cfdsfemmpi_b200 import Batch
    from cfdsfemmpi_b200.surrogate import attach_shared, train_shared
    cases = meshgen.batch_cases(count=3, n_lo=8, n_hi=14, dt=0.05, steps=20, seed=7)
    pairs = [(m, c) for m, c, _, _ in cases]
    conds = [float(np.log(re) / np.log(5000.0)) for _, _, _, re in cases]
    kw = dict(restart=200, rtol=1e-8, pc="pbjacobi", max_it=20000)
    out = []
    for learned in (False, True):
        b = Batch(pairs, **kw)
        b.set_schedule(3, 4, 1)
        trajs = [[h.get_solution()] for h in b.handles]
        for k in range(12):
            b.step(np.full(len(pairs), 0.05 * (k + 1)))
            for i, h in enumerate(b.handles):
                trajs[i].append(h.get_solution())
        nets = []
        if learned:
            net0, shared, losses = train_shared(b.handles, trajs, conds, iters=600, lr=2e-3, seed=0, first=2)
            assert net0.num_samples == 3 * 10 and losses[-1] < losses[0]
            net0.close()
            nets = [attach_shared(h, shared, c) for h, c in zip(b.handles, conds)]
        stats = []
        for k in range(12, 16):
            st, _ = b.step(np.full(len(pairs), 0.05 * (k + 1)))
            stats.extend(s.as_dict() for s in st)
        out.append(([h.get_solution().reshape(-1, 3) for h in b.handles], stats))
        for q in nets:
            q.close()
        b.close()
    (base, _), (guided, st) = out
    assert all(s["converged"] for s in st)
    assert any(s["guess_used"] for s in st)
    for a, c in zip(guided, base):
        assert np.linalg.norm(a[:, :2] - c[:, :2]) / np.linalg.norm(c[:, :2]) < 1e-6
