"""Learned preconditioner: the network's CUDA kernels (tcgen05 convolutions,
own weight gradient, pooling, head, loss, Adam) against a CPU FP32 torch
reference, and flexible CG with the composite preconditioner against
Jacobi-PCG.

Tolerances: each kernel is checked on its own against the reference on the
same BF16 inputs (relative L2 5e-3 for BF16 outputs, 1e-5 for FP32 weight
gradients).  The whole network is compared with the reference's own BF16
rounding at the same places: forward to 2e-2 relative; parameter gradients,
which carry BF16 activation-gradient rounding through 10 layers (and FP32
atomics in an order that changes from run to run), to 2e-1 relative L2 with
a cosine above 0.98 per tensor.  The solver bar is the
solve's own: every method reaches ||b - A x|| / ||b|| <= tol.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from pic_b200 import api, deck

torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_picunet_exports_cpu():
    from pic_b200 import unet
    hdr = open(os.path.join(ROOT, "include", "picunet.h")).read()
    declared = re.findall(r"^int (unet_\w+)\(", hdr, flags=re.M)
    assert sorted(declared) == sorted(unet.EXPORTS)
    lib = unet.load()
    for name in declared:
        assert hasattr(lib, name), name


def test_static_features_cpu():
    from pic_b200 import unet
    from pic_b200.deck import Mesh
    m = Mesh(deck.config("cfg1"))
    try:
        f = unet.static_features(m).reshape(m.nnx, m.nny, 3)
        nt = m.array("node_type").reshape(m.nnx, m.nny)
        assert np.array_equal(f[..., 2] > 0.5, nt <= 0)
        c = m.nnx // 2  # disk centre: eps_r = 4, level set negative
        assert abs(f[c, c, 0] - np.log(4.0)) < 1e-6 and f[c, c, 1] < 0
        assert f[1, 1, 0] == 0.0 and f[1, 1, 1] > 0
        assert np.all(np.abs(f[..., 1]) <= 1.0)
    finally:
        m.close()


def test_reference_network_cpu():
    import unet_ref as R
    g = torch.Generator().manual_seed(0)
    params = {}
    for name, cin, cout in R.LAYERS:
        params[name + ".w"] = torch.randn(cout, 3, 3, cin, generator=g) * 0.1
        params[name + ".b"] = torch.zeros(cout)
    params["head.w"] = torch.randn(32, generator=g)
    params["head.b"] = torch.zeros(1)
    z = R.forward(params, torch.randn(2, 13, 11, 8, generator=g))
    assert z.shape == (2 * 13 * 11,)
    p = R.pool(torch.arange(15.0).reshape(1, 3, 5, 1))
    assert p.shape == (1, 2, 3, 1)
    assert p[0, 1, 2, 0].item() == 14.0 and p[0, 0, 0, 0].item() == (0 + 1 + 5 + 6) / 4


# --------------------------------------------------------------------------
gpu = pytest.mark.gpu


def _bf(t):
    return t.to(torch.bfloat16)


def P(t):
    return C.c_void_p(t.data_ptr())


def _conv(lib, op, x, w, d, bias=None):
    from pic_b200 import unet
    n, h, ww, c = x.shape if op == unet.UNET_FPROP_RELU else d.shape
    k = w.shape[0]
    need = C.c_size_t(0)
    assert lib.unet_conv(op, n, h, ww, c, k, None, None, None, None, None, 0, C.byref(need), None) == 0
    ws = torch.zeros(max(need.value, 256), dtype=torch.uint8, device="cuda")
    rc = lib.unet_conv(op, n, h, ww, c, k, P(x), P(w), P(d), P(bias) if bias is not None else None, P(ws),
                       ws.numel(), None, None)
    assert rc == 0
    torch.cuda.synchronize()


def _rel(a, b):
    a = a.double().cpu()
    b = b.double().cpu()
    return float((a - b).norm() / max(float(b.norm()), 1e-30))


@gpu
@pytest.mark.parametrize("c,k,h,w", [(8, 32, 37, 45), (32, 64, 19, 23), (192, 64, 19, 23), (128, 128, 10, 12)])
def test_conv_fprop_matches_cpu(c, k, h, w):
    from pic_b200 import unet
    import torch.nn.functional as F
    lib = unet.load()
    g = torch.Generator().manual_seed(c + k)
    x = torch.randn(2, h, w, c, generator=g)
    wt = torch.randn(k, 3, 3, c, generator=g) * (2.0 / (9 * c)) ** 0.5
    b = torch.randn(k, generator=g) * 0.1
    xb, wb, bb = _bf(x).cuda(), _bf(wt).cuda(), _bf(b).cuda()
    y = torch.zeros(2, h, w, k, dtype=torch.bfloat16, device="cuda")
    _conv(lib, unet.UNET_FPROP_RELU, xb, wb, y, bias=bb)
    xr, wr, br = xb.float().cpu(), wb.float().cpu(), bb.float().cpu()
    ref = torch.relu(F.conv2d(xr.permute(0, 3, 1, 2), wr.permute(0, 3, 1, 2), padding=1)
                     + br[None, :, None, None]).permute(0, 2, 3, 1)
    got = y.float().cpu()
    assert (got - ref).abs().max().item() <= 8e-3 * ref.abs().max().item() + 1e-6
    assert _rel(got, ref) < 5e-3


@gpu
@pytest.mark.parametrize("c,k,h,w", [(32, 32, 37, 45), (192, 64, 19, 23), (64, 128, 10, 12)])
def test_conv_dgrad_and_wgrad_match_cpu(c, k, h, w):
    from pic_b200 import unet
    import torch.nn.functional as F
    lib = unet.load()
    g = torch.Generator().manual_seed(7 * c + k)
    x = _bf(torch.randn(2, h, w, c, generator=g)).float()
    wt = _bf(torch.randn(k, 3, 3, c, generator=g) * 0.1).float()
    dy = _bf(torch.randn(2, h, w, k, generator=g)).float()
    xr = x.clone().requires_grad_(True)
    wr = wt.clone().requires_grad_(True)
    F.conv2d(xr.permute(0, 3, 1, 2), wr.permute(0, 3, 1, 2), padding=1).permute(0, 2, 3, 1).backward(dy)
    dx = torch.zeros(2, h, w, c, dtype=torch.bfloat16, device="cuda")
    _conv(lib, unet.UNET_DGRAD, _bf(dy).cuda(), _bf(wt).cuda(), dx)
    assert _rel(dx.float(), xr.grad) < 5e-3
    dw = torch.zeros(k, 3, 3, c, dtype=torch.float32, device="cuda")
    xd, dyd = _bf(x).cuda(), _bf(dy).cuda()
    assert lib.unet_wgrad(2, h, w, c, k, P(xd), P(dyd), P(dw), None) == 0
    torch.cuda.synchronize()
    assert _rel(dw, wr.grad) < 1e-5


@gpu
def test_rms_features_output():
    from pic_b200 import unet
    import unet_ref as R
    lib = unet.load()
    h, w = 33, 29
    g = torch.Generator().manual_seed(3)
    r = torch.randn(h * w, generator=g, dtype=torch.float64)
    mask = (torch.rand(h * w, generator=g) > 0.2).to(torch.int32)
    feat = torch.randn(h * w * 3, generator=g)
    rd, md, fd = r.cuda(), mask.cuda(), feat.cuda()
    scratch = torch.zeros(unet.UNET_RMS_SCRATCH, dtype=torch.float64, device="cuda")
    sc = torch.zeros(2, dtype=torch.float64, device="cuda")
    s_ref = float(torch.sqrt((r * r * (mask > 0)).sum() / (mask > 0).sum()))
    for _ in range(2):  # the ticket re-arms itself
        assert lib.unet_rms(h * w, P(rd), P(md), P(scratch), P(sc), None) == 0
        torch.cuda.synchronize()
        assert abs(float(sc[0]) - s_ref) <= 1e-12 * s_ref
    x = torch.zeros(h * w * 8, dtype=torch.bfloat16, device="cuda")
    assert lib.unet_features(h, w, P(rd), P(sc), P(fd), P(x), None) == 0
    z = torch.randn(h * w, generator=g).cuda()
    out = torch.zeros(h * w, dtype=torch.float64, device="cuda")
    assert lib.unet_output(h * w, P(z), P(sc), P(md), P(out), None) == 0
    torch.cuda.synchronize()
    assert torch.equal(x.float().cpu().reshape(-1, 8), R.features(r, float(sc[0]), feat))
    o_ref = float(sc[0]) * z.double().cpu() * (mask > 0)
    assert torch.allclose(out.cpu(), o_ref, rtol=1e-15, atol=0)


@gpu
def test_backward_ops_match_cpu():
    """ReLU/bias, pooling, upsample-concat and head backward kernels on BF16
    inputs against the CPU reference's autograd."""
    import unet_ref as R
    from pic_b200 import unet
    lib = unet.load()
    g = torch.Generator().manual_seed(9)
    n, h, w = 2, 13, 11
    h2, w2 = 7, 6
    for c in (32, 96):  # relu backward + bias gradient (96: 12 channel groups)
        y = _bf(torch.relu(torch.randn(n, h, w, c, generator=g)))
        dy = _bf(torch.randn(n, h, w, c, generator=g))
        yd, dyd = y.cuda(), dy.cuda()
        db = torch.zeros(c, device="cuda")
        assert lib.unet_relu_bwd(n * h * w, c, P(yd), P(dyd), P(db), None) == 0
        torch.cuda.synchronize()
        ref = dy.float() * (y.float() > 0)
        assert torch.equal(dyd.float().cpu(), ref)
        assert torch.allclose(db.cpu(), ref.sum(dim=(0, 1, 2)), rtol=1e-5, atol=1e-4)
    x = torch.randn(n, h, w, 32, generator=g).requires_grad_(True)
    gp = _bf(torch.randn(n, h2, w2, 32, generator=g)).float()
    R.pool(x).backward(gp)
    dx = torch.zeros(n, h, w, 32, dtype=torch.bfloat16, device="cuda")
    assert lib.unet_pool_bwd(n, h, w, 32, P(_bf(gp).cuda()), P(dx), 0, None) == 0
    xf = _bf(x.detach()).cuda()
    yp = torch.zeros(n, h2, w2, 32, dtype=torch.bfloat16, device="cuda")
    assert lib.unet_pool(n, h, w, 32, P(xf), P(yp), None) == 0
    torch.cuda.synchronize()
    assert _rel(dx.float(), x.grad) < 4e-3
    assert _rel(yp.float(), R.pool(xf.float().cpu())) < 4e-3
    lo = torch.randn(n, h2, w2, 64, generator=g).requires_grad_(True)
    sk = torch.randn(n, h, w, 32, generator=g).requires_grad_(True)
    gu = _bf(torch.randn(n, h, w, 96, generator=g)).float()
    R.upcat(lo, sk).backward(gu)
    dlo = torch.zeros(n, h2, w2, 64, dtype=torch.bfloat16, device="cuda")
    dsk = torch.zeros(n, h, w, 32, dtype=torch.bfloat16, device="cuda")
    assert lib.unet_upcat_bwd(n, h, w, 64, 32, P(_bf(gu).cuda()), P(dlo), P(dsk), 0, None) == 0
    lob, skb = _bf(lo.detach()).cuda(), _bf(sk.detach()).cuda()
    yu = torch.zeros(n, h, w, 96, dtype=torch.bfloat16, device="cuda")
    assert lib.unet_upcat(n, h, w, 64, 32, P(lob), P(skb), P(yu), None) == 0
    torch.cuda.synchronize()
    assert _rel(dlo.float(), lo.grad) < 4e-3 and torch.equal(dsk.float().cpu(), sk.grad)
    assert torch.equal(yu.float().cpu(), R.upcat(lob.float().cpu(), skb.float().cpu()))
    yh = _bf(torch.randn(n * h * w, 32, generator=g)).float()
    wh = torch.randn(32, generator=g).requires_grad_(True)
    bh = torch.zeros(1).requires_grad_(True)
    yr = yh.clone().requires_grad_(True)
    gz = torch.randn(n * h * w, generator=g)
    (yr @ wh + bh).backward(gz)
    dyh = torch.zeros(n * h * w, 32, dtype=torch.bfloat16, device="cuda")
    dwh = torch.zeros(32, device="cuda")
    dbh = torch.zeros(1, device="cuda")
    assert lib.unet_head_bwd(n * h * w, 32, P(_bf(yh).cuda()), P(wh.detach().cuda()), P(gz.cuda()), P(dyh),
                             P(dwh), P(dbh), None) == 0
    torch.cuda.synchronize()
    assert _rel(dyh.float(), yr.grad) < 4e-3
    assert torch.allclose(dwh.cpu(), wh.grad, rtol=1e-4, atol=1e-3)
    assert torch.allclose(dbh.cpu(), bh.grad, rtol=1e-4, atol=1e-3)


def _net_and_ref(n, h, w, seed=0):
    from pic_b200 import unet
    net = unet.UNet(seed=seed)
    for name, v in net.params.items():  # non-zero biases so their gradients matter
        if name.endswith(".b") and not name.startswith("head"):
            v["p"].uniform_(-0.05, 0.05)
            v["bf"].copy_(v["p"].to(torch.bfloat16))
    net._ensure(n, h, w)
    ref = {}
    for name, v in net.params.items():
        ref[name] = (v["p"] if name.startswith("head") else v["bf"].float()).detach().cpu().clone()
    torch.cuda.synchronize()
    return net, ref


@gpu
def test_unet_forward_backward_match_cpu_autograd():
    import unet_ref as R
    n, h, w = 2, 37, 45
    net, ref = _net_and_ref(n, h, w)
    g = torch.Generator().manual_seed(11)
    x = torch.zeros(n, h, w, 8)
    x[..., :4] = torch.randn(n, h, w, 4, generator=g)
    x = x.to(torch.bfloat16).float()
    net.a["x0"].copy_(x.to(torch.bfloat16))
    z = net.forward().clone()
    torch.cuda.synchronize()
    for v in ref.values():
        v.requires_grad_(True)
    zr = R.forward(ref, x)
    assert _rel(z, zr.detach()) < 2e-2
    gz = torch.randn(n * h * w, generator=g)
    (zr * gz).sum().backward()
    net.zero_grad()
    net.gz.copy_(gz)
    net.backward()
    torch.cuda.synchronize()
    for name, v in net.params.items():
        a, b = v["g"].double().cpu().reshape(-1), ref[name].grad.double().reshape(-1)
        cos = float(a @ b / (a.norm() * b.norm()))
        assert _rel(a, b) < 2e-1 and cos > 0.98, (name, _rel(a, b), cos)


@gpu
def test_adam_matches_torch():
    from pic_b200 import unet
    lib = unet.load()
    g = torch.Generator().manual_seed(5)
    p0 = torch.randn(1000, generator=g)
    pt = p0.clone().requires_grad_(True)
    opt = torch.optim.Adam([pt], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    p, m, v = p0.cuda(), torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    pb = torch.zeros(1000, dtype=torch.bfloat16, device="cuda")
    for t in range(1, 4):
        grad = torch.randn(1000, generator=g)
        pt.grad = grad.clone()
        opt.step()
        gd = grad.cuda()
        assert lib.unet_adam(1000, P(p), P(gd), P(m), P(v), P(pb), 1e-2, 0.9, 0.999, 1e-8, t, None) == 0
    torch.cuda.synchronize()
    assert torch.allclose(p.cpu(), pt.detach(), rtol=1e-5, atol=1e-6)
    assert torch.equal(pb.cpu(), p.cpu().to(torch.bfloat16))


# ---- flexible CG with the composite preconditioner ------------------------

def _sim(ncells=128, ppc=4, seed=0, tol=1e-10):
    from pic_b200.simulation import Simulation
    cfg = deck.config("cfg1", ncx=ncells, ncy=ncells, ppc=ppc, seed=seed, pcg_tol=tol)
    sim = Simulation(cfg)
    sim.initial_fields()
    return sim


def _solve_from(sim, phi0, solver):
    api.check(sim.lib.pic_set_solver(solver), "pic_set_solver")
    sim.set_field("phi", phi0)
    st = api.SolveStats()
    api.check(sim.lib.pic_ife_solve(None, 0.0, C.byref(st)), "pic_ife_solve")
    return st, sim.field("phi")


def _true_rel_residual(sim):
    nt = sim.mesh.array("node_type")
    mask = torch.tensor((nt > 0).astype(np.float64), device="cuda")
    phi = torch.tensor(sim.field("phi"), device="cuda") * mask
    ax = torch.empty_like(phi)
    b = torch.tensor(sim.field("b"), device="cuda") * mask
    torch.cuda.synchronize()
    api.check(sim.lib.pic_apply_operator(P(phi), P(ax)), "op")
    torch.cuda.synchronize()
    return float(((b - ax) * mask).norm() / b.norm())


@gpu
def test_fcg_falls_back_to_jacobi_pcg():
    sim = _sim(ncells=64)
    try:
        calls = []

        def bad(r, z, user):  # a failing preconditioner
            calls.append(1)
            return 1

        cb = api.PRECOND_FN(bad)
        api.check(sim.lib.pic_set_preconditioner(cb, None), "set")
        zero = np.zeros(sim.mesh.nn)
        st_j, phi_j = _solve_from(sim, zero, api.PIC_SOLVER_JPCG)
        st_f, phi_f = _solve_from(sim, zero, api.PIC_SOLVER_FCG_UNET)
        assert calls and st_f.fallback == 5
        assert np.array_equal(phi_f, phi_j) and st_f.iterations == st_j.iterations
        api.check(sim.lib.pic_set_solver(api.PIC_SOLVER_JPCG), "set")
    finally:
        sim.close()


@gpu
@pytest.mark.parametrize("window", [1, 4])
def test_fcg_with_jacobi_callback_matches_pcg(window):
    """FCG with z = D^-1 r (a fixed SPD preconditioner) is Jacobi-PCG in exact
    arithmetic: same iteration count to within a few."""
    sim = _sim(ncells=64)
    try:
        nt = sim.mesh.array("node_type")
        diag = sim.mesh.array("a_diag")
        dfull = np.ones(sim.mesh.nn)
        dfull[nt > 0] = diag[nt[nt > 0] - 1]
        dfull = torch.tensor(dfull, device="cuda")
        mask = torch.tensor((nt > 0).astype(np.float64), device="cuda")
        st_ = C.c_void_p()
        api.check(sim.lib.pic_cuda_stream(C.byref(st_)), "stream")
        ts = torch.cuda.ExternalStream(st_.value)
        from pic_b200.unet import DeviceArray
        torch.cuda.synchronize()

        def jac(r, z, user):
            with torch.cuda.stream(ts):
                rv = torch.as_tensor(DeviceArray(r, sim.mesh.nn), device="cuda")
                zv = torch.as_tensor(DeviceArray(z, sim.mesh.nn), device="cuda")
                torch.div(rv * mask, dfull, out=zv)
            return 0

        cb = api.PRECOND_FN(jac)
        api.check(sim.lib.pic_set_preconditioner(cb, None), "set")
        api.check(sim.lib.pic_set_fcg_window(window), "window")
        zero = np.zeros(sim.mesh.nn)
        st_j, phi_j = _solve_from(sim, zero, api.PIC_SOLVER_JPCG)
        st_f, phi_f = _solve_from(sim, zero, api.PIC_SOLVER_FCG_UNET)
        assert st_f.fallback == 0
        assert abs(st_f.iterations - st_j.iterations) <= max(3, st_j.iterations // 20)
        assert np.abs(phi_f - phi_j).max() <= 1e-7 * np.abs(phi_j).max()
        assert _true_rel_residual(sim) <= sim.cfg.pcg_tol * 1.0001
        api.check(sim.lib.pic_set_solver(api.PIC_SOLVER_JPCG), "set")
    finally:
        sim.close()


@gpu
def test_learned_preconditioner_gain_and_tolerance():
    """Trained online on the simulation's own solves, the network cuts flexible
    CG's iterations against the same stages without it, and every solve meets
    the tolerance on its true residual."""
    from pic_b200 import unet
    sim = _sim(ncells=128)
    try:
        lp = unet.LearnedPreconditioner(sim, seed=0, crop=96, batch=4, lr=2e-3, coarse_cells=16)
        for _ in range(30):  # warm-up: Jacobi-PCG steps, pairs harvested, online training
            lp.before_step()
            sim.step()
            lp.after_step(train_iters=8)
        assert lp.losses[-1] < lp.losses[0]
        zero = np.zeros(sim.mesh.nn)
        tol = sim.cfg.pcg_tol
        st_j, phi_j = _solve_from(sim, zero, api.PIC_SOLVER_JPCG)
        assert _true_rel_residual(sim) <= tol * 1.0001
        lp.set_learned(False)
        st_c, phi_c = _solve_from(sim, zero, api.PIC_SOLVER_FCG_UNET)
        assert st_c.fallback == 0 and _true_rel_residual(sim) <= tol * 1.0001
        lp.set_learned(True)
        st_l, phi_l = _solve_from(sim, zero, api.PIC_SOLVER_FCG_UNET)
        assert st_l.fallback == 0, lp.error
        assert _true_rel_residual(sim) <= tol * 1.0001
        scale = np.abs(phi_j).max()
        assert np.abs(phi_l - phi_j).max() <= 1e-6 * scale and np.abs(phi_c - phi_j).max() <= 1e-6 * scale
        print(f"\nJacobi-PCG {st_j.iterations} it; FCG smoothing+coarse {st_c.iterations} it; "
              f"+ learned {st_l.iterations} it; loss {lp.losses[0]:.3f} -> {lp.losses[-1]:.3f}")
        assert st_l.iterations < st_c.iterations < st_j.iterations
    finally:
        sim.close()


@gpu
def test_fcg_graphs_match_eager():
    """Captured FCG iterations (CUDA graphs) give the same solve, bit for
    bit, as the kernel-by-kernel path."""
    from pic_b200.simulation import Simulation
    out = []
    for flag in ("0", "1"):
        os.environ["PIC_FCG_GRAPHS"] = flag
        try:
            sim = Simulation(deck.config("cfg1", ncx=128, ncy=128, ppc=2, pcg_tol=1e-10))
        finally:
            del os.environ["PIC_FCG_GRAPHS"]
        try:
            sim.initial_fields()
            api.check(sim.lib.pic_set_precond_stages(1, 2.0 / 3.0, 0), "stages")
            api.check(sim.lib.pic_coarse_setup(sim.mesh.ptr, 16), "coarse")
            api.check(sim.lib.pic_set_fcg_window(2), "window")
            st, phi = _solve_from(sim, np.zeros(sim.mesh.nn), api.PIC_SOLVER_FCG_UNET)
            assert st.fallback == 0 and _true_rel_residual(sim) <= sim.cfg.pcg_tol * 1.0001
            out.append((st.iterations, phi))
            api.check(sim.lib.pic_set_solver(api.PIC_SOLVER_JPCG), "set")
        finally:
            sim.close()
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])


@gpu
def test_persistent_fcg_matches_graph_path():
    """The one-kernel FCG (window 1, classical stages) and the graph-launched
    iterations reach the same tolerance in the same number of iterations to
    within a few (their restriction sums in a different order)."""
    from pic_b200.simulation import Simulation
    out = []
    for flag in ("0", "1"):
        os.environ["PIC_FCG_PERSISTENT"] = flag
        try:
            sim = Simulation(deck.config("cfg1", ncx=256, ncy=256, ppc=2, pcg_tol=1e-10))
        finally:
            del os.environ["PIC_FCG_PERSISTENT"]
        try:
            sim.initial_fields()
            sim.set_solver("fcg", coarse_cells=32, window=1)
            st, phi = _solve_from(sim, np.zeros(sim.mesh.nn), api.PIC_SOLVER_FCG_UNET)
            assert st.fallback == 0 and _true_rel_residual(sim) <= sim.cfg.pcg_tol * 1.0001
            out.append((st.iterations, phi))
            api.check(sim.lib.pic_set_solver(api.PIC_SOLVER_JPCG), "set")
        finally:
            sim.close()
    assert abs(out[0][0] - out[1][0]) <= 2
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-7 * np.abs(out[0][1]).max()
