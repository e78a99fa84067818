"""Path-replay adjoint (rtb_render_backward) against central finite differences and the FP64
CPU restatement.

Loss: L = sum over pixels and channels of (I - T)^2, accumulated in FP64, with T rendered from
perturbed albedos; dL/dI = 2 (I - T).  Finite differences are central (h = 1e-3) with common
random numbers (same frame seed); for diffuse-only materials the sampled paths do not depend on
albedo or emission, so the image is a polynomial in them and the FD is smooth.  64 parameters
are drawn uniformly from all albedo and emission components (bench.fd_check).  Tolerance:
relative error <= 1e-2 on every drawn parameter whose FD is at least 1e-2 of its group's
typical gradient (the median non-zero magnitude); the rest (including parameters of
primitives no path reaches, whose FD and gradient are both exactly zero) are reported apart
and held to an absolute error of 1e-3 of that typical gradient (near 1e-4 of it, a central
difference of an FP32 image is at its noise floor: measured 1.0e-4 on the benchmark scene).  The benchmark's own configuration (4,096 primitives, 512x512,
32 spp, depth 6) is checked in full, as is a smaller scene against the FP64 CPU adjoint.
"""
import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth
from rtb200.diff import DifferentiableScene, render_function
from rtb200.tracer import Context

pytestmark = pytest.mark.gpu


def _setup(torch, n=600, w=64, h=48, spp=8, depth=4):
    s = synth.hetero_scene(n, 41, synth.WORKLOAD_IDS["test"], 30)
    wl = synth.Workload("adj", s, synth.camera_looking_z((0.0, 0.0, -2.9), w / h), w, h, spp, depth,
                        frame_seed=77, frame_index=2)
    ctx = Context(0)
    ds = DifferentiableScene(ctx, s, w, h, spp, depth, wl.camera, wl.frame_index, wl.frame_seed)
    return ctx, ds, wl


def _render(torch, ds, albedo, emission):
    ds.set_parameters(albedo, emission)
    img = torch.empty(ds.width * ds.height * 3, dtype=torch.float32, device="cuda")
    ds.render_into(img.data_ptr())
    torch.cuda.synchronize()
    return img.cpu().numpy()


def _grads(torch, ds, adj):
    a = torch.from_numpy(np.ascontiguousarray(adj, dtype=np.float32)).cuda()
    ga = torch.empty(ds.count * 3, dtype=torch.float32, device="cuda")
    ge = torch.empty(ds.count * 3, dtype=torch.float32, device="cuda")
    ds.backward_into(a.data_ptr(), ga.data_ptr(), ge.data_ptr())
    torch.cuda.synchronize()
    return ga.cpu().numpy().reshape(-1, 3), ge.cpu().numpy().reshape(-1, 3)


def _check_fd(fd):
    print("\nFD check: %d parameters; %d large (max rel err %.3g, median %.3g); %d small "
          "(max abs err / typical gradient %.3g, %d exactly zero)"
          % (fd["parameters"], fd["large"]["count"], fd["large"]["max_rel_err"],
             fd["large"]["median_rel_err"], fd["small"]["count"],
             fd["small"]["max_abs_err_over_scale"], fd["small"]["exact_zero"]))
    for i, grp, g, f, scale in fd["rows"]:
        print("  %6d %s grad %+.6e fd %+.6e rel %.2e" % (i, "albedo  " if grp == 0 else "emission",
                                                          g, f, abs(g - f) / max(abs(f), 1e-300)))
    assert fd["parameters"] == 64
    assert fd["large"]["count"] >= 16
    assert fd["large"]["max_rel_err"] <= 1e-2
    assert fd["small"]["max_abs_err_over_scale"] <= 1e-3


def test_adjoint_c5_config_finite_differences_on_uniform_parameters():
    """The differentiable benchmark configuration in full: 4,096 mixed primitives each with
    its own material, 512x512, 32 spp, depth 6; target rendered with albedos perturbed by
    N(0, 0.05) (12-uniform sum), clamped to [0, 1]."""
    torch = pytest.importorskip("torch")
    w = synth.adjoint_workload()
    ctx = Context(0)
    ds = DifferentiableScene(ctx, w.scene, w.width, w.height, w.spp, w.max_depth, w.camera,
                             w.frame_index, w.frame_seed)
    try:
        alb0, emi0 = ds.albedo(), ds.emission()
        st = synth.Stream(1, synth.WORKLOAD_IDS["adjoint"], 1, 7)
        u12 = st.uniform(12 * alb0.size).reshape(-1, 3, 12)
        target_alb = np.clip(alb0 + 0.05 * (u12.sum(axis=2) - 6.0) * (alb0 > 0), 0.0, 1.0)
        target = _render(torch, ds, target_alb, emi0).astype(np.float64)
        img = _render(torch, ds, alb0, emi0)
        ga, ge = _grads(torch, ds, 2.0 * (img.astype(np.float64) - target))
        g = np.concatenate([ga.reshape(-1), ge.reshape(-1)]).astype(np.float64)

        def loss(alb, emi):
            return float(np.sum((_render(torch, ds, alb, emi).astype(np.float64) - target) ** 2))

        import bench
        fd = bench.fd_check(g, ga.size, loss, alb0, emi0, 64, np.random.default_rng(1))
        _check_fd(fd)
    finally:
        ds.close()
        ctx.close()


def test_adjoint_matches_finite_differences_and_fp64_cpu():
    torch = pytest.importorskip("torch")
    ctx, ds, wl = _setup(torch)
    try:
        alb0, emi0 = ds.albedo(), ds.emission()
        st = synth.Stream(5, synth.WORKLOAD_IDS["test"], 31, 1)
        noise = (st.uniform(12 * alb0.size).reshape(-1, 3, 12).sum(axis=2) - 6.0) * 0.05
        target_alb = np.clip(alb0 + noise * (alb0 > 0), 0.0, 1.0)
        target = _render(torch, ds, target_alb, emi0)
        img = _render(torch, ds, alb0, emi0)
        adj = 2.0 * (img.astype(np.float64) - target)
        ga, ge = _grads(torch, ds, adj)

        def loss(alb, emi):
            im = _render(torch, ds, alb, emi).astype(np.float64)
            return float(np.sum((im - target) ** 2))

        g = np.concatenate([ga.reshape(-1), ge.reshape(-1)]).astype(np.float64)
        import bench
        fd = bench.fd_check(g, ga.size, loss, alb0, emi0, 64, np.random.default_rng(3))
        _check_fd(fd)
        big = np.array([r[0] for r in fd["rows"] if abs(r[3]) >= bench.FD_SMALL * r[4] > 0])

        # FP64 CPU restatement of the same adjoint (same paths except where the host and
        # CUDA sin/cos differ by an ulp)
        ds.set_parameters(alb0, emi0)
        bvh = oracle.build_bvh(wl.scene)
        ca, ce = oracle.adjoint(wl, adj.astype(np.float32), bvh)
        gc = np.concatenate([ca.reshape(-1), ce.reshape(-1)])
        rel = np.abs(g[big] - gc[big]) / np.abs(gc[big])
        assert np.median(rel) <= 1e-4 and np.max(rel) <= 1e-2, (np.median(rel), np.max(rel))
    finally:
        ds.close()
        ctx.close()


def test_autograd_function_forward_backward():
    torch = pytest.importorskip("torch")
    ctx, ds, wl = _setup(torch, n=300, w=32, h=24, spp=4, depth=3)
    try:
        F = render_function()
        alb = torch.tensor(ds.albedo(), requires_grad=True)
        emi = torch.tensor(ds.emission(), requires_grad=True)
        img = F.apply(alb, emi, ds)
        direct = _render(torch, ds, ds.albedo(), ds.emission())
        np.testing.assert_array_equal(img.detach().cpu().numpy(), direct)
        loss = (img ** 2).sum()
        loss.backward()
        ga, ge = _grads(torch, ds, 2.0 * direct)
        np.testing.assert_allclose(alb.grad.cpu().numpy(), ga, rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(emi.grad.cpu().numpy(), ge, rtol=1e-5, atol=1e-7)
    finally:
        ds.close()
        ctx.close()


def test_host_buffer_backward_matches_device_backward():
    """rtb_render_backward_sample (host buffers, the entry a Java Function binds) gives the
    device entry's gradients (FP32 atomics gather them, so to 1e-5 relative)."""
    torch = pytest.importorskip("torch")
    ctx, ds, wl = _setup(torch, n=300, w=32, h=24, spp=4, depth=3)
    try:
        import ctypes as C
        from rtb200 import native as N
        img = _render(torch, ds, ds.albedo(), ds.emission())
        adj = (2.0 * img).astype(np.float32)
        ga, ge = _grads(torch, ds, adj)
        ha = np.zeros(ds.count * 3, np.float32)
        he = np.zeros(ds.count * 3, np.float32)
        ctx.check(ctx.lib.rtb_render_backward_sample(ctx.handle, ds.res.handle, C.byref(ds.cam),
                                                     C.byref(ds.params), N.fptr(adj),
                                                     N.fptr(ha), N.fptr(he)))
        np.testing.assert_allclose(ha.reshape(-1, 3), ga, rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(he.reshape(-1, 3), ge, rtol=1e-5, atol=1e-7)
    finally:
        ds.close()
        ctx.close()
