"""The discrete adjoint on the GPU (bh_gpu_adjoint / bh_gpu_adjoint_rays).

  - per-ray gradients of the kernel equal the CPU-compiled adjoint's;
  - on the 512^2 gradient workload (a = 0.7, 50 deg, 0.2 Eddington, r_out
    25 M against a target rendered at 0.75, 53 deg, 0.22, 27 M) the gradient
    matches central finite differences of the binary64 forward render with a
    relative step of 1e-4: to 1e-3 over the pixels whose ray ends in the
    same event in both perturbed renders (same class, continuously moving end
    point: the discrete adjoint holds each ray's events fixed), and over the
    whole frame for the Eddington ratio, which moves no edge;
  - the loss is the sum of squared luminance differences of the render;
  - repeated calls give identical bits;
  - the edge term: d/d r_out (the edge term alone) and the whole spin and
    inclination gradients (per-ray terms of the images of order one and two
    plus the edge term) against central differences of a supersampled render
    (64^2 pixels of 8 x 8 samples, where a finite step moves thousands of
    samples across the disc's edges).
"""
import copy
import ctypes as C
import math
import os

import numpy as np
import pytest

from blackhole_b200 import abi, workloads
from blackhole_b200.gpu import BHError

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-3      # relative, against central finite differences
FD_REL_STEP = 1e-4


def _with(cfg, k, v):
    c = copy.deepcopy(cfg)
    if k == 0:
        c.spin = v
    elif k == 1:
        c.cam.theta = v
    elif k == 2:
        c.eddington = v
    else:
        c.disc_r_out = v
    return c


def _params(cfg):
    return [cfg.spin, cfg.cam.theta, cfg.eddington, cfg.disc_r_out]


def _lum(renderer, cfg):
    return renderer.render(cfg)[..., 1]


@pytest.fixture(scope="module")
def c4(renderer):
    cfg = workloads.adjoint_512()
    target = _lum(renderer, workloads.adjoint_512(target=True)).astype(np.float32)
    g, per_ray, ray_y = renderer.adjoint(cfg, target, per_ray=True)
    return cfg, target, g, per_ray, ray_y


def test_loss_is_the_sum_of_squared_luminance_differences(renderer, c4):
    cfg, target, g, per_ray, ray_y = c4
    Y = _lum(renderer, cfg)
    loss = float(np.sum((Y - target.astype(np.float64)) ** 2))
    assert g["loss"] == pytest.approx(loss, rel=1e-12)
    # The adjoint's own binary64 forward pass reproduces the render's
    # luminances (its right-hand side is written without the render kernel's
    # angle-addition and single-reciprocal forms, so rays can differ at the
    # integration tolerance, and a ray whose event sits at rounding distance
    # from a class boundary can end in the other class).
    close = np.isclose(ray_y, Y.reshape(-1), rtol=1e-6, atol=1e-12 * Y.max())
    assert close.mean() > 0.9995
    assert g["rays"] == cfg.width * cfg.height
    assert g["disc_rays"] > 0 and g["sky_rays"] > 0
    # the r_out derivative is the edge term alone
    assert math.isfinite(g["d_r_out"]) and g["d_r_out"] != 0.0
    assert g["edge_cells"] > 0 and g["edge_candidates"] >= g["edge_cells"] // 2
    assert float(per_ray[:, 3].sum()) == 0.0


@pytest.mark.parametrize("k,name", [(0, "d_spin"), (1, "d_inclination"), (2, "d_eddington")])
def test_gradient_matches_central_differences(renderer, c4, k, name):
    cfg, target, g, per_ray, _ = c4
    v = _params(cfg)[k]
    h = FD_REL_STEP * abs(v)
    cp, cm = _with(cfg, k, v + h), _with(cfg, k, v - h)
    t = target.astype(np.float64)
    lp = (_lum(renderer, cp) - t) ** 2
    lm = (_lum(renderer, cm) - t) ** 2
    r0, rp, rm = renderer.trace_rays(cfg), renderer.trace_rays(cp), renderer.trace_rays(cm)
    w0, wp, wm = r0["what"], rp["what"], rm["what"]
    Y = _lum(renderer, cfg).reshape(-1)
    same = np.isclose(c4[4], Y, rtol=1e-6, atol=1e-12 * Y.max())   # adjoint forward agrees with the render
    # The same event in both perturbed renders: same class, and the final
    # radius moved continuously (a ray whose first disc crossing passes the
    # inner edge sees the far side of the disc instead: same class, other
    # crossing, a jump in the frame the discrete adjoint does not contain).
    r_end0, r_endp, r_endm = r0["y"][:, 1], rp["y"][:, 1], rm["y"][:, 1]
    cont = np.abs(r_endp - r_endm) <= 1e-3 * np.abs(r_end0)
    stable = ((wp == w0) & (wm == w0) & same & cont).reshape(lp.shape)
    fd = float(np.sum((lp - lm)[stable])) / (2 * h)
    adj = float(np.sum(per_ray[:, k].reshape(lp.shape)[stable]))
    assert adj == pytest.approx(fd, rel=GRAD_TOL), (name, adj, fd, int((~stable).sum()))
    # the frame total is the sum of the per-ray contributions of images of
    # order one and two and the edge term; the rest is held out
    edge = {0: g["edge_spin"], 1: g["edge_inclination"], 2: 0.0}[k]
    held = {0: g["held_spin"], 1: g["held_inclination"], 2: 0.0}[k]
    assert g[name] - edge + held == pytest.approx(float(per_ray[:, k].sum()), rel=1e-12, abs=1e-300)
    if k == 2:
        assert ((wp == w0) & (wm == w0)).all()
        fd_all = float(np.sum(lp - lm)) / (2 * h)
        assert g[name] == pytest.approx(fd_all, rel=GRAD_TOL)


def test_repeated_calls_are_bitwise_identical(renderer, c4):
    cfg, target, g, per_ray, _ = c4
    g2, per_ray2, _ = renderer.adjoint(cfg, target, per_ray=True)
    for key in ("loss", "d_spin", "d_inclination", "d_eddington", "d_r_out", "edge_spin", "edge_inclination",
                "edge_cells", "edge_candidates"):
        assert g2[key] == g[key]
    assert np.array_equal(per_ray, per_ray2)


def test_kernel_rays_match_the_cpu_adjoint(renderer):
    from blackhole_b200.build import CHECK_LIB, build_check

    if not os.path.exists(CHECK_LIB):
        build_check()
    lib = C.CDLL(CHECK_LIB)
    D = C.POINTER(C.c_double)
    lib.bhx_ray.argtypes = [C.POINTER(abi.bh_render_config), C.c_longlong, C.c_double, C.c_int, C.c_int, D]
    cfg = workloads.adjoint_512()
    cfg.width = cfg.height = 48
    target = np.zeros((48, 48), dtype=np.float32)
    Y = _lum(renderer, cfg)
    _, per_ray, _ = renderer.adjoint(cfg, target, per_ray=True)
    order = abi.work_order(48, 48, 1)          # ray id -> trace_rays index
    for rid in range(0, 48 * 48, 97):
        idx = order[rid]
        w = 2.0 * Y.reshape(-1)[idx]
        out = np.zeros(9)
        c = cfg.to_c()
        assert lib.bhx_ray(C.byref(c), rid, w, 0, 0, out.ctypes.data_as(D)) == abi.OK
        assert np.allclose(per_ray[idx], out[1:5], rtol=1e-6, atol=1e-12 * np.abs(out[1:5]).max())


def test_unsupported_scene_and_bad_target_are_refused(renderer):
    cfg = workloads.adjoint_512()
    cfg.width = cfg.height = 16
    with pytest.raises(ValueError):
        renderer.adjoint(cfg, np.zeros(10, dtype=np.float32))
    cfg.sun_enabled = True
    with pytest.raises(BHError) as e:
        renderer.adjoint(cfg, np.zeros((16, 16), dtype=np.float32))
    assert e.value.code == abi.ERR_UNSUPPORTED


def test_autograd_wrapper_returns_the_adjoint(renderer, c4):
    torch = pytest.importorskip("torch")
    from blackhole_b200.autograd import luminance_loss

    cfg, target, g, _, _ = c4
    params = torch.tensor(_params(cfg), dtype=torch.float64, requires_grad=True)
    loss = luminance_loss(params, target, cfg, renderer)
    loss.backward()
    assert float(loss.detach()) == g["loss"]
    assert params.grad.tolist() == [g["d_spin"], g["d_inclination"], g["d_eddington"], g["d_r_out"]]


@pytest.mark.parametrize("k,name", [(0, "d_spin"), (1, "d_inclination")])
def test_photon_ring_crop_gradient_matches_central_differences(renderer, k, name):
    """The adjoint of the photon-ring frame (a = 0.998, 75 deg, centred on the
    critical curve) on a 1024^2 crop, against central differences with
    relative step 1e-4, over the rays whose event is the same in both
    perturbed renders."""
    cfg = workloads.photon_ring_crop(1024)
    target = _lum(renderer, workloads.photon_ring_crop(1024, target=True)).astype(np.float32)
    g, per_ray, ray_y = renderer.adjoint(cfg, target, per_ray=True)
    v = _params(cfg)[k]
    h = FD_REL_STEP * abs(v)
    cp, cm = _with(cfg, k, v + h), _with(cfg, k, v - h)
    t = target.astype(np.float64)
    lp = (_lum(renderer, cp) - t) ** 2
    lm = (_lum(renderer, cm) - t) ** 2
    r0, rp, rm = renderer.trace_rays(cfg), renderer.trace_rays(cp), renderer.trace_rays(cm)
    Y = _lum(renderer, cfg).reshape(-1)
    same = np.isclose(ray_y, Y, rtol=1e-6, atol=1e-12 * Y.max())
    cont = np.abs(rp["y"][:, 1] - rm["y"][:, 1]) <= 1e-3 * np.abs(r0["y"][:, 1])
    stable = ((rp["what"] == r0["what"]) & (rm["what"] == r0["what"]) & same & cont).reshape(lp.shape)
    fd = float(np.sum((lp - lm)[stable])) / (2 * h)
    adj = float(np.sum(per_ray[:, k].reshape(lp.shape)[stable]))
    assert adj == pytest.approx(fd, rel=GRAD_TOL), (name, adj, fd, int((~stable).sum()))


def _supersampled(n, s, target=False):
    cfg = workloads.adjoint_512(target=target)
    cfg.width = cfg.height = n
    cfg.sqrt_spp = s
    return cfg


@pytest.fixture(scope="module")
def supersampled(renderer):
    cfg = _supersampled(64, 8)
    T = _lum(renderer, _supersampled(64, 8, target=True)).astype(np.float32)
    return cfg, T, renderer.adjoint(cfg, T)


def _fd(renderer, cfg, T, k, h):
    t = T.astype(np.float64)
    v = _params(cfg)[k]
    lp = float(np.sum((_lum(renderer, _with(cfg, k, v + h)) - t) ** 2))
    lm = float(np.sum((_lum(renderer, _with(cfg, k, v - h)) - t) ** 2))
    return (lp - lm) / (2 * h)


def test_r_out_edge_term_matches_supersampled_differences(renderer, supersampled):
    """d loss / d r_out of a 64^2 frame of 8 x 8 samples per pixel (the
    edge term: the outer edge's motion across the image) against central
    differences with a step of 0.25 M, which moves every sample whose
    crossing lies within 0.25 M of r_out across the edge; 2 % tolerance."""
    cfg, T, g = supersampled
    fd = _fd(renderer, cfg, T, 3, 0.25)
    assert g["d_r_out"] == pytest.approx(fd, rel=0.02), (g["d_r_out"], fd, g["edge_cells"])


@pytest.mark.parametrize("k,name", [(0, "d_spin"), (1, "d_inclination")])
def test_whole_gradient_matches_supersampled_differences(renderer, supersampled, k, name):
    """The spin and inclination gradients of the same frame (the per-ray
    terms of images of order one and two and the edge term of both disc
    edges) against central differences with a step of 0.01; 5 % tolerance.
    Without the edge term the inclination gradient has the wrong sign here:
    the disc's outer edge sweeping across the image dominates it."""
    cfg, T, g = supersampled
    fd = _fd(renderer, cfg, T, k, 1e-2)
    assert g[name] == pytest.approx(fd, rel=0.05), (name, g[name], fd)
    if k == 1:
        interior = g[name] - g["edge_inclination"]
        assert np.sign(interior) != np.sign(fd)


def test_gradient_descent_recovers_the_scene(renderer):
    """The gradient drives an optimiser to the scene that made the target:
    from (a, inclination, Eddington ratio, r_out) = (0.8, 54 deg, 0.24, 28 M)
    to the target's (0.7, 50 deg, 0.2, 25 M) on a 64^2 frame of 4 x 4 samples
    per pixel, with Adam over 150 steps (parameters scaled to comparable
    sizes).  r_out moves only through the edge term."""
    torch = pytest.importorskip("torch")
    from blackhole_b200.autograd import luminance_loss

    def frame(a, inc, edd, r_out):
        c = workloads.adjoint_512()
        c.width = c.height = 64
        c.sqrt_spp = 4
        c.spin, c.cam.theta, c.eddington, c.disc_r_out = a, math.radians(inc), edd, r_out
        return c

    truth = (0.7, 50.0, 0.2, 25.0)
    start = (0.8, 54.0, 0.24, 28.0)
    target = _lum(renderer, frame(*truth)).astype(np.float32)
    cfg = frame(*start)
    scale = torch.tensor([0.1, 0.05, 0.05, 2.0], dtype=torch.float64)
    z = (torch.tensor([start[0], math.radians(start[1]), start[2], start[3]], dtype=torch.float64) / scale)
    z.requires_grad_(True)
    opt = torch.optim.Adam([z], lr=0.05)
    first = None
    for _ in range(150):
        opt.zero_grad()
        loss = luminance_loss(z * scale, target, cfg, renderer)
        loss.backward()
        opt.step()
        first = float(loss.detach()) if first is None else first
    a, inc, edd, r_out = (z * scale).detach().tolist()
    with torch.no_grad():
        final = float(luminance_loss(z * scale, target, cfg, renderer))
    assert final < 1e-3 * first
    assert abs(a - 0.7) < 2e-3 and abs(math.degrees(inc) - 50.0) < 0.05
    assert abs(edd - 0.2) < 1e-3 and abs(r_out - 25.0) < 0.05
