"""GPU tests of the voxel-grid form (`psc_render_grid`) and its adjoint
(`psc_adjoint`) at the differentiation workload's full size: 256x256x64
Worley grid over 20x20x2 km, 512x512 view, 96 + 6 steps, checkpoint every 16.

Checked against the FP64 oracle (oracle/oracle_grid.cpp): the forward image,
the loss, the full gradient (an independent reverse sweep over all stored
steps) and Richardson-extrapolated central differences of the FP64 loss on
64 seeded voxels.  The finite-difference step is 1e-3 of the grid's largest
value (5e-5 1/m) and half of it: at 1e-3 1/m itself the loss is so curved in
empty voxels next to cloud edges (each such voxel turns into a new
scatterer) that the plain central difference's truncation error exceeds the
derivative, while the extrapolated difference agrees with the FP64 adjoint
to ~1e-9.  The target is the oracle's render of the grid with 5 % Gaussian
noise on every value."""
import ctypes as C

import numpy as np
import pytest

from pedalsky_b200 import capi, scenes
from pedalsky_b200 import grid as GR
from pedalsky_b200.capi import PscError, call
from pedalsky_b200.subsystem import subsystem_for_scene

from . import _gpu
from ._metrics import composite, rel_stats

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prob(oracle, oracle_noise):
    torch = _gpu.torch_cuda()
    sc = scenes.grid_512()
    luts = oracle.bake_luts(sc.frame, sc.world)
    G = sc.extra["grid"]
    spec = dict(sc.extra["grid_spec"])
    Lt, Tt = oracle.grid_render(sc, oracle_noise, luts, scenes.grid_target_values(G), spec)
    tgt = (Lt + sc.background * Tt).astype(np.float32)
    sub = subsystem_for_scene(sc, luts=luts, noise=oracle_noise)
    P = GR.GridProblem(sc, G)
    P.set_target(tgt)
    cache = {}
    yield dict(sc=sc, luts=luts, G=G, spec=spec, tgt=tgt, sub=sub, P=P, torch=torch, cache=cache)
    sub.close()


def _oracle_adjoint(oracle, noise, p, exit_t):
    key = ("adj", exit_t)
    if key not in p["cache"]:
        sp = dict(p["spec"], exit_transmittance=exit_t)
        p["cache"][key] = oracle.grid_adjoint(p["sc"], noise, p["luts"], p["G"], sp,
                                              p["sc"].background, p["tgt"], threads=8)
    return p["cache"][key]


def _gpu_adjoint(p, exit_t, k=16, rows=None):
    P = p["P"]
    P.spec.update(exit_transmittance=exit_t, checkpoint_every=k)
    P.zero_grad()
    for r in (rows or [None]):
        P.adjoint(p["sub"].handle, rows=r)
    p["torch"].cuda.synchronize()
    return P.grad.cpu().numpy().astype(np.float64), P.acc.cpu().numpy()


def test_grid_forward_matches_fp64_oracle(oracle, oracle_noise, prob):
    sc, P = prob["sc"], prob["P"]
    P.spec.update(exit_transmittance=0.01)
    P.render(prob["sub"].handle)
    prob["torch"].cuda.synchronize()
    L, T = P.L.cpu().numpy(), P.T.cpu().numpy()
    Lo, To = oracle.grid_render(sc, oracle_noise, prob["luts"], prob["G"], prob["spec"])
    st = rel_stats(composite(L, T, sc.background), composite(Lo, To, sc.background))
    print("grid forward vs FP64:", st)
    assert st["p999"] <= 1e-4 and st["max"] <= 1e-3, st
    assert (T[..., :3] < 0.5).mean() > 0.05  # the view does see cloud


@pytest.mark.parametrize("exit_t", [0.01, 0.0])
def test_adjoint_matches_fp64_gradient(oracle, oracle_noise, prob, exit_t):
    g, acc = _gpu_adjoint(prob, exit_t)
    go, gso, lo = _oracle_adjoint(oracle, oracle_noise, prob, exit_t)
    l2 = np.linalg.norm(g - go) / np.linalg.norm(go)
    act = np.abs(go) > 1e-2 * np.abs(go).max()
    r = np.abs(g - go)[act] / np.abs(go)[act]
    print(f"exit {exit_t}: rel L2 {l2:.3g}, active {act.sum()}, rel median {np.median(r):.3g}, "
          f"p99 {np.quantile(r, 0.99):.3g}; loss {acc[0]} vs {lo}; d/dscale {acc[1]} vs {gso}")
    assert act.sum() > 1000
    assert l2 <= 2e-3, l2
    assert np.median(r) <= 2e-3
    assert abs(acc[0] - lo) <= 1e-5 * lo
    assert abs(acc[1] - gso) <= 5e-3 * abs(gso)


def test_adjoint_matches_central_differences(oracle, oracle_noise, prob):
    """64 seeded voxels among those the image depends on, no early exit."""
    g, acc = _gpu_adjoint(prob, 0.0)
    go, gso, _ = _oracle_adjoint(oracle, oracle_noise, prob, 0.0)
    sp = dict(prob["spec"], exit_transmittance=0.0)
    flat = np.abs(go).ravel()
    rng = np.random.default_rng(1)
    vox = rng.choice(np.flatnonzero(flat > 1e-4 * flat.max()), 64, replace=False)
    fd, _, npx = oracle.grid_fd_richardson(prob["sc"], oracle_noise, prob["luts"], prob["G"], sp,
                                           prob["sc"].background, prob["tgt"], vox,
                                           1e-3 * float(prob["G"].max()))
    assert (npx > 0).all()
    a, b = g.ravel()[vox], go.ravel()[vox]
    rel = np.abs(a - fd) / np.abs(fd)
    print(f"GPU vs FD: median {np.median(rel):.3g}, max {rel.max():.3g}, "
          f"max abs / max|grad| {np.abs(a - fd).max() / flat.max():.3g}")
    np.testing.assert_allclose(b, fd, rtol=1e-4)                       # the oracle itself
    assert np.all(np.abs(a - fd) <= 5e-3 * np.abs(fd) + 5e-4 * flat.max())
    assert np.median(rel) <= 2e-3
    # density_scale, over the FP32 values actually applied
    hi, lo = np.float32(1 + 1e-5), np.float32(1 - 1e-5)
    lp = oracle.grid_loss(prob["sc"], oracle_noise, prob["luts"], prob["G"],
                          dict(sp, density_scale=float(hi)), prob["sc"].background, prob["tgt"])
    lm = oracle.grid_loss(prob["sc"], oracle_noise, prob["luts"], prob["G"],
                          dict(sp, density_scale=float(lo)), prob["sc"].background, prob["tgt"])
    fds = (lp - lm) / (float(hi) - float(lo))
    assert abs(fds - gso) <= 1e-4 * abs(fds)
    assert abs(acc[1] - fds) <= 5e-3 * abs(fds)


def test_checkpoint_interval_and_row_bands_do_not_change_the_gradient(prob):
    base, acc = _gpu_adjoint(prob, 0.01)
    nb = np.linalg.norm(base)
    for k in (4, 8, 32):
        gk, ak = _gpu_adjoint(prob, 0.01, k=k)
        assert np.linalg.norm(gk - base) <= 1e-5 * nb, k
        assert abs(ak[0] - acc[0]) <= 1e-9 * acc[0]
    gb, ab = _gpu_adjoint(prob, 0.01, rows=[(0, 200), (200, 512)])
    assert np.linalg.norm(gb - base) <= 1e-5 * nb
    assert abs(ab[0] - acc[0]) <= 1e-9 * acc[0]
    assert abs(ab[1] - acc[1]) <= 1e-5 * abs(acc[1])


def test_grid_argument_errors(prob):
    P, h = prob["P"], prob["sub"].handle
    P.spec.update(exit_transmittance=0.01, checkpoint_every=16)
    for k in (0, 33, 2):  # 96 steps at k = 2 need 48 checkpoints (> 32)
        P.spec["checkpoint_every"] = k
        with pytest.raises(PscError) as e:
            P.adjoint(h)
        assert e.value.code == -1
    P.spec["checkpoint_every"] = 16
    bad = P.grid()
    bad.values = None
    v = capi.View(8, 8, None, P.L.data_ptr(), None, None)
    with pytest.raises(PscError):
        call("psc_render_grid", h, C.byref(bad), C.byref(v), None)
    bad = P.grid()
    bad.exit_transmittance = 1.0
    with pytest.raises(PscError):
        call("psc_render_grid", h, C.byref(bad), C.byref(v), None)
    with pytest.raises(PscError):  # adjoint without a target buffer
        call("psc_adjoint", h, C.byref(P.grid()), C.byref(v), C.c_void_p(P.bg.data_ptr()), None,
             C.c_void_p(P.grad.data_ptr()), C.c_void_p(P.acc.data_ptr() + 8),
             C.c_void_p(P.acc.data_ptr()), None)


def test_layer_range_gradient_matches_central_differences(oracle, oracle_noise):
    """d loss / d base_m and d loss / d top_m of the layer (psc_layer_gradient)
    on a 128x128 view of the same grid scene, no early exit, against
    Richardson-extrapolated central differences (1 m and 0.5 m) of the FP64
    oracle's loss; and row bands add up to the whole view."""
    import dataclasses
    torch = _gpu.torch_cuda()
    sc = scenes.grid_512(128, 128)
    luts = oracle.bake_luts(sc.frame, sc.world)
    G = sc.extra["grid"]
    spec = dict(sc.extra["grid_spec"], exit_transmittance=0.0)
    Lt, Tt = oracle.grid_render(sc, oracle_noise, luts, scenes.grid_target_values(G), spec)
    tgt = (Lt + sc.background * Tt).astype(np.float32)
    sub = subsystem_for_scene(sc, luts=luts, noise=oracle_noise)
    try:
        P = GR.GridProblem(sc, G, spec=spec)
        P.set_target(tgt)
        out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
        P.layer_gradient(sub.handle, out)
        bands = torch.zeros(2, dtype=torch.float64, device="cuda:0")
        P.layer_gradient(sub.handle, bands, rows=(0, 50))
        P.layer_gradient(sub.handle, bands, rows=(50, 128))
        torch.cuda.synchronize()
        g = out.cpu().numpy()
        gb = bands.cpu().numpy()
    finally:
        sub.close()

    def loss(d_base, d_top):
        layers = (capi.CloudLayerGpu * 8).from_buffer_copy(sc.layers)
        layers[0].base_m = float(np.float32(sc.layers[0].base_m + d_base))
        layers[0].top_m = float(np.float32(sc.layers[0].top_m + d_top))
        s2 = dataclasses.replace(sc, layers=layers)
        return oracle.grid_loss(s2, oracle_noise, luts, G, spec, sc.background, tgt)

    fd = []
    for e_base, e_top in ((1.0, 0.0), (0.0, 1.0)):
        d1 = (loss(e_base, e_top) - loss(-e_base, -e_top)) / 2.0
        d2 = (loss(e_base / 2, e_top / 2) - loss(-e_base / 2, -e_top / 2)) / 1.0
        fd.append((4.0 * d2 - d1) / 3.0)
    fd = np.array(fd)
    rel = np.abs(g - fd) / np.abs(fd)
    print(f"\nlayer gradient d/dbase, d/dtop: GPU {g}, FD {fd}, rel {rel}")
    assert np.all(np.abs(fd) > 0)
    assert np.all(rel <= 2e-2), (g, fd)
    assert np.allclose(gb, g, rtol=1e-5, atol=0)
