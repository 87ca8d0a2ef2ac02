"""CPU checks of the voxel-grid oracle that the GPU adjoint is tested against:
its FP64 reverse-mode gradient agrees with central finite differences of its
own FP64 loss (Richardson-extrapolated), the finite differences need only the
pixels the voxel touches, and row-band gradients summed over two gloo ranks
equal the single-process gradient (the adjoint's multi-GPU exchange)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pedalsky_b200 import scenes, sharding

SMALL = dict(width=48, height=40, grid_shape=(48, 12, 48), steps=24)


def _problem(oracle, noise, exit_t=0.0):
    sc = scenes.grid_512(**SMALL)
    luts = oracle.bake_luts(sc.frame, sc.world)
    G = sc.extra["grid"]
    spec = dict(sc.extra["grid_spec"], exit_transmittance=exit_t)
    Lt, Tt = oracle.grid_render(sc, noise, luts, scenes.grid_target_values(G), spec)
    tgt = (Lt + sc.background * Tt).astype(np.float32)
    return sc, luts, G, spec, tgt


@pytest.fixture(scope="module")
def small(oracle, oracle_noise):
    return _problem(oracle, oracle_noise)


def test_grid_values_follow_the_spec():
    G = scenes.worley_grid(64, 16, 64, seed=0)
    assert G.shape == (16, 64, 64) and G.dtype == np.float32
    assert G.min() == 0.0 and 0.04 < G.max() <= 0.05
    assert 0.02 < (G > 0).mean() < 0.6
    assert np.array_equal(G, scenes.worley_grid(64, 16, 64, seed=0))
    Gt = scenes.grid_target_values(G)
    assert (Gt >= 0).all() and np.allclose(Gt[G == 0], 0)
    rel = (Gt[G > 0] - G[G > 0]) / G[G > 0]
    assert abs(rel.std() - 0.05) < 0.005


def test_oracle_adjoint_matches_extrapolated_central_differences(oracle, oracle_noise, small):
    sc, luts, G, spec, tgt = small
    grad, gs, loss = oracle.grid_adjoint(sc, oracle_noise, luts, G, spec, sc.background, tgt)
    assert loss > 0 and np.isfinite(grad).all()
    # the reported loss is the oracle's forward loss
    l_fwd = oracle.grid_loss(sc, oracle_noise, luts, G, spec, sc.background, tgt)
    assert abs(loss - l_fwd) <= 1e-12 * l_fwd
    rng = np.random.default_rng(5)
    flat = np.abs(grad).ravel()
    active = np.flatnonzero(flat > 1e-3 * flat.max())
    vox = rng.choice(active, 16, replace=False)
    eps = 1e-3 * float(G.max())
    fd, _, npx = oracle.grid_fd_richardson(sc, oracle_noise, luts, G, spec, sc.background, tgt,
                                           vox, eps)
    assert (npx > 0).all()
    a = grad.ravel()[vox]
    np.testing.assert_allclose(a, fd, rtol=2e-4, atol=1e-6 * flat.max())
    assert abs(_scale_fd(oracle, oracle_noise, sc, luts, G, spec, tgt, 1e-5) - gs) <= 1e-5 * abs(gs)


def _scale_fd(oracle, noise, sc, luts, G, spec, tgt, e):
    """Central difference in density_scale over the FP32 values actually applied."""
    hi, lo = np.float32(1 + e), np.float32(1 - e)
    lp = oracle.grid_loss(sc, noise, luts, G, dict(spec, density_scale=float(hi)), sc.background, tgt)
    lm = oracle.grid_loss(sc, noise, luts, G, dict(spec, density_scale=float(lo)), sc.background, tgt)
    return (lp - lm) / (float(hi) - float(lo))


def test_fd_over_touched_pixels_equals_full_image_difference(oracle, oracle_noise, small):
    sc, luts, G, spec, tgt = small
    grad, _, _ = oracle.grid_adjoint(sc, oracle_noise, luts, G, spec, sc.background, tgt)
    v = int(np.argmax(np.abs(grad)))
    eps = 1e-4
    fd, npx = oracle.grid_fd(sc, oracle_noise, luts, G, spec, sc.background, tgt, [v], eps)
    flat = G.ravel().copy()
    vals = []
    for d in (eps, -eps):
        flat[v] = np.float32(G.ravel()[v] + d)
        vals.append(oracle.grid_loss(sc, oracle_noise, luts, flat.reshape(G.shape), spec,
                                     sc.background, tgt))
    flat[v] = G.ravel()[v]
    h = float(np.float32(G.ravel()[v] + eps)) - float(np.float32(G.ravel()[v] - eps))
    assert 0 < npx[0] < sc.width * sc.height
    assert abs(fd[0] - (vals[0] - vals[1]) / h) <= 1e-9 * abs(fd[0])


def test_early_exit_truncates_the_march_consistently(oracle, oracle_noise):
    sc, luts, G, spec, tgt = _problem(oracle, oracle_noise, exit_t=0.01)
    grad, gs, loss = oracle.grid_adjoint(sc, oracle_noise, luts, G, spec, sc.background, tgt)
    l_fwd = oracle.grid_loss(sc, oracle_noise, luts, G, spec, sc.background, tgt)
    assert abs(loss - l_fwd) <= 1e-12 * l_fwd
    # a step small enough that no pixel changes its exit step
    assert abs(_scale_fd(oracle, oracle_noise, sc, luts, G, spec, tgt, 1e-6) - gs) <= 1e-4 * abs(gs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _band_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import pyoracle as po
        noise = po.bake_noise()
        sc, luts, G, spec, tgt = _problem(po, noise)
        band = sharding.row_bands(sc.height, world)[rank]
        g, gs, loss = po.grid_adjoint(sc, noise, luts, G, spec, sc.background, tgt, threads=2,
                                      rows=(band.y0, band.y1))
        grad = torch.from_numpy(g)
        acc = torch.tensor([loss, gs], dtype=torch.float64)
        sharding.allreduce_gradient(grad, acc)
        q.put((rank, grad.numpy(), acc.numpy()))
    finally:
        dist.destroy_process_group()


def test_row_band_gradients_all_reduce_to_the_whole_image(oracle, oracle_noise, small):
    sc, luts, G, spec, tgt = small
    grad, gs, loss = oracle.grid_adjoint(sc, oracle_noise, luts, G, spec, sc.background, tgt)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_band_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, g, acc in res:
        np.testing.assert_allclose(g, grad, rtol=1e-12, atol=1e-12 * np.abs(grad).max())
        assert abs(acc[0] - loss) <= 1e-12 * loss and abs(acc[1] - gs) <= 1e-12 * abs(gs)
