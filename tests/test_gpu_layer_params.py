"""GPU tests of the procedural march's layer-parameter gradient
(`psc_layer_param_gradient`): d loss / d coverage, shape_bias, detail_bias,
density_scale, base_m and top_m of one layer of the three-layer precision
scene (Cu
1500-2300 m, As 4000-5000 m, Ci 8000-9000 m; 128 primary + 6 light steps)
at 160x90, PLAIN schedule, FP32 storage, exact filtering.

The reference is the FP64 oracle (oracle/oracle_march.cpp): its loss
(sum((L + background T - target)^2) / (3 pixels)) differentiated by
Richardson-extrapolated central differences (steps e and e/2, with the
float32-rounded parameter values) of the march with its discontinuous tests
held (`oracle_render_frozen`: the layer hits and their order, the early
exits, the 1e-3 density threshold and the AP opacity test replay the
outcomes of the unperturbed march).  The
tangent differentiates the march with those outcomes held too; the plain
central differences of the march as it branches differ from both by the
jumps of the samples that cross the 1e-3 threshold within the step (+3 %
for layer 0's coverage, +30 % for layer 1's on this scene), a term that does
not vanish as the step shrinks and that no pathwise derivative carries.

Two targets, each the oracle's render of the same scene with some of layer
0's parameters moved: its density parameters (coverage +0.04, shape_bias
+0.15, detail_bias -0.10, density_scale x1.15) for their derivatives, its
altitude range (base +40 m, top -60 m) for d / d base and d / d top, so that
each derivative is a coherent sum over the pixels rather than a small
difference of large ones.  The diurnal modulation is on (strength 1, sun at
35 degrees), through which the shape and detail biases act on the
convective cumulus layer; it is 0 for the non-convective altostratus layer.

The range derivatives pass through the trilinear noise taps, whose weights
are piecewise linear in position: the loss has a kink wherever a sample or
light tap crosses a texel boundary, so central differences over metres
average the slope over many kinks (-2753 over 1 m for the cumulus base
against -2650 ... -2658 over 8 ... 1 mm).  They are therefore taken over 8,
4, 2 and 1 mm (the branch-held image in double, so that millimetre steps
resolve, each step the float32-rounded parameter values' own difference),
and the tangent must lie within 2 % of their median (measured on the B200:
0.15-0.9 %)."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from pedalsky_b200 import capi, scenes
from pedalsky_b200.capi import PscError
from pedalsky_b200.layer_grad import PARAMS, layer_param_gradient
from pedalsky_b200.subsystem import subsystem_for_scene

from . import _gpu

pytestmark = pytest.mark.gpu

W, H = 160, 90
FIELDS = ("coverage", "shape_bias", "detail_bias", "density_scale", "base_m", "top_m")
NP = len(FIELDS)


def _moved(sc, layer, deltas):
    layers = (capi.CloudLayerGpu * 8).from_buffer_copy(sc.layers)
    for name, d in deltas.items():
        setattr(layers[layer], name, float(np.float32(getattr(sc.layers[layer], name) + d)))
    return dataclasses.replace(sc, layers=layers)


@pytest.fixture(scope="module")
def prob(oracle, oracle_noise):
    torch = _gpu.torch_cuda()
    sc = scenes.precision_1080p(W, H, storage=capi.STORAGE_F32, schedule=capi.SCHED_PLAIN,
                                filt=capi.FILTER_EXACT)
    sc.params.diurnal_strength = 1.0
    luts = oracle.bake_luts(sc.frame, sc.world)
    moved = _moved(sc, 0, dict(coverage=0.04, shape_bias=0.15, detail_bias=-0.10,
                               density_scale=0.15 * sc.layers[0].density_scale))
    Lt, Tt = oracle.render(moved, oracle_noise, luts, threads=8)
    tgt = (Lt + sc.background * Tt).astype(np.float32)
    moved_r = _moved(sc, 0, dict(base_m=40.0, top_m=-60.0))
    Lr, Tr = oracle.render(moved_r, oracle_noise, luts, threads=8)
    tgt_r = (Lr + sc.background * Tr).astype(np.float32)
    sub = subsystem_for_scene(sc, luts=luts, noise=oracle_noise)
    dev = torch.device("cuda", 0)
    bg = torch.from_numpy(np.ascontiguousarray(sc.background, np.float32)).to(dev)
    tg = torch.from_numpy(tgt).to(dev)
    tg_r = torch.from_numpy(tgt_r).to(dev)
    depth = torch.from_numpy(np.ascontiguousarray(sc.depth, np.float32)).to(dev)
    yield dict(sc=sc, luts=luts, tgt=tgt, tgt_r=tgt_r, sub=sub, bg=bg, tg=tg, tg_r=tg_r, depth=depth,
               torch=torch)
    sub.close()


def _gpu_grad(p, layer, rows=None, target="tg"):
    torch = p["torch"]
    g = torch.zeros(NP, dtype=torch.float64, device="cuda:0")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    for r0, r1 in rows or [(0, H)]:
        view = capi.View(W, r1 - r0, p["depth"][r0:].data_ptr(), None, None, None, W, H, 0, r0)
        layer_param_gradient(p["sub"].handle, view, layer, p["bg"][r0:], p[target][r0:], g, loss)
    torch.cuda.synchronize()
    return g.cpu().numpy(), float(loss.cpu().numpy()[0])


def _oracle_loss(oracle, noise, p, sc, frozen=True, target="tgt"):
    if frozen:
        L, T, misses = oracle.render_frozen(p["sc"], sc, noise, p["luts"], threads=8)
        assert misses == 0
    else:
        L, T = oracle.render(sc, noise, p["luts"], threads=8)
    I = L.astype(np.float64)[..., :3] + p["sc"].background[..., :3].astype(np.float64) * T[..., :3]
    return float(np.sum((I - p[target][..., :3].astype(np.float64)) ** 2) / (3.0 * W * H))


def _richardson(oracle, noise, p, layer, name, e, frozen=True, target="tgt"):
    x = float(getattr(p["sc"].layers[layer], name))

    def cd(h):
        lo, hi = np.float32(x - h), np.float32(x + h)
        f_hi = _oracle_loss(oracle, noise, p, _moved(p["sc"], layer, {name: float(hi) - x}), frozen, target)
        f_lo = _oracle_loss(oracle, noise, p, _moved(p["sc"], layer, {name: float(lo) - x}), frozen, target)
        return (f_hi - f_lo) / (float(hi) - float(lo))

    return (4.0 * cd(e / 2) - cd(e)) / 3.0


def test_layer_parameter_gradient_matches_fp64_central_differences(oracle, oracle_noise, prob):
    g, loss = _gpu_grad(prob, 0)
    ref_loss = _oracle_loss(oracle, oracle_noise, prob, prob["sc"])
    steps = dict(coverage=2e-3, shape_bias=2e-2, detail_bias=5e-3,
                 density_scale=2e-3 * prob["sc"].layers[0].density_scale)
    fd = np.array([_richardson(oracle, oracle_noise, prob, 0, n, steps[n]) for n in FIELDS[:4]])
    g = g[:4]
    fd_plain = _richardson(oracle, oracle_noise, prob, 0, "coverage", steps["coverage"], frozen=False)
    rel = np.abs(g - fd) / np.abs(fd)
    print(f"\nlayer 0 d loss / d {PARAMS}:\n  GPU {g}\n  FD  {fd}\n  rel {rel}\n"
          f"  loss GPU {loss:.9e} oracle {ref_loss:.9e}\n"
          f"  coverage by central differences of the branching march: {fd_plain:.6e}")
    assert PARAMS == FIELDS
    assert np.all(np.abs(fd) > 0)
    assert np.all(rel <= 5e-3), (g, fd)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss


def _central(oracle, noise, p, layer, name, h, target):
    x = float(getattr(p["sc"].layers[layer], name))
    lo, hi = np.float32(x - h), np.float32(x + h)
    f_hi = _oracle_loss(oracle, noise, p, _moved(p["sc"], layer, {name: float(hi) - x}), True, target)
    f_lo = _oracle_loss(oracle, noise, p, _moved(p["sc"], layer, {name: float(lo) - x}), True, target)
    return (f_hi - f_lo) / (float(hi) - float(lo))


@pytest.mark.parametrize("layer", [0, 1])
def test_altitude_range_gradient_matches_fp64_central_differences(oracle, oracle_noise, prob, layer):
    """The tangent lies within 2 % of the median of the FP64 central
    differences over 8, 4, 2 and 1 mm."""
    g, _ = _gpu_grad(prob, layer, target="tg_r")
    for k, name in ((4, "base_m"), (5, "top_m")):
        fd = np.array([_central(oracle, oracle_noise, prob, layer, name, h, "tgt_r")
                       for h in (8e-3, 4e-3, 2e-3, 1e-3)])
        mid = float(np.median(fd))
        print(f"\nlayer {layer} d loss / d {name}: GPU {g[k]:.6g}, FD at 8/4/2/1 mm {fd}, "
              f"rel to the median {abs(g[k] - mid) / abs(mid):.2e}")
        assert abs(mid) > 0
        assert abs(g[k] - mid) <= 2e-2 * abs(mid), (g[k], fd)


def test_biases_have_no_effect_on_a_non_convective_layer(oracle, oracle_noise, prob):
    g, _ = _gpu_grad(prob, 1)
    print(f"\nlayer 1 (altostratus) gradient {g}")
    assert g[1] == 0.0 and g[2] == 0.0
    assert g[0] != 0.0 and g[3] != 0.0
    fd = np.array([_richardson(oracle, oracle_noise, prob, 1, n, e) for n, e in
                   (("coverage", 2e-3), ("density_scale", 2e-3 * prob["sc"].layers[1].density_scale))])
    got = g[[0, 3]]
    print(f"  FD coverage, density_scale {fd}\n  rel {np.abs(got - fd) / np.abs(fd)}")
    assert np.all(np.abs(got - fd) <= 5e-3 * np.abs(fd)), (got, fd)


def test_row_bands_add_up_to_the_whole_view(prob):
    g, loss = _gpu_grad(prob, 0)
    gb, lb = _gpu_grad(prob, 0, rows=[(0, 37), (37, 64), (64, H)])
    assert np.allclose(gb, g, rtol=1e-5, atol=0)
    assert abs(lb - loss) <= 1e-5 * loss


def test_argument_errors(prob):
    torch = prob["torch"]
    g = torch.zeros(NP, dtype=torch.float64, device="cuda:0")
    view = capi.View(W, H, prob["depth"].data_ptr(), None, None, None, 0, 0, 0, 0)
    with pytest.raises(PscError):
        layer_param_gradient(prob["sub"].handle, view, 3, prob["bg"], prob["tg"], g)
    with pytest.raises(PscError):
        capi.call("psc_layer_param_gradient", prob["sub"].handle, C.byref(view), 0, None,
                  C.c_void_p(prob["tg"].data_ptr()), C.c_void_p(g.data_ptr()), None, None)


@pytest.mark.parametrize("variant", ["cone", "kahan"])
def test_light_path_variants(oracle, oracle_noise, variant):
    """The cone light sampling (cloud_march.wgsl:599-666) and the Kahan
    option: the cumulus coverage and top derivatives against the FP64
    branch-held central differences, as above."""
    torch = _gpu.torch_cuda()
    sc = scenes.precision_1080p(W, H, storage=capi.STORAGE_F32, schedule=capi.SCHED_PLAIN,
                                filt=capi.FILTER_EXACT, kahan=int(variant == "kahan"))
    sc.params.diurnal_strength = 1.0
    if variant == "cone":
        sc.params.cone_light_sampling = 1
    luts = oracle.bake_luts(sc.frame, sc.world)
    moved = _moved(sc, 0, dict(coverage=0.04, top_m=-60.0))
    Lt, Tt = oracle.render(moved, oracle_noise, luts, threads=8)
    tgt = (Lt + sc.background * Tt).astype(np.float32)
    sub = subsystem_for_scene(sc, luts=luts, noise=oracle_noise)
    try:
        dev = torch.device("cuda", 0)
        p = dict(sc=sc, luts=luts, tgt=tgt, sub=sub, torch=torch,
                 bg=torch.from_numpy(np.ascontiguousarray(sc.background, np.float32)).to(dev),
                 tg=torch.from_numpy(tgt).to(dev),
                 depth=torch.from_numpy(np.ascontiguousarray(sc.depth, np.float32)).to(dev))
        g, _ = _gpu_grad(p, 0)
        fd_cov = _richardson(oracle, oracle_noise, p, 0, "coverage", 2e-3)
        fd_top = np.array([_central(oracle, oracle_noise, p, 0, "top_m", h, "tgt") for h in (4e-3, 2e-3, 1e-3)])
        mid = float(np.median(fd_top))
        print(f"\n[{variant}] coverage GPU {g[0]:.6e} FD {fd_cov:.6e}; top GPU {g[5]:.6g} FD {fd_top}")
        assert abs(g[0] - fd_cov) <= 5e-3 * abs(fd_cov)
        assert abs(g[5] - mid) <= 2e-2 * abs(mid)
    finally:
        sub.close()
