"""CPU tests of the oracle's branch-held march (`oracle_render_frozen`), the
reference the layer-parameter gradient is checked against: replaying a
march's own branch outcomes reproduces it bit for bit; with another scene's
parameters the replay follows the recorded path (no missing outcomes), and
its loss is smooth in the parameter (central differences at e and e/2 agree
to a few 1e-3), unlike the branching march, whose differences carry the
jumps of the samples crossing the 1e-3 density threshold."""
import dataclasses

import numpy as np

from pedalsky_b200 import capi, scenes

W, H = 64, 36


def _scene():
    sc = scenes.precision_1080p(W, H, storage=capi.STORAGE_F32, schedule=capi.SCHED_PLAIN,
                                filt=capi.FILTER_EXACT)
    sc.params.diurnal_strength = 1.0
    return sc


def _moved(sc, layer, name, d):
    layers = (capi.CloudLayerGpu * 8).from_buffer_copy(sc.layers)
    setattr(layers[layer], name, float(np.float32(getattr(sc.layers[layer], name) + d)))
    return dataclasses.replace(sc, layers=layers)


def test_replay_of_its_own_branches_is_the_march(oracle, oracle_noise):
    sc = _scene()
    luts = oracle.bake_luts(sc.frame, sc.world)
    L0, T0 = oracle.render(sc, oracle_noise, luts, threads=4)
    L1, T1, misses = oracle.render_frozen(sc, sc, oracle_noise, luts, threads=4)
    assert misses == 0
    assert np.array_equal(L0, L1.astype(np.float32)) and np.array_equal(T0, T1.astype(np.float32))


def test_branch_held_loss_is_smooth_in_coverage(oracle, oracle_noise):
    sc = _scene()
    luts = oracle.bake_luts(sc.frame, sc.world)
    tgt = sc.background * 0.5

    def loss(d, frozen):
        s2 = _moved(sc, 1, "coverage", d)
        if frozen:
            L, T, misses = oracle.render_frozen(sc, s2, oracle_noise, luts, threads=4)
            assert misses == 0
        else:
            L, T = oracle.render(s2, oracle_noise, luts, threads=4)
        I = L[..., :3].astype(np.float64) + sc.background[..., :3] * T[..., :3]
        return float(np.sum((I - tgt[..., :3]) ** 2))

    x = sc.layers[1].coverage

    def cd(e, frozen):
        hi, lo = np.float32(x + e), np.float32(x - e)
        return (loss(float(hi) - x, frozen) - loss(float(lo) - x, frozen)) / (float(hi) - float(lo))

    a, b = cd(2e-3, True), cd(1e-3, True)
    print(f"\nbranch-held d loss / d coverage: {a:.6e} (e = 2e-3), {b:.6e} (e = 1e-3); "
          f"branching march {cd(2e-3, False):.6e}")
    assert abs(a - b) <= 5e-3 * abs(b)
