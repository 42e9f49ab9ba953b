"""Batched rendering (gg_render_batch): many scenes of uneven size in one
persistent launch of the mixed-precision kernel, replayed from a CUDA graph,
with an autotuned kernel variant.

A batched scene is traced with the same per-ray arithmetic as the scene on
its own (its parameters are the same numbers; only which warp runs which ray
differs), so its image must equal the single-scene render byte for byte.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from gargantua_b200 import abi, workloads
from gargantua_b200.gr_core import Kerr


def test_batch_scene_generator_ranges_and_determinism():
    a = workloads.batch_scenes(64, seed=0)
    b = workloads.batch_scenes(64, seed=0)
    assert [(s.width, s.metric.spin, s.camera.position[1]) for s in a] == \
        [(s.width, s.metric.spin, s.camera.position[1]) for s in b]
    for k, s in enumerate(a):
        assert 0.0 <= s.metric.spin <= 0.998
        assert 10.0 <= s.camera.position[1] <= 100.0
        assert math.radians(5.0) <= s.camera.position[2] <= math.radians(89.0)
        assert s.width == s.height and s.width % 64 == 0 and 64 <= s.width <= 512
        assert 15.0 <= s.disk.r_outer <= 40.0
        assert s.options.sky.seed == k
    assert workloads.batch_scenes(4, seed=1)[0].metric.spin != a[0].metric.spin


def test_batch_variant_table(gglib):
    """The autotuner's grid: refill period, register budget, block size (64,
    128, 256 threads) and samples per queue claim (16, 32, 64), each variant
    within the SM's 2,048 threads and 228 KB of shared memory (12 slots of
    16 B plus 16 B per thread, 1 KB reserved per CTA)."""
    vs = [abi.batch_variant(v) for v in range(abi.GG_BATCH_VARIANTS)]
    assert len(set(vs)) == len(vs)
    assert {v[2] for v in vs} == {64, 128, 256} and {v[3] for v in vs} == {16, 32, 64}
    for period, ctas, block, chunk in vs:
        assert period in (4, 8, 16, 32) and block % 32 == 0
        assert block * ctas <= 2048
        assert 65536 // (block * ctas) >= 64  # registers per thread
        assert ctas * (block * (12 * 16 + 16) + 1024 + 128) <= 228 * 1024
    with pytest.raises(abi.GargantuaError):
        abi.batch_variant(abi.GG_BATCH_VARIANTS)
    assert len(abi.batch_variant_names()) == abi.GG_BATCH_VARIANTS


def _small_batch(n=6):
    return workloads.batch_scenes(n, seed=3, max_side=128)


@pytest.mark.gpu
def test_large_batch_with_hand_back_matches_single_renders(renderer):
    """A batch above 2^20 samples hands rays that leave the FP64 band back to
    FP32; those rays then take different (equally accurate) steps than in the
    single-round renders of the small scenes, so images agree on all but a
    few pixels."""
    scenes = workloads.batch_scenes(40, seed=5, max_side=512)
    assert sum(s.n_samples for s in scenes) >= 1 << 20
    imgs = renderer.render_batch(scenes)
    st = renderer.stats()
    assert st.rays == sum(s.n_samples for s in scenes) and st.fp64_rays > 0
    same = total = 0
    for sc, img in zip(scenes, imgs):
        ref, _ = renderer.render(sc)
        px = (img == ref).all(axis=2)
        same += int(px.sum())
        total += px.size
    assert same / total > 0.9995, same / total


@pytest.mark.gpu
def test_batch_equals_single_scene_renders(renderer):
    """Below 2^20 samples a batch and single renders both run one FP64 round,
    so every ray takes the same steps."""
    scenes = _small_batch()
    imgs = renderer.render_batch(scenes)
    st = renderer.stats()
    assert st.rays == sum(s.n_samples for s in scenes)
    attempts = 0
    for sc, img in zip(scenes, imgs):
        ref, _ = renderer.render(sc)
        attempts += renderer.stats().attempts
        assert np.array_equal(img, ref)
    assert st.attempts == attempts


@pytest.mark.gpu
def test_batch_scenes_against_oracle(renderer, oracle_mod):
    """The batch held to the FP64 oracle directly, not only through the
    single-scene renders: each scene of a small batch (mixed precision)
    against the oracle's render of the same scene with the same stepper in
    FP64.  The batch returns images only, so the bar is on the bytes: within
    one step of 255 on 99.9 % of the pixels, as the single mixed renders are
    held to the FP64 kernel."""
    scenes = workloads.batch_scenes(10, seed=4, max_side=256)
    ref = workloads.batch_scenes(10, seed=4, max_side=256, precision=abi.GG_PREC_FP64)
    imgs = renderer.render_batch(scenes)
    close = exact = total = 0
    for img, sc in zip(imgs, ref):
        want, _ = oracle_mod.render(sc)
        d = np.abs(img.astype(int) - want.astype(int)).max(axis=2)
        close += int((d <= 1).sum())
        exact += int((d == 0).sum())
        total += d.size
    assert close / total >= 0.999, (close, total)
    assert exact / total >= 0.99, (exact, total)


@pytest.mark.gpu
def test_batch_graph_replay_with_new_parameters(renderer):
    scenes = _small_batch()
    first = renderer.render_batch(scenes)
    again = renderer.render_batch(scenes)  # replays the cached graph
    assert all(np.array_equal(x, y) for x, y in zip(first, again))
    # same shape, new spin and camera distance: the graph is reused, the
    # scene table it uploads is new
    scenes[2].metric = Kerr(1.0, 0.5)
    scenes[2].camera.position = (0.0, 33.0, scenes[2].camera.position[2], 0.0)
    changed = renderer.render_batch(scenes)
    ref, _ = renderer.render(scenes[2])
    assert np.array_equal(changed[2], ref)
    assert not np.array_equal(changed[2], first[2])
    assert np.array_equal(changed[0], first[0])


@pytest.mark.gpu
def test_batch_autotune_variants_agree(renderer):
    scenes = _small_batch(4)
    best, ms = renderer.batch_autotune(scenes)
    assert 0 <= best < abi.GG_BATCH_VARIANTS
    assert all(m > 0 for m in ms) and ms[best] == min(ms)
    outs = []
    for v in range(abi.GG_BATCH_VARIANTS):
        renderer.batch_set_variant(v)
        outs.append(renderer.render_batch(scenes))
    for o in outs[1:]:
        assert all(np.array_equal(x, y) for x, y in zip(o, outs[0]))
    renderer.batch_set_variant(best)


@pytest.mark.gpu
def test_batch_rejects_unsupported(renderer):
    scenes = _small_batch(3)
    fp64 = workloads.batch_scenes(3, seed=3, max_side=128, precision=abi.GG_PREC_FP64)
    with pytest.raises(abi.GargantuaError) as e:
        renderer.render_batch(fp64)
    assert e.value.status == abi.GG_ERR_UNSUPPORTED
    mixed_kinds = scenes[:2] + [workloads.schwarzschild_thin_256(
        precision=abi.GG_PREC_MIXED, stepper=abi.GG_STEPPER_DP45)]
    with pytest.raises(abi.GargantuaError) as e:
        renderer.render_batch(mixed_kinds)
    assert e.value.status == abi.GG_ERR_UNSUPPORTED
    # the context stays usable
    imgs = renderer.render_batch(scenes)
    assert len(imgs) == 3
