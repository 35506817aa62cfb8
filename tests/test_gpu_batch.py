"""The batched form on the GPU: cameras of different sizes, spp, bounces and skies rendered by one
graph-captured launch give, camera for camera, the image `lw_render_hq` gives for the same inputs
(1e-4 relative per pixel), and the autotuner leaves a valid tuning."""

import numpy as np
import pytest

from lumenwright_b200 import batch as BT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


def small_cameras():
    cams = BT.c3_cameras(n=6, seed=11)
    sizes = [(64, 36), (96, 54), (160, 90), (48, 27), (128, 72), (80, 45)]
    for c, (w, h), spp in zip(cams, sizes, [4, 8, 2, 16, 3, 5]):
        c.width, c.height, c.spp = w, h, spp
    return cams


def test_batch_matches_separate_renders(ctx):
    hq, jobs = BT.c3_jobs(ctx, small_cameras())
    ctx.upload_hq_scene(hq)
    outs = ctx.batch_prepare(jobs)
    ctx.batch_run()
    ctx.batch_read()
    for (p, sky, spp), got in zip(jobs, outs):
        want = ctx.render_hq(p, sky, spp)
        ok = np.abs(got - want) <= 1e-4 * np.maximum(np.abs(got), np.abs(want)) + 1e-6
        assert ok.all(), (int(p["frame"][0]), np.abs(got - want).max())
    # A second replay of the same graph gives the same images.
    first = [o.copy() for o in outs]
    ctx.batch_run()
    ctx.batch_read()
    for a, b in zip(first, outs):
        assert np.array_equal(a, b)


def test_batch_cameras_match_the_oracle(ctx):
    # Directly against the oracle: the batch's cameras (the two times of day, game-sky maps and
    # Chunky's cache) from one graph launch against the oracle's CPU-backend loop (f64 sums / spp)
    # over the same inputs, every pixel within 1e-4 relative.
    from oracle import oracle as O
    hq, jobs = BT.c3_jobs(ctx, small_cameras())
    ctx.upload_hq_scene(hq)
    outs = ctx.batch_prepare(jobs)
    ctx.batch_run()
    ctx.batch_read()
    checked = set()
    for (p, sky, spp), got in zip(jobs, outs):
        kind = "maps" if float(p["sky_map"][0]) >= 1.0 else "cache"
        if kind in checked:
            continue
        checked.add(kind)
        w, h = int(p["frame"][0]), int(p["frame"][1])
        v = O.OracleScene(p, hq.grid, hq.models, hq.quads, hq.atlas, hq.emitters, hq.emitter_grid, sky)
        want = v.render_mean(0, 0, w, h, spp)
        ok = np.abs(got - want) <= 1e-4 * np.maximum(np.abs(got), np.abs(want)) + 1e-6
        print(f"batch camera {w}x{h} at {spp} spp ({kind}): {ok.mean():.6f} within 1e-4")
        assert ok.all(), (w, h, np.abs(got - want).max())
    assert checked == {"maps", "cache"}


def test_a_batch_in_passes_gives_the_separate_renders_bit_for_bit(ctx, monkeypatch):
    # With the item sums capped small the wavefront batch runs in several passes of one-sample
    # items (each an equal slice of every camera's samples): each camera's image is lw_render_hq's
    # (one-sample items, the same order of additions) bit for bit.
    monkeypatch.setenv("LUMENWRIGHT_BATCH_SUMS_MB", "1")
    hq, jobs = BT.c3_jobs(ctx, small_cameras())
    ctx.upload_hq_scene(hq)
    ctx.set_tuning(threads=128, budget=0, sub=0, engine=0, paths=0)
    total = sum(int(p["frame"][0]) * int(p["frame"][1]) * spp for p, _, spp in jobs)
    assert total * 16 > 2 * (1 << 20)  # at least three passes (one camera has fewer spp than passes)
    outs = ctx.batch_prepare(jobs)
    ctx.batch_run()
    ctx.batch_read()
    for (p, sky, spp), got in zip(jobs, outs):
        want = ctx.render_hq(p, sky, spp)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), int(p["frame"][0])


def test_autotuner_picks_a_tuning(ctx, tmp_path):
    hq, jobs = BT.c3_jobs(ctx, small_cameras())
    ctx.upload_hq_scene(hq)
    tuner = BT.Autotuner(ctx, cache_dir=str(tmp_path), trial_fraction=1.0)
    best, entry = tuner.tune(jobs)
    assert best["engine"] in (0, 1) and len(entry["trials"]) == len(BT.Autotuner.candidates())
    again, _ = tuner.tune(jobs)  # from the cache
    now = ctx.get_tuning()
    assert again == best and {k: now[k] for k in best} == best
    ctx.set_tuning(threads=128, budget=0, sub=0, engine=0, paths=0)


def test_batch_engines_give_the_same_images(ctx):
    # The batched wavefront (one graph whose loop node runs the shade/trace iterations on the
    # device) and the batched megakernel take the same items: equal images, bit for bit.
    from lumenwright_b200.native import ENGINE_MEGAKERNEL, ENGINE_WAVEFRONT
    hq, jobs = BT.c3_jobs(ctx, small_cameras())
    ctx.upload_hq_scene(hq)
    ctx.set_tuning(engine=ENGINE_MEGAKERNEL)
    outs = ctx.batch_prepare(jobs)
    ctx.batch_run()
    ctx.batch_read()
    want = [o.copy() for o in outs]
    ctx.set_tuning(engine=ENGINE_WAVEFRONT)
    got = ctx.batch_prepare(jobs)
    ctx.batch_run()
    ctx.batch_read()
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    # replayed again: the loop starts over from the cleared slots
    first = [o.copy() for o in got]
    ctx.batch_run()
    ctx.batch_read()
    for a, b in zip(first, got):
        assert np.array_equal(a, b)
