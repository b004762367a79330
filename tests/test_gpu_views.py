"""Many views per step (cgs_execute_views): eager per-view launches and CUDA
graph replays both reproduce, bit for bit, what single frames render for the
same cage state; a replay whose tile entries outgrow the captured key
buffers renders the affected views again and the graph is rebuilt."""
import numpy as np
import pytest

from cindergs_b200 import GpuPipelineState, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    st = GpuPipelineState(0)
    wl, cams, comps = workloads.multiview_cage(n=40_000, views=6)
    st.upload_scene(wl.scene)
    cages = wl.bind(st)
    yield st, wl, cages, cams, comps
    st.close()


def images_np(imgs):
    return [t.cpu().numpy().view(np.uint8).reshape(t.shape[0], t.shape[1], 4) for t in imgs]


def single_frames(st, wl, cages, cams, comps):
    out = []
    for cam, comp in zip(cams, comps):
        st.execute_frame_gpu(wl.scene, cages, cam, comp, force_stage3=True)
        out.append(st.readback_framebuffer_rgba8(comp.screen_width, comp.screen_height))
    return out


def test_eager_views_match_single_frames(setup):
    st, wl, cages, cams, comps = setup
    wl.step()
    imgs = st.view_images(comps)
    stats = st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=False)
    assert not stats["graph_replayed"] and not stats["graph_captured"]
    assert stats["total_tile_entries"] > 0
    got = images_np(imgs)
    ref = single_frames(st, wl, cages, cams, comps)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g, r)


def test_graph_replays_match(setup):
    st, wl, cages, cams, comps = setup
    imgs = st.view_images(comps)
    wl.step()
    first = st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=True)
    assert first["graph_captured"] and not first["graph_replayed"]
    for step in range(3):
        wl.step()  # the cage moves: Stage 1 runs inside the replay
        stats = st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=True)
        assert stats["graph_replayed"] and not stats["graph_captured"], stats
        got = images_np(imgs)
        ref = single_frames(st, wl, cages, cams, comps)
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g, r)


def test_replay_overflow_renders_again(setup):
    st, wl, cages, cams, comps = setup
    imgs = st.view_images(comps)
    rest = wl.cage.mesh.rest_vertices.copy()
    sim = wl.cage.simulator
    sim.current_positions = rest.copy()
    st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=True)  # capture at rest
    stats = st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=True)
    assert stats["graph_replayed"]
    # a cage three times as large: every bound splat grows, entries outgrow
    # the captured capacity
    c = rest.mean(axis=0)
    sim.current_positions = ((rest - c) * 3.0 + c).astype(np.float32)
    stats = st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=True)
    assert stats["graph_replayed"] and stats["views_rerendered"] > 0, stats
    got = images_np(imgs)
    ref = single_frames(st, wl, cages, cams, comps)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g, r)
    again = st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=True)
    assert again["graph_captured"], again  # rebuilt with the grown capacity
    sim.current_positions = rest.copy()


def test_autotuned_views_render_the_same(setup):
    """Per-view digit widths and entry-sort methods chosen by the autotuner
    on the reference's 16x16 tiles give the same images as the defaults; with
    tile shapes tuned too, the replayed graph gives the images of an eager
    batch with the same choices."""
    from cindergs_b200 import _abi, autotune
    st, wl, cages, cams, comps = setup
    wl.step()
    best = autotune.tune_views(st, wl.scene, cages, cams, comps, repeats=1,
                               tile_shapes=(_abi.TILE_16X16,))
    assert set(best) == {(c.screen_width, c.screen_height) for c in comps}
    tss, rbs, ess = autotune.per_view(best, comps)
    assert set(tss) == {_abi.TILE_16X16}
    a, b = st.view_images(comps), st.view_images(comps)
    st.execute_views(wl.scene, cages, cams, comps, a, use_graph=False)
    st.execute_views(wl.scene, cages, cams, comps, b, use_graph=True, radix_bits=rbs,
                     entry_sort=ess, tile_shape=tss)
    for x, y in zip(images_np(a), images_np(b)):
        np.testing.assert_array_equal(x, y)
    best = autotune.tune_views(st, wl.scene, cages, cams, comps, repeats=1)
    tss, rbs, ess = autotune.per_view(best, comps)
    st.execute_views(wl.scene, cages, cams, comps, a, use_graph=False, radix_bits=rbs,
                     entry_sort=ess, tile_shape=tss)
    for _ in range(2):  # capture, then replay
        st.execute_views(wl.scene, cages, cams, comps, b, use_graph=True, radix_bits=rbs,
                         entry_sort=ess, tile_shape=tss)
        for x, y in zip(images_np(a), images_np(b)):
            np.testing.assert_array_equal(x, y)
