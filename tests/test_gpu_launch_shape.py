"""Launch shapes (cgs_ctx_set_launch_shape: Stage 2 block size, binning
blocks per SM, tile-range grid) change how the frame's kernels are launched,
never what they compute: every shape the autotuner may pick renders the
oracle's frame bit for bit (Stage 2 records, Stage 3 lists), and values
outside the documented ranges are rejected."""
import itertools

import numpy as np
import pytest

from cindergs_b200 import GpuPipelineState, autotune, random_scene
from cindergs_b200 import _abi
from helpers import assert_stage23_exact, compositor, config0_camera, gpu_buffers, oracle_frame

pytestmark = pytest.mark.gpu


def test_every_launch_shape_renders_the_same_frame():
    st = GpuPipelineState(0)
    try:
        scene = random_scene(100_000, seed=0)
        cam = config0_camera(1280, 720)
        comp = compositor(1280, 720, cam, deg=3, bg=(0.0, 0.0, 0.0, 1.0))
        o = oracle_frame(scene, cam, comp)
        ch = autotune.LAUNCH_CHOICES
        for pt, bb, rb in itertools.product(ch["project_threads"], ch["bin_blocks_per_sm"],
                                            ch["ranges_blocks"]):
            st.set_launch_shape(pt, bb, rb)
            t = st.execute_frame_gpu(scene, None, cam, comp, force_stage3=True, write_f32=True)
            assert t.total_tile_entries == o["entries"]
            assert_stage23_exact(gpu_buffers(st), o)
            img = st.readback_framebuffer_f32(1280, 720)
            assert float(np.abs(img - o["rgba_f32"]).max()) <= 2e-3
        shape, ms = autotune.tune_launch_shape(st, scene, None, cam, comp, repeats=1)
        assert set(shape) == set(ch) and ms > 0
        for bad in ((300, 0, 0), (0, 9, 0), (0, 0, 70000)):
            with pytest.raises(_abi.CgsError) as e:
                st.set_launch_shape(*bad)
            assert e.value.code == _abi.CGS_E_ARG
    finally:
        st.close()
