"""The quantized scene ingest (cgs_scene_upload_quantized) renders exactly
what the dequantized scene renders when uploaded with f16 SH planes."""
import numpy as np
import pytest

from cindergs_b200 import (CameraUniforms, CompositorUniforms, GpuPipelineState,
                           QuantizedGaussianSceneSoa, random_scene)
from cindergs_b200 import _abi

pytestmark = pytest.mark.gpu


def frame(st, scene, w=960, h=544):
    cam = CameraUniforms.from_look_at((0.3, 0.5, 3.5), (0, 0, 0), (0, 1, 0), np.deg2rad(60), w, h,
                                      0.2)
    comp = CompositorUniforms(w, h, (0, 0, 0, 1), tuple(float(x) for x in cam.eye()), 3)
    st.execute_frame_gpu(scene, None, cam, comp, force_stage3=True)
    img = st.readback_framebuffer_rgba8(w, h)
    keys = st.read_buffer(_abi.BUF_SORTED_KEYS, np.uint32)
    return img, keys


@pytest.mark.parametrize("degree", [3, 1])
def test_quantized_matches_dequantized(degree):
    st = GpuPipelineState(0)
    s = random_scene(30_000, seed=5, box=1.0)
    q = QuantizedGaussianSceneSoa.from_soa(s, degree)
    d = q.to_soa()
    d.sh_coeffs = d.sh_coeffs.astype(np.float16)
    st.upload_scene(q)
    img_q, keys_q = frame(st, q)
    st.upload_scene(d)
    img_d, keys_d = frame(st, d)
    np.testing.assert_array_equal(img_q, img_d)
    np.testing.assert_array_equal(keys_q, keys_d)
    assert img_q[..., :3].max() > 0
    st.close()
