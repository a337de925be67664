"""An XML scene file drives the CUDA path: the XML copy of the icosphere
configuration renders the same image and the same gradients as the
programmatic scene (same samples)."""
import pytest
import torch

from tensorray_b200 import api, scene_xml
from tests.test_scene_xml import config1_xml

pytestmark = pytest.mark.gpu


def test_xml_scene_renders_like_the_programmatic_scene(built_lib, tmp_path):
    path, ref_spec = config1_xml(str(tmp_path), 64, 48)
    out = []
    for spec in (scene_xml.load_xml(path), ref_spec):
        scene = api.Scene(spec)
        scene.configure()
        opts = api.RenderOptions(3, 3, 8, 8, 8, 8, 8)
        img = api.PathTracer().renderC(scene, opts).clone()
        scene.clear_grads()
        for cls in (api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator,
                    api.IndirectEdgeIntegrator, api.PixelBoundaryIntegrator):
            cls().renderD(scene, opts, img * 0 + 1)
        out.append((img, scene.get_grads()["positions"].clone()))
    (ia, ga), (ib, gb) = out
    torch.testing.assert_close(ia, ib, rtol=1e-6, atol=1e-7)
    # the gradients differ only by the order of float atomic additions
    assert float((ga - gb).norm() / gb.norm()) <= 1e-5
    assert float((ga - gb).abs().max()) <= 1e-4 * float(gb.abs().max())
