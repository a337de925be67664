"""Central finite differences of the full gradient (all five integrators) on
64 seeded random parameters of the 100K-triangle configuration: 32 vertex
coordinates of the displaced sphere and 32 texel channels of its 512x512
albedo texture. The pattern is the reference's ValidateBackwardDiff
(LibTensorRay/Tensor/Tensor.h:2968-3021: central differences against the
reverse-mode gradient) with the render-level recipe of
example/validation/validate_gpu.py:103-132 (forward renders with the same
seeds on either side).

Loss: L = sum(w * I) for a fixed weight image w ~ U[0.25, 1].

Scene scale. The reference offsets every ray by a fixed 1e-2
(SHADOW_EPSILON, LibTensorRay/Renderer/Config.h:35). The displaced sphere's
edges are about 0.016 long and its bumps self-occlude near the limb, so at
unit scale the primary-edge term's far-side ray skips surface closer than
1e-2 behind a silhouette edge. That biases the term there, in the reference's
algorithm and so in this path, which reproduces it (at vertex 7909, dL/dI = 1,
1024 spp x 8 seeds: gradient (9.0, 9.4, 3.0) +- (1.4, 2.2, 0.6) against FD
(-1.25, -2.07, -0.85) +- 0.04). Scaling every length by 10 leaves the image
unchanged and makes the offset negligible. The same vertex then gives
(-0.16, -0.17, -0.08) +- (0.14, 0.22, 0.06) against FD
(-0.13, -0.21, -0.09). The check therefore runs on the configuration
scaled by 10, with the vertex step scaled to match: 1e-2 there is 1e-3 at
unit scale. Texels have no length and keep eps = 1e-3.

Criteria. Texels enter no boundary term, and the gradient and the finite
difference use the same samples, so they agree per seed to float rounding:
relative L2 over the 32 channels <= 2e-2 for every seed. Vertex gradients
combine interior and boundary estimators with independent noise. Each
coordinate gets a paired z-score over 16 seeds, (mean of AD - FD) / its
standard error. Every |z| must be <= 5 and the mean z^2 <= 3 (about 1.15
for unbiased, normal errors with 15 degrees of freedom; the estimators'
heavier tails push it up a little)."""
import copy

import numpy as np
import pytest
import torch

from tensorray_b200 import api, scenes
from tests.helpers import PARITY_LOG

pytestmark = pytest.mark.gpu

R = 512
D = 5
SCALE = 10.0
SEEDS = 16
SPP = 64
EPS_VERTEX = 1e-3 * SCALE
EPS_TEXEL = 1e-3
INTEGRATORS = (api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator, api.IndirectEdgeIntegrator,
               api.PixelBoundaryIntegrator)


def scaled(spec, k):
    """The same scene with every length (meshes and camera position) times k;
    the rendered image does not change (area-light radiance is per area)."""
    sc = copy.deepcopy(spec)
    for m in sc.meshes:
        m.positions = (m.positions * np.float32(k)).astype(np.float32)
    c = sc.cameras[0]
    sc.cameras = [scenes.CameraSpec(tuple(float(x) * k for x in c.pos), c.target, c.up, c.width, c.height, c.fov)]
    return sc


@pytest.fixture(scope="module")
def fd_scene(built_lib):
    spec = scaled(scenes.config2_scene(R, R, tris=100_000), SCALE)
    scene = api.Scene(spec)
    scene.configure()
    g = torch.Generator().manual_seed(3)
    w = (0.25 + 0.75 * torch.rand(R, R, 3, generator=g)).to(scene.device)
    return spec, scene, w


def _grads(scene, w, seed, spp):
    opts = api.RenderOptions(seed, D, spp, spp, spp, spp, spp)
    scene.clear_grads()
    for cls in INTEGRATORS:
        cls().renderD(scene, opts, w)
    g = scene.get_grads()
    return g["positions"].clone(), g["texels"].clone()


def _loss(scene, w, seed):
    img = api.PathTracer().renderC(scene, api.RenderOptions(seed, D, SPP, 0, 0, 0, 0))
    return float((img * w).double().sum())


def _pick(grad, n, rng, limit=None):
    """n seeded (index, channel) pairs among rows with a nonzero pilot gradient."""
    rows = grad[:limit] if limit else grad
    cand = torch.nonzero(rows.abs().sum(1) > 0).reshape(-1).cpu().numpy()
    assert len(cand) >= n
    return rng.choice(cand, n, replace=False), rng.integers(0, 3, n)


def test_cfg2_gradient_matches_central_fd_on_64_parameters(fd_scene):
    spec, scene, w = fd_scene
    nv_sphere = len(spec.meshes[0].positions)
    pilot_p, pilot_t = _grads(scene, w, 1000, 16)
    rng = np.random.default_rng(7)
    vs, va = _pick(pilot_p, 32, rng, nv_sphere)
    ts, tc = _pick(pilot_t, 32, rng)

    ad_v = np.zeros((SEEDS, 32))
    ad_t = np.zeros((SEEDS, 32))
    for s in range(SEEDS):
        gp, gt = _grads(scene, w, s, SPP)
        ad_v[s] = gp[vs, va].double().cpu().numpy()
        ad_t[s] = gt[ts, tc].double().cpu().numpy()

    raw = scene._raw_positions.clone()
    fd_v = np.zeros((SEEDS, 32))
    for i in range(32):
        for sgn in (1.0, -1.0):
            p = raw.clone()
            p[vs[i], va[i]] += sgn * EPS_VERTEX
            scene.set_vertex_positions(p)
            scene.configure()
            for s in range(SEEDS):
                fd_v[s, i] += sgn * _loss(scene, w, s) / (2 * EPS_VERTEX)
    scene.set_vertex_positions(raw)
    scene.configure()

    tex = torch.as_tensor(np.ascontiguousarray(spec.textures[0]), device=scene.device).reshape(-1, 3).clone()
    texel_seeds = 4
    fd_t = np.zeros((texel_seeds, 32))
    for i in range(32):
        for sgn in (1.0, -1.0):
            t = tex.clone()
            t[ts[i], tc[i]] += sgn * EPS_TEXEL
            scene.set_texels(t)
            for s in range(texel_seeds):
                fd_t[s, i] += sgn * _loss(scene, w, s) / (2 * EPS_TEXEL)
    scene.set_texels(tex)

    # texels: same samples on both sides, per seed
    rel_t = [float(np.linalg.norm(ad_t[s] - fd_t[s]) / np.linalg.norm(fd_t[s])) for s in range(texel_seeds)]
    PARITY_LOG.append(("cfg2 x10 FD, 32 texel channels", "rel L2/seed", max(rel_t),
                       "eps 1e-3, same seeds on both sides"))
    # vertices: paired z-scores over the seeds
    dd = ad_v - fd_v
    z = dd.mean(0) / (dd.std(0, ddof=1) / np.sqrt(SEEDS))
    PARITY_LOG.append(("cfg2 x10 FD, 32 vertex coords", "mean z^2", float((z ** 2).mean()),
                       f"max |z| {float(np.abs(z).max()):.2f}, 16 seeds x {SPP} spp, eps 1e-3 (unit scale)"))
    assert max(rel_t) <= 2e-2, rel_t
    assert float(np.abs(z).max()) <= 5.0, (z.round(2).tolist(), ad_v.mean(0).tolist(), fd_v.mean(0).tolist())
    assert float((z ** 2).mean()) <= 3.0, z.round(2).tolist()
