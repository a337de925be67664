"""CPU tests that pin the oracle before it is trusted as the GPU checker:
closed-form answers, the reference's finite-difference-vs-AD pattern and the
reference's primitive-op goldens."""
import math

import numpy as np
import torch

from oracle import tr_oracle as O
from tensorray_b200 import scenes


def _plane_light_scene(width=8, height=8, albedo=0.5):
    spec = scenes.SceneSpec()
    spec.bsdfs = [scenes.BsdfSpec(scenes.DIFFUSE, (albedo,) * 3)]
    gp, gf = scenes.quad((0.0, -1.0, 0.0), 5.0, up=True)
    spec.meshes.append(scenes.MeshSpec(gp, gf, bsdf=0))
    lp, lf = scenes.quad((0.0, 1.0, 0.0), 0.5, up=False)
    spec.lights.append((10.0, 10.0, 10.0))
    spec.meshes.append(scenes.MeshSpec(lp, lf, bsdf=0, light=0))
    spec.cameras = [scenes.CameraSpec((0.0, 2.0, 3.0), (0.0, -1.0, 0.0), (0.0, 1.0, 0.0), width, height, 30.0)]
    return spec


def polygon_irradiance(x, n, verts, radiance):
    """Lambert's closed form for the irradiance from a uniform polygonal
    emitter: E = L/2 * sum_i angle_i * (n . unit(cross(v_i, v_i+1)))."""
    E = 0.0
    k = len(verts)
    for i in range(k):
        a = verts[i] - x
        b = verts[(i + 1) % k] - x
        a /= np.linalg.norm(a)
        b /= np.linalg.norm(b)
        ang = math.acos(max(-1.0, min(1.0, float(a @ b))))
        c = np.cross(a, b)
        c /= np.linalg.norm(c)
        E += ang * float(c @ n)
    return abs(E) * radiance / 2.0


def test_direct_lighting_matches_lambert_polygon_formula():
    spec = _plane_light_scene()
    sc = O.OracleScene(spec, requires_grad=())
    c = spec.cameras[0]
    cam = O.camera_matrices(c.pos, c.target, c.up, c.width, c.height, c.fov)
    spp, D = 512, 1
    smp = O.uniform_table(3, 2 + 5 * D, c.width * c.height * spp)
    with torch.no_grad():
        img = O.path_tracer(sc, cam, spp, D, smp)
    # analytic outgoing radiance at every sampled primary hit
    N = c.width * c.height * spp
    slots = torch.arange(N)
    pix = slots % (c.width * c.height)
    d = O.camera_ray_dir(cam, pix % c.width, pix // c.width, smp[0], smp[1])
    org = torch.from_numpy(cam["pos"]).expand(N, 3).contiguous()
    tri, u, v, t = sc.intersect(org, d, O.SHADOW_EPS, O.RAY_MAX)
    assert bool((tri < 2).all()) and bool((tri >= 0).all())  # every ray lands on the ground
    hits = (org + t[:, None] * d).numpy().astype(np.float64)
    light = spec.meshes[1].positions.astype(np.float64)
    verts = [light[0], light[1], light[2], light[3]]
    n = np.array([0.0, 1.0, 0.0])
    Lo = np.array([0.5 / math.pi * polygon_irradiance(h, n, verts, 10.0) for h in hits[:: 97]])
    ref_mean = Lo.mean()
    # the estimator at the same hits, averaged over all pixels
    est = float(img[:, 0].mean())
    ref_all = np.array([0.5 / math.pi * polygon_irradiance(h, n, verts, 10.0) for h in hits]).reshape(-1)
    ref_img = np.zeros(c.width * c.height)
    np.add.at(ref_img, pix.numpy(), ref_all / spp)
    assert abs(est - ref_img.mean()) < 0.01 * ref_img.mean(), (est, ref_img.mean(), ref_mean)


def test_oracle_ad_matches_central_fd_for_light_translation():
    """ValidateBackwardDiff pattern (Tensor.h:2968-3021): central FD with step
    1e-3 against reverse mode, with the samples held fixed."""
    spec = _plane_light_scene(6, 6)
    sc = O.OracleScene(spec, requires_grad=("translation",))
    c = spec.cameras[0]
    cam = O.camera_matrices(c.pos, c.target, c.up, c.width, c.height, c.fov)
    spp, D = 16, 1
    smp = O.uniform_table(4, 2 + 5 * D, c.width * c.height * spp)
    dLdI = torch.ones(c.width * c.height, 3)
    g, _ = O.grads(sc, cam, 0, spp, D, smp, dLdI)
    ad = g["translation"][1].double()
    eps = 1e-3
    fd = []
    base = sc.translation.detach().clone()
    for k in range(3):
        vals = []
        for s in (+1, -1):
            with torch.no_grad():
                sc.translation.copy_(base)
                sc.translation[1, k] += s * eps
                sc.configure()
                vals.append(float(O.path_tracer(sc, cam, spp, D, smp).double().sum()))
        fd.append((vals[0] - vals[1]) / (2 * eps))
    with torch.no_grad():
        sc.translation.copy_(base)
    fd = torch.tensor(fd, dtype=torch.float64)
    err = (ad - fd).abs()
    assert bool((err < 2e-2 * fd.abs().max() + 1e-3).all()), (ad.tolist(), fd.tolist())


def test_vector_cross_golden():
    # Utils.cpp UtilityTest "Test 12": VectorCross([3,4,5], [6,7,8])
    a = torch.tensor([[3.0, 4.0, 5.0]])
    b = torch.tensor([[6.0, 7.0, 8.0]])
    assert O.cross(a, b).tolist() == [[-3.0, 6.0, -3.0]]


def test_watertight_shared_edge_hits_exactly_once():
    # two triangles sharing the edge x = 0 in the plane z = 0
    P0 = torch.tensor([[0.0, -1.0, 0.0], [0.0, -1.0, 0.0]])
    P1 = torch.tensor([[0.0, 1.0, 0.0], [1.0, 0.0, 0.0]])
    P2 = torch.tensor([[-1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    ys = torch.linspace(-0.9, 0.9, 257)
    org = torch.stack([torch.zeros_like(ys), ys, torch.full_like(ys, 1.0)], -1)
    dirs = torch.tensor([[0.0, 0.0, -1.0]]).expand_as(org).contiguous()
    tri, u, v, t = O.intersect_brute(P0, P1, P2, org, dirs, 1e-4, 1e30)
    assert bool((tri >= 0).all())
    assert bool((t == 1.0).all())
    # hits exactly on the shared edge resolve to the lower triangle id
    assert bool((tri == 0).all())


def test_intersect_misses_and_parallel():
    P0 = torch.tensor([[0.0, 0.0, 0.0]])
    P1 = torch.tensor([[1.0, 0.0, 0.0]])
    P2 = torch.tensor([[0.0, 1.0, 0.0]])
    org = torch.tensor([[2.0, 2.0, 1.0], [0.2, 0.2, 1.0], [0.2, 0.2, 1.0], [0.2, 0.2, -1.0]])
    dirs = torch.tensor([[0.0, 0.0, -1.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0], [0.0, 0.0, 1.0]])
    tri, u, v, t = O.intersect_brute(P0, P1, P2, org, dirs, 1e-4, 1e30)
    assert tri.tolist() == [-1, -1, -1, 0]
    assert abs(float(t[3]) - 1.0) < 1e-7 and abs(float(u[3]) - 0.2) < 1e-6 and abs(float(v[3]) - 0.2) < 1e-6


def test_edges_follow_processEdges():
    # a quad = two triangles: 5 unique edges, one interior
    F = np.array([[0, 2, 1], [0, 3, 2]])
    E = O.build_edges(F)
    assert E.shape == (5, 5)
    interior = E[E[:, 3] >= 0]
    assert interior.tolist() == [[0, 2, 0, 1, 1]]
    assert (E[:, 0] < E[:, 1]).all()


def test_hash_sampler_range_and_moments():
    s = O.hash_uniform(1, 0, 0, np.arange(1 << 16, dtype=np.uint64))
    assert s.min() >= 2.0 ** -24 and s.max() <= 1 - 2.0 ** -24
    assert abs(float(s.mean()) - 0.5) < 5e-3
    assert abs(float((s * s).mean()) - 1.0 / 3.0) < 5e-3


def test_camera_center_ray_points_at_target():
    cam = O.camera_matrices((0, 0, 4), (0, 0, 0), (0, 1, 0), 256, 256, 45.0)
    d = O.camera_ray_dir(cam, torch.tensor([127]), torch.tensor([127]), torch.tensor([1.0]), torch.tensor([1.0]))
    assert torch.allclose(d, torch.tensor([[0.0, 0.0, -1.0]]), atol=1e-6)
    # top-left pixel looks up and to the world's -x (left-handed LookAt, Matrix.cpp:181-209)
    d0 = O.camera_ray_dir(cam, torch.tensor([0]), torch.tensor([0]), torch.tensor([0.0]), torch.tensor([0.0]))
    assert float(d0[0, 0]) < 0 and float(d0[0, 1]) > 0
    half = math.atan2(float(d0[0, 1]), -float(d0[0, 2]))
    assert abs(half - math.radians(22.5)) < 1e-5


def test_culled_ray_queries_equal_brute_force():
    """The oracle's cluster culling (TriangleClusters) is conservative: the
    same hits, barycentrics and distances as the test over every triangle,
    for random rays and for rays leaving surface points (the set-up rays of
    the boundary terms)."""
    from tensorray_b200 import scenes
    osc = O.OracleScene(scenes.config2_scene(8, 8, tris=20000), requires_grad=())
    g = torch.Generator().manual_seed(1)
    org = (torch.rand(600, 3, generator=g) - 0.5) * 4
    p = osc.pos.detach()
    tri = torch.randint(0, osc.idx.shape[0], (600,), generator=g)
    surf = (p[osc.idx[tri, 0]] + p[osc.idx[tri, 1]] + p[osc.idx[tri, 2]]) / 3
    org = torch.cat([org, surf])
    d = torch.nn.functional.normalize(torch.randn(1200, 3, generator=g), dim=1)
    assert osc.idx.shape[0] >= O.CULL_MIN_TRIANGLES
    P = [p[osc.idx[:, k]] for k in range(3)]
    culled = osc.intersect(org, d, O.SHADOW_EPS, O.RAY_MAX)
    brute = O.intersect_brute(*P, org, d, O.SHADOW_EPS, O.RAY_MAX)
    assert int((brute[0] >= 0).sum()) > 300
    for a, b in zip(culled, brute):
        assert torch.equal(a, b)


def test_guiding_tree_refinement_partitions_the_sample_cube():
    """AQ refinement (the oracle's _aq_points / _aq_refine): after two passes
    the leaves still tile the (edge, light) sample cube, i.e. their volumes
    sum to the depth-0 tree's and every leaf lies inside its edge's
    interval; the leaf limit holds; and a threshold nothing exceeds leaves the
    depth-0 tree unchanged."""
    from tensorray_b200 import scenes
    osc = O.OracleScene(scenes.config1_scene(16, 16), requires_grad=())
    with torch.no_grad():
        osc.configure()
    E = osc.edges.shape[0]
    g0 = O.aq_guide(osc, 3, 2, 0.1)
    g2 = O.aq_guide(osc, 3, 2, 0.1, depth=2, max_size=E + 150, thold=1e-5)
    b0, b2 = g0["box"].double(), g2["box"].double()
    vol = lambda b: ((b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2])).sum()
    n2 = b2.shape[1]
    assert E < n2 <= E + 150
    assert abs(float(vol(b2)) - float(vol(b0))) < 1e-6
    cdf = osc.sec_cdf.double()
    lo = torch.cat([torch.zeros(1, dtype=torch.float64), cdf[:-1]])
    e = g2["edge"]
    assert bool((b2[0] >= lo[e] - 1e-7).all() and (b2[3] <= cdf[e] + 1e-7).all())
    assert bool((b2[1] >= 0).all() and (b2[4] <= 1).all() and (b2[2] >= 0).all() and (b2[5] <= 1).all())
    assert bool((b2[3] >= b2[0]).all() and (b2[4] > b2[1]).all() and (b2[5] > b2[2]).all())
    same = O.aq_guide(osc, 3, 2, 0.1, depth=2, max_size=E + 150, thold=1e30)
    assert torch.equal(same["box"], g0["box"]) and torch.equal(same["cdf"], g0["cdf"])
