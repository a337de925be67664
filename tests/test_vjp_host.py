"""The hand-written reverse-mode adjoints (factor_vjp / eval_inner_vjp /
tangent_vjp, xdotn_grad, camera_factor_grad) against forward-mode dual
numbers evaluating the same factor code, on random inputs on the host: both
BSDFs, both coordinate_system branches, unnormalised shading normals. The
harness is compiled with nvcc from the library sources (no GPU needed)."""
import os
import subprocess

import pytest

from tensorray_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def harness_exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("vjp") / "vjp_harness")
    src = os.path.join(HERE, "native", "vjp_harness.cu")
    scene = os.path.join(build.CSRC, "scene.cu")
    cmd = [build._nvcc(), "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "--expt-relaxed-constexpr", "--extended-lambda", src, scene, "-o", out, "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        pytest.fail("nvcc failed:\n" + res.stderr[-2000:])
    return out


@pytest.fixture(scope="module")
def harness(harness_exe):
    run = subprocess.run([harness_exe], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    return {l.split()[0]: (int(l.split()[1]), float(l.split()[2])) for l in run.stdout.strip().splitlines()}


@pytest.mark.parametrize("name,tol", [("factor_vjp", 1e-4), ("factor_value", 1e-5), ("xdotn_grad", 5e-4),
                                      ("camera_factor_grad", 1e-5)])
def test_reverse_mode_matches_dual_numbers(harness, name, tol):
    cases, worst = harness[name]
    assert cases > 10000
    assert worst < tol, f"{name}: worst relative error {worst:.3e}"


def test_bsdf_adjoint_matches_autograd_of_the_oracle(harness_exe, tmp_path):
    """eval_inner_vjp, the library's hand-written reverse mode of the BSDF
    value (Diffuse.cpp:37-41, Microfacet.cpp:37-79), against torch autograd
    of the oracle's independent restatement (tr_oracle.eval_inner) in float64,
    on 2000 seeded cases (a tenth with a direction below the horizon).

    Each output (value, gradients with respect to the two local directions
    and the albedo) is measured by its error relative to the float64 result,
    and so is the same autograd run in float32. Near grazing directions
    (cos ~ 1e-3) the gradient's 1/q^2 terms cancel, and both float32
    computations are then about 1e-4 off. The hand-written adjoint must be as
    accurate as float32 autograd: its median, 99th percentile and largest
    error within 2x, 3x and 2x of autograd's (measured: 3.6e-8, 5.2e-6 and
    1.02e-4 against 3.5e-8, 2.9e-6 and 1.03e-4)."""
    from types import SimpleNamespace

    import numpy as np
    import torch

    from oracle import tr_oracle as O
    rng = np.random.default_rng(4)
    n = 2000
    c = np.zeros((n, 17), np.float32)
    c[:, 0] = rng.integers(0, 2, n)
    c[:, 1] = rng.uniform(0.05, 1.0, n)
    c[:, 2:5] = rng.uniform(0, 1, (n, 3))
    c[:, 5:8] = rng.uniform(0, 1, (n, 3))
    for cols in (slice(8, 11), slice(11, 14)):
        v = rng.normal(size=(n, 3))
        v[:, 2] = np.abs(v[:, 2]) * np.where(rng.random(n) < 0.9, 1.0, -1.0)
        c[:, cols] = v / np.linalg.norm(v, axis=1, keepdims=True)
    c[:, 14:17] = rng.normal(size=(n, 3))
    fi, fo = tmp_path / "in.bin", tmp_path / "out.bin"
    fi.write_bytes(np.int32(n).tobytes() + c.tobytes())
    subprocess.run([harness_exe, "eval_inner_vjp", str(fi), str(fo)], check=True, timeout=120)
    out = np.fromfile(str(fo), np.float32).reshape(n, 12)

    def autograd(i, dtype):
        b = SimpleNamespace(type=int(c[i, 0]), roughness=float(c[i, 1]),
                            specular=tuple(float(x) for x in c[i, 2:5]))
        kd, lo, li = (torch.tensor(c[i:i + 1, a:a + 3], dtype=dtype, requires_grad=True) for a in (5, 8, 11))
        B = O.eval_inner(b, kd, lo, li)
        B.backward(torch.tensor(c[i:i + 1, 14:17], dtype=B.dtype))
        zero = torch.zeros(1, 3, dtype=B.dtype)
        return [B.detach()[0]] + [(t.grad if t.grad is not None else zero)[0] for t in (lo, li, kd)]

    e_lib, e_f32 = [], []
    for i in range(n):
        r64, r32 = autograd(i, torch.float64), autograd(i, torch.float32)
        for j in range(4):
            ref = r64[j].numpy()
            scale = max(np.abs(ref).max(), 1e-6)
            e_lib.append(np.abs(out[i, 3 * j:3 * j + 3] - ref).max() / scale)
            e_f32.append(np.abs(r32[j].double().numpy() - ref).max() / scale)
    e_lib, e_f32 = np.array(e_lib), np.array(e_f32)
    assert np.median(e_lib) <= 2 * np.median(e_f32) + 1e-9
    assert np.percentile(e_lib, 99) <= 3 * np.percentile(e_f32, 99)
    assert e_lib.max() <= 2 * e_f32.max(), (e_lib.max(), e_f32.max())


def test_xdotn_adjoint_matches_autograd_of_the_oracle(harness_exe, tmp_path):
    """xdotn_grad, the library's reverse mode of the boundary terms' xDotN
    (RayIntersectAD, Utils.cpp:288-297, then n . (w P0 + u P1 + v P2) with
    detached vertices), against float64 autograd of the same composition of
    the oracle's ray_intersect_ad and normalize, on 2000 seeded rays towards
    random triangles. Value and the gradients with respect to the ray's two
    points and the three vertices are as accurate as float32 autograd: median,
    99th percentile and largest error within 2x, 3x and 2x of autograd's
    (measured: 3.2e-7, 1.2e-4 and 8.2e-3 against 3.6e-7, 1.2e-4 and 8.2e-3;
    the tail is rays nearly parallel to their triangle)."""
    import numpy as np
    import torch

    from oracle import tr_oracle as O
    rng = np.random.default_rng(8)
    n = 2000
    c = np.zeros((n, 19), np.float32)
    P0 = rng.normal(size=(n, 3))
    P1, P2 = P0 + rng.normal(size=(n, 3)), P0 + rng.normal(size=(n, 3))
    bary = rng.dirichlet([1, 1, 1], n)
    hit = bary[:, :1] * P0 + bary[:, 1:2] * P1 + bary[:, 2:3] * P2
    org = hit + rng.normal(size=(n, 3)) * 2
    target = org + (hit - org) * rng.uniform(0.3, 0.9, (n, 1))
    c[:, 0:3], c[:, 3:6], c[:, 6:9], c[:, 9:12], c[:, 12:15] = org, target, P0, P1, P2
    nn = rng.normal(size=(n, 3))
    c[:, 15:18] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    c[:, 18] = rng.normal(size=n)
    fi, fo = tmp_path / "in.bin", tmp_path / "out.bin"
    fi.write_bytes(np.int32(n).tobytes() + c.tobytes())
    subprocess.run([harness_exe, "xdotn_grad", str(fi), str(fo)], check=True, timeout=120)
    out = np.fromfile(str(fo), np.float32).reshape(n, 16)

    def autograd(i, dtype):
        pts = [torch.tensor(c[i:i + 1, a:a + 3], dtype=dtype, requires_grad=True) for a in (0, 3, 6, 9, 12)]
        o, tg, p0, p1, p2 = pts
        u, v = O.ray_intersect_ad(O.normalize(tg - o), o, p0, p1 - p0, p2 - p0)
        w = 1.0 - u - v
        u2 = w[:, None] * p0.detach() + u[:, None] * p1.detach() + v[:, None] * p2.detach()
        x = O.dot(torch.tensor(c[i:i + 1, 15:18], dtype=dtype), u2)
        (x * float(c[i, 18])).sum().backward()
        return [x.detach()] + [p.grad[0] for p in pts]

    e_lib, e_f32 = [], []
    for i in range(n):
        r64, r32 = autograd(i, torch.float64), autograd(i, torch.float32)
        got = [out[i, 0:1]] + [out[i, 1 + 3 * j:4 + 3 * j] for j in range(5)]
        for g, a, b in zip(got, r64, r32):
            ref = a.numpy()
            scale = max(np.abs(ref).max(), 1e-6)
            e_lib.append(np.abs(g - ref).max() / scale)
            e_f32.append(np.abs(b.double().numpy() - ref).max() / scale)
    e_lib, e_f32 = np.array(e_lib), np.array(e_f32)
    assert np.median(e_lib) <= 2 * np.median(e_f32) + 1e-9
    assert np.percentile(e_lib, 99) <= 3 * np.percentile(e_f32, 99)
    assert e_lib.max() <= 2 * e_f32.max(), (e_lib.max(), e_f32.max())


def test_camera_factor_adjoint_matches_autograd_of_the_oracle(harness_exe, tmp_path):
    """camera_factor_grad, the library's reverse mode of EvalFilter's factor
    G / Detach(G) * J (Camera.cpp:279-303), against float64 autograd of the
    oracle's camera_factor on 2000 seeded points, normals and weights, with
    the library's camera. As accurate as float32 autograd: median, 99th
    percentile and largest error within 2x, 3x and 2x of autograd's
    (measured: 3.6e-8, 8.1e-7 and 6.2e-6 against 4.2e-8, 8.2e-7 and 6.2e-6)."""
    import numpy as np
    import torch

    from oracle import tr_oracle as O
    from tensorray_b200 import api
    rng = np.random.default_rng(9)
    cam = api.Camera((1.0, 2.0, 5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 320, 200, 40.0)
    m32 = cam.matrices()
    m64 = {k: (np.asarray(v, np.float64) if isinstance(v, np.ndarray) else v) for k, v in m32.items()}
    n = 2000
    c = np.zeros((n, 7), np.float32)
    c[:, 0:3] = rng.normal(0, 1.0, (n, 3))
    ng = rng.normal(size=(n, 3))
    c[:, 3:6] = ng / np.linalg.norm(ng, axis=1, keepdims=True)
    c[:, 6] = rng.normal(size=n)
    fi, fo = tmp_path / "in.bin", tmp_path / "out.bin"
    fi.write_bytes(np.int32(n).tobytes() + bytes(cam.c) + c.tobytes())
    subprocess.run([harness_exe, "camera_factor_grad", str(fi), str(fo)], check=True, timeout=120)
    out = np.fromfile(str(fo), np.float32).reshape(n, 7)

    def autograd(i, dtype, mats):
        p = torch.tensor(c[i:i + 1, 0:3], dtype=dtype, requires_grad=True)
        g = torch.tensor(c[i:i + 1, 3:6], dtype=dtype, requires_grad=True)
        J = torch.ones(1, dtype=dtype, requires_grad=True)
        (O.camera_factor(mats, p, g, J) * float(c[i, 6])).sum().backward()
        return [p.grad[0], g.grad[0], J.grad]

    e_lib, e_f32 = [], []
    for i in range(n):
        r64, r32 = autograd(i, torch.float64, m64), autograd(i, torch.float32, m32)
        for got, a, b in zip([out[i, 0:3], out[i, 3:6], out[i, 6:7]], r64, r32):
            ref = a.numpy()
            scale = max(np.abs(ref).max(), 1e-6)
            e_lib.append(np.abs(got - ref).max() / scale)
            e_f32.append(np.abs(b.double().numpy() - ref).max() / scale)
    e_lib, e_f32 = np.array(e_lib), np.array(e_f32)
    assert np.median(e_lib) <= 2 * np.median(e_f32) + 1e-9
    assert np.percentile(e_lib, 99) <= 3 * np.percentile(e_f32, 99)
    assert e_lib.max() <= 2 * e_f32.max(), (e_lib.max(), e_f32.max())


def test_path_factor_adjoint_matches_autograd_of_the_oracle(harness_exe, tmp_path):
    """factor_vjp, the library's reverse mode of the NEE / continuation factor
    of EvalRadianceDirect (Integrator.cpp:186-267),
    F = B(kd, wo, wi) |ns.wi| |nz.wi| / d^2 J K with the BSDF in the frame
    coordinate_system builds around the unnormalised shading normal, against
    float64 autograd of the same factor composed from the oracle's
    coordinate_system, bsdf_eval, normalize and dot, on 2000 seeded diffuse
    and GGX vertices. Value and the gradients with respect to the previous
    vertex, the vertex, the shading normal, the albedo, the next point, its
    normal and J are as accurate as float32 autograd: median, 99th percentile
    and largest error within 2x, 3x and 2x of autograd's (measured: 1.6e-7,
    6.6e-6 and 2.8e-3 against 1.6e-7, 6.7e-6 and 2.5e-2)."""
    from types import SimpleNamespace

    import numpy as np
    import torch

    from oracle import tr_oracle as O
    rng = np.random.default_rng(12)
    n = 2000

    def unit(m):
        v = rng.normal(size=(m, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    c = np.zeros((n, 30), np.float32)
    c[:, 0] = (np.arange(n) % 3 != 0).astype(np.float32)
    c[:, 1] = rng.uniform(0.1, 0.9, n)
    c[:, 2:5] = [0.04, 0.05, 0.5]
    ns = unit(n) * 0.3 + np.array([0.0, 1.0, 0.0])
    nsu = ns / np.linalg.norm(ns, axis=1, keepdims=True)
    ns = nsu * rng.uniform(0.9, 1.0, (n, 1))                      # unnormalised shading normals
    x = rng.uniform(-1, 1, (n, 3))
    c[:, 5:8] = x + (nsu + unit(n) * 0.8) * rng.uniform(1, 2, (n, 1))
    c[:, 8:11], c[:, 11:14] = x, ns
    c[:, 14:17] = [0.3, 0.5, 0.7]
    c[:, 17:20] = x + (nsu + unit(n) * 0.8) * rng.uniform(0.5, 2.5, (n, 1))
    c[:, 20:23] = unit(n)
    c[:, 23] = rng.uniform(0.5, 1.5, n)
    c[:, 24:27] = rng.uniform(0.1, 10, (n, 3))
    c[:, 27:30] = rng.normal(size=(n, 3))
    fi, fo = tmp_path / "in.bin", tmp_path / "out.bin"
    fi.write_bytes(np.int32(n).tobytes() + c.tobytes())
    subprocess.run([harness_exe, "factor_vjp", str(fi), str(fo)], check=True, timeout=120)
    out = np.fromfile(str(fo), np.float32).reshape(n, 22)

    def autograd(i, dtype):
        b = SimpleNamespace(type=int(c[i, 0]), roughness=float(c[i, 1]), specular=tuple(float(v) for v in c[i, 2:5]))
        xp, xx, nsv, kd, zz, nz = (torch.tensor(c[i:i + 1, a:a + 3], dtype=dtype, requires_grad=True)
                                   for a in (5, 8, 11, 14, 17, 20))
        J = torch.tensor(c[i:i + 1, 23], dtype=dtype, requires_grad=True)
        wo = -O.normalize(xx - xp)
        t, bb = O.coordinate_system(nsv)
        wi = zz - xx
        d2 = O.dot(wi, wi)
        wi = wi / torch.sqrt(d2)[:, None]
        G = O.dot(nz, -wi).abs() / d2
        bv = O.bsdf_eval(b, (t, bb, nsv), None, kd, wo, wi, False) * O.dot(nsv, wi).abs()[:, None]
        F = bv * (J * G)[:, None] * torch.tensor(c[i:i + 1, 24:27], dtype=dtype)
        (F * torch.tensor(c[i:i + 1, 27:30], dtype=dtype)).sum().backward()
        zero = torch.zeros(1, 3, dtype=dtype)
        return [F.detach()[0]] + [(q.grad if q.grad is not None else zero)[0]
                                  for q in (xp, xx, nsv, kd, zz, nz)] + [J.grad]

    e_lib, e_f32 = [], []
    for i in range(n):
        r64, r32 = autograd(i, torch.float64), autograd(i, torch.float32)
        got = [out[i, 0:3]] + [out[i, 3 + 3 * j:6 + 3 * j] for j in range(6)] + [out[i, 21:22]]
        for g, a, b in zip(got, r64, r32):
            ref = a.numpy()
            scale = max(np.abs(ref).max(), 1e-6)
            e_lib.append(np.abs(g - ref).max() / scale)
            e_f32.append(np.abs(b.double().numpy() - ref).max() / scale)
    e_lib, e_f32 = np.array(e_lib), np.array(e_f32)
    assert np.median(e_lib) <= 2 * np.median(e_f32) + 1e-9
    assert np.percentile(e_lib, 99) <= 3 * np.percentile(e_f32, 99)
    assert e_lib.max() <= 2 * e_f32.max(), (e_lib.max(), e_f32.max())
