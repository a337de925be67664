"""The library's shading functions, compiled for the host by nvcc from
csrc/shading.cuh (tests/native/shading_harness.cu), against the oracle's
restatements on seeded cases that include grazing and below-horizon
directions, roughness from 0.01 to 1 and samples at 0, 1/2 and the ends of
(0, 1):

- cosine_hemisphere (Utils.cpp:70-95), disk_concentric (Utils.cpp:97-115),
  coordinate_system (Utils.cpp:118-140), out_dir_valid and the GGX visible-
  normal sample (BSDF.cpp:272-302) agree bit for bit, NaNs included;
- eval_inner (Diffuse.cpp:37-41, Microfacet.cpp:37-79) and bsdf_pdf_local
  agree within 1e-6 relative per case: the Fresnel term's exp and a few
  divisions round differently in libm and in torch (largest seen: 2.1e-7 and
  2.5e-7);
- the sensor functions, Camera::sampleDirect (Camera.cpp:399-416), the
  boundary-ray direction (Camera.cpp:379-397), WriteToImage's pixel
  (Camera.cpp:418-431) and EvalFilter's factor (Camera.cpp:279-303), agree
  bit for bit on the library's camera;
- the counter-hash sampler and discrete sampling with sample reuse agree bit
  for bit.

The device build of the same functions is checked against the oracle by the
GPU parity tests; this adds per-function coverage of the edge cases without
a GPU."""
import os
import subprocess
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import tr_oracle as O
from tensorray_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))
N = 20000
N_BSDF = 1500      # cases that go through the oracle's per-material calls


@pytest.fixture(scope="module")
def harness_exe(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("shading_exe") / "shading_harness")
    cmd = [build._nvcc(), "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "--expt-relaxed-constexpr", os.path.join(HERE, "native", "shading_harness.cu"), "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        pytest.fail("nvcc failed:\n" + res.stderr[-2000:])
    return exe


@pytest.fixture(scope="module")
def harness_out(harness_exe, tmp_path_factory):
    d = tmp_path_factory.mktemp("shading")
    c = _cases()
    fi, fo = str(d / "in.bin"), str(d / "out.bin")
    with open(fi, "wb") as f:
        f.write(np.int32(N).tobytes())
        f.write(c.tobytes())
    subprocess.run([harness_exe, fi, fo], check=True, timeout=120)
    return c, np.fromfile(fo, np.float32).reshape(N, 19)


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _cases() -> np.ndarray:
    """Records of the harness: type, roughness, spec[3], kd[3], wo[3], wi[3],
    s0, s1, n[3], ng[3]."""
    rng = np.random.default_rng(0)
    c = np.zeros((N, 22), np.float32)
    c[:, 0] = rng.integers(0, 2, N)
    c[:, 1] = np.where(rng.random(N) < 0.1, rng.choice([0.01, 0.05, 1.0], N), rng.uniform(0.02, 1.0, N))
    c[:, 2:5] = rng.uniform(0, 1, (N, 3))
    c[:, 5:8] = rng.uniform(0, 1, (N, 3))
    wo, wi = _unit(rng, N), _unit(rng, N)
    g = rng.random(N) < 0.1                       # grazing and horizon outgoing directions
    wo[g, 2] = rng.choice([1e-4, -1e-4, 1e-7, 0.0], g.sum())
    wo[g] /= np.linalg.norm(wo[g], axis=1, keepdims=True)
    c[:, 8:11], c[:, 11:14] = wo, wi
    s = rng.random((N, 2))
    e = rng.random(N) < 0.05                      # samples at the edges of (0, 1)
    s[e] = rng.choice([0.0, 0.5, 1 - 2 ** -24, 2 ** -24], (e.sum(), 2))
    c[:, 14:16] = s
    c[:, 16:19] = rng.normal(size=(N, 3))
    c[:, 19:22] = _unit(rng, N)
    return c


def _t(a):
    return torch.as_tensor(np.ascontiguousarray(a))


def _bits_equal(ours, ref):
    ours = np.ascontiguousarray(ours, np.float32)
    ref = np.ascontiguousarray(ref, np.float32)
    same = (ours.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(ours) & np.isnan(ref))
    return bool(same.all())


def test_sampling_warps_and_frames_are_bit_identical(harness_out):
    c, out = harness_out
    s0, s1 = _t(c[:, 14]), _t(c[:, 15])
    assert _bits_equal(out[:, 4:7], O.cosine_hemisphere(s0, s1).numpy())
    dx, dy = O.disk_concentric(s0, s1)
    assert _bits_equal(out[:, 7:9], np.stack([dx.numpy(), dy.numpy()], 1))
    t, b = O.coordinate_system(_t(c[:, 16:19]))
    assert _bits_equal(out[:, 12:15], t.numpy()) and _bits_equal(out[:, 15:18], b.numpy())
    valid = np.zeros(N, np.float32)
    for typ in (0, 1):
        m = c[:, 0] == typ
        valid[m] = O.out_dir_valid(SimpleNamespace(type=typ), _t(c[m, 16:19]), _t(c[m, 19:22]),
                                   _t(c[m, 11:14])).numpy()
    assert np.array_equal(out[:, 18], valid)


def test_bsdf_value_pdf_and_visible_normal_sample(harness_out):
    c, out = harness_out
    worst_eval = worst_pdf = 0.0
    for i in range(N_BSDF):
        b = SimpleNamespace(type=int(c[i, 0]), roughness=float(c[i, 1]), specular=tuple(float(x) for x in c[i, 2:5]))
        kd, wo, wi = _t(c[i:i + 1, 5:8]), _t(c[i:i + 1, 8:11]), _t(c[i:i + 1, 11:14])
        ev = O.eval_inner(b, kd, wo, wi).numpy()[0].astype(np.float64)
        pdf = float(O.bsdf_pdf_local(b, wo, wi)[0])
        worst_eval = max(worst_eval, float(np.abs(out[i, 0:3] - ev).max() / max(np.abs(ev).max(), 1e-30)))
        worst_pdf = max(worst_pdf, abs(float(out[i, 3]) - pdf) / max(abs(pdf), 1e-30))
        if c[i, 10] > 0:
            vs = O.vndf_sample(wo, np.float32(c[i, 1]), _t(c[i:i + 1, 14]), _t(c[i:i + 1, 15])).numpy()[0]
            assert _bits_equal(out[i, 9:12], vs), i
    assert worst_eval <= 1e-6 and worst_pdf <= 1e-6, (worst_eval, worst_pdf)


def test_sensor_functions_are_bit_identical(harness_exe, tmp_path):
    from tensorray_b200 import api
    from tests.helpers import oracle_camera_from
    rng = np.random.default_rng(3)
    cam = api.Camera((1.0, 2.0, 5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 320, 200, 40.0)
    oc = oracle_camera_from(cam)
    n = 20000
    c = np.zeros((n, 9), np.float32)
    c[:, 0:3] = rng.normal(0, 2, (n, 3))                       # points in front of and behind the camera
    ng = rng.normal(size=(n, 3))
    c[:, 3:6] = ng / np.linalg.norm(ng, axis=1, keepdims=True)
    c[:, 6] = rng.uniform(0.5, 2, n)
    c[:, 7:9] = rng.uniform(-0.1, 1.1, (n, 2))                 # sensor coordinates, some off the film
    fi, fo = tmp_path / "cin.bin", tmp_path / "cout.bin"
    fi.write_bytes(np.int32(n).tobytes() + bytes(cam.c) + c.tobytes())
    subprocess.run([harness_exe, "camera", str(fi), str(fo)], check=True, timeout=120)
    out = np.fromfile(str(fo), np.float32).reshape(n, 10)
    qx, qy, valid, pixel, sval = O.sample_direct(oc, _t(c[:, 0:3]))
    assert _bits_equal(out[:, 0], qx.numpy()) and _bits_equal(out[:, 1], qy.numpy())
    assert np.array_equal(out[:, 2], valid.numpy().astype(np.float32))
    assert np.array_equal(out[:, 3], pixel.numpy().astype(np.float32))
    assert _bits_equal(out[:, 4], sval.numpy())
    assert _bits_equal(out[:, 5:8], O.sensor_ray_dir(oc, _t(c[:, 7]), _t(c[:, 8])).numpy())
    assert np.array_equal(out[:, 8], O.image_pixel(oc, _t(c[:, 7]), _t(c[:, 8])).numpy().astype(np.float32))
    assert _bits_equal(out[:, 9], O.camera_factor(oc, _t(c[:, 0:3]), _t(c[:, 3:6]), _t(c[:, 6])).numpy())


def test_sample_sources_are_bit_identical(harness_exe, tmp_path):
    """The counter-hash sampler every path reads its uniforms from
    (hash_uniform) over 15,200 (seed, term, dimension, slot) tuples, slots 0
    and 2^32 - 1 among them; and Distribution1D::SampleDiscrete with
    ReuseSample (Distribution.cu:37-48, Distribution.cpp:37-43) over CDFs of
    1-300 entries with zero-weight runs, at random samples, at the CDF's own
    values and at 0, 1 and the ends of (0, 1)."""
    rng = np.random.default_rng(5)
    recs, ref = [], []
    for _ in range(50):
        seed, term, dim = (int(x) for x in rng.integers(0, 2 ** 32, 3, dtype=np.uint64))
        slots = np.concatenate([rng.integers(0, 2 ** 32, 300, dtype=np.uint64),
                                np.array([0, 1, 2 ** 32 - 1, 2 ** 31], np.uint64)])
        recs += [(seed, term, dim, int(s)) for s in slots]
        ref.append(O.hash_uniform(seed, term, dim, slots))
    recs, ref = np.array(recs, np.uint32), np.concatenate(ref).astype(np.float32)
    fi, fo = tmp_path / "hin.bin", tmp_path / "hout.bin"
    fi.write_bytes(np.int32(len(recs)).tobytes() + recs.tobytes())
    subprocess.run([harness_exe, "hash", str(fi), str(fo)], check=True, timeout=120)
    assert _bits_equal(np.fromfile(str(fo), np.float32), ref)

    for _ in range(30):
        n = int(rng.integers(1, 300))
        f = rng.uniform(0, 1, n).astype(np.float32)
        f[rng.random(n) < 0.3] = 0
        f[0] = f[0] if f.sum() > 0 else 1.0
        cdf, integral = O.cdf_of(torch.as_tensor(f))
        u = np.concatenate([rng.random(500).astype(np.float32), cdf.numpy()[:50],
                            np.array([0.0, 1.0, 2 ** -24, 1 - 2 ** -24], np.float32)])
        fi, fo = tmp_path / "din.bin", tmp_path / "dout.bin"
        fi.write_bytes(np.int32(n).tobytes() + cdf.numpy().astype(np.float32).tobytes()
                       + np.int32(len(u)).tobytes() + u.tobytes())
        subprocess.run([harness_exe, "discrete", str(fi), str(fo)], check=True, timeout=120)
        raw = np.fromfile(str(fo), np.uint8).reshape(-1, 8)
        idx = raw[:, :4].copy().view(np.int32).ravel()
        reuse = raw[:, 4:].copy().view(np.float32).ravel()
        ri, _, rr = O.sample_discrete(cdf, integral, torch.as_tensor(f), torch.as_tensor(u))
        assert np.array_equal(idx, ri.numpy()) and _bits_equal(reuse, rr.numpy())
