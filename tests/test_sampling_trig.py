"""The sampling code's sin/cos/acos (csrc/common.cuh: sincos_det, acos_det)
against the oracle's numpy restatement, bit for bit, and against float64
libm within one float ulp. The CPU case runs the host build of the same
source; the GPU case runs it in a kernel and also bounds the distance to
CUDA's own sinf/cosf/acosf."""
import os
import subprocess

import numpy as np
import pytest

from oracle import tr_oracle as O
from tensorray_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))


def _inputs():
    g = np.random.default_rng(5)
    ang = g.uniform(-2 * np.pi - 0.5, 2 * np.pi + 0.5, 200_000)
    unit = g.uniform(-1.0, 1.0, 200_000)
    edge = np.array([0.0, -0.0, 1.0, -1.0, 0.5, -0.5, np.pi / 4, -np.pi / 4, np.pi / 2, np.pi, 2 * np.pi,
                     1.0000001, -1.0000001, 1e-30, 0.99999994, -0.99999994])
    near = np.concatenate([k * np.pi / 4 + g.uniform(-1e-6, 1e-6, 2000) for k in range(-8, 9)])
    return np.concatenate([ang, unit, edge, near]).astype(np.float32)


def _compile(tmp):
    out = os.path.join(tmp, "trig_harness")
    cmd = [build._nvcc(), "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "--expt-relaxed-constexpr", "-fmad=false", os.path.join(HERE, "native", "trig_harness.cu"),
           "-o", out, "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        pytest.fail("nvcc failed:\n" + res.stderr[-2000:])
    return out


def _run(tmp, device):
    exe = _compile(tmp)
    x = _inputs()
    inp = os.path.join(tmp, "x.f32")
    x.tofile(inp)
    args = [exe, inp, os.path.join(tmp, "out")] + (["device"] if device else [])
    res = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    host = np.fromfile(os.path.join(tmp, "out.host.f32"), np.float32).reshape(-1, 3)
    dev = np.fromfile(os.path.join(tmp, "out.dev.f32"), np.float32).reshape(2, -1, 3) if device else None
    return x, host, dev


def _oracle(x):
    s, c = O.sincos_det(x)
    return np.stack([s.numpy(), c.numpy(), O.acos_det(x).numpy()], -1)


def _ulps(a, ref64):
    ref = ref64.astype(np.float32)
    ok = np.isfinite(ref64)
    return np.abs(a[ok].astype(np.float64) - ref64[ok]) / np.spacing(np.abs(ref[ok]))


def _check_accuracy(x, out):
    xd = x.astype(np.float64)
    assert _ulps(out[:, 0], np.sin(xd)).max() <= 1.0
    assert _ulps(out[:, 1], np.cos(xd)).max() <= 1.0
    with np.errstate(invalid="ignore"):
        ref = np.arccos(xd)
    assert np.array_equal(np.isnan(out[:, 2]), np.isnan(ref))
    assert _ulps(out[:, 2], ref).max() <= 1.0


def test_host_trig_matches_oracle_bits(tmp_path):
    x, host, _ = _run(str(tmp_path), device=False)
    np.testing.assert_array_equal(host.view(np.uint32), _oracle(x).view(np.uint32))
    _check_accuracy(x, host)


@pytest.mark.gpu
def test_device_trig_matches_oracle_bits(tmp_path):
    x, host, dev = _run(str(tmp_path), device=True)
    ours, cuda = dev[0], dev[1]
    np.testing.assert_array_equal(ours.view(np.uint32), _oracle(x).view(np.uint32))
    np.testing.assert_array_equal(ours.view(np.uint32), host.view(np.uint32))
    _check_accuracy(x, ours)
    # CUDA's single-precision functions are accurate to a few ulp; ours sit
    # within that distance of them
    for k in range(3):
        ok = np.isfinite(ours[:, k]) & np.isfinite(cuda[:, k]) & (np.abs(ours[:, k]) > 1e-6)
        d = np.abs(ours[ok, k].astype(np.float64) - cuda[ok, k]) / np.spacing(np.abs(ours[ok, k]))
        assert d.max() <= 4.0, (k, float(d.max()))
