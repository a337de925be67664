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
def harness(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("vjp") / "vjp_harness")
    src = os.path.join(HERE, "native", "vjp_harness.cu")
    scene = os.path.join(build.CSRC, "scene.cu")
    cmd = [build._nvcc(), "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "--expt-relaxed-constexpr", "--extended-lambda", src, scene, "-o", out, "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        pytest.fail("nvcc failed:\n" + res.stderr[-2000:])
    run = subprocess.run([out], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    return {l.split()[0]: (int(l.split()[1]), float(l.split()[2])) for l in run.stdout.strip().splitlines()}


@pytest.mark.parametrize("name,tol", [("factor_vjp", 1e-4), ("factor_value", 1e-5), ("xdotn_grad", 5e-4),
                                      ("camera_factor_grad", 1e-5)])
def test_reverse_mode_matches_dual_numbers(harness, name, tol):
    cases, worst = harness[name]
    assert cases > 10000
    assert worst < tol, f"{name}: worst relative error {worst:.3e}"
