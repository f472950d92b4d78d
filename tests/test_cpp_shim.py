"""The C++ shim include/sil/ddc_compat.hpp: it and a reference-style call
site (tests/cpp/shim_example.cpp) compile; on a GPU the call site's outputs
match the oracle (d bit-exact, Laplacian 1e-12, solve to 1e-10, the
general-metric staged Laplacian and codifferential 1e-12)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"
EXAMPLE = os.path.join(ROOT, "tests", "cpp", "shim_example.cpp")


def _gxx():
    return shutil.which("g++")


@pytest.mark.skipif(_gxx() is None, reason="no g++")
def test_shim_and_example_compile():
    subprocess.check_call([_gxx(), "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"), EXAMPLE])


@pytest.mark.skipif(_gxx() is None, reason="no g++")
def test_environment_overrides(tmp_path):
    """The reference's SIMILIE_* overrides: applied where the library has the
    feature, refused with SIL_ERR_UNSUPPORTED where it has not (no GPU call)."""
    exe = str(tmp_path / "shim_env")
    subprocess.check_call([_gxx(), "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "shim_env.cpp"),
                           "-o", exe])
    env = {k: v for k, v in os.environ.items() if not k.startswith("SIMILIE_")}
    out = subprocess.run([exe], check=True, capture_output=True, text=True, env=env).stdout
    assert out.strip().endswith("env ok"), out


@pytest.mark.gpu
def test_example_matches_the_oracle(tmp_path):
    lib = os.path.join(ROOT, "similie_b200", "libsil_b200.so")
    assert os.path.exists(lib), "build the library first"
    exe = str(tmp_path / "shim_example")
    subprocess.check_call([_gxx(), "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(CUDA, "include"), EXAMPLE, "-o", exe, lib,
                           "-L", os.path.join(CUDA, "lib64"), "-lcudart",
                           "-Wl,-rpath," + os.path.dirname(lib) + ":" + os.path.join(CUDA, "lib64")])
    out = subprocess.run([exe, str(tmp_path)], check=True, capture_output=True, text=True).stdout.split("\n")
    it, conv, rel = out[0].split()
    assert int(conv) == 1 and float(rel) <= 1e-10
    assert out[1].startswith("error 1")       # k = 3 on a 2D field: SIL_ERR_INVALID
    tag, it2, conv2, rel2, nnz = out[2].split()
    assert tag == "assembled" and int(conv2) == 1 and float(rel2) <= 1e-10
    assert int(it2) < int(it)                  # SSOR needs fewer iterations than Jacobi
    ref_nnz = O.assemble2d(33, 33, rd_mu(tmp_path)).nnz  # up to entries cancelling to exactly zero in one arithmetic
    assert abs(int(nnz) - ref_nnz) <= ref_nnz // 100
    rd = lambda name: np.fromfile(str(tmp_path / name), dtype=np.float64)
    nx, ny = 12, 9
    phi = rd("phi.bin").reshape(nx, ny, 1)
    ref = np.zeros((nx, ny, 2))
    O.coboundary(phi, ref, 0)
    np.testing.assert_array_equal(rd("dphi.bin").reshape(nx, ny, 2), ref)
    xs = 0.1 * np.arange(nx) + 0.002 * np.arange(nx) ** 2
    ys = 0.15 * np.arange(ny)
    lap = O.laplacian(2, 0, O.position_from_coords([xs, ys]), phi)
    np.testing.assert_allclose(rd("lap.bin").reshape(nx - 1, ny - 1, 1), lap, rtol=1e-12, atol=1e-12 * np.abs(lap).max())
    n = 33
    r = rd("rhs.bin") - O.mag2d_apply(n, n, rd("mu.bin"), rd("sol.bin"))
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(rd("rhs.bin"))
    r2 = rd("rhs.bin") - O.mag2d_apply(n, n, rd("mu.bin"), rd("sol_ssor.bin"))
    assert np.linalg.norm(r2) <= 2e-10 * np.linalg.norm(rd("rhs.bin"))
    # general-metric staged Laplacian and codifferential through the shim
    assert out[3] == "metric ok"
    mx, my = 10, 8
    pos, met, w1 = rd("pos.bin").reshape(mx, my, 2), rd("met.bin").reshape(mx, my, 4), rd("w1.bin").reshape(mx, my, 2)
    lap1 = O.laplacian(2, 1, pos, w1, metric=met)
    got = rd("lap1.bin").reshape(mx - 1, my - 1, 2)
    assert np.max(np.abs(got - lap1)) <= 1e-12 * np.max(np.abs(lap1))
    cod = O.codifferential(2, 1, pos, w1, metric=met)
    got = rd("cod.bin").reshape(mx, my, 1)
    assert np.max(np.abs(got - cod)) <= 1e-12 * np.max(np.abs(cod))


def rd_mu(tmp_path):
    return np.fromfile(str(tmp_path / "mu.bin"), dtype=np.float64)
