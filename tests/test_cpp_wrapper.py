"""The C++ drop-in (include/mpm/mpm.hpp) compiles against the C ABI and links
to libmpm_b200.so; without a GPU its constructor throws the no-device status."""
import shutil
import subprocess

import pytest

from conftest import ROOT, has_gpu

SRC = r'''
#include <cstdio>
#include <vector>
#include "mpm/mpm.hpp"
struct Vec2 { float x, y; };
int main() {
    mpm_params p;
    mpm_params_default(&p, 2);
    p.width = 32; p.height = 32; p.border_margin = 3;
    std::vector<Vec2> pos = {{10.f, 10.f}, {10.5f, 10.25f}}, vel = {{0.f, -1.f}, {0.f, -1.f}};
    std::vector<float> vol = {0.25f, 0.25f};
    try {
        using Solver = mpm::BasicSolver<Vec2>;
        Solver solver(p, pos, vel, vol);
        for (int i = 0; i < 10; ++i) solver.Step();
        const std::vector<Vec2>& out = solver.GetParticlePositions();
        std::printf("ok %zu %.6f %.6f\n", out.size(), out[0].x, out[0].y);
        return 0;
    } catch (const std::exception& e) {
        std::printf("error %s\n", e.what());
        return 3;
    }
}
'''


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    from mpm_snow_sim2d_b200.build import LIB, build
    build()
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("cpp")
    (d / "main.cpp").write_text(SRC)
    exe = d / "drop_in"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(d / "main.cpp"), str(LIB),
                    f"-Wl,-rpath,{LIB.parent}", "-o", str(exe)], check=True)
    return exe


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_cpp_drop_in_reports_no_device(program):
    res = subprocess.run([str(program)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 3
    assert "no usable sm_100" in res.stdout


@pytest.mark.gpu
def test_cpp_drop_in_steps_on_gpu(program):
    res = subprocess.run([str(program)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    _, n, x, y = res.stdout.split()
    assert int(n) == 2 and abs(float(x) - 10.0) < 0.1 and float(y) < 10.0
