"""Host-compiled unit tests of device math (no GPU): the exact jump-ahead
through the walk's rounded running sums, built from the same header the
kernels include."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_dda_jump_matches_sequential_sums(tmp_path):
    exe = tmp_path / "test_dda_jump"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", str(exe),
                           os.path.join(HERE, "cpp", "test_dda_jump.cpp")])
    out = subprocess.run([str(exe), "30000"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert " 0 failures" in out.stdout


def test_cpp_dropin_header_compiles():
    """include/cublox/OccupancyGrid.hpp compiles against the C ABI header."""
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    inc = os.path.join(here, "..", "include")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", inc,
                        os.path.join(here, "cpp", "header_compiles.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
