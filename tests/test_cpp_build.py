"""The C++ wrapper header (include/fcib_solver.hpp) and the driver that uses it compile with g++ and link
against the engine library; no GPU needed (the driver is run by tests/test_gpu_cpp.py)."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "cpp"))


def test_cpp_driver_builds(tmp_path):
    import build as cpp_build
    from forte_b200 import build

    build.build()
    exe = cpp_build.build(str(tmp_path))
    assert os.access(exe, os.X_OK)
