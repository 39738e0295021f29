"""The C++ drop-in header, compiled and run the way a reference caller would
use it (tests/cpp/test_dropin.cpp)."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

pytestmark = pytest.mark.gpu


def test_cpp_dropin(cuda, tmp_path):
    import cassandra_b200

    cassandra_b200.load()
    exe = tmp_path / "test_dropin"
    cmd = ["g++", "-std=c++20", "-O2", f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include",
           str(ROOT / "tests" / "cpp" / "test_dropin.cpp"), "-o", str(exe), f"-L{ROOT / 'cassandra_b200'}",
           "-lcassandra_b200", "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{ROOT / 'cassandra_b200'}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "ALL OK" in res.stdout
