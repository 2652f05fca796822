"""The C++ host API over the C ABI (include/fi_sqlops.hpp), run on the GPU:
tests/cpp/host_api_test.cpp partitions, joins and checks the reference's
argument errors through the C++ classes that mirror the reference's Rust
API (GpuRadixPartitioner, PartitionOffsets, PartitionedRelation,
CudaRadixJoin)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_cpp_host_api():
    r = subprocess.run(["make", "-s", "-C", os.path.join(HERE, "cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([os.path.join(HERE, "cpp", "_build", "host_api_test")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host api ok" in r.stdout
