"""NVTX ranges of the library's entry points, on the CPU.

Every entry point that issues device work opens an NVTX range named after itself for
the call's duration, so that a profiler groups the kernels under the call. This test
attaches a minimal NVTX tool (tests/nvtx_probe.c, built here with gcc) through
NVTX_INJECTION64_PATH in a child process, calls entry points that finish on the host
(the OBJ reader, and calls refused for their arguments), and reads the ranges back."""
import os
import shutil
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

CHILD = r"""
import ctypes, sys
sys.path.insert(0, sys.argv[1])
import cpt
n = ctypes.c_uint32()
assert cpt.lib.cpt_obj_load(sys.argv[2].encode(), 1.0, None, 0.7, None, None, 0, ctypes.byref(n)) == cpt.OK
assert n.value == 1
b = cpt.Bvh()
assert cpt.lib.cpt_lbvh_build(None, 100, None, 30, ctypes.byref(b), None, 0, 0, None) == cpt.ERR_INVALID_ARGUMENT
assert cpt.lib.cpt_trace(None, None, 1, 0, None, None, None) == cpt.ERR_INVALID_ARGUMENT
assert cpt.lib.cpt_lbvh_split(None, 1.0, 0, None, 0, None, 0, None) == cpt.ERR_INVALID_ARGUMENT
assert cpt.lib.cpt_resolve(None, 8, 8, 0, None, None) == cpt.ERR_INVALID_ARGUMENT
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc to build the NVTX probe")
def test_entry_points_open_named_ranges(tmp_path):
    probe = str(tmp_path / "libnvtx_probe.so")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["gcc", "-shared", "-fPIC", "-O1", f"-I{cuda_inc}", "-o", probe,
                    os.path.join(ROOT, "tests", "nvtx_probe.c")], check=True)
    obj = tmp_path / "tri.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    log = tmp_path / "ranges.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=probe, CPT_NVTX_LOG=str(log))
    subprocess.run([sys.executable, "-c", CHILD, PKG, str(obj)], check=True, env=env, timeout=300)
    lines = log.read_text().split("\n")[:-1]
    assert lines == ["push cpt_obj_load", "pop", "push cpt_lbvh_build", "pop", "push cpt_trace", "pop",
                     "push cpt_lbvh_split", "pop", "push cpt_resolve", "pop"]
