"""The header-only C++ adapter (include/cmpmc_b200/run_events_gpu.hpp) compiles against the
reference's own headers and links the C ABI library. Runs where the reference headers are
available (the oracle build host); without a device the run stops at context creation."""
import os
import subprocess

import pytest

from tests.helpers import ROOT, has_gpu

REF_INCLUDE = "/root/reference/include"


@pytest.mark.skipif(not os.path.isdir(REF_INCLUDE), reason="reference headers not present")
def test_adapter_compiles_links_and_runs(tmp_path):
    exe = tmp_path / "shim_example"
    lib_dir = os.path.join(ROOT, "cmpmc_b200", "_lib")
    cmd = ["g++", "-std=c++20", "-O1", "-pthread", f"-I{REF_INCLUDE}", f"-I{os.path.join(ROOT, 'include')}",
           os.path.join(ROOT, "tests", "shim_example.cpp"), f"-L{lib_dir}", "-lcmpmc_b200", f"-Wl,-rpath,{lib_dir}",
           "-o", str(exe)]
    subprocess.run(cmd, check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    if has_gpu():
        assert r.returncode == 0, r.stdout + r.stderr
    else:
        assert r.returncode == 3 and "no CUDA device" in r.stdout, r.stdout + r.stderr
