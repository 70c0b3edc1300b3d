"""The C++ drop-in (include/cmpmc_b200/run_events_gpu.hpp): tests/shim_example.cpp changes
only the namespace of the reference's run_events call sites and checks the device results
against the reference's CPU run_events (plain form event by event, batched form within
statistics). oracle/Makefile builds it, against the reference's headers, into
oracle/_ref/shim_example, next to the other oracle programs; the binary travels with the
built library, so the GPU run needs no reference sources."""
import os
import subprocess

import pytest

from tests.helpers import ROOT, has_gpu

SHIM = os.path.join(ROOT, "oracle", "_ref", "shim_example")


def _run():
    if not os.path.exists(SHIM):
        pytest.skip("oracle/_ref/shim_example not built (make -C oracle ref needs the reference headers)")
    return subprocess.run([SHIM], capture_output=True, text=True, timeout=900)


def test_shim_refuses_to_run_without_device():
    if has_gpu():
        pytest.skip("a device is present")
    r = _run()
    assert r.returncode == 3 and "no CUDA device" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_shim_drop_in_matches_reference_cpu():
    r = _run()
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shim checks passed" in r.stdout
