"""The drop-in: tn::relax_cl (libv2m_relax_cl.so) called by the reference
pipeline's own dispatch over the reference's types (tests/dropin_driver.cpp).

CPU: without a device relax_cl throws std::runtime_error and the pipeline's
fallback (restore the seeds, relax_cpu) produces the reference result.
GPU: relax_cl runs on the device and its nodes equal relax_cpu's bit for bit;
and a failure injected on the host in the middle of a run (V2M_CUDA_FAIL_AT)
takes the pipeline's fallback with the seeds restored.
"""
import os
import subprocess

import pytest

from trussnet_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "_bin", "dropin_driver")

needs_driver = pytest.mark.skipif(not os.path.exists(DRIVER), reason="drop-in driver not built (needs the reference)")


def run(env=None, dim=40, iters=30):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([DRIVER, str(dim), str(iters)], capture_output=True, text=True, env=e, timeout=600)
    assert r.returncode == 0, r.stderr
    fields = dict(kv.split("=") for kv in r.stdout.split())
    return fields, r.stderr


@needs_driver
@pytest.mark.skipif(_lib.load().v2m_cuda_device_count() > 0, reason="a CUDA device is present")
def test_fallback_without_device():
    f, err = run()
    assert f["path"] == "cpu-fallback"
    assert "relax_cl failed" in err and "no CUDA device" in err
    assert f["identical"] == "1"


@needs_driver
@pytest.mark.gpu
def test_dropin_on_device_equals_relax_cpu():
    f, err = run()
    assert f["path"] == "cuda", err
    assert f["identical"] == "1"
    a, b = f["iters"].split("/")
    assert a == b


@needs_driver
@pytest.mark.gpu
@pytest.mark.parametrize("where", ["create", "rebuild", "iterate:10", "readback"])
def test_injected_fault_restores_seeds_and_falls_back(where):
    """A failure of the library in the middle of a run on a live device
    (V2M_CUDA_FAIL_AT: the host code fails as a CUDA call would; nothing is done
    to the GPU) reaches the pipeline's dispatch as std::runtime_error; it
    restores the seeds and runs relax_cpu, so the result equals relax_cpu's.
    At readback the positions were already written into the pipeline's nodes
    when the failure came: the restore is what makes the result right."""
    f, err = run({"V2M_CUDA_FAIL_AT": where})
    assert f["path"] == "cpu-fallback", err
    assert "injected fault at " + where.split(":")[0] in err
    assert f["identical"] == "1"
