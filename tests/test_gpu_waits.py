"""Failure detection on the GPU without a fault: the library's bounded mbarrier wait (the one its
bulk-copy staging and tensor-core kernels use) is made to run out on a barrier that nothing
completes; the kernel reports CLEO_ERR_TIMEOUT to the host and returns, and the device then runs
an ordinary SDM step that matches the oracle."""
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.sdm import make_sdm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


def test_bounded_wait_reports_timeout_and_device_stays_usable(lib):
    assert lib.cleo_b200_check_bounded_wait(1 << 12) == abi.CODE["CLEO_ERR_TIMEOUT"]
    assert lib.cleo_b200_check_bounded_wait(0) == abi.CODE["CLEO_ERR_ARGUMENT"]
    assert lib.cleo_b200_check_bounded_wait((1 << 24) + 1) == abi.CODE["CLEO_ERR_ARGUMENT"]
    w = W.uneven3d(ndims=(6, 5, 4), seed=41)
    w["params"].exec_mode = abi.EXEC_BATCHED
    g = make_sdm(w, lib=lib)
    o = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    for s in range(2):
        g.run_step(s * w["tstep"], (s + 1) * w["tstep"])
        o.run_step(s * w["tstep"], (s + 1) * w["tstep"])
    g.check()
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=1e-12, what="after")
    g.close()
