"""CLEO's own RunCLEO with the B200 SDMMethods (include/cleo_b200_sdmmethods.hpp) on the GPU.

The harness (oracle/adapter_harness.cpp) runs RunCLEO's whole call sequence (create_supers and
create_gbxs from initial conditions, prepare_to_timestep, then start_step / coupldyn_step /
sdm_step / proceed_to_next_step: runcleo.hpp:126-175, 220-227) with prescribed coupled dynamics
that change every gridbox's temperature and vapour at every coupling step, and an observer that
records the domain superdroplets and gridbox states. With the B200 specialisation of SDMMethods:
* against the same RunCLEO with CLEO's own SDMMethods (its sources compiled here): order, gridbox
  indices, multiplicities and ids bit for bit, every double within 1e-12 relative (CLEO's host
  libm against correctly rounded pow/exp);
* with the states held fixed, against the correctly rounded oracle's stepping: every observation
  bit for bit;
* a failure of the step surfaces as the C++ exception the adapter throws.
"""
import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from test_adapter import domain_only, oracle_observations, same_observation, with_cleo_volumes

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not K.adapter_available(),
                                 reason="adapter harness absent (needs CLEO's sources to build)")]

MODES = [abi.EXEC_PLAIN, abi.EXEC_BATCHED]
MODE_IDS = ["plain", "batched"]


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_runcleo_b200_matches_runcleo_cleo(lib, mode):
    w = W.uneven3d(ndims=(8, 12, 10), seed=43)
    w["params"].exec_mode = mode
    b = K.run_cleo(w, 2000, 500, b200=1, amp=1.0)
    c = K.run_cleo(w, 2000, 500, b200=0, amp=1.0)
    assert [o[0] for o in b] == [o[0] for o in c] == [0, 500, 1000, 1500, 2000]
    for x, y in zip(b, c):
        same_observation((x[0], domain_only(x[1]), x[2]), (y[0], domain_only(y[1]), y[2]),
                         f"t={x[0]}", rtol=1e-12)
    assert b[-1][1]["n_domain"] > 0


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_runcleo_b200_is_the_oracle_bit_for_bit(lib, mode):
    w = W.uneven3d(ndims=(8, 12, 10), seed=44)
    w["params"].exec_mode = mode
    b = K.run_cleo(w, 1500, 300, b200=1)
    o = K.oracle_lib(cr=True)
    K.oracle_threads(o)
    ref = oracle_observations(o, with_cleo_volumes(w, b[0][2]), 1500, 300)
    assert [x[0] for x in b] == [x[0] for x in ref]
    for x, y in zip(b, ref):
        same_observation((x[0], domain_only(x[1]), x[2]), (y[0], domain_only(y[1]), y[2]),
                         f"t={x[0]}")


def test_runcleo_b200_reports_a_failure(lib):
    from test_oracle import _err_case
    w = _err_case({}, dict(wvel_lo=50.0, wvel_hi=50.0))
    with pytest.raises(RuntimeError, match=r"status 8 "):
        K.run_cleo(w, 300, 100, b200=1, nspacedims=1)
