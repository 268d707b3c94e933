"""The allocation-free gridbox sort (cleo_b200_sort_by_gridbox_static) against the context's sort.

For callers that cannot allocate device memory while they run, the library offers one sort whose
scratch lives in a static device array. As such a caller would, the checks first make the set-up
call (n = 0) that loads the array onto the device at start-up; then they call the sort through the
C ABI twice in a row, on two different populations, and compare each result bit for bit with the
order that the context's own sort (cleo_b200_upload_supers) produces for the same superdroplets;
then they check that sizes beyond the array's limit are refused. Kept in a file of its own that
pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

from cleo_b200 import abi, workloads as W
from cleo_b200.sdm import make_sdm

pytestmark = pytest.mark.gpu

LIMIT = 1 << 20


def shuffled_population(seed, ndims):
    w = W.uneven3d(ndims=ndims, seed=seed)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(len(w["supers"]["xi"]))
    sd = {k: np.ascontiguousarray(v[perm]) for k, v in w["supers"].items()}
    out = rng.random(len(perm)) < 0.03  # some superdroplets outside the domain
    sd["sdgbxindex"][out] = abi.OOB
    w["supers"] = sd
    return w


def test_static_sort_matches_context_sort_twice():
    import torch
    assert torch.cuda.is_available()
    lib = abi.load_library()
    stream = torch.cuda.current_stream()
    # start-up: the set-up call, before any other device memory of this test is taken
    assert lib.cleo_b200_sort_by_gridbox_static(None, 0, 0, None, None, None) == 0
    for call, (seed, ndims) in enumerate(((41, (8, 16, 16)), (42, (12, 20, 10)))):
        w = shuffled_population(seed, ndims)
        sd = w["supers"]
        n = len(sd["xi"])
        ngbxs = int(w["grid"]["ngbxs"])
        assert n <= LIMIT
        ctx_sort = make_sdm(w, lib=lib).download_supers()  # the context's sort
        nd = ctx_sort["n_domain"]
        gbx = torch.tensor(sd["sdgbxindex"].astype(np.int64), device="cuda").to(torch.int32)
        order = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        gstart = torch.full((ngbxs + 2,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = lib.cleo_b200_sort_by_gridbox_static(
            C.c_void_p(gbx.data_ptr()), n, ngbxs, C.c_void_p(order.data_ptr()),
            C.c_void_p(gstart.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        o = order.cpu().numpy().astype(np.int64)
        gs = gstart.cpu().numpy().astype(np.int64)
        assert np.array_equal(np.sort(o), np.arange(n)), call  # a permutation
        ids = sd["sdid"][o]
        assert np.array_equal(ids[:nd], ctx_sort["sdid"][:nd]), call  # same stable order
        assert gs[ngbxs] == nd and gs[ngbxs + 1] == n, call
        counts = np.bincount(np.minimum(sd["sdgbxindex"], ngbxs).astype(np.int64),
                             minlength=ngbxs + 1)
        assert np.array_equal(np.diff(gs), counts), call


def test_static_sort_rejects_sizes_beyond_limit():
    import torch
    lib = abi.load_library()
    gbx = torch.zeros(8, dtype=torch.int32, device="cuda")
    order = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = lib.cleo_b200_sort_by_gridbox_static(C.c_void_p(gbx.data_ptr()), LIMIT + 1, 4,
                                              C.c_void_p(order.data_ptr()), None, None)
    assert abi.STATUS[rc] == "CLEO_ERR_CAPACITY"
