"""The condensation surrogate on the GPU: gradients of the training kernels against the FP64
numpy restatement, the tcgen05 inference against the mma.sync and FP32 check paths, training
on pairs from the solver, and the seeded solves against the CPU oracle.

Bars: gradient per parameter group within 1e-4 of the group's largest FP64 gradient (FP32
arithmetic over up to 4096 samples); inference paths within 1e-4 of the target scale of each
other (same BF16 operands, FP32 accumulation in a different order) and within 1e-2 (max) /
1e-4 (mean) of the FP64 restatement; seeded solves within 1e-12 relative of the oracle solved
from the reference guess at the same tight tolerance.
"""
import ctypes as C
import copy

import numpy as np
import pytest

import checkers as K
import mlp_numpy as M
from cleo_b200 import abi, workloads as W
from cleo_b200.config import make_params
from cleo_b200.sdm import SDM, CleoError, make_sdm
from cleo_b200.surrogate import Surrogate, condensation_solve, to_device, train_surrogate

pytestmark = pytest.mark.gpu

TIGHT = dict(maxniters=200, rtol=0.0, atol=1e-8)


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


def _solver(lib, nr_seed=abi.NRSEED_REFERENCE, **tol):
    p = make_params(condtstep=1.0, nr_seed=nr_seed, **(tol or TIGHT))
    return SDM(p, W.cartesian_grid((1, 1, 1), (1.0, 1.0, 1.0), nspacedims=0), 1, lib=lib)


@pytest.fixture(scope="module")
def trained(lib):
    solver = _solver(lib)
    sur, info = train_surrogate(solver, n_pairs=1 << 17, chunk=1 << 18, steps=3000, batch=8192,
                                lr=2e-3,
                                seed=11, lib=lib)
    yield sur, info
    sur.close()
    solver.close()


def _feats(lib, n, seed):
    import torch
    sur = Surrogate(seed=seed, lib=lib)
    dev = to_device(W.condsolve(n, seed=seed))
    f, _, _ = sur.features(dev, want_direct=False)
    t = torch.randn(n, dtype=torch.float32, device="cuda", generator=torch.Generator(
        device="cuda").manual_seed(seed))
    sur.fit_normalisation(f, t)
    return sur, f, t


def test_features_match_restatement(lib):
    import torch
    w = W.condsolve(5000, seed=3)
    sur = Surrogate(seed=1, lib=lib)
    f, _, direct = sur.features(to_device(w))
    f = f.cpu().numpy().astype(np.float64)
    akoh = 3.3e-7 / (273.15 * 1e-6) / w["temp"]
    from cleo_b200.config import MR0, Mr_sol, RHO0
    bkoh = 4.3e-6 * RHO0 / MR0 * w["msol"] * 2.0 / Mr_sol
    exp = np.stack([np.log(w["radius"]), np.log(w["msol"]), w["s_ratio"] - 1.0, w["temp"],
                    w["press"], w["delt"], np.log(3.0 * bkoh / akoh)], axis=1)
    # single-precision logarithms of single-precision arguments: a few float ulps of max(1, |x|)
    assert np.all(np.abs(f - exp) <= 1e-6 * np.maximum(1.0, np.abs(exp)))
    d = direct.cpu().numpy()
    assert set(np.unique(d)) <= {0, 1} and 0 < d.mean() < 1
    torch.cuda.synchronize()


def test_loss_grad_matches_fp64(lib):
    sur, f, t = _feats(lib, 4096, seed=5)
    p, nrm = sur.get_params()
    g, loss = sur.loss_grad(f, t)
    l64, g64 = M.loss_grad(p, nrm, f.cpu().numpy(), t.cpu().numpy())
    g = g.cpu().numpy()
    for name, (lo, hi) in M.GROUPS.items():
        scale = np.max(np.abs(g64[lo:hi]))
        err = np.max(np.abs(g[lo:hi] - g64[lo:hi]))
        assert err <= 1e-4 * scale + 1e-9, (name, err, scale)
    assert abs(float(loss.item()) - l64) <= 1e-5 * l64
    sur.close()


@pytest.mark.parametrize("n", [1, 127, 129, 100003])
def test_inference_paths_agree(lib, n):
    sur, f, _ = _feats(lib, n, seed=9)
    p, nrm = sur.get_params()
    y = {path: sur.infer(f, path).cpu().numpy().astype(np.float64)
         for path in (abi.MLP_TCGEN05, abi.MLP_MMA_SYNC, abi.MLP_FP32)}
    ref = M.infer_bf16(p, nrm, f.cpu().numpy())
    scale = float(nrm[15])
    for path, v in y.items():
        assert np.all(np.isfinite(v)), path
        assert np.max(np.abs(v - ref)) <= 1e-2 * scale, (path, np.max(np.abs(v - ref)))
        assert np.mean(np.abs(v - ref)) <= 1e-4 * scale, (path, np.mean(np.abs(v - ref)))
    for path in (abi.MLP_MMA_SYNC, abi.MLP_FP32):
        d = np.max(np.abs(y[abi.MLP_TCGEN05] - y[path]))
        assert d <= 1e-4 * scale, (path, d)
    sur.close()


def test_training_lowers_loss(trained):
    sur, info = trained
    loss = info["loss"]
    assert info["n_pairs"] == 1 << 17 and info["n_pairs"] > 0.2 * info["n_drawn"]
    assert np.all(np.isfinite(loss))
    assert loss[-100:].mean() < 0.05 * loss[:10].mean(), (loss[:10].mean(), loss[-100:].mean())


def test_seeded_solve_matches_oracle_and_saves_iterations(lib, trained):
    import torch
    sur, _ = trained
    w = W.condsolve(1 << 16, seed=78)  # a population whose solves all converge (oracle rc 0)
    dev = to_device(w)
    plain = _solver(lib)
    seeded = _solver(lib, nr_seed=abi.NRSEED_MLP)
    assert lib.cleo_b200_set_surrogate(seeded.ctx, sur.handle) == 0
    r_plain, it_plain = condensation_solve(plain, dev)
    r_seed, it_seed = condensation_solve(seeded, dev)
    _, _, direct = sur.features(dev)
    p = make_params(condtstep=1.0, **TIGHT)
    rc, r_orc, it_orc = K.condsolve(K.oracle_lib(), "oc", p, w)
    assert rc == 0
    r_plain, r_seed = r_plain.cpu().numpy(), r_seed.cpu().numpy()
    it_plain = it_plain.cpu().numpy().astype(np.int64)
    it_seed = it_seed.cpu().numpy().astype(np.int64)
    d = direct.cpu().numpy().astype(bool)
    assert K.max_rel(r_plain, r_orc) <= 1e-12
    assert np.array_equal(it_plain, it_orc.astype(np.int64))
    assert K.max_rel(r_seed, r_orc) <= 1e-12
    # the seed only enters the direct branch
    assert np.array_equal(it_seed[~d], it_plain[~d])
    assert it_seed[d].sum() < 0.6 * it_plain[d].sum(), (it_seed[d].mean(), it_plain[d].mean())
    # the oracle's seeded solve (same seeds) gives the same iterations and radii
    f, _, _ = sur.features(dev, want_direct=False)
    t = sur.infer(f).double().cpu().numpy()
    seed_r2 = w["radius"] ** 2 * np.exp(t)
    rc2, r_os, it_os = K.condsolve(K.oracle_lib(), "oc", p, w, seed_rsqrd=seed_r2)
    assert rc2 == 0 and K.max_rel(r_seed, r_os) <= 1e-12
    torch.cuda.synchronize()
    plain.close()
    seeded.close()


@pytest.mark.parametrize("ndims", [(6, 5, 4), (8, 16, 16)])
def test_sdm_seeded_batched_matches_oracle(lib, trained, ndims):
    sur, _ = trained
    w = W.uneven3d(ndims=ndims, seed=4)
    for k, v in TIGHT.items():
        setattr(w["params"], k, v)
    wg = dict(w)
    wg["params"] = copy.copy(w["params"])
    wg["params"].nr_seed = abi.NRSEED_MLP
    wg["params"].exec_mode = abi.EXEC_BATCHED
    g = make_sdm(wg, lib=lib)
    assert lib.cleo_b200_set_surrogate(g.ctx, sur.handle) == 0
    o = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    ts = w["tstep"]
    for s in range(3):
        g.run_step(s * ts, (s + 1) * ts)
        o.run_step(s * ts, (s + 1) * ts)
    g.check()
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=1e-12, what="seeded")
    _, ig = g.download_budgets()
    _, io = o.download_budgets()
    print(f"Newton iterations, seeded {int(ig.sum())} vs reference guess {int(io.sum())}")


def test_seeded_step_needs_a_surrogate(lib):
    w = W.uneven3d(ndims=(4, 4, 4), seed=1)
    w["params"].nr_seed = abi.NRSEED_MLP
    g = make_sdm(w, lib=lib)
    with pytest.raises(CleoError) as ei:
        g.run_step(0, w["tstep"])
    assert ei.value.name == "CLEO_ERR_MLP"
    w["params"].exec_mode = abi.EXEC_PLAIN
    with pytest.raises(CleoError) as ei:
        make_sdm(w, lib=lib)
    assert ei.value.name == "CLEO_ERR_ARGUMENT"
