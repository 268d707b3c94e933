"""Host side of the condensation surrogate (no reference counterpart).

The reference's implicit-Euler condensation solver (libs/superdrops/impliciteuler.cpp:35-54)
starts every Newton-Raphson iteration from ImplicitIterations::initialguess
(impliciteuler.cpp:156-170). This module trains a 7 -> 64 -> 64 -> 1 GELU multilayer perceptron
on pairs that the solver itself produces, on the GPU with the library's own forward/backward and
Adam kernels, and attaches it to a context so that ``nr_seed = NRSEED_MLP`` starts the Newton
iteration of the direct branch from the predicted post-step r^2. FP64 Newton polishing to the
solver's own convergence test still decides every result.

Torch tensors are only device-memory plumbing here; all arithmetic runs in libcleo_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .sdm import CleoError

FEATURES = ("log r", "log msol", "s_ratio - 1", "T", "p", "delt", "log(3 b / a)")
INPUTS = ("radius", "msol", "temp", "press", "s_ratio", "delt")


def _p(t):
    return C.c_void_p(t.data_ptr())


class Surrogate:
    """A surrogate model on the current CUDA device (cleo_b200_mlp_* of include/cleo_b200.h)."""

    def __init__(self, seed: int = 0, stream=None, lib: C.CDLL | None = None):
        import torch
        self.lib = lib if lib is not None else abi.load_library()
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        self.stream = C.c_void_p(int(stream) if not isinstance(stream, C.c_void_p)
                                 else stream.value)
        self._m = C.c_void_p()
        self._check(self.lib.cleo_b200_mlp_create(self.stream, int(seed) & (2**64 - 1),
                                                  C.byref(self._m)), "mlp_create")

    @property
    def handle(self):
        return self._m

    def _check(self, rc, where):
        if rc != 0:
            raise CleoError(rc, where=f"in {where}")

    def close(self):
        if self._m:
            self.lib.cleo_b200_mlp_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters ----
    def get_params(self):
        p = np.zeros(abi.MLP_NPARAMS, dtype=np.float32)
        nrm = np.zeros(abi.MLP_NNORM, dtype=np.float32)
        fp = C.POINTER(C.c_float)
        self._check(self.lib.cleo_b200_mlp_get_params(self._m, p.ctypes.data_as(fp),
                                                      nrm.ctypes.data_as(fp)), "mlp_get_params")
        return p, nrm

    def set_params(self, params: np.ndarray, norm: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        nrm = np.ascontiguousarray(norm, dtype=np.float32)
        assert p.size == abi.MLP_NPARAMS and nrm.size == abi.MLP_NNORM
        fp = C.POINTER(C.c_float)
        self._check(self.lib.cleo_b200_mlp_set_params(self._m, p.ctypes.data_as(fp),
                                                      nrm.ctypes.data_as(fp)), "mlp_set_params")

    # ---- data ----
    def features(self, dev: dict, radius_new=None, want_direct: bool = True):
        """Raw features (n x 7 float32), optional target log(r_new^2/r^2) and direct-branch mask."""
        import torch
        n = int(dev["radius"].numel())
        feats = torch.empty((n, abi.MLP_NFEATURES), dtype=torch.float32, device="cuda")
        tgt = torch.empty(n, dtype=torch.float32, device="cuda") if radius_new is not None else None
        direct = torch.empty(n, dtype=torch.uint8, device="cuda") if want_direct else None
        rc = self.lib.cleo_b200_mlp_features(
            self._m, n, *[_p(dev[k]) for k in INPUTS],
            _p(radius_new) if radius_new is not None else None, _p(feats),
            _p(tgt) if tgt is not None else None, _p(direct) if direct is not None else None)
        self._check(rc, "mlp_features")
        return feats, tgt, direct

    def fit_normalisation(self, feats, target):
        self._check(self.lib.cleo_b200_mlp_fit_normalisation(self._m, int(target.numel()),
                                                             _p(feats), _p(target)),
                    "mlp_fit_normalisation")

    # ---- training ----
    def loss_grad(self, feats, target):
        import torch
        g = torch.empty(abi.MLP_NPARAMS, dtype=torch.float32, device="cuda")
        loss = torch.empty(1, dtype=torch.float32, device="cuda")
        self._check(self.lib.cleo_b200_mlp_loss_grad(self._m, int(target.numel()), _p(feats),
                                                     _p(target), _p(g), _p(loss)),
                    "mlp_loss_grad")
        return g, loss

    def train(self, feats, target, steps: int, batch: int = 8192, lr: float = 2e-3,
              seed: int = 1):
        import torch
        hist = torch.empty(max(int(steps), 1), dtype=torch.float32, device="cuda")
        self._check(self.lib.cleo_b200_mlp_train(self._m, int(target.numel()), _p(feats),
                                                 _p(target), int(steps), int(batch),
                                                 float(lr), int(seed), _p(hist)), "mlp_train")
        return hist

    def infer(self, feats, path: int = abi.MLP_TCGEN05):
        import torch
        n = int(feats.shape[0])
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        self._check(self.lib.cleo_b200_mlp_infer(self._m, n, _p(feats), _p(out), int(path)),
                    "mlp_infer")
        return out


def condensation_solve(sdm, dev: dict, allow=()):
    """cleo_b200_condensation_solve on device tensors: (new radius, Newton iterations).

    A device-side failure raises CleoError unless its status name is in ``allow`` (every droplet
    is still solved; a droplet that did not converge keeps its last iterate)."""
    import torch
    n = int(dev["radius"].numel())
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    nit = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = sdm.lib.cleo_b200_condensation_solve(sdm.ctx, n, *[_p(dev[k]) for k in INPUTS],
                                              _p(out), _p(nit))
    if rc != 0:
        raise CleoError(rc, where="in condensation_solve")
    err = sdm.status()
    if err.code != 0 and abi.STATUS.get(err.code) not in allow:
        raise CleoError(err.code, err.gbxindex, err.index, where="in condensation_solve")
    return out, nit


def to_device(inputs: dict) -> dict:
    import torch
    return {k: torch.tensor(np.ascontiguousarray(inputs[k]), dtype=torch.float64, device="cuda")
            for k in INPUTS}


def train_surrogate(solver_sdm, n_pairs: int = 1 << 24, steps: int = 20000, batch: int = 8192,
                    lr: float = 2e-3, seed: int = 101, model_seed: int = 7, lib=None,
                    chunk: int = 1 << 24):
    """Train a surrogate on n_pairs pairs that ``solver_sdm``'s condensation solver generates.

    The inputs follow the independent-droplet population of ``workloads.condsolve``, drawn in
    chunks (seeds seed, seed + 1, ...) until n_pairs droplets whose solve takes the direct branch
    (the branch a seed applies to) and converges have been collected; exactly n_pairs are kept.
    Returns (surrogate, info dict with the loss history and the training-set size).
    """
    import torch
    from . import workloads as W
    sur = Surrogate(seed=model_seed, lib=lib)
    fs, ts = [], []
    have, drawn, k = 0, 0, 0
    while have < n_pairs:
        inputs = to_device(W.condsolve(chunk, seed=seed + k))
        # a rare droplet whose Newton iteration cannot meet the tolerance (the reference would
        # abort on it) is marked in the iteration counts and left out
        r_new, nit = condensation_solve(solver_sdm, inputs, allow=("CLEO_ERR_NR_NOCONVERGE",))
        feats, tgt, direct = sur.features(inputs, radius_new=r_new)
        ok = (nit.view(torch.int32) >= 0)  # the failure bit is the sign bit
        keep = direct.bool() & ok
        fs.append(feats[keep])
        ts.append(tgt[keep])
        have += int(keep.sum())
        drawn += chunk
        k += 1
        del inputs, r_new, nit, feats, tgt, direct
    feats = torch.cat(fs)[:n_pairs].contiguous()
    tgt = torch.cat(ts)[:n_pairs].contiguous()
    del fs, ts
    if solver_sdm.status().code != 0:  # the droplets left out above recorded their failure
        solver_sdm.lib.cleo_b200_clear_status(solver_sdm.ctx)
    sur.fit_normalisation(feats, tgt)
    hist = sur.train(feats, tgt, steps=steps, batch=batch, lr=lr, seed=seed)
    torch.cuda.synchronize()
    return sur, {"n_pairs": int(tgt.numel()), "n_drawn": drawn,
                 "loss": hist.cpu().numpy(), "feats": feats, "target": tgt}


def _main(argv=None):
    """Time the three inference paths on n droplets of the independent-droplet population with a
    randomly initialised surrogate: python -m cleo_b200.surrogate --infer N"""
    import argparse
    import torch
    from . import workloads as W
    ap = argparse.ArgumentParser()
    ap.add_argument("--infer", type=int, default=1 << 22)
    ap.add_argument("--repeat", type=int, default=2)
    a = ap.parse_args(argv)
    sur = Surrogate(seed=3)
    f, _, _ = sur.features(to_device(W.condsolve(a.infer, seed=5)), want_direct=False)
    sur.fit_normalisation(f, torch.randn(a.infer, device="cuda"))
    for name, path in (("tcgen05", abi.MLP_TCGEN05), ("mma_sync", abi.MLP_MMA_SYNC),
                       ("fp32", abi.MLP_FP32)):
        for _ in range(a.repeat):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            sur.infer(f, path)
            e1.record()
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        print(f"{name}: {ms:.3f} ms, {a.infer / ms / 1e6:.3f} G samples/s")
    sur.close()


if __name__ == "__main__":
    _main()
