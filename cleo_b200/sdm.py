"""SDMMethods-shaped host driver over the context C API.

Mirrors what RunCLEO does with SDMMethods (libs/runcleo/runcleo.hpp:304-322,
libs/runcleo/sdmmethods.hpp:244-332): create the domain, hand it the superdroplets and gridbox
states, call ``run_step(t_mdl, t_next)`` per coupling step, read the state back at observation
steps. The reference aborts on invalid physics (Kokkos::abort); here a non-zero status raises
:class:`CleoError` carrying the reference abort site's code.

By default the context is the CUDA library (``libcleo_b200.so``). Any library exposing the same
context API under another prefix can be passed in (the tests use this for the CPU checkers).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class CleoError(RuntimeError):
    def __init__(self, code: int, gbxindex: int = abi.OOB, index: int = 0, where: str = ""):
        self.code = int(code)
        self.name = abi.STATUS.get(self.code, f"code {self.code}")
        self.gbxindex = int(gbxindex)
        self.index = int(index)
        super().__init__(f"{self.name} (gridbox {self.gbxindex}, superdroplet {self.index}) {where}")


class SDM:
    """One domain: superdroplets, gridbox states and maps on one device (or CPU checker)."""

    def __init__(self, params: abi.Params, grid: dict, capacity: int, lib: C.CDLL | None = None,
                 prefix: str = "cleo_b200"):
        self.lib = lib if lib is not None else abi.load_library()
        self.prefix = prefix
        self.params = params
        self.grid = grid
        self.capacity = int(capacity)
        self.ngbxs = int(grid["ngbxs"])
        self._grid_struct = abi.grid_struct(grid)
        self._ctx = C.c_void_p()
        rc = self._f("create")(C.byref(params), C.byref(self._grid_struct), self.capacity,
                               C.byref(self._ctx))
        if rc != 0:
            raise CleoError(rc, where="in create")

    def _f(self, name):
        return getattr(self.lib, f"{self.prefix}_{name}")

    @property
    def ctx(self):
        return self._ctx

    def close(self):
        if self._ctx:
            self._f("destroy")(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, where):
        if rc != 0:
            err = abi.Error()
            self._f("status")(self._ctx, C.byref(err))
            code = err.code if err.code != 0 else rc
            raise CleoError(code, err.gbxindex, err.index, where)

    def upload_supers(self, sd: dict):
        arrs = {name: np.ascontiguousarray(sd[name], dtype=dt) for name, dt in abi.SUPERS_FIELDS}
        n = int(arrs["xi"].shape[0])
        s = abi.supers_struct(arrs)
        self._check(self._f("upload_supers")(self._ctx, C.byref(s), n), "in upload_supers")
        self.n_total = n

    def upload_state(self, st: dict):
        arrs = {f: np.ascontiguousarray(st[f], dtype=np.float64) for f in abi.STATE_FIELDS}
        s = abi.state_struct(arrs)
        self._check(self._f("upload_state")(self._ctx, C.byref(s)), "in upload_state")

    def upload_state_async(self, st: dict):
        """cleo_b200_upload_state_async: the states are taken by the next run_step (the arrays
        are kept alive until then)."""
        arrs = {f: np.ascontiguousarray(st[f], dtype=np.float64) for f in abi.STATE_FIELDS}
        s = abi.state_struct(arrs)
        self._check(self._f("upload_state_async")(self._ctx, C.byref(s)),
                    "in upload_state_async")
        self._staged = arrs

    def download_budgets_async(self, cond_mass: np.ndarray, nr_iters: np.ndarray):
        """Enqueue the budgets' copy into the given arrays (float64 and uint64 of ngbxs); they
        hold the values after synchronize()."""
        assert cond_mass.dtype == np.float64 and nr_iters.dtype == np.uint64
        self._check(self._f("download_budgets_async")(
            self._ctx, C.c_void_p(cond_mass.ctypes.data), C.c_void_p(nr_iters.ctypes.data)),
            "in download_budgets_async")

    def synchronize(self):
        self._check(self._f("synchronize")(self._ctx), "in synchronize")

    def run_step(self, t_mdl: int, t_next: int):
        """SDMMethods::run_step(t_mdl, t_next): enqueue one coupling step."""
        self._check(self._f("step")(self._ctx, int(t_mdl), int(t_next)), "in step")

    def status(self) -> abi.Error:
        err = abi.Error()
        self._f("status")(self._ctx, C.byref(err))
        return err

    def check(self):
        err = self.status()
        if err.code != 0:
            raise CleoError(err.code, err.gbxindex, err.index, "after step")

    def download_supers(self) -> dict:
        out = {name: np.zeros(self.capacity, dtype=dt) for name, dt in abi.SUPERS_FIELDS}
        s = abi.supers_struct(out)
        nd, nt = C.c_size_t(), C.c_size_t()
        self._check(self._f("download_supers")(self._ctx, C.byref(s), C.byref(nd), C.byref(nt)),
                    "in download_supers")
        res = {k: v[: nt.value] for k, v in out.items()}
        res["n_domain"] = nd.value
        res["n_total"] = nt.value
        return res

    def download_state(self) -> dict:
        out = {f: np.zeros(self.ngbxs, dtype=np.float64) for f in abi.STATE_FIELDS}
        s = abi.state_struct(out)
        self._check(self._f("download_state")(self._ctx, C.byref(s)), "in download_state")
        return out

    def download_budgets(self):
        cm = np.zeros(self.ngbxs, dtype=np.float64)
        it = np.zeros(self.ngbxs, dtype=np.uint64)
        self._check(self._f("download_budgets")(self._ctx, abi.ptr(cm, C.c_double),
                                                abi.ptr(it, C.c_uint64)), "in download_budgets")
        return cm, it

    def monitors_begin(self):
        """before_timestepping of the SDMMonitor members selected by params.monitors."""
        self._check(self._f("monitors_begin")(self._ctx), "in monitors_begin")

    def download_monitors(self, reset: bool = False) -> dict:
        """Accumulated mass-moment changes (micro/motion, all/rain) and precipitation."""
        out = {name: np.zeros(self.ngbxs, dtype=dt) for name, dt in abi.MONITOR_FIELDS}
        m = abi.monitors_struct(out)
        self._check(self._f("download_monitors")(self._ctx, C.byref(m), int(bool(reset))),
                    "in download_monitors")
        return out


def make_sdm(workload: dict, lib=None, prefix="cleo_b200", params=None) -> SDM:
    """Create, upload supers and states of a workload dict (see :mod:`cleo_b200.workloads`)."""
    p = params if params is not None else workload["params"]
    sdm = SDM(p, workload["grid"], len(workload["supers"]["xi"]), lib=lib, prefix=prefix)
    sdm.upload_state(workload["state"])
    sdm.upload_supers(workload["supers"])
    return sdm


def _main(argv=None):
    """Run SDM steps of a synthetic workload on the GPU and print the per-stage CUDA-event times
    of the last step:  python -m cleo_b200.sdm --workload uneven3d --ndims 32 64 64 --steps 4

    Every step is complete (motion, re-sort, condensation, collisions); nothing is skipped.
    """
    import argparse
    import json

    from . import workloads as W
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="uneven3d",
                    choices=["uneven3d", "bubble3d", "rainshaft", "box"],
                    help="rainshaft: the 1x1x256 column of 256 superdroplets per gridbox; box: "
                         "the Golovin box model of 8192 superdroplets (--ndims ignored)")
    ap.add_argument("--ndims", type=int, nargs=3, default=(32, 64, 64))
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--plain", action="store_true", help="the plain schedule (default batched)")
    ap.add_argument("--launch-config", type=int, nargs=4, default=None,
                    help="pass-A block, pass-A CTAs per SM, warp-kernel gridbox limit, "
                         "CTAs per SM of the warp kernel's 64-slot variant "
                         "(cleo_b200_set_launch_config)")
    a = ap.parse_args(argv)
    if a.workload == "rainshaft":
        w = W.rainshaft()
    elif a.workload == "box":
        w = W.box_golovin()
    else:
        build = W.uneven3d if a.workload == "uneven3d" else W.bubble3d
        w = build(ndims=tuple(a.ndims))
    w["params"].exec_mode = abi.EXEC_PLAIN if a.plain else abi.EXEC_BATCHED
    g = make_sdm(w)
    if a.launch_config is not None:
        cfg = (C.c_int32 * 4)(*a.launch_config)
        g._check(g.lib.cleo_b200_set_launch_config(g.ctx, cfg), "in set_launch_config")
    ts = w["tstep"]
    for s in range(a.steps - 1):
        g.run_step(s * ts, (s + 1) * ts)
    lib = g.lib
    lib.cleo_b200_set_profiling(g.ctx, 1)
    g.run_step((a.steps - 1) * ts, a.steps * ts)
    g.check()
    ms = (C.c_double * 8)()
    cnt = (C.c_uint64 * 8)()
    lib.cleo_b200_stage_times(g.ctx, ms, cnt)
    names = ("motion", "sort", "microphysics", "condensation", "collisions")
    print(json.dumps({"workload": a.workload, "ndims": list(a.ndims),
                      "superdroplets": int(g.download_supers()["n_domain"]),
                      "stages_ms": {n: ms[k] for k, n in enumerate(names)}}))
    g.close()


if __name__ == "__main__":
    _main()
