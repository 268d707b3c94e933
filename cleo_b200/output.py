"""Superdroplet output: CLEO's SuperdropsObserver + TimeObserver datasets (Zarr v2).

:class:`SuperdropsZarr` wraps the library's native writer (cleo_b200_zarr_* of
include/cleo_b200.h). At an observation the domain superdroplets are gathered and converted on
the GPU, copied once into pinned host memory and written as ragged 1-D arrays, with the files
and bytes CLEO's own observers write (observers/superdrops_observer.hpp:485-490,
observers/time_observer.hpp:141-144, zarr/simple_dataset.hpp:44-292). :func:`read_dataset` reads
such a dataset back with numpy (the reference reads it with xarray/zarr, which this package
does not need).
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import abi
from .sdm import CleoError


def _vars_mask(variables) -> int:
    if variables is None:
        return abi.OBS_ALL
    m = 0
    for v in variables:
        if v not in abi.OBS_VARS:
            raise ValueError(f"unknown superdroplet output variable {v!r}")
        m |= abi.OBS_VARS[v][0]
    return m


class SuperdropsZarr:
    """A dataset written by TimeObserver >> SuperdropsObserver(variables)."""

    def __init__(self, path, maxchunk: int, interval: int = 1, variables=None,
                 lib: C.CDLL | None = None):
        self.lib = lib if lib is not None else abi.load_library()
        self.path = os.fspath(path)
        self.variables = tuple(v for v in abi.OBS_VARS if _vars_mask(variables) & abi.OBS_VARS[v][0])
        self._z = C.c_void_p()
        rc = self.lib.cleo_b200_zarr_open(self.path.encode(), int(maxchunk), int(interval),
                                          _vars_mask(variables), C.byref(self._z))
        if rc != 0:
            raise CleoError(rc, where="in zarr_open")

    def observe(self, sdm, t_mdl: int):
        """Observation of a context's domain superdroplets at model step t_mdl."""
        rc = self.lib.cleo_b200_zarr_observe(self._z, sdm.ctx, int(t_mdl))
        if rc != 0:
            raise CleoError(rc, where="in zarr_observe")

    def observe_host(self, t_mdl: int, supers: dict):
        """Observation of host superdroplets (SoA dict of the C ABI's field names, in the order
        to write), converted to the output types as the reference's Collect* functors do."""
        n = len(supers["sdgbxindex"]) if "sdgbxindex" in supers else len(supers["radius"])
        src = {"sdId": "sdid", "sdgbxindex": "sdgbxindex", "xi": "xi", "radius": "radius",
               "msol": "msol", "coord3": "coord3", "coord1": "coord1", "coord2": "coord2"}
        arrs = {v: np.ascontiguousarray(np.asarray(supers[src[v]]).astype(abi.OBS_VARS[v][1]))
                for v in self.variables}
        o = abi.obs_struct(arrs)
        rc = self.lib.cleo_b200_zarr_observe_host(self._z, int(t_mdl), C.byref(o), n)
        if rc != 0:
            raise CleoError(rc, where="in zarr_observe_host")

    def close(self):
        if self._z:
            z, self._z = self._z, C.c_void_p()
            rc = self.lib.cleo_b200_zarr_close(z)
            if rc != 0:
                raise CleoError(rc, where="in zarr_close")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gather_supers(sdm, variables=None) -> dict:
    """The domain superdroplets of a context as output-typed host arrays (GPU gather)."""
    n = C.c_size_t()
    mask = _vars_mask(variables)
    rc = sdm.lib.cleo_b200_gather_supers(sdm.ctx, mask, C.byref(abi.ObsSupers()), 0, C.byref(n))
    if rc not in (0, abi.CODE["CLEO_ERR_CAPACITY"]):
        raise CleoError(rc, where="in gather_supers")
    cap = n.value
    arrs = {v: np.empty(max(cap, 1), dtype=dt) for v, (bit, dt) in abi.OBS_VARS.items()
            if mask & bit}
    o = abi.obs_struct(arrs)
    rc = sdm.lib.cleo_b200_gather_supers(sdm.ctx, mask, C.byref(o), cap, C.byref(n))
    if rc != 0:
        raise CleoError(rc, where="in gather_supers")
    return {v: a[:n.value] for v, a in arrs.items()}


def read_array(path, name) -> np.ndarray:
    """A 1-D array of a dataset: its chunks concatenated and cut to its shape."""
    d = os.path.join(os.fspath(path), name)
    with open(os.path.join(d, ".zarray")) as f:
        meta = json.load(f)
    (shape,), (chunk,) = meta["shape"], meta["chunks"]
    dt = np.dtype(meta["dtype"])
    out = np.empty(shape, dtype=dt)
    for c in range((shape + chunk - 1) // chunk):
        data = np.fromfile(os.path.join(d, str(c)), dtype=dt)
        lo = c * chunk
        hi = min(lo + chunk, shape)
        out[lo:hi] = data[:hi - lo]
    return out


def read_dataset(path) -> dict:
    """time, raggedcount and every superdroplet variable of a dataset, plus 'offsets' (the
    first superdroplet of each observation in the ragged arrays)."""
    path = os.fspath(path)
    out = {"time": read_array(path, "time"), "raggedcount": read_array(path, "raggedcount")}
    for v in abi.OBS_VARS:
        if os.path.isdir(os.path.join(path, v)):
            out[v] = read_array(path, v)
    out["offsets"] = np.concatenate([[0], np.cumsum(out["raggedcount"], dtype=np.int64)])
    return out


def attrs(path, name) -> dict:
    with open(os.path.join(os.fspath(path), name, ".zattrs")) as f:
        return json.load(f)


def _main(argv=None):
    """Throughput of observations of the uneven 3-D workload on the GPU:
    python -m cleo_b200.output --ndims 64 128 128 --obs 2 --dir /tmp/sdout

    Prints one JSON line: the gather kernels alone (device time, CUDA events on the context's
    stream), gather + copy to pinned host memory, and whole observations (gather, copy, files).
    """
    import argparse
    import json as _json
    import shutil
    import tempfile
    import time

    import torch

    from . import workloads as W
    from .sdm import make_sdm
    ap = argparse.ArgumentParser()
    ap.add_argument("--ndims", type=int, nargs=3, default=(64, 128, 128))
    ap.add_argument("--obs", type=int, default=2)
    ap.add_argument("--maxchunk", type=int, default=1 << 24)
    ap.add_argument("--dir", default=None)
    a = ap.parse_args(argv)
    w = W.uneven3d(ndims=tuple(a.ndims), seed=3)
    w["params"].exec_mode = abi.EXEC_BATCHED
    g = make_sdm(w, lib=abi.load_library())
    g.run_step(0, w["tstep"])
    lib = g.lib
    stream = torch.cuda.ExternalStream(lib.cleo_b200_stream(g.ctx))
    n = C.c_size_t()
    empty = abi.ObsSupers()
    lib.cleo_b200_gather_supers(g.ctx, abi.OBS_ALL, C.byref(empty), 0, C.byref(n))  # warm-up
    nsd = n.value
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kern = []
    for _ in range(5):
        e0.record(stream)
        lib.cleo_b200_gather_supers(g.ctx, abi.OBS_ALL, C.byref(empty), 0, C.byref(n))
        e1.record(stream)
        e1.synchronize()
        kern.append(e0.elapsed_time(e1))
    pinned = {v: torch.empty(nsd, dtype={np.uint32: torch.int32, np.uint64: torch.int64,
                                         np.float32: torch.float32}[dt]).pin_memory()
              for v, (_, dt) in abi.OBS_VARS.items()}
    o = abi.obs_struct({v: t.numpy().view(abi.OBS_VARS[v][1]) for v, t in pinned.items()})
    copy = []
    for _ in range(3):
        t0 = time.perf_counter()
        rc = lib.cleo_b200_gather_supers(g.ctx, abi.OBS_ALL, C.byref(o), nsd, C.byref(n))
        copy.append((time.perf_counter() - t0) * 1e3)
        assert rc == 0, rc
    root = a.dir or tempfile.mkdtemp(prefix="sdout")
    obs = []
    try:
        with SuperdropsZarr(os.path.join(root, "ds"), a.maxchunk, 1, lib=lib) as z:
            for k in range(a.obs):
                t0 = time.perf_counter()
                z.observe(g, k)
                obs.append((time.perf_counter() - t0) * 1e3)
    finally:
        shutil.rmtree(root, ignore_errors=True)
    out_bytes = 36 * nsd
    in_bytes = 60 * nsd
    print(_json.dumps({
        "superdroplets": nsd, "output_bytes_per_superdroplet": 36,
        "gather_kernels_ms": min(kern),
        "gather_kernels_GBps": (in_bytes + out_bytes) / min(kern) / 1e6,
        "gather_and_copy_ms": min(copy), "copy_GBps": out_bytes / min(copy) / 1e6,
        "observation_ms": obs, "observation_superdroplets_per_s": nsd / (min(obs) / 1e3),
        "maxchunk": a.maxchunk}))
    g.close()


if __name__ == "__main__":
    _main()
