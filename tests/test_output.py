"""Superdroplet output on the CPU: the oracle's restatement of CLEO's Zarr writing against
CLEO's own observers (SimpleDataset<FSStore>, TimeObserver >> SuperdropsObserver, compiled in
oracle/_ref), and the library's native writer (host observations) against both, byte for byte;
the numpy reader, variable subsets and the error cases.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi
from cleo_b200.output import SuperdropsZarr, attrs, read_dataset
from cleo_b200.sdm import CleoError

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import zarr_writer as ZW  # noqa: E402

needs_ref = pytest.mark.skipif(not K.ref_available(), reason="reference build absent")


def _ref_writer():
    lib = K.ref_lib()
    lib.ref_zarr_open.argtypes = [C.c_char_p, C.c_size_t, C.c_uint32, C.POINTER(C.c_void_p)]
    lib.ref_zarr_open.restype = C.c_int
    lib.ref_zarr_observe_supers.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t]
    lib.ref_zarr_observe_supers.restype = C.c_int
    lib.ref_zarr_close.argtypes = [C.c_void_p]
    lib.ref_zarr_close.restype = None
    return lib


def _sequence(seed):
    """maxchunk, interval and observations [(t_mdl, supers)] covering exact multiples of the
    chunk, one-off sizes, empty observations and skipped (off-interval) steps."""
    rng = np.random.default_rng(seed)
    maxchunk = int(rng.choice([1, 2, 3, 5, 7, 16, 1000]))
    interval = int(rng.choice([1, 2, 3]))
    obs = []
    for t in range(int(rng.integers(0, 12))):
        n = int(rng.choice([0, 1, maxchunk, max(maxchunk - 1, 0), maxchunk + 1, 2 * maxchunk,
                            int(rng.integers(0, 40))]))
        radius = np.exp(rng.normal(0, 3, n))
        sd = {"sdgbxindex": rng.integers(0, 10, n).astype(np.uint32),
              "xi": rng.integers(1, 2 ** 62, n).astype(np.uint64),
              "radius": radius, "msol": np.minimum(np.exp(rng.normal(-20, 3, n)), radius ** 3),
              "coord3": rng.random(n) * 3, "coord1": rng.random(n), "coord2": rng.random(n),
              "sdid": rng.integers(0, 2 ** 40, n).astype(np.uint64)}
        obs.append((t * int(rng.choice([1, 1, 2])), sd))
    return maxchunk, interval, obs


def _write_ref(path, maxchunk, interval, obs):
    lib = _ref_writer()
    z = C.c_void_p()
    assert lib.ref_zarr_open(os.fspath(path).encode(), maxchunk, interval, C.byref(z)) == 0
    for t, sd in obs:
        s = abi.supers_struct(sd)
        assert lib.ref_zarr_observe_supers(z, t, C.byref(s), len(sd["xi"])) == 0
    lib.ref_zarr_close(z)


def _write_oracle(path, maxchunk, interval, obs, variables=tuple(ZW.VARIABLES)):
    o = ZW.SuperdropsDataset(os.fspath(path), maxchunk, interval, variables)
    for t, sd in obs:
        o.observe(t, sd)
    o.close()


def _write_native(path, maxchunk, interval, obs, variables=None):
    with SuperdropsZarr(path, maxchunk, interval, variables) as z:
        for t, sd in obs:
            z.observe_host(t, sd)


@needs_ref
@pytest.mark.parametrize("seed", range(24))
def test_oracle_writer_matches_reference(tmp_path, seed):
    maxchunk, interval, obs = _sequence(seed)
    _write_ref(tmp_path / "ref", maxchunk, interval, obs)
    _write_oracle(tmp_path / "orc", maxchunk, interval, obs)
    a, b = ZW.tree(tmp_path / "ref"), ZW.tree(tmp_path / "orc")
    assert sorted(a) == sorted(b)
    for k in a:
        assert a[k] == b[k], k


@pytest.mark.parametrize("seed", range(24))
def test_native_writer_matches_oracle(tmp_path, seed):
    maxchunk, interval, obs = _sequence(seed)
    _write_oracle(tmp_path / "orc", maxchunk, interval, obs)
    _write_native(tmp_path / "lib", maxchunk, interval, obs)
    a, b = ZW.tree(tmp_path / "orc"), ZW.tree(tmp_path / "lib")
    assert sorted(a) == sorted(b)
    for k in a:
        assert a[k] == b[k], k


@needs_ref
def test_native_writer_matches_reference_large(tmp_path):
    """Observations large enough for the native writer's one-thread-per-array path."""
    rng = np.random.default_rng(5)
    obs = []
    for t in range(3):
        n = 1_100_000 + 77 * t
        sd = {"sdgbxindex": rng.integers(0, 5000, n).astype(np.uint32),
              "xi": rng.integers(1, 2 ** 40, n).astype(np.uint64), "radius": rng.random(n) + 0.5,
              "msol": rng.random(n) * 1e-3, "coord3": rng.random(n), "coord1": rng.random(n),
              "coord2": rng.random(n), "sdid": np.arange(n, dtype=np.uint64) * 7}
        obs.append((t, sd))
    _write_ref(tmp_path / "ref", 250_000, 1, obs)
    _write_native(tmp_path / "lib", 250_000, 1, obs)
    a, b = ZW.tree(tmp_path / "ref"), ZW.tree(tmp_path / "lib")
    assert sorted(a) == sorted(b)
    for k in a:
        assert a[k] == b[k], k


def test_reader_and_subset(tmp_path):
    maxchunk, _, obs = 4, 1, _sequence(3)[2]
    variables = ("sdId", "radius", "xi")
    _write_native(tmp_path / "ds", maxchunk, 1, obs, variables)
    _write_oracle(tmp_path / "orc", maxchunk, 1, obs, variables)
    assert ZW.tree(tmp_path / "ds") == ZW.tree(tmp_path / "orc")
    ds = read_dataset(tmp_path / "ds")
    assert set(ds) == {"time", "raggedcount", "offsets", "sdId", "radius", "xi"}
    counts = [len(sd["xi"]) for _, sd in obs]
    assert list(ds["raggedcount"]) == counts
    assert np.array_equal(ds["time"], np.array([t / 1e5 for t, _ in obs], dtype=np.float32))
    for k, (_, sd) in enumerate(obs):
        lo, hi = ds["offsets"][k], ds["offsets"][k + 1]
        assert np.array_equal(ds["radius"][lo:hi], sd["radius"].astype(np.float32))
        assert np.array_equal(ds["xi"][lo:hi], sd["xi"])
        assert np.array_equal(ds["sdId"][lo:hi], sd["sdid"].astype(np.uint32))
    a = attrs(tmp_path / "ds", "radius")
    assert a == {"_ARRAY_DIMENSIONS": ["superdroplets"], "units": "micro-m",
                 "scale_factor": 1.0, "sample_dimension": "superdroplets"}


def test_no_observations(tmp_path):
    _write_native(tmp_path / "a", 8, 1, [])
    _write_oracle(tmp_path / "b", 8, 1, [])
    assert ZW.tree(tmp_path / "a") == ZW.tree(tmp_path / "b")
    ds = read_dataset(tmp_path / "a")
    assert ds["time"].size == 0 and ds["radius"].size == 0


def test_errors(tmp_path):
    with pytest.raises(CleoError) as e:
        SuperdropsZarr(tmp_path / "x", 0)
    assert e.value.name == "CLEO_ERR_ARGUMENT"
    with pytest.raises(ValueError):
        SuperdropsZarr(tmp_path / "x", 4, variables=("mass",))
    blocker = tmp_path / "file"
    blocker.write_text("not a directory")
    with pytest.raises(CleoError) as e:
        SuperdropsZarr(blocker / "ds", 4)
    assert e.value.name == "CLEO_ERR_IO"
    # XiFunc aborts on a multiplicity of 2^64 - 1 (superdrops_observer.hpp:229-234)
    z = SuperdropsZarr(tmp_path / "xi", 4)
    n = 3
    sd = {"sdgbxindex": np.zeros(n, np.uint32), "xi": np.array([1, 2 ** 64 - 1, 3], np.uint64),
          "radius": np.ones(n), "msol": np.ones(n) * 1e-3, "coord3": np.zeros(n),
          "coord1": np.zeros(n), "coord2": np.zeros(n), "sdid": np.arange(n, dtype=np.uint64)}
    with pytest.raises(CleoError) as e:
        z.observe_host(0, sd)
    assert e.value.name == "CLEO_ERR_XI_OUTPUT"
    z.close()
