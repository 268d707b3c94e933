"""CPU restatement of CLEO's superdroplet output path (TEST INFRASTRUCTURE ONLY).

Only the tests use this module: it checks the library's native Zarr writer and its GPU gather.
It restates, in numpy, what CLEO's SuperdropsObserver and TimeObserver write into a
SimpleDataset<FSStore>, file by file:

* dataset: ``.zgroup`` (ZarrGroup, zarr/zarr_group.hpp:49-53) and ``.zattrs``
  (SimpleDataset ctor, zarr/simple_dataset.hpp:68-73);
* one 1-D Zarr v2 array per variable (ZarrArray, zarr/zarr_array.hpp:82-346): a host buffer of
  ``maxchunk`` elements, reset to the type's maximum (zarr/buffer.hpp:57-66), filled by each
  write; whole chunks are stored under ``<name>/<chunk number>`` (zarr/chunks.hpp:88-106,
  193-215); a full buffer is stored at the start of the next write (zarr_array.hpp:146-162) and a
  partly filled one, padding included, when the array is finished (zarr_array.hpp:207-216);
* ``.zarray`` metadata (zarr/zarr_metadata.cpp:32-81) and ``.zattrs`` metadata
  (zarr/xarray_metadata.cpp:35-170; scale factors printed as std::scientific with 6 digits);
  the last ``.zarray`` write, when an array is destroyed (xarray_zarr_array.hpp:139-143), holds
  its final shape: the number of observations for "time" and "raggedcount", the number of
  elements written for a ragged superdroplet array (set_ragged_arrayshape,
  xarray_zarr_array.hpp:91-98);
* the observation (ParallelWriteSupers::operator(), observers/parallel_write_data.hpp:240-246):
  the domain superdroplets' variables as 4-byte unsigned (sdgbxindex, sdId), 8-byte unsigned (xi)
  and 4-byte float (radius, msol, coord3, coord1, coord2) values (superdrops_observer.hpp:139-464),
  then their count in "raggedcount" (RaggedCount, superdrops_observer.hpp:48-96); "time" holds
  float(step2dimlesstime(t_mdl)) (time_observer.hpp:57-64, initialise/timesteps.hpp:56-59) and
  is written before the superdroplets (TimeObserver >> SuperdropsObserver).
"""
from __future__ import annotations

import os

import numpy as np

TIME0 = 1000.0
COORD0 = TIME0 * 1.0
R0 = 1e-6
P0, TEMP0, CP0 = 100000.0, 273.15, 1004.64
RHO0 = P0 / (CP0 * TEMP0)
MASS0grams = R0 * R0 * R0 * RHO0 * 1000

# name: (dtype, units, scale factor or None for integers)   (superdrops_observer.hpp:163-470)
VARIABLES = {
    "sdId": ("<u4", "", None),
    "sdgbxindex": ("<u4", "", None),
    "xi": ("<u8", "", None),
    "radius": ("<f4", "micro-m", R0 * 1e6),
    "msol": ("<f4", "g", MASS0grams),
    "coord3": ("<f4", "m", COORD0),
    "coord1": ("<f4", "m", COORD0),
    "coord2": ("<f4", "m", COORD0),
}
# the SoA field each variable is collected from
SOURCE = {"sdId": "sdid", "sdgbxindex": "sdgbxindex", "xi": "xi", "radius": "radius",
          "msol": "msol", "coord3": "coord3", "coord1": "coord1", "coord2": "coord2"}

ZGROUP = '{\n  "zarr_format": 2\n}'
DATASET_ZATTRS = ('{\n  "creator": "Clara Bayley",\n  "title": "Dataset from CLEO is Xarray and '
                  'NetCDF compatible Zarr Group of Arrays"\n}')


def _write(path: str, data: bytes):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "wb") as f:
        f.write(data)


def zarray_json(shape: int, chunk: int, dtype: str) -> str:
    return ('{\n  "shape": [%d],\n  "chunks": [%d],\n  "dtype": "%s",\n  "order": "C",\n'
            '  "compressor": null,\n  "fill_value": null,\n  "filters": null,\n'
            '  "zarr_format": 2\n}' % (shape, chunk, dtype))


def zattrs_json(dim: str, units: str, scale, sampledim: str | None) -> str:
    s = '{\n  "_ARRAY_DIMENSIONS": ["%s"],\n  "units": "%s"' % (dim, units)
    if scale is not None:
        s += ',\n  "scale_factor": %.6e' % scale
    if sampledim is not None:
        s += ',\n  "sample_dimension": "%s"' % sampledim
    return s + "\n}"


class Array1D:
    """ZarrArray + XarrayZarrArray of one dimension."""

    def __init__(self, root, name, dtype, chunk, dim, units, scale, sampledim):
        self.root, self.name, self.dtype, self.chunk = root, name, np.dtype(dtype), chunk
        self.nchunks = 0
        self.buf = None
        self._reset()
        _write(self._p(".zarray"), zarray_json(0, chunk, dtype).encode())
        _write(self._p(".zattrs"), zattrs_json(dim, units, scale, sampledim).encode())

    def _p(self, key):
        return os.path.join(self.root, self.name, key)

    def _reset(self):
        if self.dtype.kind == "f":
            mx = np.finfo(self.dtype).max
        else:
            mx = np.iinfo(self.dtype).max
        self.buf = np.full(self.chunk, mx, dtype=self.dtype)
        self.fill = 0

    def _store(self, data):
        _write(self._p(str(self.nchunks)), np.ascontiguousarray(data, dtype=self.dtype).tobytes())
        self.nchunks += 1

    def append(self, data):
        data = np.asarray(data, dtype=self.dtype).ravel()
        k = min(self.chunk - self.fill, data.size)
        self.buf[self.fill:self.fill + k] = data[:k]
        self.fill += k
        rest = data[k:]
        if self.fill == self.chunk:  # a full buffer is stored before the rest of the data
            self._store(self.buf)
            self._reset()
        nwhole = rest.size // self.chunk
        for c in range(nwhole):
            self._store(rest[c * self.chunk:(c + 1) * self.chunk])
        tail = rest[nwhole * self.chunk:]
        if tail.size:  # the buffer was stored and reset above
            self.buf[:tail.size] = tail
            self.fill = tail.size

    def append_one(self, value):
        if self.fill == self.chunk:
            self._store(self.buf)
            self._reset()
        self.buf[self.fill] = value
        self.fill += 1

    def total(self):
        return self.nchunks * self.chunk + self.fill

    def finish(self, shape):
        _write(self._p(".zarray"), zarray_json(shape, self.chunk, self.dtype.str).encode())
        if self.fill > 0:
            self._store(self.buf)


class SuperdropsDataset:
    """A dataset written by TimeObserver >> SuperdropsObserver(variables)."""

    def __init__(self, root, maxchunk, interval, variables=tuple(VARIABLES)):
        self.root, self.interval = root, int(interval)
        _write(os.path.join(root, ".zgroup"), ZGROUP.encode())
        _write(os.path.join(root, ".zattrs"), DATASET_ZATTRS.encode())
        self.time = Array1D(root, "time", "<f4", maxchunk, "time", "s", TIME0, None)
        self.ntimes = 0
        self.vars = {}
        for name in VARIABLES:  # the examples' order of creation does not change any file
            if name in variables:
                dt, units, scale = VARIABLES[name]
                self.vars[name] = Array1D(root, name, dt, maxchunk, "superdroplets", units,
                                          scale, "superdroplets")
        self.count = Array1D(root, "raggedcount", "<u4", maxchunk, "time", "", None,
                             "superdroplets")

    def observe(self, t_mdl: int, supers: dict):
        """at_start_step with the domain superdroplets (SoA dict of the C ABI's fields)."""
        if t_mdl % self.interval != 0:
            return
        self.ntimes += 1
        self.time.append_one(np.float32(np.float64(t_mdl) / 100000.0))
        n = len(supers["sdgbxindex"])
        if "xi" in self.vars and n and np.any(np.asarray(supers["xi"], np.uint64)
                                              == np.iinfo(np.uint64).max):
            raise OverflowError("superdroplet multiplicity too large")
        for name, arr in self.vars.items():
            src = np.asarray(supers[SOURCE[name]])
            arr.append(src.astype(arr.dtype))  # static_cast: truncation / round to nearest
        self.count.append_one(np.uint32(n))

    def close(self):
        self.time.finish(self.ntimes)
        for arr in self.vars.values():
            arr.finish(arr.total())
        self.count.finish(self.ntimes)


def tree(root) -> dict:
    """{relative path: bytes} of every file under root."""
    out = {}
    for d, _, files in os.walk(root):
        for f in files:
            p = os.path.join(d, f)
            with open(p, "rb") as fh:
                out[os.path.relpath(p, root)] = fh.read()
    return out
