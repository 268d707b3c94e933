"""CLEO's binary input files, read straight into the structure-of-arrays the C ABI takes.

* Layout (libs/initialise/readbinary.{hpp,cpp}; written by cleopy/writebinary.py): four
  little-endian u32 [first data byte, global metadata string bytes, number of variables, bytes
  of metadata per variable], the global metadata string, then per variable 3 x u32 [first
  byte, bytes per datapoint, number of datapoints], 2 chars [type, units] and an f64 scale
  factor, then the data.
* Gridbox boundaries (GbxBoundsFromBinary, gbx_bounds_from_binary.cpp:24-215): variables
  ndims (u64 x 3: nz, nx, ny), gbxidxs (u32), gbxbounds (f64, 6 per gridbox: coord3 {lower,
  upper}, coord1 {..}, coord2 {..}); area = dx dy, volume = dz dx dy.
* Superdroplets (InitAllSupersFromBinary::read_initdata_binary,
  init_all_supers_from_binary.cpp:60-75): sdgbxindex (u32), xi (u64), radius, msol, coord3,
  coord1, coord2 (f64); absent coordinates read as 0.
* Coupled dynamics from files (CartesianDynamics, fromfile_cartesian_dynamics.cpp): one f64
  variable per file, all time steps in a row; press, temp, qvap, qcond at gridbox centres, wvel
  on coord3 faces ((nz+1) nx ny per step), uvel on coord1 faces (nz (nx+1) ny), vvel on coord2
  faces (nz nx (ny+1)); a gridbox's {lower, upper} face values as get_wvel / get_uvel / get_vvel
  index them; FromFileComms::update_gridbox_state (fromfilecomms.cpp:40-52) copies them into the
  gridbox state every coupling step.

All values stay in CLEO's dimensionless units (the files' scale factors re-dimensionalise).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .config import LLIM, ULIM, _finite_nghbrs, _periodic_nghbrs


@dataclass
class VarMeta:
    b0: int        # first byte of the variable's data
    bsize: int     # bytes per datapoint
    nvar: int      # number of datapoints
    vtype: bytes   # struct type character
    units: bytes
    scale_factor: float


def read_binary(path) -> tuple[str, list[VarMeta], bytes]:
    """Global metadata string, per-variable metadata and the raw file (readbinary.cpp:27-103)."""
    raw = Path(path).read_bytes()
    if len(raw) < 16:
        raise ValueError(f"{path}: not a CLEO binary file")
    d0byte, charbytes, nvars, mbytes = struct.unpack_from("<4I", raw, 0)
    metastr = raw[16:16 + charbytes].decode("latin-1")
    metas = []
    pos = 16 + charbytes
    for _ in range(nvars):
        b0, bsize, nvar = struct.unpack_from("<3I", raw, pos)
        vtype, units = raw[pos + 12:pos + 13], raw[pos + 13:pos + 14]
        (scale,) = struct.unpack_from("<d", raw, pos + 14)
        metas.append(VarMeta(b0, bsize, nvar, vtype, units, scale))
        pos += mbytes
    return metastr, metas, raw


def var_from_binary(raw: bytes, meta: VarMeta, dtype) -> np.ndarray:
    """vector_from_binary (readbinary.hpp:83-90)."""
    dt = np.dtype(dtype).newbyteorder("<")
    return np.frombuffer(raw, dtype=dt, count=meta.nvar, offset=meta.b0).astype(dtype)


def gridfile(path, nspacedims: int) -> dict:
    """Maps of an undecomposed Cartesian domain from a gridbox-boundaries file, in the form
    config.cartesian_grid returns (plus 'volume', the per-gridbox volume)."""
    _, meta, raw = read_binary(path)
    ndims = var_from_binary(raw, meta[0], np.uint64)
    idxs = var_from_binary(raw, meta[1], np.uint32)
    bounds = var_from_binary(raw, meta[2], np.float64)
    nz, nx, ny = (int(v) for v in ndims)
    ngbxs = nz * nx * ny
    if bounds.size != 6 * idxs.size or idxs.size != ngbxs:
        raise ValueError(f"{path}: gridbox indices and bounds are not consistent")
    b = np.empty((ngbxs, 6))
    b[idxs] = bounds.reshape(-1, 6)  # get_coordXgbxbounds looks gridboxes up by index
    g = {"ngbxs": ngbxs, "ndims": (nz, nx, ny)}
    for k, name in enumerate(("coord3", "coord1", "coord2")):
        if nspacedims > k:
            g[name + "lo"] = np.ascontiguousarray(b[:, 2 * k])
            g[name + "hi"] = np.ascontiguousarray(b[:, 2 * k + 1])
        else:  # unused direction: null bounds (createcartesianmaps.cpp:38-45)
            g[name + "lo"] = np.full(ngbxs, LLIM)
            g[name + "hi"] = np.full(ngbxs, ULIM)
    idx = np.arange(ngbxs, dtype=np.uint64)
    selfn = idx.astype(np.uint32)
    g["back3"], g["fwd3"] = _finite_nghbrs(idx, 1, nz) if nspacedims >= 1 else (selfn, selfn)
    g["back1"], g["fwd1"] = (_periodic_nghbrs(idx, nz, nx) if nspacedims >= 2
                             else (selfn.copy(), selfn.copy()))
    g["back2"], g["fwd2"] = (_periodic_nghbrs(idx, nz * nx, ny) if nspacedims >= 3
                             else (selfn.copy(), selfn.copy()))
    for k in ("back3", "fwd3", "back1", "fwd1", "back2", "fwd2"):
        g[k] = np.ascontiguousarray(g[k], dtype=np.uint32)
    dz, dx, dy = b[:, 1] - b[:, 0], b[:, 3] - b[:, 2], b[:, 5] - b[:, 4]
    g["gbxarea"] = np.ascontiguousarray(dx * dy)
    g["volume"] = np.ascontiguousarray(dz * dx * dy)
    return g


def initsupers(path, nspacedims: int, maxnsupers: int | None = None) -> dict:
    """Superdroplets of an initialisation file, as the supers dict of the C ABI (sdid = 0, 1, ...,
    as Superdrop::IDType::Gen hands them out)."""
    _, meta, raw = read_binary(path)
    n = meta[0].nvar
    if maxnsupers is not None and maxnsupers < n:
        raise ValueError(f"fewer superdroplets ({maxnsupers}) than the file holds ({n})")
    sd = {"sdgbxindex": var_from_binary(raw, meta[0], np.uint32),
          "xi": var_from_binary(raw, meta[1], np.uint64),
          "radius": var_from_binary(raw, meta[2], np.float64),
          "msol": var_from_binary(raw, meta[3], np.float64)}
    for k, name in enumerate(("coord3", "coord1", "coord2")):
        sd[name] = (var_from_binary(raw, meta[4 + k], np.float64)
                    if len(meta) > 4 + k and nspacedims > k else np.zeros(n))
    sd["sdid"] = np.arange(n, dtype=np.uint64)
    for v in sd.values():
        if v.size != n:
            raise ValueError(f"{path}: superdroplet attributes of different lengths")
    return sd


class FromFileDynamics:
    """Thermodynamics and winds for every coupling step from CLEO's per-variable files."""

    FIELDS = ("press", "temp", "qvap", "qcond", "wvel", "uvel", "vvel")

    def __init__(self, paths: dict, ndims, nspacedims: int, nsteps: int):
        self.nz, self.nx, self.ny = (int(v) for v in ndims)
        self.nspacedims = int(nspacedims)
        self.data = {}
        for f in self.FIELDS[:4]:
            _, meta, raw = read_binary(paths[f])
            self.data[f] = var_from_binary(raw, meta[0], np.float64)
        winds = {1: ("wvel",), 2: ("wvel", "uvel"), 3: ("wvel", "uvel", "vvel")}.get(
            self.nspacedims, ())
        for f in winds:
            _, meta, raw = read_binary(paths[f])
            self.data[f] = var_from_binary(raw, meta[0], np.float64)
        ng = self.nz * self.nx * self.ny
        for f in self.FIELDS[:4]:
            if self.data[f].size < ng * nsteps:
                raise ValueError(f"{f}: fewer values than {nsteps} steps of {ng} gridboxes")
        self.step = 0

    def state(self, volume) -> dict:
        """Gridbox states of the current step, in the state dict of the C ABI."""
        nz, nx, ny = self.nz, self.nx, self.ny
        ng = nz * nx * ny
        ii = np.arange(ng)
        k, i, j = ii % nz, (ii // nz) % nx, ii // (nz * nx)  # kijfromindex
        st = {"volume": np.ascontiguousarray(volume, dtype=np.float64)}
        pos = self.step * ng
        for f in self.FIELDS[:4]:
            st[f] = np.ascontiguousarray(self.data[f][pos:pos + ng])
        zero = np.zeros(ng)
        st["wvel_lo"], st["wvel_hi"] = zero, zero.copy()
        st["uvel_lo"], st["uvel_hi"] = zero.copy(), zero.copy()
        st["vvel_lo"], st["vvel_hi"] = zero.copy(), zero.copy()
        if "wvel" in self.data:  # get_wvel_from_binary
            p = self.step * (nz + 1) * nx * ny + nx * (nz + 1) * j + (nz + 1) * i + k
            st["wvel_lo"], st["wvel_hi"] = self.data["wvel"][p], self.data["wvel"][p + 1]
        if "uvel" in self.data:  # get_uvel_from_binary
            p = self.step * nz * (nx + 1) * ny + (nx + 1) * nz * j + nz * i + k
            st["uvel_lo"], st["uvel_hi"] = self.data["uvel"][p], self.data["uvel"][p + nz]
        if "vvel" in self.data:  # get_vvel_from_binary
            p = self.step * nz * nx * (ny + 1) + ii
            st["vvel_lo"], st["vvel_hi"] = self.data["vvel"][p], self.data["vvel"][p + nx * nz]
        return {key: np.ascontiguousarray(v, dtype=np.float64) for key, v in st.items()}

    def advance(self):
        """CartesianDynamics::increment_position (one coupling step)."""
        self.step += 1
