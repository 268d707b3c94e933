"""Writes small CLEO binary input files with the reference's own writer (cleopy/writebinary.py,
loaded from the CLEO sources) in the layouts of cleopy's create_gbxboundaries.py (gridbox
bounds), create_initsuperdrops.py (superdroplets) and create_thermodynamics.py (one variable
per coupled-dynamics file, all time steps in a row; winds on the gridbox faces), and saves the
arrays that went into them to binaries.npz. The readers of cleo_b200/binaryio.py are checked
against these files (and, where the reference build exists, against CLEO's C++ readers).

    python tests/golden/make_binaries.py [/path/to/CLEO]
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# CLEO's sources: the first argument, else $CLEO_SRC, else a checkout named "reference" beside
# this repository
CLEO = (sys.argv[1] if len(sys.argv) > 1 else
        os.environ.get("CLEO_SRC", os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(
            os.path.abspath(__file__)))), "..", "reference")))
COORD0 = 1000.0
R0 = 1e-6
MASS0 = R0 ** 3 * (100000.0 / (1004.64 * 273.15))
NDIMS = (4, 3, 2)  # nz, nx, ny
NSTEPS = 3


def load_writer():
    spec = importlib.util.spec_from_file_location(
        "writebinary", os.path.join(CLEO, "cleopy", "writebinary.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.writebinary


def typed(a, t):
    return [t(v) for v in np.asarray(a).ravel()]


def main():
    writebinary = load_writer()
    nz, nx, ny = NDIMS
    ng = nz * nx * ny
    zedges = np.array([0.0, 20.0, 45.0, 75.0, 110.0]) / COORD0  # uneven z spacing
    xedges = np.array([0.0, 30.0, 60.0, 90.0]) / COORD0
    yedges = np.array([0.0, 25.0, 50.0]) / COORD0
    idx = np.arange(ng)
    iz, ix, iy = idx % nz, (idx // nz) % nx, idx // (nz * nx)
    bounds = np.stack([zedges[iz], zedges[iz + 1], xedges[ix], xedges[ix + 1], yedges[iy],
                       yedges[iy + 1]], axis=1)
    grid = os.path.join(HERE, "dimlessGBxboundaries.dat")
    ndims = np.array([nz, nx, ny], dtype=np.uint64)
    data = typed(ndims, np.uint) + typed(idx, np.uintc) + typed(bounds, np.double)
    writebinary(grid, data, [3, ng, 6 * ng], [np.uint, np.uintc, np.double],
                [b" ", b" ", b"m"], np.array([1.0, 1.0, COORD0]), "gridbox boundaries")

    rng = np.random.default_rng(42)
    nsd = 60
    gbx = rng.integers(0, ng, nsd).astype(np.uint32)
    xi = rng.integers(1, 10 ** 9, nsd).astype(np.uint64)
    radius = np.exp(rng.uniform(np.log(0.05), np.log(80.0), nsd))
    msol = np.exp(rng.uniform(np.log(1e-6), np.log(1e-3), nsd))
    b = bounds[gbx]
    coord3 = b[:, 0] + rng.uniform(0.05, 0.95, nsd) * (b[:, 1] - b[:, 0])
    coord1 = b[:, 2] + rng.uniform(0.05, 0.95, nsd) * (b[:, 3] - b[:, 2])
    coord2 = b[:, 4] + rng.uniform(0.05, 0.95, nsd) * (b[:, 5] - b[:, 4])
    sup = os.path.join(HERE, "dimlessSDsinit.dat")
    data = (typed(gbx, np.uintc) + typed(xi, np.uint) + typed(radius, np.double) +
            typed(msol, np.double) + typed(coord3, np.double) + typed(coord1, np.double) +
            typed(coord2, np.double))
    writebinary(sup, data, [nsd] * 7, [np.uintc, np.uint] + [np.double] * 5,
                [b" ", b" ", b"m", b"g", b"m", b"m", b"m"],
                np.array([1.0, 1.0, R0, MASS0, COORD0, COORD0, COORD0]),
                "Variables in this file are Superdroplet attributes:"
                " [sdgbxindex, xi, radius, msol, coord3, coord1, coord2]")

    dyn = {}
    sizes = {"press": ng, "temp": ng, "qvap": ng, "qcond": ng, "wvel": (nz + 1) * nx * ny,
             "uvel": nz * (nx + 1) * ny, "vvel": nz * nx * (ny + 1)}
    lo_hi = {"press": (0.7, 1.0), "temp": (1.0, 1.1), "qvap": (0.005, 0.015),
             "qcond": (0.0, 0.001), "wvel": (-0.002, 0.002), "uvel": (-0.003, 0.003),
             "vvel": (-0.001, 0.001)}
    for name, n in sizes.items():
        lo, hi = lo_hi[name]
        v = rng.uniform(lo, hi, n * NSTEPS)
        dyn[name] = v
        writebinary(os.path.join(HERE, f"dimless_{name}.dat"), typed(v, np.double),
                    [n * NSTEPS], [np.double], [b" "], np.array([1.0]), name)
    np.savez(os.path.join(HERE, "binaries.npz"), ndims=ndims, bounds=bounds, gbx=gbx, xi=xi,
             radius=radius, msol=msol, coord3=coord3, coord1=coord1, coord2=coord2,
             nsteps=NSTEPS, **{f"dyn_{k}": v for k, v in dyn.items()})


if __name__ == "__main__":
    main()
