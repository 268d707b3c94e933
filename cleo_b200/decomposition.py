"""Domain decomposition of the SDM step over ranks: the host logic of a multi-GPU run in which
each rank (one process per GPU) owns a slab of gridboxes and the superdroplets in it.

The reference decomposes its domain over MPI ranks (libs/cartesiandomain/cartesian_decomposition.hpp:40-140)
and, after every motion step, sends each superdroplet that moved into another rank's gridboxes to
that rank (CartesianTransportAcrossDomain, libs/cartesiandomain/movement/
cartesian_transport_across_domain.hpp:66-239: per-peer counts with MPI_Alltoall, then the
superdroplets' fields with MPI_Isend/Irecv, then the local sort). Here:

* a rank owns a contiguous range of gridbox indexes, whole rows of constant coord2 index (the
  index is iz + nz (ix + nx iy), doubly_periodic_domain.hpp:41-70, so rows of iy are contiguous);
* every rank holds the whole grid (bounds, neighbours, face winds and thermodynamic state are per
  gridbox and small) and steps only its own superdroplets: motion moves them over the whole grid,
  then the emigrants — superdroplets now in another rank's gridboxes — are packed into one array
  per destination and exchanged (counts first, then the records, over the process group; NCCL
  over NVLink between GPUs, gloo on CPU), and the microphysics runs on the rank's gridboxes;
* the received superdroplets are placed so that the rank's next sort gives exactly the order of
  the single-domain run: a rank's superdroplets sit at lower positions of the global array than
  every higher rank's, so immigrants from lower ranks go before the rank's own superdroplets and
  immigrants from higher ranks after them, each group in its source order; a stable sort by
  gridbox then puts, in every gridbox, the arrivals from lower positions first, its stayers, and
  the arrivals from higher positions, as the single-domain stable sort does.

Superdroplets that left the domain stay with the rank that held them (the out-of-domain store
has no order to keep). A gridbox's state is only changed by the rank that owns it; the other
ranks' copies of it see no superdroplets and stay as they were.
"""
from __future__ import annotations

import numpy as np

from . import abi

FIELDS = tuple(name for name, _ in abi.SUPERS_FIELDS)


def slab_ranges(ndims, world: int):
    """Gridbox index ranges [lo, hi) of the ranks: rows of constant coord2 index (ny of them,
    nz * nx gridboxes each) split into world near-equal contiguous groups."""
    nz, nx, ny = (int(v) for v in ndims)
    if world < 1 or world > ny:
        raise ValueError(f"{world} ranks for {ny} rows of gridboxes")
    per_row = nz * nx
    cuts = [(ny * r) // world for r in range(world + 1)]
    return [(cuts[r] * per_row, cuts[r + 1] * per_row) for r in range(world)]


def owner(gbx: np.ndarray, ranges) -> np.ndarray:
    """The rank owning each gridbox index (indexes past the last range: -1, out of the domain)."""
    his = np.array([hi for _, hi in ranges], dtype=np.int64)
    r = np.searchsorted(his, gbx.astype(np.int64), side="right")
    return np.where(r < len(ranges), r, -1)


def take(sd: dict, idx: np.ndarray) -> dict:
    return {f: sd[f][idx] for f in FIELDS}


def concat(parts) -> dict:
    parts = [p for p in parts if len(p["xi"])]
    if not parts:
        return {name: np.zeros(0, dtype=dt) for name, dt in abi.SUPERS_FIELDS}
    return {f: np.concatenate([p[f] for p in parts]) for f in FIELDS}


def split(sd: dict, n_domain: int, rank: int, ranges):
    """A rank's superdroplets after motion (in-domain ones first, in their order, as the
    download gives them): (kept, emigrants by destination rank, out-of-domain). `kept` holds the
    rank's in-domain superdroplets still in its gridboxes."""
    gbx = sd["sdgbxindex"][:n_domain]
    dest = owner(gbx, ranges)
    idx = np.arange(n_domain)
    kept = take(sd, idx[dest == rank])
    out = {r: take(sd, idx[dest == r]) for r in range(len(ranges)) if r != rank}
    grave = take(sd, np.arange(n_domain, len(sd["xi"])))
    return kept, out, grave


def pack(sd: dict) -> np.ndarray:
    """The records as an (n, 8) array of 64-bit words (field order of FIELDS)."""
    n = len(sd["xi"])
    w = np.empty((n, len(FIELDS)), dtype=np.uint64)
    for k, f in enumerate(FIELDS):
        a = np.ascontiguousarray(sd[f])
        w[:, k] = a.astype(np.uint64) if a.dtype == np.uint32 else a.view(np.uint64)
    return w


def unpack(w: np.ndarray) -> dict:
    out = {}
    for k, (f, dt) in enumerate(abi.SUPERS_FIELDS):
        col = np.ascontiguousarray(w[:, k])
        out[f] = col.astype(np.uint32) if dt == np.uint32 else col.view(dt)
    return out


def exchange(out: dict, rank: int, world: int, dist) -> dict:
    """Every rank's emigrants to their destinations: the counts of every pair first (an
    all-gather of each rank's counts), then each nonempty pair's records by point-to-point
    send/receive. Returns the immigrants by source rank. Every rank makes the same collective
    calls in the same order."""
    import torch
    counts = torch.tensor([len(out[r]["xi"]) if r != rank else 0 for r in range(world)],
                          dtype=torch.int64)
    table = [torch.zeros(world, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(table, counts)
    reqs, bufs = [], {}
    for src in range(world):
        n = int(table[src][rank])
        if src != rank and n > 0:
            bufs[src] = torch.empty((n, len(FIELDS)), dtype=torch.int64)
            reqs.append(dist.irecv(bufs[src], src=src))
    sends = []
    for dst in range(world):
        if dst != rank and int(table[rank][dst]) > 0:
            t = torch.from_numpy(pack(out[dst]).view(np.int64))
            sends.append(t)
            reqs.append(dist.isend(t, dst=dst))
    for q in reqs:
        q.wait()
    return {src: unpack(b.numpy().view(np.uint64)) for src, b in bufs.items()}


def qcond_of_gridboxes(sd: dict, state: dict, lo: int, hi: int) -> np.ndarray:
    """qcond of the gridboxes [lo, hi) from the superdroplets in them (in array order, which the
    stable sort keeps within each gridbox): effect_on_hydrometeor_states
    (movesupersindomain.hpp:95-136), which CLEO applies after the transport across ranks and the
    sort; a rank applies it to its gridboxes once the immigrants are in. Same expressions as the
    library's: condensate_mass (superdrop_attrs.hpp:208-218) x xi summed in order, over the
    gridbox's volume, over the dry air density (thermodynamic_equations.hpp)."""
    from .config import CP0, MR0, R0, RHO_L, RHO_SOL, RHO0, VOL0
    pi = 3.141592653589793238462643383279502884
    rgas_univ = 8.314462618
    Rgas_dry = (rgas_univ / MR0) / CP0
    Rgas_v = (rgas_univ / 0.01801528) / CP0
    Rho_l, Rho_sol = RHO_L / RHO0, RHO_SOL / RHO0
    massconst = 4.0 / 3.0 * pi * Rho_l
    density_factor = 1.0 - Rho_l / Rho_sol
    tot = np.zeros(hi - lo, dtype=np.float64)
    gbx = sd["sdgbxindex"]
    for k in range(len(gbx)):  # in order: each gridbox's terms added as the sequential loop does
        g = int(gbx[k])
        if not lo <= g < hi:
            continue
        r, msol = float(sd["radius"][k]), float(sd["msol"][k])
        m = msol * density_factor
        m += massconst * (r * r * r)
        tot[g - lo] += max(0.0, m - msol) * float(sd["xi"][k])
    R0cubed_VOL0 = R0 * R0 * R0 / VOL0
    out = np.empty(hi - lo)
    for j in range(hi - lo):
        g = lo + j
        rho_cond = tot[j] / state["volume"][g] * R0cubed_VOL0
        rgas_equiv = Rgas_dry + Rgas_v * state["qvap"][g]
        rho_dry = state["press"][g] / (rgas_equiv * state["temp"][g])
        out[j] = rho_cond / rho_dry
    return out


def merge(kept: dict, immigrants: dict, grave: dict, rank: int) -> dict:
    """The rank's superdroplets for its next upload: immigrants from lower ranks (in rank order),
    its own, immigrants from higher ranks, then its out-of-domain ones."""
    lower = [immigrants[r] for r in sorted(immigrants) if r < rank]
    higher = [immigrants[r] for r in sorted(immigrants) if r > rank]
    return concat(lower + [kept] + higher + [grave])
