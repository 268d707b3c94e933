"""Generate the golden fixtures from CLEO's own hot-path sources (run where they are available).

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture holds the inputs of one small configuration and the state the reference build
(oracle/_ref/libcleo_ref.so: CLEO's sources compiled unmodified against the Kokkos-API shim)
reaches after a number of SDM steps. tests/test_golden.py checks the oracle against them, so the
oracle stays pinned where the reference sources are not available.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import checkers as K  # noqa: E402
from cleo_b200 import abi, workloads as W  # noqa: E402
from cleo_b200.config import make_params  # noqa: E402
from cleo_b200.sdm import make_sdm  # noqa: E402
from test_oracle import VARIANTS  # noqa: E402

GOLDEN_STEPS = {
    "box_golovin_nulls": 12, "box_coalbure_cke": 20, "box_coalbure_ts": 20,
    "box_breakup_const": 20, "rain_sediment_out": 40, "rain_alter_thermo": 25,
    "bubble_flow_wrap": 20, "uneven3d_xyz_winds": 12,
}


def save_step_fixture(name, build, nsteps):
    ref = K.ref_lib()
    w = build()
    b = make_sdm(w, lib=ref, prefix="ref")
    for s in range(nsteps):
        b.run_step(s * w["tstep"], (s + 1) * w["tstep"])
    d = b.download_supers()
    st = b.download_state()
    cm, _ = b.download_budgets()
    out = {"nsteps": nsteps, "tstep": w["tstep"], "params": np.frombuffer(bytes(w["params"]), np.uint8)}
    for k, v in w["grid"].items():
        out["grid_" + k] = np.asarray(v)
    for k, v in w["state"].items():
        out["in_state_" + k] = v
    for k, v in w["supers"].items():
        out["in_sd_" + k] = v
    for k, v in d.items():
        out["out_sd_" + k] = np.asarray(v)
    for k, v in st.items():
        out["out_state_" + k] = v
    out["out_cond_mass"] = cm
    np.savez_compressed(os.path.join(HERE, f"step_{name}.npz"), **out)


def save_condsolve_fixture():
    ref = K.ref_lib()
    w = W.condsolve(3000, seed=77)
    out = {k: w[k] for k in ("radius", "msol", "temp", "press", "s_ratio", "delt")}
    for tag, (mx, rt, at) in {"reftol": (50, 0.0, 0.01), "tight": (200, 0.0, 1e-10)}.items():
        p = make_params(condtstep=1.0, maxniters=mx, rtol=rt, atol=at)
        rc, r, _ = K.condsolve(ref, "ref", p, w)
        assert rc == 0
        out[f"params_{tag}"] = np.frombuffer(bytes(p), np.uint8)
        out[f"out_{tag}"] = r
    np.savez_compressed(os.path.join(HERE, "condsolve.npz"), **out)


def save_terminalv_fixture():
    ref = K.ref_lib()
    r = np.exp(np.linspace(np.log(1e-3), np.log(5e4), 300))
    out = {"radius": r}
    for kind in (abi.TV_SIMMEL, abi.TV_ROGERSYAU, abi.TV_ROGERSGK):
        out[f"tv_{kind}"] = np.array([ref.ref_terminal_velocity(kind, x) for x in r])
    np.savez_compressed(os.path.join(HERE, "terminalv.npz"), **out)


if __name__ == "__main__":
    assert K.ref_available(), "build the reference first: make -C oracle ref"
    for name, build, _ in VARIANTS:
        if name in GOLDEN_STEPS:
            save_step_fixture(name, build, GOLDEN_STEPS[name])
    save_condsolve_fixture()
    save_terminalv_fixture()
    print("fixtures written to", HERE)
