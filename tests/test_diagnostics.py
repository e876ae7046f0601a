"""FP64 diagnostics (psb_diagnostics): mass, momentum, kinetic and potential
energy, and the density-error mean and max of the current state.

Known answers, from the downloaded FP32 state summed in FP64 with numpy:
the same sums to 1e-12 relative (only the summation order differs); the
mass is n m exactly; a batch's per-scene entries add up to the whole; and
two calls give identical results (fixed reduction order, no atomics).
"""
import numpy as np
import pytest

import psb_project_b200 as P


def numpy_diag(state, sc, g):
    m = sc.mass
    v = state["vel"].astype(np.float64)
    x = state["pos"].astype(np.float64)
    rho = state["density"].astype(np.float64)
    err = np.abs(rho - sc.rho0) / sc.rho0
    return {"mass": m * len(v), "momentum": list(m * v.sum(0)), "kinetic": 0.5 * m * np.sum(v * v),
            # the step's gravity is stored in FP32
            "potential": -m * np.sum(x @ np.asarray(g, np.float32).astype(np.float64)), "density_err_mean": err.mean(),
            "density_err_max": err.max()}


def close(a, b, rel=1e-12, scale=None):
    s = scale if scale is not None else max(abs(b), 1e-300)
    return abs(a - b) <= rel * s


def check(got, want, scale_v):
    assert got["mass"] == pytest.approx(want["mass"], rel=1e-15)
    for a, b in zip(got["momentum"], want["momentum"]):
        assert close(a, b, scale=want["mass"] * scale_v * 1e-3 + 1e-300) or close(a, b)
    assert close(got["kinetic"], want["kinetic"])
    assert close(got["potential"], want["potential"])
    assert close(got["density_err_mean"], want["density_err_mean"])
    assert got["density_err_max"] == want["density_err_max"]


@pytest.mark.gpu
def test_diagnostics_match_numpy_fp64():
    sc = P.dam_break((16, 14, 12), 0.01, (0.5, 0.4, 0.4), 0.02, dt=5e-4, seed=31)
    with P.Simulation(sc) as sim:
        sim.upload(P.scene_positions(sc))
        sim.presolve(16)
        sim.step(10)
        st = sim.download()
        d1 = sim.diagnostics()
        d2 = sim.diagnostics()
    assert d1 == d2
    want = numpy_diag(st, sc, sc.gravity)
    vmax = float(np.abs(st["vel"]).max())
    check(d1, want, vmax)
    assert d1["kinetic"] > 0 and d1["density_err_max"] > 0


@pytest.mark.gpu
def test_batch_diagnostics_per_scene():
    scenes = P.batch_scenes(n_scenes=3, seed=32, n_range=(300, 2500), side=(0.3, 0.5), dt=5e-4,
                            warm_start=P.WARM_ZERO)
    with P.BatchSimulation(scenes) as b:
        b.set_graph(True)
        b.upload(P.batch_positions(scenes))
        b.step(6)
        st = b.download()
        per = b.diagnostics(per_scene=True)
        whole = b.diagnostics()
    assert len(per) == 3
    for k, sc in enumerate(scenes):
        part = {key: b.split(st[key])[k] for key in ("pos", "vel", "density")}
        check(per[k], numpy_diag(part, sc, sc.gravity), float(np.abs(part["vel"]).max()))
    assert whole["mass"] == pytest.approx(sum(d["mass"] for d in per), rel=1e-15)
    assert whole["kinetic"] == pytest.approx(sum(d["kinetic"] for d in per), rel=1e-12)
    assert whole["density_err_max"] == max(d["density_err_max"] for d in per)
