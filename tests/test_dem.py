"""DEM (PSB_DEM): known answers on the FP64 oracle and GPU parity.

The reference's DEM step (CudaSystem::update, CudaSystem.cpp:207-224) is
pinned oracle-to-reference in test_oracle_vs_reference.py. Here:
  * config profile, two spheres head-on without gravity: the linear
    spring-dashpot with c_n from dashpot_from_restitution rebounds at the
    restitution e (the damped half-period result), and momentum is kept;
  * a sphere released above the floor bounces and settles at the
    projection bound, r above the face;
  * GPU against the oracle, reference and config profiles, each step from
    the GPU's own FP32 state (tolerances as in test_gpu_parity.py: positions
    4 ulps + 1e-5 of the displacement, velocities 3e-5 of the field max,
    contact force 1e-5 of its max, neighbour counts bit-exact).
"""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import runtime as R


def two_spheres(e, dt=1e-5):
    sc = P.dem_block((2, 1, 1), 0.05, (0.4, 0.4, 0.4), (1.0, 1.0, 1.0), 0.01, restitution=e, dt=dt, jitter=0.0)
    return sc.replace(gravity=(0.0, 0.0, 0.0))


@pytest.mark.parametrize("e", [0.3, 0.8])
def test_head_on_rebound_at_restitution(e):
    sc = two_spheres(e)
    pos = np.array([[0.45, 0.5, 0.5], [0.48, 0.5, 0.5]])
    vel = np.array([[0.5, 0.0, 0.0], [-0.5, 0.0, 0.0]])
    o = oracle.OracleSim(sc, pos, vel)
    for _ in range(4000):     # 0.04 s: contact lasts ~2.3 ms
        o.step()
    assert o.vel[0, 0] < 0 < o.vel[1, 0]
    assert abs(o.vel[1, 0] / 0.5 - e) < 0.02 * e + 2e-3
    assert abs(o.vel[:, 0].sum()) < 1e-12


def test_sphere_settles_on_floor():
    sc = P.dem_block((1, 1, 1), 0.05, (0.5, 0.05, 0.5), (1.0, 1.0, 1.0), 0.01, dt=1e-4, jitter=0.0)
    o = oracle.OracleSim(sc, np.array([[0.5, 0.05, 0.5]]))
    for _ in range(3000):
        o.step()
    assert abs(o.pos[0, 1] - 0.01) < 1e-6
    assert abs(o.vel[0, 1]) < 1e-2


def ref_dem_scene():
    return P.dem_block((8, 8, 8), 0.02, (0.1, 0.1, 0.1), (0.5, 0.5, 0.5), 0.01, profile=P.PROFILE_REF,
                       spring=20.0, h=0.025, dt=1e-3, seed=4, jitter=2e-3)


def config_dem_scene():
    # spacing below the diameter: the lattice starts in contact
    return P.dem_block((10, 8, 9), 0.0195, (0.2, 0.05, 0.2), (1.0, 1.0, 1.0), 0.01, dt=1e-4, seed=6, jitter=2e-4)


def rel_norm(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["ref", "config"])
def test_gpu_dem_steps_match_oracle(which):
    sc = ref_dem_scene() if which == "ref" else config_dem_scene()
    pos = P.scene_positions(sc)
    vel = np.random.default_rng(2).normal(0.0, 0.2, (sc.n, 3)).astype(np.float32)
    with P.Simulation(sc) as sim:
        sim.upload(pos, vel, vel)
        orc = oracle.OracleSim(sc, pos, vel, vel, float_state=True)
        for _ in range(5):
            x0 = orc.pos.copy()
            sim.step(1)
            orc.step()
            out = sim.download()
            ulp = np.spacing(np.float32(np.max(np.abs(orc.pos))))
            disp = np.max(np.abs(orc.pos - x0))
            assert np.max(np.abs(out["pos"] - orc.pos)) <= 4 * float(ulp) + 1e-5 * disp
            assert rel_norm(out["vel"], orc.vel) <= 3e-5
            assert np.array_equal(sim.read_field(R.FIELD_NBR_COUNT), orc.nbr)
            f = sim.read_field(R.FIELD_FORCE_NP)
            assert rel_norm(f, orc.f_np) <= 1e-5
            orc.pos[:] = out["pos"]
            orc.vel[:] = out["vel"]
