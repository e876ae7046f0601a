"""Fluid-DEM coupling through boundary particles (config C1).

Every DEM sphere is one boundary particle of the fluid at its centre; the
fluid's reaction on it (psb_boundary_forces: minus the mirrored-pressure
forces it exerts) is the sphere's external force in the next DEM step
(psb_set_external_force).

Known answers:
  * the reaction is the oracle's sum (FP32 against FP64: 1e-5 of the
    largest force), and a DEM step with an external force is the oracle's;
  * a sphere of 2500 kg/m^3 released inside a settled fluid sinks, and
    slower than it falls in air: its mean acceleration over the first 20 ms
    lies between 0.15 g and 0.9 g. Buoyancy alone would give
    g (1 - rho0/rho_s) = 0.6 g and a sphere's added mass 0.5 g; the point
    sphere also meets the fluid's pressure response as it starts to move,
    and the oracle measures 0.33 g. Free fall (no coupling) gives g and a
    floating sphere a negative value; both fail;
  * spheres above the fluid fall freely until they reach it.
On the oracle (CPU) the same coupled loop runs in FP64.
"""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P

G = 9.81
SETTLE = 200


def tank():
    sc = P.dam_break((16, 20, 16), 0.01, (0.16, 0.3, 0.16), 0.02, dt=5e-4, seed=51, jitter=1e-4)
    pos = P.scene_positions(sc)
    centre = np.array([0.085, 0.095, 0.085], np.float32)
    keep = np.linalg.norm(pos - centre, axis=1) > 0.012
    sphere = P.dem_block((1, 1, 1), 0.02, centre - 0.01, (0.16, 0.3, 0.16), 0.01, density=2500.0, dt=5e-4,
                         jitter=0.0)
    return sc.replace(n=int(keep.sum())), pos[keep], sphere, centre


def test_oracle_coupled_sphere_sinks_slower_than_free_fall():
    sc, pos, sph, centre = tank()
    fluid = oracle.OracleSim(sc, pos.astype(np.float64), boundary=centre[None].astype(np.float64))
    fluid.presolve(64)
    for _ in range(SETTLE):             # the fluid closes around the sphere held still
        fluid.step()
    ball = oracle.OracleSim(sph, centre[None].astype(np.float64))
    steps = 40
    for _ in range(steps):
        fluid.P.n_bnd = 1
        fluid.bnd_pos[:] = ball.pos
        fluid.bnd_psi[:] = oracle.boundary_psi(sc, fluid.bnd_pos)
        fluid.step()
        f = oracle.boundary_reaction(sc, fluid.pos, fluid.p, fluid.bnd_pos)
        ball.set_external_force(f)
        ball.step()
    a = -ball.vel[0, 1] / (steps * float(sph.dt))
    assert 0.15 * G < a < 0.9 * G, a / G


@pytest.mark.gpu
def test_gpu_reaction_matches_oracle():
    sc, pos, sph, centre = tank()
    bnd = np.array([centre, centre + [0.03, 0.02, 0.0], centre - [0.0, 0.04, 0.03]], np.float32)
    with P.Simulation(sc) as sim:
        sim.upload(pos)
        sim.set_boundary(bnd)
        sim.presolve(32)
        sim.step(2)
        st = sim.download()
        got = sim.boundary_forces()
    want = oracle.boundary_reaction(sc, st["pos"].astype(np.float64), st["pressure"].astype(np.float64),
                                    bnd.astype(np.float64))
    assert np.abs(want).max() > 1e-3
    assert np.max(np.abs(got - want)) <= 1e-5 * np.abs(want).max()


@pytest.mark.gpu
def test_gpu_dem_external_force_matches_oracle():
    sph = P.dem_block((6, 5, 4), 0.025, (0.1, 0.1, 0.1), (0.4, 0.4, 0.4), 0.01, dt=5e-4, seed=52)
    pos = P.scene_positions(sph)
    f = np.random.default_rng(3).normal(0, 0.05, (sph.n, 3)).astype(np.float32)
    with P.Simulation(sph) as sim:
        sim.upload(pos)
        sim.set_external_force(f)
        sim.step(3)
        got = sim.download()
    ref = oracle.OracleSim(sph, pos.astype(np.float64), float_state=True)
    ref.set_external_force(f.astype(np.float64))
    for _ in range(3):
        ref.step()
    # the DEM parity tolerances (test_dem.py): velocities 3e-5 of the field
    # max, positions 4 ulps + 1e-5 of the displacement
    assert np.max(np.abs(got["vel"] - ref.vel)) <= 3e-5 * np.abs(ref.vel).max()
    ulp = np.spacing(np.float32(np.abs(ref.pos).max()))
    disp = np.abs(ref.pos - pos).max()
    assert np.max(np.abs(got["pos"] - ref.pos)) <= 4 * float(ulp) + 1e-5 * disp


@pytest.mark.gpu
def test_gpu_coupled_sphere_sinks_slower_than_free_fall():
    sc, pos, sph, centre = tank()
    steps = 40
    with P.Simulation(sc) as fluid, P.Simulation(sph) as ball:
        fluid.upload(pos)
        fluid.set_boundary(centre[None])
        fluid.presolve(64)
        fluid.step(SETTLE)                   # the fluid closes around the sphere held still
        ball.upload(centre[None])
        P.FluidDemCoupling(fluid, ball).step(steps)
        v = ball.download()["vel"][0]
    a = -v[1] / (steps * float(sph.dt))
    assert 0.15 * G < a < 0.9 * G, a / G
    with P.Simulation(sph) as free:          # the same sphere without the fluid falls at g
        free.upload(centre[None])
        free.step(steps)
        vf = free.download()["vel"][0]
    assert abs(-vf[1] / (steps * float(sph.dt)) - G) < 1e-3 * G


@pytest.mark.gpu
def test_gpu_c1_spheres_fall_freely_above_the_fluid():
    fl, sp = P.c1_scenes(fluid_n=(16, 16, 16), dem_n=(4, 4, 4))
    with P.Simulation(fl) as fluid, P.Simulation(sp) as balls:
        fluid.upload(P.scene_positions(fl))
        fluid.presolve(16)
        balls.upload(P.scene_positions(sp))
        c = P.FluidDemCoupling(fluid, balls)
        c.step(10)
        v = balls.download()["vel"]
        assert np.all(c.last_force == 0)                # 2 cm above the fluid: no interaction yet
    assert np.allclose(v[:, 1], -G * 10 * float(sp.dt), rtol=1e-4)
