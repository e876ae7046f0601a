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
  * spheres above the fluid fall freely until they reach it;
  * a sheet of 400 spheres (as heavy as the water below it) dropped on a
    tank: with the spheres' motion solved inside the corrector (implicit
    coupling) the corrector keeps converging, the water stays calm after
    the impact and the sheet sinks; the staggered exchange instead throws
    the water about at tens of m/s and runs the corrector to its cap on
    most steps (the added-mass instability of explicit partitioned
    coupling).
On the oracle (CPU) the same coupled loop runs in FP64.
"""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import runtime as R

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


def sheet_drop():
    """A 7,056-particle tank under a 10 x 4 x 10 sheet of 2500 kg/m^3
    spheres (4.2 kg against 7.1 kg of water) 2 cm above its surface."""
    box = (0.21, 0.6, 0.21)
    fl = P.dam_break((21, 16, 21), 0.01, box, 0.02, dt=1e-3, mass=1e-3, seed=3)
    sp = P.dem_block((10, 4, 10), 0.021, (0.0, 0.18, 0.0), box, 0.01, density=2500.0, k_n=1e4, restitution=0.3,
                     dt=1e-3, seed=5)
    return fl, sp


def run_sheet(implicit, steps):
    fl, sp = sheet_drop()
    bpos = P.scene_positions(sp).astype(np.float64)
    fluid = oracle.OracleSim(fl, P.scene_positions(fl).astype(np.float64), boundary=bpos + [0.0, 10.0, 0.0])
    fluid.presolve(64)
    for _ in range(50):                 # the tank settles, the spheres far away
        fluid.step()
    balls = oracle.OracleSim(sp, bpos)
    c = oracle.Coupling(fl, fluid, sp, balls, implicit=implicit)
    its, vmax, v99 = [], [], []
    for _ in range(steps):
        st, _ = c.step()
        its.append(st.iters)
        speed = np.linalg.norm(fluid.vel, axis=1)
        vmax.append(speed.max())
        v99.append(np.percentile(speed, 99))
    return np.array(its), np.array(vmax), np.array(v99), bpos, balls.pos


def test_oracle_implicit_coupling_keeps_a_dropped_sheet_stable():
    its, vmax, v99, b0, b1 = run_sheet(True, 200)
    assert its.mean() <= 8 and np.count_nonzero(its >= 50) <= 2, (its.mean(), np.count_nonzero(its >= 50))
    # the sheet hits at t ~ 0.07 s and the water it displaces streams up
    # through its pores; 99% of the water stays below 3 m/s (a few droplets
    # splash faster)
    assert v99.max() < 3.0, v99.max()
    assert b1[:, 1].mean() < b0[:, 1].mean() - 0.02            # it sinks


def test_oracle_staggered_coupling_fails_on_the_same_sheet():
    its, vmax, _, _, _ = run_sheet(False, 300)
    assert np.count_nonzero(its >= 50) > 50 and vmax.max() > 50.0, (np.count_nonzero(its >= 50), vmax.max())


@pytest.mark.gpu
def test_gpu_implicit_coupling_matches_oracle():
    """Implicit coupled steps of a sphere sinking in the settled tank, each
    from the GPU's state against the FP64 oracle from the same state (fluid
    and sphere). The corrector count must agree unless the deciding error
    lies within 2e-6 of eta (then the compared fields differ by one
    correction and the step is skipped). The fluid is held to the multi-
    correction config tolerances (pressure 1e-4 of the field max, density
    1e-5 element-wise plus the shift of x* by the pressure error), the
    pressure with the boundary tests' addition: each correction adds
    delta (rho* - rho0), and the FP32 Kahan densities agree with FP64 to
    ~2e-7 relative, so k corrections can move it by k delta 2e-7 rho0; near
    the sphere the predicted sphere position, stored in FP32 like x*, adds
    its terms with the weight psi_b / m (~5 fluid masses), so the bound
    there is (1 + psi_b / m) times that. The
    sphere's velocity change is dt (f + F) / m with F the reaction, a sum of
    the pressures of the ~30 fluid particles around the sphere, each within
    1e-4 of the field max while they carry about a third of it: F, and the
    velocity change with it, is held to 1e-3 of itself (plus 1e-6 of the
    velocity for its FP32 storage)."""
    sc, pos, sph, centre = tank()
    compared = 0
    with P.Simulation(sc) as fluid, P.Simulation(sph) as ball:
        fluid.upload(pos)
        fluid.set_boundary(centre[None])
        fluid.presolve(64)
        fluid.step(SETTLE)
        ball.upload(centre[None])
        c = P.FluidDemCoupling(fluid, ball)
        for _ in range(4):
            fs, bs = fluid.download(), ball.download()
            c.step(1)
            st = fluid.stats()
            got_f, got_b = fluid.download(), ball.download()
            ofl = oracle.OracleSim(sc, fs["pos"], fs["vel"], fs["vel_half"], fs["pressure"],
                                   boundary=bs["pos"].astype(np.float64))
            oball = oracle.OracleSim(sph, bs["pos"].astype(np.float64), bs["vel"], bs["vel_half"])
            so, _ = oracle.Coupling(sc, ofl, sph, oball).step()
            if st.iters != so.iters:
                assert abs(so.err[min(st.iters, so.iters)] - sc.eta) <= 2e-6, (st.iters, so.iters)
                continue
            compared += 1
            dv = np.abs(oball.vel[0] - bs["vel"][0]).max()
            assert np.max(np.abs(got_b["vel"][0] - oball.vel[0])) <= 1e-3 * dv + 1e-6 * np.abs(oball.vel).max()
            psi_m = float(oracle.boundary_psi(sc, bs["pos"].astype(np.float64))[0]) / sc.mass
            p_abs = max(so.iters, 1) * oracle.pci_delta(sc) * 2e-7 * sc.rho0 * (1.0 + psi_m)
            assert np.max(np.abs(got_f["pressure"] - ofl.p)) <= max(1e-4 * np.abs(ofl.p).max(), p_abs)
            assert np.max(np.abs(got_f["density"] - ofl.rho) / ofl.rho) <= 1e-4
    assert compared >= 2


@pytest.mark.gpu
def test_gpu_c1_implicit_spheres_sink_and_corrector_converges():
    """The C1 set-up at test size (4,096 fluid particles, 64 spheres): 250
    implicit coupled steps. The spheres enter the fluid and sink below its
    initial surface, every value stays finite, and the corrector converges
    on at least 90% of the steps."""
    fl, sp = P.c1_scenes(fluid_n=(16, 16, 16), dem_n=(4, 4, 4))
    its = []
    with P.Simulation(fl) as fluid, P.Simulation(sp) as balls:
        fluid.upload(P.scene_positions(fl))
        fluid.presolve(16)
        balls.upload(P.scene_positions(sp))
        c = P.FluidDemCoupling(fluid, balls)
        for _ in range(250):
            c.step(1)
            its.append(fluid.stats().iters)
        b = balls.download()
        f = fluid.download()
    its = np.array(its)
    assert np.isfinite(f["pos"]).all() and np.isfinite(f["vel"]).all() and np.isfinite(b["pos"]).all()
    assert b["pos"][:, 1].mean() < 16 * 0.01, b["pos"][:, 1].mean()
    assert np.count_nonzero(its >= fl.max_iters) <= 25, np.count_nonzero(its >= fl.max_iters)


@pytest.mark.gpu
def test_gpu_boundary_motion_and_dem_forces_refuse_bad_calls():
    """psb_set_boundary_motion needs a boundary set, a positive finite mass
    and a config-profile PCISPH single scene; psb_dem_forces a DEM context.
    The refused calls change nothing: the context still steps."""
    sc, pos, sph, centre = tank()
    with P.Simulation(sc) as fluid, P.Simulation(sph) as ball:
        fluid.upload(pos)
        v = np.zeros((1, 3), np.float32)
        with pytest.raises(R.PsbError) as e:
            fluid.set_boundary_motion(v, v, 0.01)         # no boundary yet
        assert e.value.status == R.ESTATE
        fluid.set_boundary(centre[None])
        for bad in (0.0, -1.0, float("nan"), float("inf")):
            with pytest.raises(R.PsbError) as e:
                fluid.set_boundary_motion(v, v, bad)
            assert e.value.status == R.EINVAL
        with pytest.raises(R.PsbError) as e:
            fluid.dem_forces()                             # not a DEM context
        assert e.value.status == R.EINVAL
        ball.upload(centre[None])
        f = ball.dem_forces()                              # gravity alone for one sphere
        assert np.allclose(f, [[0.0, -G * float(sph.mass), 0.0]], rtol=1e-6)
        fluid.set_boundary_motion(v, f, float(sph.mass))
        fluid.set_boundary_motion(None)                    # static again
        fluid.step(1)
        assert fluid.stats().converged == 1
