"""Emission mid-run: the reference's emitters (src/Kernel/Emitters/*) and
particles appended to a resident state (PCI_SPHSystem::emitParticles and
_initialize(begin, N), PciSphSystem.cpp:50-160).

The reference's emitters need its Particle, SimulationData and GL geometry
classes, so they are restated in the oracle, loop for loop, rather than
compiled; these tests pin both restatements to each other and to what the
reference's loops imply:
CPU:
  * the library's host generator (psb_emitter_positions) equals the
    oracle's, bit for bit, for every type and two emissions;
  * known answers: the box is a float lattice of step 2 particle_radius
    inside its bounds, whose far faces appear only when the float
    accumulation lands on them; every sphere and cylinder layer starts
    with five coincident points at r = 0 (its angle loop runs 0 .. 2 pi
    inclusive); heart points satisfy |res| <= 0.001; ellipsoid points lie
    at the centre's height within the offsets' bounds; mesh points lie in
    their triangles; random emissions differ between emissions and repeat
    for the same seed;
GPU:
  * psb_emit appends at ids n .. n + k - 1 with density and pressure 0 and
    the SPH half-step velocity 0 (a DEM sphere's is its velocity);
  * emitters inside steps: a reference-profile PCISPH dam break with a box
    emitter, and DEM with sphere and ellipsoid emitters (drawn on the
    device), each step against the oracle that appends the same particles
    and steps (the parity suite's tolerances);
  * emissions beyond the capacity fail the step before it changes anything.
"""
import ctypes

import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import emitters as E
from psb_project_b200 import runtime as R


def cases():
    return {
        "box": E.box((0.1, 0.2, 0.3), (0.05, 0.03, 0.04), 0.005, world=(0.01, 0.0, -0.02)),
        "box_fine": E.box((0.0, 0.0, 0.0), (0.1, 0.1, 0.1), 0.0033),
        "sphere": E.sphere((0.0, 0.05, 0.0), 0.05, 0.01),
        "sphere_big": E.sphere((0.0, 0.0, 0.0), 0.1, 0.007),
        "cylinder": E.cylinder((0.2, 0.1, 0.3), (0, 1, 0), 0.05, 0.1, 0.004),
        "ellipsoid": E.ellipsoid((0.1, 0.1, 0.1), 0.2, 0.1, 100, seed=3),
        "mesh": E.mesh([[0, 0, 0], [1, 0, 0], [0, 0, 1], [0, 1, 0]], [[0, 1, 2], [0, 2, 3]], 50, seed=4),
        "heart": E.heart(),
    }


def orc_positions(e, emission=0):
    return oracle.emitter_positions(e.type, e.v, e.particle_radius, e.count, e.faces, e.seed, emission)


@pytest.mark.parametrize("name", sorted(cases()))
def test_host_generator_matches_oracle(name):
    e = cases()[name]
    for emission in (0, 3):
        a, b = E.positions(e, emission), orc_positions(e, emission)
        assert a.shape == b.shape and a.shape[0] > 0
        assert np.array_equal(a, b)


def test_box_is_a_float_lattice():
    e = E.box((0.1, 0.2, 0.3), (0.05, 0.03, 0.04), 0.005)
    p = E.positions(e)
    lo = np.array([0.075, 0.185, 0.28])
    hi = np.array([0.125, 0.215, 0.32])
    step = np.float32(0.005) * np.float32(2)
    counts = []
    for a in range(3):
        u = np.unique(p[:, a])
        assert u[0] == np.float32(lo[a])                     # the near face is always there
        assert np.allclose(np.diff(u), 0.01, atol=1e-6)
        # the far face only when the float accumulation lands on or below it
        assert float(u[-1]) <= hi[a] < float(np.float32(u[-1] + step))
        counts.append(len(u))
    assert p.shape[0] == np.prod(counts)


def test_rings_start_with_five_centre_points():
    for e in (E.sphere((0.0, 0.0, 0.0), 0.05, 0.01), E.cylinder((0.0, 0.1, 0.0), (0, 1, 0), 0.03, 0.05, 0.01)):
        p = E.positions(e)
        first = p[:5]
        assert np.all(first == first[0])                   # theta = 0, pi/2, pi, 3 pi/2, 2 pi at r = 0
        assert not np.array_equal(p[5], first[0])


def test_heart_points_on_the_surface():
    p = E.positions(E.heart()).astype(np.float64)
    x, y, z = p.T
    res = (x * x + 2 * y * y + z * z - 1) ** 3 - x * x * z ** 3
    assert np.all(np.abs(res) <= 0.001 + 1e-5)


def test_random_emitters():
    e = E.ellipsoid((0.1, 0.3, 0.1), 0.2, 0.1, 2000, seed=7)
    p0, p1 = E.positions(e, 0), E.positions(e, 1)
    assert not np.array_equal(p0, p1) and np.array_equal(p0, E.positions(e, 0))
    assert np.all(p0[:, 1] == np.float32(0.3))
    assert np.all(np.abs(p0[:, 0] - 0.1) <= 0.1 + 0.002 + 1e-6) and np.all(np.abs(p0[:, 2] - 0.1) <= 0.05 + 0.001 + 1e-6)
    assert abs(p0[:, 0].mean() - 0.1) < 0.01
    m = E.mesh([[0, 0, 0], [1, 0, 0], [0, 0, 1]], [[0, 1, 2]], 500, seed=8)
    q = E.positions(m, 0).astype(np.float64)
    assert np.all(q[:, 0] >= -1e-7) and np.all(q[:, 2] >= -1e-7) and np.all(q[:, 0] + q[:, 2] <= 1 + 1e-6)
    assert np.all(q[:, 1] == 0)


def test_bad_emitter_rejected():
    with pytest.raises(R.PsbError):
        E.positions(E.Emitter(9, []))


@pytest.mark.parametrize("bad", [
    E.box([0, 0, 0], [0.1, 0.1, 0.1], 0.0),                   # step 0: the lattice loop would not advance
    E.box([0, 0, 0], [0.1, 0.1, 0.1], -0.01),
    E.box([0, 0, 0], [0.1, 0.1, 0.1], float("nan")),
    E.box([0, 0, 0], [float("inf"), 0.1, 0.1], 0.01),
    E.box([0, 0, 0], [0.1, float("nan"), 0.1], 0.01),
    E.box([1e6, 0, 0], [0.1, 0.1, 0.1], 1e-3),               # step below a float ulp at 1e6
    E.box([0, 0, 0], [10.0, 10.0, 10.0], 1e-3),              # 1.25e14 points
    E.sphere([0, 0, 0], 0.5, 0.0),
    E.sphere([0, 1e12, 0], 0.5, 1e-5),                       # step below a double ulp at 1e12
    E.sphere([0, 0, 0], 100.0, 1e-3),
    E.cylinder([0, 0, 0], [0, 1, 0], 0.2, 1.0, 0.0),
    E.cylinder([0, 0, 0], [0, float("inf"), 0], 0.2, 1.0, 0.01),
    E.cylinder([0, 0, 0], [0, 1, 0], 50.0, 50.0, 1e-3),
    E.ellipsoid([0, 0, 0], 1.0, 1.0, -1),
    E.mesh([[0, 0, 0], [1, 0, 0], [0, 0, 1]], [[0, 1, 2]] * 4096, 1 << 20),
])
def test_degenerate_emitter_rejected_without_generating(bad):
    """Emitters whose generator loops would never end, or whose one emission
    would pass the int32 particle count, fail with PSB_EINVAL at once."""
    with pytest.raises(R.PsbError):
        E.positions(bad)


def test_bound_admits_the_ordinary_emitters():
    for e in (E.box([0.3, 0.2, 0.1], [0.2, 0.1, 0.3], 0.005), E.sphere([0.1, 0.0, 0.2], 0.15, 0.01),
              E.cylinder([0, 0.4, 0], [0, 1, 0], 0.1, 0.3, 0.01), E.box([5.0, 5.0, 5.0], [0.0, 0.0, 0.0], 0.01)):
        assert E.positions(e).shape[0] >= 1


# ---- GPU ---------------------------------------------------------------------------

def _compare(got, ref, x0_pos, v_tol=3e-5):
    disp = np.abs(ref.pos[:x0_pos.shape[0]] - x0_pos).max() if x0_pos.shape[0] else 0.0
    ulp = float(np.spacing(np.float32(np.abs(ref.pos).max())))
    assert np.max(np.abs(got["pos"] - ref.pos)) <= 4 * ulp + 1e-5 * max(disp, 1e-3)
    assert np.max(np.abs(got["vel_half"] - ref.vel_half)) <= v_tol * max(1.0, np.abs(ref.vel_half).max())


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["pcisph", "dem"])
def test_gpu_emit_appends(method):
    if method == "pcisph":
        sc = P.ref_scene((8, 8, 8), seed=31)
    else:
        sc = P.dem_block((6, 6, 6), 0.03, (0.05, 0.05, 0.05), (0.5, 0.5, 0.5), 0.01, dt=1e-4, seed=32)
    pos = P.scene_positions(sc)
    k = 20
    with P.Simulation(sc.replace(n=sc.n + 2 * k)) as sim:
        sim.upload(pos)
        sim.step(1)
        before = sim.download()
        new = np.random.default_rng(0).uniform(0.12, 0.2, (k, 3)).astype(np.float32)
        vel = np.tile(np.float32([0.3, -0.1, 0.2]), (k, 1))
        sim.emit(new, vel)
        got = sim.download()
        assert sim.n == sc.n + k
        assert np.array_equal(got["pos"][:sc.n], before["pos"]) and np.array_equal(got["pos"][sc.n:], new)
        assert np.array_equal(got["vel"][sc.n:], vel)
        want_vh = vel if method == "dem" else np.zeros_like(vel)
        assert np.array_equal(got["vel_half"][sc.n:], want_vh)
        assert np.all(got["density"][sc.n:] == 0) and np.all(got["pressure"][sc.n:] == 0)
        sim.step(2)
        with pytest.raises(R.PsbError):
            sim.emit(np.zeros((k + 1, 3), np.float32) + 0.1)


@pytest.mark.gpu
def test_gpu_pcisph_box_emitter_matches_oracle():
    sc = P.ref_scene((12, 10, 8), seed=33)
    e = E.box((0.2, 0.2, 0.15), (0.03, 0.02, 0.03), 0.005, velocity=(0.5, 0.0, 0.0), duration=3)
    per = E.positions(e).shape[0]
    pos = P.scene_positions(sc)
    with P.Simulation(sc.replace(n=sc.n + 3 * per)) as sim:
        sim.upload(pos)
        sim.add_emitter(e)
        ref = oracle.OracleSim(sc, pos.astype(np.float64), float_state=True)
        for step in range(5):
            x0 = sim.download()
            for key, a in (("pos", ref.pos), ("vel", ref.vel), ("vel_half", ref.vel_half)):
                a[:] = x0[key]
            if step < 3:
                ref.append(E.positions(e, step), vel=np.tile(e.velocity, (per, 1)))
            sim.step(1)
            ref.step()
            got = sim.download()
            assert sim.n == sc.n + min(step + 1, 3) * per
            _compare(got, ref, x0["pos"])


@pytest.mark.gpu
def test_gpu_dem_emitters_match_oracle():
    # the block stays below y = 0.09; the sphere emitter's layers (its y
    # enters sqrt(R^2 - y^2) as an absolute coordinate) fill y = 0.15 .. 0.3
    sc = P.dem_block((5, 4, 5), 0.025, (0.05, 0.0, 0.05), (0.6, 0.6, 0.6), 0.01, dt=2e-4, seed=34)
    es = [E.sphere((0.3, 0.45, 0.3), 0.3, 0.02, velocity=(0.0, -0.5, 0.0), duration=2),
          E.ellipsoid((0.3, 0.45, 0.3), 0.4, 0.4, 16, velocity=(0.1, 0.0, 0.0), duration=3, seed=11)]
    per = [E.positions(x).shape[0] for x in es]
    pos = P.scene_positions(sc)
    with P.Simulation(sc.replace(n=sc.n + 2 * per[0] + 3 * per[1])) as sim:
        sim.upload(pos)
        for x in es:
            sim.add_emitter(x)
        ref = oracle.OracleSim(sc, pos.astype(np.float64), float_state=True)
        for step in range(4):
            x0 = sim.download()
            ref.pos[:] = x0["pos"]
            ref.vel[:] = x0["vel"]
            ref.vel_half[:] = x0["vel_half"]
            for x, k in zip(es, per):
                if step < x.duration:
                    v = np.tile(x.velocity, (k, 1))
                    ref.append(E.positions(x, step), vel=v, vel_half=v)
            sim.step(1)
            ref.step()
            got = sim.download()
            _compare(got, ref, x0["pos"])
            assert np.max(np.abs(got["vel"] - ref.vel)) <= 3e-5 * max(1.0, np.abs(ref.vel).max())


@pytest.mark.gpu
def test_gpu_emission_beyond_capacity_fails_cleanly():
    sc = P.ref_scene((6, 6, 6), seed=35)
    e = E.box((0.2, 0.2, 0.2), (0.02, 0.02, 0.02), 0.005, duration=5)
    per = E.positions(e).shape[0]
    with P.Simulation(sc.replace(n=sc.n + per + per // 2)) as sim:
        sim.upload(P.scene_positions(sc))
        sim.add_emitter(e)
        sim.step(1)
        assert sim.n == sc.n + per
        before = sim.download()
        with pytest.raises(R.PsbError):
            sim.step(1)
        assert sim.n == sc.n + per
        assert np.array_equal(sim.download()["pos"], before["pos"])
        sim.clear_emitters()
        sim.step(1)
