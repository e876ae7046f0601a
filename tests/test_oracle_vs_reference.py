"""The oracle against the reference's own kernels executed on the CPU
(oracle/_ref: the reference's .cu kernel sources compiled as host code).
Skipped where oracle/_ref has not been built (no reference tree)."""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_neighbour_counts_and_density(seed):
    sc = P.ref_scene(seed=seed, jitter=2e-3)
    pos = oracle.scene_positions(sc).astype(np.float64)
    ref = oracle.RefSim(sc, pos)
    rc = ref.search()
    oc, ol = oracle.neighbors(sc, pos)
    assert np.array_equal(rc, oc)
    assert rel(oracle.density(sc, pos, oc, ol, clamp=False), ref.density_pci()) < 1e-13


def test_random_cloud_counts():
    """Uniform random positions: every pair distance is arbitrary, so the
    cut-off test sees many near-h pairs."""
    sc = P.ref_scene()
    rng = np.random.default_rng(3)
    pos = rng.uniform(0.0, 0.3, size=(3000, 3)).astype(np.float32).astype(np.float64)
    sc = sc.replace(n=pos.shape[0])
    ref = oracle.RefSim(sc, pos)
    assert np.array_equal(ref.search(), oracle.neighbors(sc, pos, with_lists=False)[0])


@pytest.mark.parametrize("method", [P.PCISPH, P.WCSPH])
def test_steps_match(method):
    sc = P.ref_scene(method=method, nxyz=(10, 14, 8), box=(0.25, 0.3, 0.2), seed=5)
    pos = oracle.scene_positions(sc).astype(np.float64)
    ref = oracle.RefSim(sc, pos)
    orc = oracle.OracleSim(sc, pos)
    for _ in range(6):
        ref.pcisph_update() if method == P.PCISPH else ref.wcsph_update()
        orc.step()
        assert rel(orc.pos, ref.get("pos", 3)) < 1e-12
        assert rel(orc.vel_half, ref.get("vel_ap", 3)) < 1e-9
        assert rel(orc.rho, ref.get("density", 1)) < 1e-12
        assert rel(orc.p, ref.get("pressure", 1)) < 1e-9


def dem_ref_scene(seed=4):
    """Reference-profile DEM block: interaction radius h = 0.025 over a
    0.02 lattice, so every sphere has listed neighbours in contact range."""
    return P.dem_block((8, 8, 8), 0.02, (0.1, 0.1, 0.1), (0.5, 0.5, 0.5), 0.01, profile=P.PROFILE_REF,
                       spring=20.0, damping=0.01, shear=0.005, attraction=0.002, h=0.025, dt=1e-3, seed=seed,
                       jitter=2e-3)


def test_dem_steps_match():
    """CudaSystem::update (collideParticles, integrateEuler, collisionBox)
    against the oracle's DEM step, 6 steps from random velocities."""
    sc = dem_ref_scene()
    pos = oracle.scene_positions(sc).astype(np.float64)
    vel = np.random.default_rng(1).normal(0.0, 0.2, (sc.n, 3))
    ref = oracle.RefSim(sc, pos, vel)
    orc = oracle.OracleSim(sc, pos, vel)
    for _ in range(6):
        # neighbour counts at the step's start positions: the reference's
        # search against the oracle's walk, then against the list its step uses
        counts = ref.search()
        assert np.array_equal(counts, oracle.neighbors(sc, orc.pos, with_lists=False)[0])
        ref.dem_update()
        orc.step()
        assert np.array_equal(orc.nbr, counts)
        assert rel(orc.pos, ref.get("pos", 3)) < 1e-12
        assert rel(orc.vel, ref.get("vel", 3)) < 1e-12
