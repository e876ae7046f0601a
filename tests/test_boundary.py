"""Static boundary particles (Akinci et al. 2012; psb_set_boundary).

Known answers, on the oracle (no GPU):
  * psi_b = rho0 / sum_k W_bk exactly; inside a slab thicker than two
    kernel reaches, a boundary particle sampled on the fluid's rest lattice
    sees a full lattice neighbourhood, so psi_b = m to rounding;
  * fluid resting on a two-spacing slab: every fluid layer beyond the first
    has exactly the rest density; the first one lies 4.5% over it (the
    slab's top layer stands in for the solid below it as well; the
    corrector holds the fluid a little off the wall in response);
  * the mirrored pressure pushes a pressurised fluid particle away from the
    wall, and a dam break around a sphere never enters the sphere.
On the GPU: psi against the oracle (FP32 against FP64, 1e-6) and a few
steps of a dam break around a sphere against the oracle, at the config
profile's multi-correction tolerance (1e-4 of the field max).
"""
import ctypes

import numpy as np
import pytest

import oracle
import psb_project_b200 as P

S, H = 0.01, 0.02


def lat(nx, ny, nz, org, sp=S):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return np.stack([i.ravel() * sp + org[0], j.ravel() * sp + org[1], k.ravel() * sp + org[2]], 1)


def scene(n=1000):
    return P.dam_break((10, 10, 10), S, (0.5, 0.5, 0.5), H, dt=5e-4, seed=1, jitter=0.0).replace(n=n)


def densities(sc, fluid, bnd):
    psi = oracle.boundary_psi(sc, bnd)
    Pp = oracle.params(sc.replace(n=len(fluid)))
    bp = np.ascontiguousarray(bnd, np.float64)
    Pp.n_bnd, Pp.bnd_pos, Pp.bnd_psi = len(bnd), bp.ctypes.data, psi.ctypes.data
    cnt, lists = oracle.neighbors(sc.replace(n=len(fluid)), fluid)
    rho = np.empty(len(fluid))
    f = np.ascontiguousarray(fluid, np.float64)
    oracle.lib().orc_density(ctypes.byref(Pp), oracle._ptr(f), oracle._ptr(cnt), oracle._ptr(np.ascontiguousarray(lists)),
                             lists.shape[1], 1, oracle._ptr(rho))
    return rho, psi


def test_psi_definition_and_full_lattice():
    sc = scene()
    bnd = lat(12, 5, 12, (0.1, 0.1, 0.1))
    psi = oracle.boundary_psi(sc, bnd)
    # psi_b sum_k W_bk = rho0
    d = np.linalg.norm(bnd[:, None, :] - bnd[None, :, :], axis=2)
    W = np.where(d < H, 315 / (64 * np.pi * H ** 9) * (H * H - d * d) ** 3, 0.0)
    assert np.allclose(psi * W.sum(1), sc.rho0, rtol=1e-12)
    # the middle layer of a 5-layer slab, away from its edges, has a full neighbourhood
    mid = (np.abs(bnd[:, 1] - 0.12) < 1e-9) & (np.abs(bnd[:, 0] - 0.155) < 0.021) & (np.abs(bnd[:, 2] - 0.155) < 0.021)
    assert np.allclose(psi[mid] / sc.mass, 1.0, rtol=1e-12)


def test_fluid_on_a_slab():
    sc = scene()
    bnd = lat(14, 2, 14, (0.1, 0.11, 0.1))
    fluid = lat(14, 6, 14, (0.1, 0.13, 0.1))
    rho, _ = densities(sc, fluid, bnd)
    ctr = (np.abs(fluid[:, 0] - 0.165) < 0.03) & (np.abs(fluid[:, 2] - 0.165) < 0.03)
    first = rho[ctr & (np.abs(fluid[:, 1] - 0.13) < 1e-9)] / sc.rho0
    second = rho[ctr & (np.abs(fluid[:, 1] - 0.14) < 1e-9)] / sc.rho0
    assert np.all(np.abs(first - 1.045) < 0.005)
    assert np.allclose(second, 1.0, rtol=1e-12)


def test_mirrored_pressure_pushes_off_the_wall():
    # fluid at uniform pressure on a slab: the boundary's own share of the
    # bottom layer's pressure force points away from the slab (+y), and
    # vanishes two spacings up
    sc = scene()
    bnd = lat(14, 2, 14, (0.1, 0.11, 0.1))
    fluid = lat(14, 4, 14, (0.1, 0.13, 0.1))
    n = len(fluid)
    rho, psi = densities(sc, fluid, bnd)
    p = np.full(n, 1000.0)
    cnt, lists = oracle.neighbors(sc.replace(n=n), fluid)
    f = np.ascontiguousarray(fluid, np.float64)
    bp = np.ascontiguousarray(bnd, np.float64)

    def force(with_boundary):
        Pp = oracle.params(sc.replace(n=n))
        if with_boundary:
            Pp.n_bnd, Pp.bnd_pos, Pp.bnd_psi = len(bnd), bp.ctypes.data, psi.ctypes.data
        out = np.zeros((n, 3))
        oracle.lib().orc_pressure_force(ctypes.byref(Pp), oracle._ptr(f), oracle._ptr(rho), oracle._ptr(p),
                                        oracle._ptr(cnt), oracle._ptr(np.ascontiguousarray(lists)), lists.shape[1],
                                        oracle._ptr(out))
        return out

    fb = force(True) - force(False)
    ctr = (np.abs(fluid[:, 0] - 0.165) < 0.03) & (np.abs(fluid[:, 2] - 0.165) < 0.03)
    bottom = ctr & (np.abs(fluid[:, 1] - 0.13) < 1e-9)
    third = ctr & (np.abs(fluid[:, 1] - 0.15) < 1e-9)
    assert np.all(fb[bottom, 1] > 0)
    assert np.allclose(fb[bottom, 0], 0, atol=1e-9 * fb[bottom, 1].max())
    assert np.all(fb[third] == 0)


def sphere_scene():
    # a 0.08 m sphere 1.5 cm from the block's face, level with it
    sc = P.dam_break((10, 16, 10), S, (0.6, 0.5, 0.4), H, dt=5e-4, seed=3, jitter=1e-4)
    centre, radius = (0.185, 0.09, 0.1), 0.08
    return sc, centre, radius, P.sphere_shell(centre, radius, S)


def test_dam_break_stays_out_of_the_sphere():
    # The collapsing block reaches the sphere after ~250 steps. The shell's
    # outer layer lies 0.07-0.08 m from the centre: with the boundary no
    # fluid particle comes closer than 0.078 m in 350 steps; without it the
    # same run puts particles inside 0.075 m.
    sc, centre, radius, bnd = sphere_scene()
    pos = oracle.scene_positions(sc).astype(np.float64)
    with_b = oracle.OracleSim(sc, pos, boundary=bnd.astype(np.float64))
    without = oracle.OracleSim(sc, pos)
    dmin = {True: np.inf, False: np.inf}
    for sim, key in ((with_b, True), (without, False)):
        sim.presolve(32)
        for _ in range(350):
            sim.step()
            dmin[key] = min(dmin[key], np.linalg.norm(sim.pos - np.asarray(centre), axis=1).min())
    assert dmin[True] > radius - 0.2 * S
    assert dmin[False] < radius - 0.5 * S


@pytest.mark.gpu
def test_gpu_psi_matches_oracle():
    sc, centre, radius, bnd = sphere_scene()
    with P.Simulation(sc) as sim:
        sim.set_boundary(bnd)
        got = sim.boundary_psi()
    want = oracle.boundary_psi(sc, bnd.astype(np.float64))
    assert np.max(np.abs(got - want) / want) < 1e-6


@pytest.mark.gpu
def test_gpu_sphere_dam_break_matches_oracle():
    """Per-step parity with the oracle (each step from the GPU's own state,
    as in tests/test_gpu_parity.py), with the sphere close enough that the
    block's face is within h of its outer layer from the first step."""
    from test_gpu_parity import TOL_P_CONFIG_PCI, TOL_V_CONFIG_PCI, _compare_step, _sync_oracle_from_gpu
    sc, _, radius, _ = sphere_scene()
    centre = (0.175, 0.09, 0.1)
    bnd = P.sphere_shell(centre, radius, S)
    pos = P.scene_positions(sc)
    d_bnd = np.min(np.linalg.norm(pos[:, None, :] - bnd[None, :, :], axis=2), axis=1)
    assert (d_bnd < H).sum() > 20          # the boundary terms are active
    sim = P.Simulation(sc)
    sim.upload(pos)
    sim.set_boundary(bnd)
    orc = oracle.OracleSim(sc, pos.astype(np.float64), float_state=True, boundary=bnd.astype(np.float64))
    for _ in range(4):
        x0 = orc.pos.copy()
        sim.step(1)
        so = orc.step()
        sg = sim.stats()
        if sg.iters == so.iters:
            # Each correction adds delta (rho* - rho0). The FP32 Kahan densities
            # agree with FP64 to ~2e-7 relative, so after k corrections the
            # pressures can differ by k delta 2e-7 rho0 (delta = 546 Pa per
            # kg/m^3 here: 0.1 Pa per correction), more than 1e-4 of the
            # field's max while the first steps' pressures are still small.
            p_abs = max(sg.iters, 1) * oracle.pci_delta(sc) * 2e-7 * sc.rho0
            p_tol = max(TOL_P_CONFIG_PCI, p_abs / max(np.max(np.abs(orc.p)), 1e-300))
            _compare_step(sim, orc, x0, p_tol=p_tol, v_tol=TOL_V_CONFIG_PCI)
        else:
            k = min(sg.iters, so.iters)
            assert abs(so.err[k] - sc.eta) <= 2e-6
        _sync_oracle_from_gpu(orc, sim.download())
    sim.close()
