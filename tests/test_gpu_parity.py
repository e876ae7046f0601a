"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Tolerances (written here, applied below):
  * cell keys, sorted order (stable on particle id) and neighbour counts:
    bit-exact;
  * density: 1e-5 relative, element-wise;
  * pressure and non-pressure forces: 1e-5 relative to the field's max
    magnitude (FP32 arithmetic against FP64; PCISPH pressure increments
    come from rho* - rho0, a cancellation, so a norm-wise bound is the
    meaningful one);
  * velocities after a step: 3e-5 of the field's max. The pressure
    acceleration is a sum of ~30 pair terms that cancel: under the
    reference's soft EOS the free surface is in tension and pair terms reach
    ~50x the net force, so ~2.4e-7 of rounding per FP32 term leaves
    ~1.5e-5 of the net (measured: 1.4e-5 WCSPH against the reference's own
    kernels, 2.1e-5 config PCISPH against the oracle);
  * positions: within 4 float ulps of the coordinate magnitude plus 1e-5 of
    the step's displacement;
  * PCISPH velocities of the few particles that one side clamped to a
    projection bound (box +- r) and the other did not are not compared: the
    projection is a threshold, a prediction within rounding of the bound
    falls on either side, and the clamped copy loses its normal velocity;
  * pressure after a multi-iteration config-profile PCISPH step: 1e-4 of its
    max. The pressure accumulates delta (rho* - rho0) over the corrections;
    an FP32 rounding of 3e-8 of a density-level term (kernel constant, wall
    term) is 3e-5 kg/m^3 of rho* - rho0, times delta ~ 34 and 4-5
    corrections: ~4e-5 of the pressure scale. The velocities of such a step
    carry that pressure's error (a_p is linear in p): 1e-4 as well;
  * reference-profile PCISPH pressure against the reference's own kernels:
    2e-5 of its max. Those kernels keep x* in FP64; the GPU stores x* in
    FP32, a half-ulp of 3.7e-9 m at 0.1 m. At h = 0.02, m = 1e-3 one pair
    moves rho by 1.6e4 kg/m^3 per metre at r = h/2, so ~30 pairs with
    independent roundings move rho* by ~5e-4 kg/m^3, 1-2e-5 of the step's
    rho* - rho0 of a few tens of kg/m^3, which the pressure increment
    inherits. The oracle, which rounds x* to FP32 like the GPU, agrees to
    1e-5 on the same step.
The oracle runs with float_state=True (it rounds every array the GPU stores
in FP32 at the same points) for multi-step comparisons.
"""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import runtime as R
from psb_project_b200.scene import PCISPH, PROFILE_CONFIG, PROFILE_REF, WCSPH

pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_V = 3e-5
TOL_P_CONFIG_PCI = 1e-4
TOL_V_CONFIG_PCI = 1e-4
TOL_P_REF_FP64 = 2e-5


def rel_norm(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def assert_positions(x_gpu, x_orc, x0):
    ulp = np.spacing(np.float32(np.max(np.abs(x_orc))))
    disp = np.max(np.abs(x_orc - x0))
    err = np.max(np.abs(np.asarray(x_gpu, np.float64) - x_orc))
    assert err <= 4 * float(ulp) + TOL * disp, (err, ulp, disp)


def small_config_scene(method=PCISPH, nxyz=(24, 20, 16), spacing=0.005, h=0.01, box=(0.5, 0.4, 0.3), dt=1e-3, seed=11):
    return P.dam_break(nxyz, spacing, box, h, method=method, dt=dt, seed=seed)


def upload(sc, pos=None):
    sim = P.Simulation(sc)
    pos = P.scene_positions(sc) if pos is None else pos
    sim.upload(pos)
    return sim, pos


# ---- grid: keys, sort, neighbours ------------------------------------------

@pytest.mark.parametrize("name", ["C0", "ref"])
def test_keys_sort_neighbours_bit_exact(name):
    sc = P.config_scene("C0") if name == "C0" else P.ref_scene()
    sim, pos = upload(sc)
    sim.build_neighbors()
    pos64 = pos.astype(np.float64)
    keys = oracle.cell_keys(sc, pos64)
    perm = oracle.sort_perm(keys)
    counts, _ = oracle.neighbors(sc, pos64, with_lists=False)
    assert np.array_equal(sim.read_field(R.FIELD_CELL_KEY), keys)
    assert np.array_equal(sim.read_field(R.FIELD_SORTED_ID), perm)
    assert np.array_equal(sim.read_field(R.FIELD_SORTED_KEY), keys[perm])
    assert np.array_equal(sim.read_field(R.FIELD_NBR_COUNT), counts)
    st = sim.stats()
    assert st.nbr_max == counts.max() and st.nbr_total == counts.sum()
    sim.close()


def test_neighbour_cutoff_borderline_pairs():
    """Pairs at float-rounded distances h*(1 +- k ulp): the FP32 guard band
    must hand them to the FP64 test and agree with the reference's
    sqrt(d.d) <= h on every one."""
    sc = P.ref_scene()
    rng = np.random.default_rng(5)
    base = rng.uniform(0.05, 0.25, size=(400, 3))
    d = rng.normal(size=(400, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    scale = sc.h * (1.0 + rng.integers(-8, 9, size=(400, 1)) * 1e-8)
    pos = np.concatenate([base, base + d * scale]).astype(np.float32)
    sc = sc.replace(n=pos.shape[0])
    sim, _ = upload(sc, pos)
    sim.build_neighbors()
    counts, _ = oracle.neighbors(sc, pos.astype(np.float64), with_lists=False)
    assert np.array_equal(sim.read_field(R.FIELD_NBR_COUNT), counts)
    ref = oracle.RefSim(sc, pos.astype(np.float64)) if oracle.ref_available() else None
    if ref is not None:
        assert np.array_equal(ref.search(), counts)
    sim.close()


def test_particles_outside_grid_are_clamped():
    sc = P.ref_scene()
    pos = P.scene_positions(sc)
    pos[:7] = np.array([[-5.0, 0.1, 0.1], [0.1, 9.0, 0.1], [0.1, 0.1, -1.0], [3, 3, 3], [np.inf, 0, 0],
                        [0.1, -np.inf, 0.1], [0.1, 0.1, 1e30]], np.float32)
    sim, _ = upload(sc, pos)
    sim.build_neighbors()
    assert sim.stats().clamped == 7
    keys = oracle.cell_keys(sc, pos.astype(np.float64))
    assert np.array_equal(sim.read_field(R.FIELD_CELL_KEY), keys)
    sim.close()


# ---- density and single steps --------------------------------------------------

@pytest.mark.parametrize("profile", [PROFILE_REF, PROFILE_CONFIG])
def test_density_at_start_positions(profile):
    sc = P.ref_scene() if profile == PROFILE_REF else small_config_scene()
    sim, pos = upload(sc)
    sim.build_neighbors()
    counts, lists = oracle.neighbors(sc, pos.astype(np.float64))
    rho = oracle.density(sc, pos.astype(np.float64), counts, lists, clamp=(profile == PROFILE_CONFIG))
    got = sim.read_field(R.FIELD_DENSITY_X).astype(np.float64)
    assert np.max(np.abs(got - rho) / rho) <= TOL
    sim.close()


def on_projection_bound(sc, x):
    """Per particle and axis: the coordinate sits exactly on a projection
    bound (box +- particle_radius, as float), where the projection clamps it."""
    x = np.asarray(x, np.float64)
    lo = (np.asarray(sc.box_min, np.float32) + np.float32(sc.particle_radius)).astype(np.float64)
    hi = (np.asarray(sc.box_max, np.float32) - np.float32(sc.particle_radius)).astype(np.float64)
    return (x == lo) | (x == hi)


def projection_disagrees(sc, x_gpu, x_orc):
    """Particles that one side clamped to a bound and the other did not: the
    projection is a threshold, and a prediction within rounding of the
    bound falls on either side of it; the clamped copy also loses its normal
    velocity. Those particles are compared by position only."""
    return np.any(on_projection_bound(sc, x_gpu) != on_projection_bound(sc, x_orc), axis=1)


def _compare_step(sim, orc, x0, p_tol=TOL, v_tol=TOL_V):
    out = sim.download()
    assert_positions(out["pos"], orc.pos, x0)
    sc = orc.scene
    keep = ~projection_disagrees(sc, out["pos"], orc.pos) if sc.method == PCISPH else np.ones(len(orc.pos), bool)
    assert (~keep).sum() <= max(2, 0.002 * len(keep))
    assert rel_norm(out["vel_half"][keep], orc.vel_half[keep]) <= v_tol
    assert rel_norm(out["vel"][keep], orc.vel[keep]) <= v_tol
    assert np.max(np.abs(out["density"] - orc.rho) / np.abs(orc.rho)) <= TOL
    assert rel_norm(out["pressure"], orc.p) <= p_tol
    assert rel_norm(sim.read_field(R.FIELD_FORCE_NP), orc.f_np) <= TOL
    assert np.array_equal(sim.read_field(R.FIELD_NBR_COUNT), orc.nbr)


def _sync_oracle_from_gpu(orc, out):
    """Per-step parity: the oracle continues from the GPU's own FP32 state."""
    orc.pos[:] = out["pos"]
    orc.vel[:] = out["vel"]
    orc.vel_half[:] = out["vel_half"]
    orc.p[:] = out["pressure"]


@pytest.mark.parametrize("method", [PCISPH, WCSPH])
def test_reference_profile_steps(method):
    """Reference-compatible physics, 3 steps. Each step starts the FP64
    oracle and the reference's own kernels (where built) from the GPU's FP32
    state, so every comparison is one step from identical inputs."""
    sc = P.ref_scene(method=method)
    sim, pos = upload(sc)
    orc = oracle.OracleSim(sc, pos, float_state=True)
    have_ref = oracle.ref_available()
    state = sim.download()
    for _ in range(3):
        x0 = orc.pos.copy()
        ref = oracle.RefSim(sc, state["pos"].astype(np.float64), state["vel"], state["vel_half"]) if have_ref else None
        sim.step(1)
        orc.step()
        _compare_step(sim, orc, x0)
        out = sim.download()
        if ref is not None:
            ref.pcisph_update() if method == PCISPH else ref.wcsph_update()
            assert rel_norm(out["vel_half"], ref.get("vel_ap", 3)) <= TOL_V
            assert rel_norm(out["vel"], ref.get("vel", 3)) <= TOL_V
            assert np.max(np.abs(out["density"] - ref.get("density", 1)) / ref.get("density", 1)) <= TOL
            assert rel_norm(out["pressure"], ref.get("pressure", 1)) <= TOL_P_REF_FP64
        _sync_oracle_from_gpu(orc, out)
        state = out
    if method == PCISPH:
        assert sim.stats().iters == 3
    sim.close()


def test_config_pcisph_steps_and_iterations():
    """Config physics (eta loop), 5 steps, each from the GPU's own state. The
    iteration counts agree unless the deciding error sits within 2e-6 of eta
    (FP32 against FP64), in which case the step is resynchronised."""
    sc = small_config_scene()
    sim, pos = upload(sc)
    orc = oracle.OracleSim(sc, pos, float_state=True)
    for _ in range(5):
        x0 = orc.pos.copy()
        sim.step(1)
        so = orc.step()
        sg = sim.stats()
        for k in range(min(so.iters, sg.iters) + 1):
            assert abs(sg.err[k] - so.err[k]) <= 1e-5, (k, sg.err[k], so.err[k])
        if sg.iters != so.iters:
            k = min(sg.iters, so.iters)
            assert abs(so.err[k] - sc.eta) <= 2e-6, (sg.iters, so.iters, so.err[k])
        else:
            assert sg.converged == so.converged
            _compare_step(sim, orc, x0, p_tol=TOL_P_CONFIG_PCI, v_tol=TOL_V_CONFIG_PCI)
        _sync_oracle_from_gpu(orc, sim.download())
    sim.close()


def test_config_wcsph_steps():
    sc = P.config_scene("C0")
    sim, pos = upload(sc)
    orc = oracle.OracleSim(sc, pos, float_state=True)
    for _ in range(3):
        x0 = orc.pos.copy()
        sim.step(1)
        orc.step()
        _compare_step(sim, orc, x0)
    sim.close()


def test_trajectory_50_steps_wcsph():
    """50 steps of the 16,384-particle WCSPH dam break: the trajectory stays
    on the FP64 oracle's to 1e-4 of the travelled distance."""
    sc = P.config_scene("C0")
    sim, pos = upload(sc)
    orc = oracle.OracleSim(sc, pos, float_state=False)
    sim.step(50)
    for _ in range(50):
        orc.step()
    out = sim.download()
    travel = np.max(np.abs(orc.pos - pos))
    err = np.max(np.abs(out["pos"] - orc.pos))
    assert err <= 1e-4 * travel + 4 * float(np.spacing(np.float32(1.0))), (err, travel)
    assert rel_norm(out["vel"], orc.vel) <= 1e-4
    sim.close()


# ---- behaviour ----------------------------------------------------------------

def test_deterministic_bitwise():
    sc = small_config_scene()
    res = []
    for _ in range(2):
        sim, _ = upload(sc)
        sim.step(3)
        out = sim.download()
        res.append(out)
        sim.close()
    for k in res[0]:
        assert np.array_equal(res[0][k].view(np.uint32), res[1][k].view(np.uint32)), k


def test_neighbour_overflow_is_a_status():
    sc = small_config_scene().replace(nbr_cap=8)
    sim, _ = upload(sc)
    with pytest.raises(R.PsbError) as e:
        sim.step(1)
    assert e.value.status == R.EOVERFLOW_NBR
    sim.close()


def test_aos_f64_roundtrip():
    sc = P.ref_scene()
    pos = P.scene_positions(sc).astype(np.float64) + 1e-9
    vel = np.random.default_rng(1).normal(size=pos.shape)
    sim = P.Simulation(sc)
    sim.upload_aos_f64(pos, vel, vel)
    out = sim.download_aos_f64()
    assert np.array_equal(out["pos"], pos.astype(np.float32).astype(np.float64))
    assert np.array_equal(out["vel"], vel.astype(np.float32).astype(np.float64))
    sim.close()


def test_noconvergence_reports_status():
    sc = small_config_scene().replace(eta=1e-9, max_iters=4)
    sim, _ = upload(sc)
    assert sim.step(1) == R.ENOCONV
    st = sim.stats()
    assert st.iters == 4 and st.converged == 0
    sim.close()


def test_bad_scene_rejected():
    sc = small_config_scene().replace(max_iters=1000)
    with pytest.raises(R.PsbError) as e:
        P.Simulation(sc)
    assert e.value.status == R.EINVAL


def test_presolve_matches_oracle():
    """Initial-pressure solve: 40 corrector passes at the start state. The
    pressure after each pass builds on the last, so the FP32 bound of the
    multi-iteration pressure applies."""
    sc = small_config_scene().replace(warm_start=P.WARM_PREVIOUS)
    sim, pos = upload(sc)
    sim.presolve(40)
    orc = oracle.OracleSim(sc, pos, float_state=True)
    orc.presolve(40)
    out = sim.download()
    assert rel_norm(out["pressure"], orc.p) <= TOL_P_CONFIG_PCI
    assert np.array_equal(out["pos"], pos)          # the state itself is untouched
    sim.close()


def test_config_pcisph_warm_started_steps():
    """Steps after a pressure pre-solve with the previous-step warm start."""
    sc = small_config_scene().replace(warm_start=P.WARM_PREVIOUS)
    sim, pos = upload(sc)
    sim.presolve(20)
    orc = oracle.OracleSim(sc, pos, float_state=True)
    orc.p[:] = sim.download()["pressure"]
    for _ in range(4):
        x0 = orc.pos.copy()
        sim.step(1)
        so = orc.step()
        sg = sim.stats()
        if sg.iters == so.iters:
            _compare_step(sim, orc, x0, p_tol=TOL_P_CONFIG_PCI, v_tol=TOL_V_CONFIG_PCI)
        else:
            k = min(sg.iters, so.iters)
            assert abs(so.err[k] - sc.eta) <= 2e-6
        _sync_oracle_from_gpu(orc, sim.download())
    sim.close()
