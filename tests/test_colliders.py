"""Collision objects: the reference's plane, sphere, cylinder, triangle mesh
and height fields (src/Kernel/Collision/*), as their kernels execute.

CPU:
  * the oracle's restatement (orc_collide) equals the reference's own
    kernels compiled for the host (oracle/_ref, through the launch each
    reference launcher makes), bit for bit, for every object type on random
    particles, moving and not;
  * known answers on the oracle: a particle falling through a floor plane
    stops where it crossed, with its normal velocity gone (elast 0) or
    reflected by (1 + r); a sphere keeps particles inside it, the swapped
    launch arguments making even container = false a container whose
    restitution divides by zero (non-finite, which psb_set_colliders
    refuses); the mesh puts a particle that sank through a floor as far
    above its start as it sank (its contact formula measures from the new
    position and applies at the old one); a height field lifts a particle
    to h(x, z) + min.y.
GPU:
  * the compat launchers (include/psb_compat.h; FP64 state, the reference's
    AoS layout) against the oracle, which equals the reference: within 1e-6
    of each particle's scale (the float arithmetic the reference keeps
    rounds differently with the GPU's fused multiply-adds);
  * the native FP32 path inside DEM steps (spheres falling onto each object)
    and a reference-profile PCISPH dam break with a floor plane, a bump and
    a sphere in the tank, each step from the GPU's own state, against the
    oracle stepping with the same objects (positions 4 ulps + 1e-5 of the
    displacement, plus 8 float ulps of the distance to a plane's corner;
    velocities 1e-4 of the field max). Not compared: particles moving
    almost parallel to a plane, whose contact point t = ((A - x).N)/(dir.N)
    is ill-conditioned in the reference's float arithmetic;
  * invalid objects are refused with PSB_EINVAL.
"""
import ctypes

import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import colliders as C
from psb_project_b200 import runtime as R

DT = 0.005


def objects():
    floor = [(-1, -0.1, -1), (1, -0.1, -1), (1, -0.1, 1), (-1, -0.1, 1)]
    mesh_v = np.array([[-1, -0.1, -1], [1, -0.1, -1], [1, -0.1, 1], [-1, -0.1, 1],
                       [-1, 0.3, -1], [1, 0.5, -1], [0, 0.4, 1]], np.float64)
    return {
        "plane": C.plane(*[(-2, 0, -2), (2, 0, -2), (2, 0, 2), (-2, 0, 2)], (0, 1, 0), elast=0.5),
        "plane_tilted": C.plane((-2, -0.2, -2), (2, 0.2, -2), (2, 0.2, 2), (-2, -0.2, 2), (-0.0995, 0.995, 0),
                                elast=0.5),
        "plane_finite": C.plane(*floor, (0, 1, 0)),
        "sphere": C.sphere((0.1, 0, 0), 0.8, elast=0.4),
        "sphere_c0": C.sphere((0.1, 0, 0), 0.8, elast=0.0, container=False),
        "cylinder_y": C.cylinder((0, 0, 0), (0, 1, 0), 0.7, 1.2),
        "cylinder_x": C.cylinder((0.05, 0.02, 0), (1, 0, 0), 0.75, 1.0),
        "mesh": C.mesh(mesh_v, [[0, 2, 1], [0, 3, 2], [4, 6, 5]]),
        "height_linear": C.height((-0.9, -0.2, -0.9), (0.9, 0, 0.9), [C.linear(0.2, -0.1)], elast=0.3),
        "height_gaussian": C.height((-0.9, -0.3, -0.9), (0.9, 0, 0.9), [C.gaussian(0.4, 0.1, -0.2, 0.3, 0.5)],
                                    elast=0.3),
        "height_periodic": C.height((-0.9, -0.1, -0.9), (0.9, 0, 0.9),
                                    [C.cosine(0.1, 4, 0.3, 0.2), C.cosine(0.05, 7, 1.1, 0.5)], elast=0.3),
    }


def particles(n=3000, seed=0, still=0):
    rng = np.random.default_rng(seed)
    xo = rng.uniform(-1, 1, (n, 3))
    v = rng.normal(0, 1, (n, 3))
    x = xo + v * 0.01
    if still:
        x[:still] = xo[:still]
    return xo, x, v


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", sorted(objects()))
def test_oracle_equals_reference_kernels(name):
    spec = objects()[name].oracle_spec()
    xo, x, v = particles(still=50)
    if spec[0] == C.PLANE:          # the reference divides by zero for a particle that did not move
        xo, x, v = particles()
    a, b, hits = oracle.collide(spec, xo, x, v, DT)
    c, d = oracle.ref_collide(spec, xo, x, v, DT, particle_radius=0.01)
    assert hits > 100
    assert np.array_equal(a, c) and np.array_equal(b, d)


def test_plane_known_answers():
    spec = C.plane((-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1), (0, 1, 0)).oracle_spec()
    xo = np.array([[0.2, 0.05, 0.3], [0.5, 0.01, -0.2], [3.0, 0.01, 0.0]])
    v = np.array([[0.1, -2.0, 0.0], [0.0, -3.0, 0.0], [0.0, -3.0, 0.0]])
    x = xo + v * 0.05
    a, b, hits = oracle.collide(spec, xo, x, v, DT)
    assert hits == 2                                        # the third lies off the quad
    t = xo[:2, 1] / -v[:2, 1]                               # where each crossed y = 0
    assert np.allclose(a[:2], xo[:2] + v[:2] * t[:, None], atol=1e-7)
    assert np.allclose(b[:2, 1], 0) and np.allclose(b[:2, [0, 2]], v[:2, [0, 2]])
    e = 0.5
    bounce = C.plane((-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1), (0, 1, 0), elast=e).oracle_spec()
    _, b2, _ = oracle.collide(bounce, xo[:1], x[:1], v[:1], DT)
    r = e * np.linalg.norm(x[0] - a[0]) / (DT * np.linalg.norm(v[0]))
    assert b2[0, 1] == pytest.approx(r * 2.0, rel=1e-6)     # v_n -> -r v_n


def test_sphere_is_always_a_container():
    for container in (True, False):
        spec = C.sphere((0, 0, 0), 0.5, elast=0.0, container=container).oracle_spec()
        xo, x, v = particles(500, seed=3)
        a, _, _ = oracle.collide(spec, xo, x, v, DT)
        assert np.all(np.linalg.norm(a, axis=1) <= 0.5 + 1e-12)
        inside = np.linalg.norm(x, axis=1) < 0.5
        assert np.array_equal(a[inside], x[inside])         # particles inside are left alone
    spec = C.sphere((0, 0, 0), 0.5, elast=0.3, container=False).oracle_spec()
    xo, x, v = particles(200, seed=4)
    _, b, hits = oracle.collide(spec, xo, x, v, DT)
    moved = np.linalg.norm(x, axis=1) > 0.5
    assert hits == moved.sum() and not np.all(np.isfinite(b[moved]))


def test_mesh_contact_formula():
    spec = C.mesh([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], [[0, 2, 1], [0, 3, 2]]).oracle_spec()
    xo = np.array([[0.1, 0.02, 0.2]])
    v = np.array([[0.0, -1.0, 0.0]])
    x = xo + v * 0.05                                       # 3 cm below the floor
    a, b, hits = oracle.collide(spec, xo, x, v, DT)
    assert hits == 1
    assert a[0, 1] == pytest.approx(0.02 + 0.03, abs=1e-12)  # above its start by the depth it sank
    assert b[0, 1] == 0.0


def test_height_field_lifts_to_surface():
    spec = C.height((-1, -0.5, -1), (1, 0, 1), [C.gaussian(0.3, 0.0, 0.0, 0.2, 0.2)]).oracle_spec()
    xo = np.array([[0.05, -0.2, 0.02], [0.5, -0.49, 0.5]])   # both end below the surface
    v = np.array([[0.0, -1.0, 0.0], [0.0, -1.0, 0.0]])
    x = xo + v * 0.02
    a, b, hits = oracle.collide(spec, xo, x, v, DT)
    h = -0.5 + 0.3 * np.exp(-(x[:, 0] ** 2 / 0.08 + x[:, 2] ** 2 / 0.08))
    assert hits == 2 and np.allclose(a[:, 1], h, rtol=1e-6)
    assert np.all(b[:, 1] > -1.0)                           # the normal part is gone


# ---- GPU ---------------------------------------------------------------------------

class Vec3(ctypes.Structure):
    _fields_ = [("e", ctypes.c_double * 3)]


# The launchers take the reference's Vector3 by value; its user-provided
# copy constructor makes the C++ ABI pass it through a hidden pointer, so a
# C caller (ctypes here) passes a pointer to the three doubles.
PV3 = ctypes.POINTER(Vec3)


def _v3(a):
    return ctypes.pointer(Vec3((ctypes.c_double * 3)(*[float(t) for t in a])))


def _compat(lib, name, spec, xo, x, v, dt, torch):
    typ, vv, elast, container, faces, terms = spec
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    to, tx, tv = d(xo), d(x), d(v)
    V = ctypes.c_void_p
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    fl, I, U = ctypes.c_float, ctypes.c_int, ctypes.c_uint
    keep = []
    if typ == C.PLANE:
        f = lib.collisionPlan_CUDA
        f.argtypes = [V, V, V, V, PV3, PV3, PV3, PV3, PV3, fl, fl, I]
        f(p(to), p(tx), p(tv), p(tv), *[_v3(vv[3 * k:3 * k + 3]) for k in range(5)], elast, dt, len(x))
    elif typ == C.SPHERE:
        f = lib.collisionSystem_Sphere_CUDA
        f.argtypes = [V, V, V, V, fl, fl, I, PV3, fl, fl, ctypes.c_bool]
        f(p(to), p(tx), p(tv), p(tv), 0.01, dt, len(x), _v3(vv[:3]), vv[3], elast, bool(container))
    elif typ == C.CYLINDER:
        f = lib.collisionCylinder_CUDA
        f.argtypes = [V, V, fl, fl, I, PV3, PV3, ctypes.c_double, ctypes.c_double, fl, ctypes.c_bool]
        f(p(tx), p(tv), 0.01, dt, len(x), _v3(vv[:3]), _v3(vv[3:6]), vv[6], vv[7], elast, True)
    elif typ == C.MESH:
        F = np.asarray(faces, np.float32).reshape(-1, 12)
        parts = [torch.as_tensor(np.ascontiguousarray(F[:, 3 * k:3 * k + 3]), device="cuda") for k in range(4)]
        keep += parts
        f = lib.collisionMesh_CUDA
        f.argtypes = [V, V, V, V, fl, fl, U, V, V, V, V, fl, I]
        f(p(to), p(tx), p(tv), p(tv), 0.01, dt, F.shape[0], *[p(t) for t in parts], elast, len(x))
    else:
        T = np.asarray(terms, np.float64).reshape(-1, 6)
        mn, mx = _v3(vv[:3]), _v3(vv[3:6])
        if T.shape[0] == 1 and T[0, 0] == C.HEIGHT_LINEAR:
            f = lib.collisionSystem_Linear_HeightFieldCollision_CUDA
            f.argtypes = [V, V, V, V, ctypes.c_double, fl, U, ctypes.c_double, ctypes.c_double, PV3, PV3, fl]
            f(p(to), p(tx), p(tv), p(tv), 0.01, dt, len(x), T[0, 1], T[0, 2], mn, mx, elast)
        elif T.shape[0] == 1 and T[0, 0] == C.HEIGHT_GAUSSIAN:
            f = lib.collisionSystem_Gaussian_HeightFieldCollision_CUDA
            f.argtypes = [V, V, V, V, ctypes.c_double, fl, U] + [ctypes.c_double] * 5 + [PV3, PV3, fl]
            f(p(to), p(tx), p(tv), p(tv), 0.01, dt, len(x), *[float(c) for c in T[0, 1:6]], mn, mx, elast)
        else:
            cols = [d(T[:, k]) for k in (1, 2, 3, 4)]
            keep += cols
            f = lib.collisionSystem_Periodic_HeightFieldCollision_CUDA
            f.argtypes = [V, V, V, V, ctypes.c_double, fl, U, U, V, V, V, V, PV3, PV3, fl]
            f(p(to), p(tx), p(tv), p(tv), 0.01, dt, len(x), T.shape[0], *[p(t) for t in cols], mn, mx, elast)
    f.restype = None
    torch.cuda.synchronize()
    return tx.cpu().numpy(), tv.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(objects()))
def test_gpu_compat_launchers_match_reference(name):
    torch = pytest.importorskip("torch")
    spec = objects()[name].oracle_spec()
    xo, x, v = particles(seed=5)
    want_x, want_v, hits = oracle.collide(spec, xo, x, v, DT)
    got_x, got_v = _compat(R.lib(), name, spec, xo, x, v, DT, torch)
    assert hits > 100
    # float arithmetic of the reference kernels (plane contact, mesh and
    # cylinder distances, the restitution factor) rounds differently with
    # the GPU's fused multiply-adds: a few float ulps of the quantities
    sx = 1.0 + np.abs(want_x - xo).max(1, keepdims=True) + np.abs(xo).max(1, keepdims=True)
    sv = 1.0 + np.abs(want_v).max(1, keepdims=True)
    assert np.all(np.abs(got_x - want_x) <= 1e-6 * sx)
    assert np.all(np.abs(got_v - want_v) <= 1e-6 * sv)


def rain_objects():
    """Objects that spheres falling from y = 0.2 .. 0.3 (x, z within 0.2
    of the axis) meet within 0.16 s."""
    floor = [(-2, 0.05, -2), (2, 0.05, -2), (2, 0.05, 2), (-2, 0.05, 2)]
    fv = np.array([[-1, 0.05, -1], [1, 0.05, -1], [1, 0.05, 1], [-1, 0.05, 1]])
    foot = ((-0.5, 0.0, -0.5), (0.5, 0.0, 0.5))
    return {
        "plane": C.plane(*floor, (0, 1, 0), elast=0.5),
        "plane_tilted": C.plane((-2, -0.15, -2), (2, 0.25, -2), (2, 0.25, 2), (-2, -0.15, 2), (-0.0995, 0.995, 0)),
        "sphere": C.sphere((0, 0.3, 0), 0.25, elast=0.4),
        "cylinder": C.cylinder((0, 0, 0), (0, 1, 0), 0.2, 2.0),
        "mesh": C.mesh(fv, [[0, 2, 1], [0, 3, 2]]),
        "height_linear": C.height(*foot, [C.linear(0.1, -0.05)], elast=0.3),
        "height_gaussian": C.height(*foot, [C.gaussian(0.06, 0.0, 0.0, 0.1, 0.1)]),
        "height_periodic": C.height(*foot, [C.cosine(0.03, 20, 0.3, 0.0), C.cosine(0.02, 31, 1.1, 0.5)], elast=0.2),
    }


def plane_slack(*objs):
    """A plane's contact point goes through float3(x - A) with A its first
    corner (PlaneCollision_Kernel.cu:22-27), so it carries a few float ulps
    of |x - A|, which fused multiply-adds round differently: 8 ulps of the
    corner's distance (2 m here)."""
    if any(o.type == C.PLANE for o in objs):
        return 8 * float(np.spacing(np.float32(3.0)))
    return 0.0


def well_conditioned(obj, x, v, sc):
    """Particles whose contact with a plane is well conditioned this DEM
    step: not behind the plane after the move, or moving at more than 0.1
    (cosine) to it. Sliding along a plane gives t = ((A - x).N)/(dir.N)
    with both terms near zero in the reference's float arithmetic."""
    keep = np.ones(x.shape[0], bool)
    if obj.type != C.PLANE:
        return keep
    g = np.asarray(sc.gravity, np.float64)
    vn = v.astype(np.float64) + g * sc.dt
    xn = x.astype(np.float64) + vn * sc.dt
    A, N = np.asarray(obj.v[:3], np.float64), np.asarray(obj.v[12:15], np.float64)
    behind = (xn - A) @ N <= 0
    cosine = np.abs(vn @ N) / np.maximum(np.linalg.norm(vn, axis=1), 1e-30)
    return ~behind | (cosine > 0.1)


def rain_scene():
    """8 x 3 x 8 spheres 5 cm apart (no contacts), box [-1, 1]^3."""
    sc = P.dem_block((8, 3, 8), 0.05, (0.8, 1.15, 0.8), (2.0, 2.0, 2.0), 0.01, dt=2e-3, seed=9, jitter=0.0)
    pos = (P.scene_positions(sc).astype(np.float64) - 1.0).astype(np.float32)
    sh = lambda a: tuple(float(t) - 1.0 for t in a)
    return sc.replace(box_min=sh(sc.box_min), box_max=sh(sc.box_max), grid_min=sh(sc.grid_min)), pos


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(rain_objects()))
def test_gpu_native_dem_steps_match_oracle(name):
    obj = rain_objects()[name]
    sc, pos = rain_scene()
    vel = np.zeros_like(pos)
    vel[:, 1] = -1.0
    acted = 0
    with P.Simulation(sc) as sim:
        sim.upload(pos, vel)
        sim.set_colliders([obj])
        ref = oracle.OracleSim(sc, pos.astype(np.float64), vel.astype(np.float64), float_state=True,
                               colliders=[obj.oracle_spec()])
        for _ in range(80):
            x0 = sim.download()
            ref.pos[:] = x0["pos"]
            ref.vel[:] = x0["vel"]
            sim.step(1)
            ref.step()
            got = sim.download()
            keep = well_conditioned(obj, x0["pos"], x0["vel"], sc)
            disp = np.abs(ref.pos - x0["pos"]).max()
            ulp = float(np.spacing(np.float32(np.abs(ref.pos).max())))
            assert np.max(np.abs(got["pos"] - ref.pos)[keep]) <= 4 * ulp + 1e-5 * disp + plane_slack(obj)
            assert np.max(np.abs(got["vel"] - ref.vel)[keep]) <= 1e-4 * max(1.0, np.abs(ref.vel).max())
            acted += int(np.sum(np.abs(ref.vel - x0["vel"] - np.array([0.0, -9.81 * sc.dt, 0.0])).max(1) > 1e-3))
    assert acted > 0


@pytest.mark.gpu
def test_gpu_pcisph_with_objects_matches_oracle():
    sc = P.ref_scene((12, 10, 8), seed=21)
    # a floor plane just under the block, a bump in the floor and a sphere
    # that cuts the block's far corners (the radial projection moves them at
    # the first step)
    objs = [C.plane((0.0, 0.0032, 0.0), (0.3, 0.0032, 0.0), (0.3, 0.0032, 0.3), (0.0, 0.0032, 0.3), (0, 1, 0)),
            C.height((0.0, 0.0, 0.0), (0.3, 0.3, 0.3), [C.gaussian(0.05, 0.15, 0.15, 0.05, 0.05)]),
            C.sphere((0.15, 0.15, 0.15), 0.2, elast=0.2)]
    pos = P.scene_positions(sc)
    with P.Simulation(sc) as sim:
        sim.upload(pos)
        sim.set_colliders(objs)
        ref = oracle.OracleSim(sc, pos.astype(np.float64), float_state=True,
                               colliders=[o.oracle_spec() for o in objs])
        for _ in range(5):
            x0 = sim.download()
            for k, a in (("pos", ref.pos), ("vel", ref.vel), ("vel_half", ref.vel_half)):
                a[:] = x0[k]
            sim.step(1)
            ref.step()
            got = sim.download()
            disp = np.abs(ref.pos - x0["pos"]).max()
            ulp = float(np.spacing(np.float32(np.abs(ref.pos).max())))
            assert np.max(np.abs(got["pos"] - ref.pos)) <= 4 * ulp + 1e-5 * disp + plane_slack(*objs)
            assert np.max(np.abs(got["vel_half"] - ref.vel_half)) <= 1e-4 * max(1.0, np.abs(ref.vel_half).max())


@pytest.mark.gpu
def test_gpu_invalid_objects_refused():
    sc = P.ref_scene((4, 4, 4), seed=22)
    with P.Simulation(sc) as sim:
        sim.upload(P.scene_positions(sc))
        bad = [C.sphere((0, 0, 0), 0.1, elast=0.5, container=False),
               C.Collider(C.MESH, [], data=np.zeros((0, 12), np.float32)),
               C.height((0, 0, 0), (1, 1, 1), [(9, 0, 0, 0, 0, 0)]),
               C.Collider(7, [0.0])]
        for b in bad:
            with pytest.raises(R.PsbError):
                sim.set_colliders([b])
        with pytest.raises(R.PsbError):
            sim.set_colliders([C.sphere((0, 0, 0), 0.1)] * 33)
        sim.set_colliders([C.sphere((0.15, 0.15, 0.15), 0.5)])
        sim.step(1)
        sim.set_colliders([])
        sim.step(1)
