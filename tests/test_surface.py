"""Iso field and marching cubes.

The reference's own kernels pin the oracle, on the CPU where oracle/_ref is
built:
  * evaluateIso_Kernel (UniformGridKernel.cu:98-138): same values to 1e-12;
  * polygonize_MarchingCube_Kernel (MarchingCube_Kernel.cu:36-160): the same
    vertex set (same edges, same interpolation) and the same triangle count;
    the triangles differ because the case table here is generated, not
    copied, so the total area is compared (1e-3).

Known answers on the oracle (no reference needed):
  * the generated table uses exactly the active edges of every case, at most
    5 triangles each;
  * on a field below the level at the grid's border, the mesh is closed
    (every edge in two triangles, never twice in the same direction) and
    every normal points toward lower values;
  * a sphere of radius R extracted from the distance field has area 4 pi R^2
    (second-order in the spacing).

On the GPU: the iso field against the oracle (1e-12 relative in the config
profile, both sum in FP64 in the same order; 1e-6 in the reference profile,
whose terms are float powf values), and the surface against the oracle:
identical triangle index lists and vertices within FP32 rounding.
"""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P

EDGE = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def blobs_field(nodes, centres, w=0.02):
    return sum(np.exp(-np.sum((nodes - c) ** 2, 1) / w) for c in centres)


def area(tri_pts):
    return 0.5 * np.linalg.norm(np.cross(tri_pts[:, 1] - tri_pts[:, 0], tri_pts[:, 2] - tri_pts[:, 0]), axis=1).sum()


def test_generated_table_uses_exactly_the_active_edges():
    ntri, tri = oracle.mc_table()
    assert ntri[0] == 0 and ntri[255] == 0 and ntri.max() <= 5
    for cs in range(256):
        act = {e for e, (a, b) in enumerate(EDGE) if ((cs >> a) & 1) != ((cs >> b) & 1)}
        used = set(int(x) for x in tri[cs][:3 * ntri[cs]])
        assert used == act, cs


def test_closed_oriented_surface():
    g = oracle.iso_grid((0, 0, 0), 0.04, (25, 25, 25))
    nodes = oracle.grid_nodes(g)
    cen = np.random.default_rng(1).uniform(0.35, 0.6, (5, 3))
    field = blobs_field(nodes, cen, w=0.01)
    v, t = oracle.marching_cubes(g, field, 0.5)
    assert len(t) > 100
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    _, cnt = np.unique(np.sort(e, 1), axis=0, return_counts=True)
    assert np.all(cnt == 2)
    _, dcnt = np.unique(e, axis=0, return_counts=True)
    assert np.all(dcnt == 1)
    n = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    c = v[t].mean(1)
    eps = 1e-4      # gradient of the same field by central differences
    grad = np.stack([(blobs_field(c + eps * np.eye(3)[a], cen, 0.01) - blobs_field(c - eps * np.eye(3)[a], cen, 0.01))
                     for a in range(3)], 1)
    assert np.mean(np.sum(n * grad, 1) < 0) > 0.999


def test_sphere_area_converges():
    R = 0.3
    errs = []
    for m in (24, 48):
        sp = 1.0 / (m - 1)
        g = oracle.iso_grid((-0.5, -0.5, -0.5), sp, (m, m, m))
        nodes = oracle.grid_nodes(g)
        v, t = oracle.marching_cubes(g, R - np.linalg.norm(nodes, axis=1), 0.0)
        errs.append(abs(area(v[t]) - 4 * np.pi * R ** 2) / (4 * np.pi * R ** 2))
    assert errs[1] < 0.01 and errs[1] < errs[0] / 2.5


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
def test_iso_field_matches_reference():
    sc = P.ref_scene(seed=3, jitter=2e-3)
    pos = oracle.scene_positions(sc).astype(np.float64)
    g = oracle.iso_grid((0.0, 0.0, 0.0), 0.011, (20, 18, 16), scale=0.65)
    ref = oracle.RefSim(sc, pos)
    want = ref.iso(g)
    got = oracle.iso_field(sc, pos, None, g)
    assert want.max() > 1.0
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


@needs_ref
def test_marching_cubes_vertices_match_reference():
    g = oracle.iso_grid((0, 0, 0), 0.05, (20, 18, 16))
    nodes = oracle.grid_nodes(g)
    field = blobs_field(nodes, np.random.default_rng(0).uniform(0.2, 0.7, (6, 3)))
    v, t = oracle.marching_cubes(g, field, 0.5)
    rv = oracle.ref_marching_cubes(g, field, 0.5)
    assert len(rv) == 3 * len(t)
    ours = np.unique(np.round(v, 12), axis=0)
    theirs = np.unique(np.round(rv, 12), axis=0)
    assert np.array_equal(ours, theirs)
    assert abs(area(v[t]) - area(rv.reshape(-1, 3, 3))) <= 1e-3 * area(rv.reshape(-1, 3, 3))


def sph_surface_case(profile):
    if profile == "ref":
        sc = P.ref_scene(seed=3, jitter=2e-3)
        g = P.iso_grid((0.0, 0.0, 0.0), 0.011, (28, 24, 20), scale=0.65)
        level = 4.0
    else:
        sc = P.dam_break((16, 14, 12), 0.005, (0.2, 0.2, 0.2), 0.01, seed=9, jitter=2e-4)
        g = P.iso_grid((0.0, 0.0, 0.0), 0.004, (30, 26, 24))
        level = 0.5
    return sc, g, level


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["ref", "config"])
def test_gpu_iso_and_surface_match_oracle(profile):
    sc, g, level = sph_surface_case(profile)
    pos = P.scene_positions(sc)
    with P.Simulation(sc) as sim:
        sim.upload(pos)
        iso = sim.iso_field(g)
        vert, tri = sim.extract_surface(g, level)
        rho = sim.read_field(P.runtime.FIELD_DENSITY)
    og = oracle.iso_grid(list(g.origin), list(g.spacing), list(g.dims), g.scale)
    want = oracle.iso_field(sc, pos.astype(np.float64), rho.astype(np.float64), og)
    tol = 1e-6 if profile == "ref" else 1e-12
    assert np.max(np.abs(iso - want)) <= tol * np.max(np.abs(want))
    # the surface of the GPU's own field: identical topology, FP32 vertices
    ov, ot = oracle.marching_cubes(og, iso, level)
    assert len(tri) > 50
    assert np.array_equal(tri, ot)
    assert np.max(np.abs(vert - ov)) <= 2 * np.spacing(np.float32(np.max(np.abs(ov))))
