"""The reference-signature layer as the reference's own classes use it.

tests/compat_link/reference_caller.cpp is written the way SPHSystem,
PCI_SPHSystem, CudaSystem, SimpleSystem and SurfaceSPH are: the reference's
types (Vector3 with its user-provided copy constructor, which the C++ ABI
passes through a hidden pointer; the polymorphic ForceExt objects;
UniformGrid; partVoisine) and every extern "C" launcher declared with the
signatures of the reference's headers. It links against libpsb.so alone.

  * CPU: it compiles, links with immediate binding (-z now) and starts, so
    every launcher those classes call resolves in the library.
  * GPU: it runs the first half of SPHSystem::update and the surface
    extraction through those launchers, and the outputs are compared with
    the reference's own kernels run as host code (oracle/_ref) on the same
    inputs: neighbour counts exact; density, pressure, the three force
    densities, normals and forcesAccum within 1e-12 of each field's max
    (device pow against glibc's, FP64, no contraction on either side); the
    two external forces within 1e-12 (the trochoid's cos of a float angle
    within 1e-6); box bounds arriving through Vector3 by value; marching-
    cubes node centres exact, iso values within 1e-6 relative (float powf
    terms, CUDA's against glibc's), the polygonizer's vertices the
    reference's as a set (the case table is generated: the same vertices
    and count per cube, the loops may be split differently) and the vertex
    normals within 1e-5.
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import runtime as R

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "compat_link", "reference_caller.cpp")
LIB_DIR = os.path.dirname(R.LIB_PATH)


def cuda_include():
    for d in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        if d and os.path.exists(os.path.join(d, "include", "vector_types.h")):
            return os.path.join(d, "include")
    pytest.skip("CUDA headers not found")


def build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = str(tmp_path / "reference_caller")
    cmd = ["g++", "-std=c++17", "-O1", "-I", cuda_include(), SRC, "-o", exe, "-L", LIB_DIR, "-lpsb",
           "-Wl,-rpath," + LIB_DIR, "-Wl,-z,now"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_reference_classes_link_against_libpsb(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe, "link"], capture_output=True, text=True, env=dict(os.environ, LD_BIND_NOW="1"))
    assert r.returncode == 0, r.stderr
    assert "37 launchers resolved" in r.stdout


def write_scene(path, sc, pos, vel, mc_dims, mc_centre, mc_len, mc_cell, scale, level, tro, bmin, bmax):
    n = pos.shape[0]
    with open(path, "wb") as f:
        f.write(struct.pack("<i", n))
        f.write(np.ascontiguousarray(pos, np.float64).tobytes())
        f.write(np.ascontiguousarray(vel, np.float64).tobytes())
        f.write(struct.pack("<7d", sc.h, sc.mass, sc.rho0, sc.k, sc.mu, sc.l, sc.sigma))
        gmin = np.asarray(sc.grid_min, np.float64)
        glen = np.asarray(sc.dims, np.float64) * np.float32(sc.cell)
        f.write(struct.pack("<3d", *(gmin + glen / 2)))
        f.write(struct.pack("<3d", *glen))
        f.write(struct.pack("<f", sc.cell))
        f.write(struct.pack("<3d", 0.0, -1.0, 0.0))
        f.write(struct.pack("<f", 9.81))
        f.write(struct.pack("<8f", *tro))
        f.write(struct.pack("<3i", *mc_dims))
        f.write(struct.pack("<3d", *mc_centre))
        f.write(struct.pack("<3d", *mc_len))
        f.write(struct.pack("<f", mc_cell))
        f.write(struct.pack("<2d", scale, level))
        f.write(struct.pack("<3d", *bmin))
        f.write(struct.pack("<3d", *bmax))
        f.write(struct.pack("<2f", sc.particle_radius, sc.dt))


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_reference_call_sequence_matches_reference_kernels(tmp_path):
    exe = build(tmp_path)
    sc = P.ref_scene(method=P.WCSPH)
    pos = oracle.scene_positions(sc).astype(np.float64)
    n = pos.shape[0]
    vel = np.random.default_rng(3).normal(0.0, 0.05, (n, 3))
    lo, hi = pos.min(0), pos.max(0)
    mc_dims = (24, 24, 24)
    mc_centre = (lo + hi) / 2
    mc_len = (hi - lo) + 4 * sc.h
    mc_cell = float(np.float32(mc_len.max() / mc_dims[0]))
    tro = (0.3, 1.0, 2.0, 0.4, 3.0, 0.5, 0.2, 0.7)        # A, lambda, k, theta, w, f, phi, time
    bmin = lo + 0.25 * (hi - lo)                            # a box cutting the block: the clamp must show
    bmax = hi - 0.25 * (hi - lo)
    scale, level = 0.65, 0.5
    write_scene(tmp_path / "in.bin", sc, pos, vel, mc_dims, mc_centre, mc_len, mc_cell, scale, level, tro, bmin, bmax)
    r = subprocess.run([exe, "run", str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    raw = open(tmp_path / "out.bin", "rb").read()
    off = 0

    def take(dtype, count, shape=None):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a.reshape(shape) if shape else a

    counts = take(np.int32, n)
    rho, p = take(np.float64, n), take(np.float64, n)
    f_press, f_visc, f_surf, normals, f_acc = [take(np.float64, 3 * n, (n, 3)) for _ in range(5)]
    f_grav = take(np.float64, 3 * n, (n, 3))
    f_tro = take(np.float64, 3 * n, (n, 3))
    box_x, box_v = take(np.float64, 3 * n, (n, 3)), take(np.float64, 3 * n, (n, 3))
    nn = int(np.prod(mc_dims))
    nodes4 = take(np.float64, 4 * nn, (nn, 4))
    nb = take(np.int32, nn)
    nv = int(nb.sum())
    verts = take(np.float64, 3 * nv, (nv, 3))
    vnorm = take(np.float64, 3 * nv, (nv, 3))
    blocks, threads, idiv, has_dev = take(np.int32, 4)
    assert off == len(raw)

    # the reference's kernels on the same inputs
    ref = oracle.RefSim(sc, pos, vel)
    assert np.array_equal(counts, ref.search())
    out = ref.densities_forces()
    assert rel(rho, out["density"]) <= 1e-12 and rel(p, out["pressure"]) <= 1e-12
    for got, key in ((f_press, "f_press"), (f_visc, "f_visc"), (f_surf, "f_surf"), (normals, "normals"),
                     (f_acc, "f_accum")):
        assert rel(got, out[key]) <= 1e-12, key
    assert rel(f_grav, oracle.ref_force_constant(out["f_accum"], out["density"], (0.0, -1.0, 0.0), 9.81)) <= 1e-12
    tro_ref = oracle.ref_force_trochoid(pos, np.zeros((n, 3)), np.full(n, sc.mass), *[np.float32(v) for v in
                                                                                     (tro[0], tro[2], tro[3], tro[4],
                                                                                      tro[6], tro[7])])
    assert rel(f_tro, tro_ref) <= 1e-6
    # box: Vector3 bounds by value; clamp into [Min + r, Max - r] and drop the normal velocity
    r_ = np.float32(sc.particle_radius)
    lo_b = (bmin.astype(np.float32) + r_).astype(np.float64)
    hi_b = (bmax.astype(np.float32) - r_).astype(np.float64)
    assert np.all(box_x >= lo_b - 1e-12) and np.all(box_x <= hi_b + 1e-12)
    inside = np.all((pos > lo_b) & (pos < hi_b), axis=1)
    assert inside.any() and (~inside).any()
    assert np.array_equal(box_x[inside], pos[inside]) and np.array_equal(box_v[inside], vel[inside])
    # surface extraction
    grid_ref = oracle.ref_mc_grid(mc_centre, *mc_len, mc_cell, mc_dims)
    assert np.array_equal(nodes4[:, :3], grid_ref[:, :3])
    iso_nodes = np.ascontiguousarray(nodes4[:, :3])
    ref_iso = oracle.RefSim(sc, pos, vel)
    iso_ref = np.zeros(nn)
    rc = oracle.ref_lib().ref_iso(ref_iso.h, oracle._ptr(iso_nodes), mc_dims[0], mc_dims[1], mc_dims[2], scale,
                                  oracle._ptr(iso_ref))
    assert rc == 0
    assert np.max(np.abs(nodes4[:, 3] - iso_ref)) <= 1e-6 * max(np.max(np.abs(iso_ref)), 1e-300)
    # the reference's polygonizer on the very node values the library produced
    vref = oracle.ref_polygonize(nodes4, mc_dims, level)
    assert nv == vref.shape[0] and nv > 0
    from scipy.spatial import cKDTree
    d1, _ = cKDTree(vref).query(verts)
    d2, _ = cKDTree(verts).query(vref)
    assert d1.max() <= 1e-9 and d2.max() <= 1e-9
    ref.set("density", out["density"])
    assert rel(vnorm, ref.vertex_normals(verts, 1.0)) <= 1e-5
    assert (blocks, threads, idiv, has_dev) == (4, 256, 4, 1)
