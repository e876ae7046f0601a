"""Files: the reference front end's export formats, and checkpoints.

CPU: every writer's output is read back here and compared with what was
written -- the Txt and XML particle formats of ParticleExporter_Txt/_XML,
the Mitsuba grid volume of _exportData (both layouts: Mitsuba's x-fastest
order and the reference's own), and the OBJ mesh of SurfaceSPH::exportOBJ
(vertex normals point out of a closed mesh). Numbers carry 9 significant
digits, so every float comes back exactly.
GPU: the context exports equal a download of the same state, and a
checkpoint continues bit for bit -- a context loaded from it and stepped on
ends where the saved one does, single scene and batch; a checkpoint does
not load into a different scene.
"""
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import psb_project_b200 as P
from psb_project_b200.runtime import PsbError


def test_txt_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    pos = rng.uniform(-1, 2, (50, 3)).astype(np.float32).astype(np.float64)
    rho = rng.uniform(900, 1100, 50).astype(np.float32)
    path = str(tmp_path / "p.txt")
    P.write_txt(path, pos, 1.25e-4, rho)
    lines = open(path).read().splitlines()
    assert lines[0] == "SPH 50" and len(lines) == 51
    for i, line in enumerate(lines[1:]):
        t = line.split()
        assert t[0] == "-p" and t[4] == "-m" and t[6] == "-d"
        assert np.array_equal(np.float32([float(v) for v in t[1:4]]), pos[i].astype(np.float32))
        assert float(t[5]) == 1.25e-4 and np.float32(float(t[7])) == rho[i]


def test_xml_structure_and_values(tmp_path):
    sc = P.config_scene("C0")
    rng = np.random.default_rng(1)
    n = 20
    pos = rng.uniform(0, 0.5, (n, 3)).astype(np.float32).astype(np.float64)
    vel = rng.normal(0, 1, (n, 3)).astype(np.float32).astype(np.float64)
    vh = rng.normal(0, 1, (n, 3)).astype(np.float32).astype(np.float64)
    nb = rng.integers(20, 40, n).astype(np.int32)
    path = str(tmp_path / "p.xml")
    P.write_xml(path, sc, pos, vel, vh, nb)
    root = ET.parse(path).getroot()
    assert root.tag == "Particles" and root.get("name") == "SPH System" and int(root.get("count")) == n
    assert float(root.get("dt")) == pytest.approx(sc.dt, rel=1e-7)
    g = root.find("Gravity")
    assert float(g.get("Y")) == -1.0 and float(g.get("Amp")) == pytest.approx(9.81, rel=1e-7)
    parts = root.findall("Particle")
    assert len(parts) == n
    for i, e in enumerate(parts):
        assert int(e.get("index")) == i and int(e.get("kernelParticles")) == nb[i]
        assert float(e.get("mass")) == sc.mass and float(e.get("interactionRadius")) == sc.h
        assert float(e.get("restDensity")) == sc.rho0 and float(e.get("viscosity")) == sc.mu
        vec = lambda tag: np.array([float(e.find(tag).get(a)) for a in "XYZ"])
        f32 = lambda a: np.asarray(a, np.float32)         # 9 digits give every float back exactly
        assert np.array_equal(f32(vec("position")), f32(pos[i])) and np.array_equal(f32(vec("velocity")), f32(vel[i]))
        assert np.array_equal(f32(vec("velocityInterAp")), f32(vh[i]))
        assert np.allclose(vec("velocityInterAv"), 2 * vel[i] - vh[i], rtol=1e-8, atol=1e-12)
        assert [c.tag for c in e] == ["position", "velocity", "velocityInterAv", "velocityInterAp", "color"]


def read_vol(path):
    b = open(path, "rb").read()
    assert b[:3] == b"VOL" and b[3] == 3
    enc, nx, ny, nz, ch = struct.unpack_from("<5I", b, 4)
    box = struct.unpack_from("<6f", b, 24)
    data = np.frombuffer(b, np.float32, offset=48)
    return enc, (nx, ny, nz), ch, box, data


def test_vol_layouts(tmp_path):
    dims = (5, 4, 3)
    field = np.arange(np.prod(dims), dtype=np.float64) * 0.5     # index i + nx (j + ny k)
    path = str(tmp_path / "a.vol")
    P.write_vol(path, field, dims, (0, 0, 0), (1, 2, 3))
    enc, res, ch, box, data = read_vol(path)
    assert enc == 1 and res == dims and ch == 1 and box == (0, 0, 0, 1, 2, 3)
    assert np.array_equal(data, field.astype(np.float32))       # Mitsuba: x fastest, as the field is stored
    with pytest.raises(PsbError):                                 # the reference's layout needs a cube
        P.write_vol(str(tmp_path / "b.vol"), field, dims, (0, 0, 0), (1, 1, 1), reference_layout=True)
    cube = (3, 3, 3)
    f3 = np.arange(27, dtype=np.float64)
    P.write_vol(str(tmp_path / "c.vol"), f3, cube, (0, 0, 0), (1, 1, 1), reference_layout=True)
    _, res, _, _, data = read_vol(str(tmp_path / "c.vol"))
    # the reference's loops: i outer, k inner over index i + n j + n^2 k
    want = [f3[i + 3 * j + 9 * k] for i in range(3) for j in range(3) for k in range(3)]
    assert res == cube and np.array_equal(data, np.float32(want))


def test_obj_closed_mesh_normals(tmp_path):
    # a tetrahedron, triangles wound counter-clockwise seen from outside
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    t = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    path = str(tmp_path / "m.obj")
    P.write_obj(path, v, t)
    lines = open(path).read().splitlines()
    vs = np.array([[float(x) for x in l.split()[1:]] for l in lines if l.startswith("v ")])
    vn = np.array([[float(x) for x in l.split()[1:]] for l in lines if l.startswith("vn ")])
    fs = [l.split()[1:] for l in lines if l.startswith("f ")]
    assert np.array_equal(vs.astype(np.float32), v) and len(vn) == 4 and len(fs) == 4
    assert [[int(x.split("//")[0]) - 1 for x in f] for f in fs] == t.tolist()
    assert all(x.split("//")[0] == x.split("//")[1] for f in fs for x in f)
    assert np.allclose(np.linalg.norm(vn, axis=1), 1, atol=1e-5)
    c = v.mean(0)
    assert np.all(np.sum((v - c) * vn, axis=1) > 0)                # outward
    with pytest.raises(PsbError):
        P.write_obj(path, v, np.array([[0, 1, 4]], np.int32))     # index out of range


def test_writers_reject_bad_arguments(tmp_path):
    """The host writers return PSB_EINVAL for negative counts, missing
    arrays, out-of-range triangle indices, negative volume dimensions, the
    reference's volume layout on a non-cubic grid, and a path that cannot be
    opened."""
    import ctypes
    from psb_project_b200 import runtime as R
    L = R.lib()
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    L.psb_write_txt.argtypes = [ctypes.c_char_p, i32, vp, ctypes.c_double, vp]
    L.psb_write_obj.argtypes = [ctypes.c_char_p, vp, i64, vp, i64]
    L.psb_write_vol.argtypes = [ctypes.c_char_p, vp, vp, vp, vp, i32]
    txt, obj, vol = (str(tmp_path / f).encode() for f in ("a.txt", "a.obj", "a.vol"))
    pos, rho = np.zeros((2, 3)), np.zeros(2, np.float32)
    assert L.psb_write_txt(txt, -1, pos.ctypes.data, 1.0, rho.ctypes.data) == 1
    assert L.psb_write_txt(txt, 2, None, 1.0, rho.ctypes.data) == 1
    assert L.psb_write_txt(str(tmp_path / "no" / "a.txt").encode(), 2, pos.ctypes.data, 1.0, rho.ctypes.data) == 1
    v, tri = np.zeros((3, 3), np.float32), np.array([[0, 1, 5]], np.int32)
    assert L.psb_write_obj(obj, v.ctypes.data, 3, tri.ctypes.data, 1) == 1
    assert L.psb_write_obj(obj, v.ctypes.data, -3, None, 0) == 1
    b = np.zeros(3, np.float32)
    assert L.psb_write_vol(vol, np.zeros(6).ctypes.data, np.array([2, 3, -1], np.int32).ctypes.data,
                           b.ctypes.data, b.ctypes.data, 0) == 1
    assert L.psb_write_vol(vol, np.zeros(24).ctypes.data, np.array([2, 3, 4], np.int32).ctypes.data,
                           b.ctypes.data, b.ctypes.data, 1) == 1

@pytest.mark.gpu
def test_exports_match_download(tmp_path):
    sc = P.dam_break((10, 8, 6), 0.01, (0.3, 0.3, 0.3), 0.02, dt=5e-4, seed=41)
    with P.Simulation(sc) as sim:
        sim.upload(P.scene_positions(sc))
        sim.step(5)
        st = sim.download()
        sim.export_txt(str(tmp_path / "s.txt"))
        sim.export_xml(str(tmp_path / "s.xml"))
    lines = open(tmp_path / "s.txt").read().splitlines()
    assert lines[0] == f"SPH {sc.n}"
    got = np.array([[float(x) for x in l.split()[1:4]] for l in lines[1:]], np.float32)
    assert np.array_equal(got, st["pos"])
    rho = np.float32([float(l.split()[7]) for l in lines[1:]])
    assert np.array_equal(rho, st["density"])
    parts = ET.parse(tmp_path / "s.xml").getroot().findall("Particle")
    vh = np.float32([[float(e.find("velocityInterAp").get(a)) for a in "XYZ"] for e in parts])
    assert np.array_equal(vh, st["vel_half"])


def _continue(make, path_in, steps):
    with make() as b:
        b.checkpoint_load(path_in)
        b.step(steps)
        return b.download(), b.steps_taken()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["single", "batch"])
def test_checkpoint_continues_bit_for_bit(tmp_path, kind):
    if kind == "single":
        sc = P.dam_break((12, 10, 8), 0.01, (0.4, 0.3, 0.3), 0.02, dt=5e-4, seed=42).replace(warm_start=P.WARM_PREVIOUS)
        make = lambda: P.Simulation(sc)
        pos = P.scene_positions(sc)
    else:
        scenes = P.batch_scenes(n_scenes=3, seed=43, n_range=(300, 2000), side=(0.3, 0.5), dt=5e-4,
                                warm_start=P.WARM_PREVIOUS)
        make = lambda: P.BatchSimulation(scenes)
        pos = P.batch_positions(scenes)
    path = str(tmp_path / "state.psbchk")
    with make() as a:
        a.upload(pos)
        a.presolve(16)
        a.step(4)
        a.checkpoint_save(path)
        a.step(6)
        want = a.download()
        steps = a.steps_taken()
    got, steps_b = _continue(make, path, 6)
    for k in ("pos", "vel", "vel_half", "pressure", "density"):
        assert np.array_equal(got[k], want[k]), k
    assert steps_b == steps


@pytest.mark.gpu
def test_checkpoint_rejects_another_scene(tmp_path):
    sc = P.dam_break((8, 8, 8), 0.01, (0.3, 0.3, 0.3), 0.02, dt=5e-4, seed=44)
    path = str(tmp_path / "s.psbchk")
    with P.Simulation(sc) as a:
        a.upload(P.scene_positions(sc))
        a.step(1)
        a.checkpoint_save(path)
    with P.Simulation(sc.replace(dt=1e-3)) as b:
        with pytest.raises(PsbError):
            b.checkpoint_load(path)
    with P.Simulation(sc.replace(n=sc.n * 2)) as c:      # a larger capacity is fine
        c.checkpoint_load(path)
        assert c.n == sc.n
