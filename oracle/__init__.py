"""ctypes bindings of the oracle (test infrastructure only).

Two checkers live under oracle/:
  * liboracle.so -- our FP64 C restatement of the hot path (psb_oracle.c);
  * _ref/libpsbref.so -- the reference's own device kernels compiled as host
    code through refshim/ (built only where the reference tree exists; the
    .so then travels with the repository).
Only tests/, the smoke check and bench.py's CPU-baseline legs import this
package. The product (psb_project_b200) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libpsbref.so")
REFCUDA_PATH = os.path.join(HERE, "_ref", "libpsbref_cuda.so")
# The reference tree's src/ directory, when it is present: PSB_REFERENCE_SRC,
# else a reference checkout beside this repository (<repo>/../reference/src).
REF_SRC = os.environ.get("PSB_REFERENCE_SRC") or os.path.join(os.path.dirname(HERE), os.pardir, "reference", "src")

ORC_MAX_ITERS = 64


def build(with_reference: bool = True) -> None:
    """Compile the oracle (and, where the reference tree exists, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if with_reference and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={REF_SRC}"], check=True)
        subprocess.run(["make", "-s", "-C", HERE, "refcuda", f"REF_SRC={REF_SRC}"], check=True)


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("box_min", ctypes.c_float * 3), ("box_max", ctypes.c_float * 3),
        ("grid_min", ctypes.c_float * 3), ("cell", ctypes.c_float), ("dims", ctypes.c_int32 * 3),
        ("h", ctypes.c_double), ("mass", ctypes.c_double), ("rho0", ctypes.c_double), ("k", ctypes.c_double),
        ("mu", ctypes.c_double), ("sigma", ctypes.c_double), ("l", ctypes.c_double),
        ("particle_radius", ctypes.c_float), ("dt", ctypes.c_float), ("gravity", ctypes.c_float * 3),
        ("profile", ctypes.c_int32), ("method", ctypes.c_int32),
        ("min_iters", ctypes.c_int32), ("max_iters", ctypes.c_int32),
        ("eta", ctypes.c_double), ("wall_k", ctypes.c_double), ("wall_c", ctypes.c_double),
        ("float_state", ctypes.c_int32), ("warm_start", ctypes.c_int32), ("spacing", ctypes.c_double),
        ("skin", ctypes.c_double), ("xsph", ctypes.c_double),
        ("dem_spring", ctypes.c_double), ("dem_damping", ctypes.c_double), ("dem_shear", ctypes.c_double),
        ("dem_attraction", ctypes.c_double),
        ("n_bnd", ctypes.c_int32), ("bnd_pos", ctypes.c_void_p), ("bnd_psi", ctypes.c_void_p),
        ("bnd_counts", ctypes.c_void_p), ("bnd_lists", ctypes.c_void_p), ("bnd_cap", ctypes.c_int32),
        ("dem_ext", ctypes.c_void_p),
        ("n_coll", ctypes.c_int32), ("coll", ctypes.c_void_p),
        ("bnd_vel", ctypes.c_void_p), ("bnd_fext", ctypes.c_void_p), ("bnd_inv_mass", ctypes.c_double),
        ("bnd_pred", ctypes.c_void_p), ("bnd_force", ctypes.c_void_p),
    ]


class OrcCollider(ctypes.Structure):
    """orc_collider: one collision object as its reference kernel executes."""
    _fields_ = [("type", ctypes.c_int32), ("container", ctypes.c_int32), ("elast", ctypes.c_float),
                ("count", ctypes.c_int32), ("v", ctypes.c_float * 16), ("faces", ctypes.c_void_p),
                ("terms", ctypes.c_void_p)]


class Colliders:
    """An orc_collider array plus the face and term arrays it points to.
    Each object: (type, v (<= 16 floats), elast, container, faces (F x 12
    float32) or None, terms (T x 6 float64) or None)."""

    def __init__(self, objs):
        self.arr = (OrcCollider * max(1, len(objs)))()
        self.keep = []
        for i, (typ, v, elast, container, faces, terms) in enumerate(objs):
            o = self.arr[i]
            o.type, o.container, o.elast = int(typ), int(bool(container)), float(elast)
            vv = list(v) + [0.0] * (16 - len(v))
            o.v[:] = [float(x) for x in vv]
            if faces is not None:
                f = np.ascontiguousarray(faces, np.float32).reshape(-1, 12)
                self.keep.append(f)
                o.faces, o.count = f.ctypes.data, f.shape[0]
            if terms is not None:
                t = np.ascontiguousarray(terms, np.float64).reshape(-1, 6)
                self.keep.append(t)
                o.terms, o.count = t.ctypes.data, t.shape[0]
        self.n = len(objs)


class OrcState(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_void_p), ("vel", ctypes.c_void_p), ("vel_ap", ctypes.c_void_p),
                ("rho", ctypes.c_void_p), ("p", ctypes.c_void_p)]


class OrcStats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("err", ctypes.c_double * (ORC_MAX_ITERS + 1)), ("nbr_total", ctypes.c_int64),
                ("nbr_max", ctypes.c_int32), ("clamped", ctypes.c_int32)]


_lib = None
_ref = None


class IsoGrid(ctypes.Structure):
    """orc_iso_grid: dims[a] nodes at origin[a] + i spacing[a], x fastest."""
    _fields_ = [("origin", ctypes.c_double * 3), ("spacing", ctypes.c_double * 3), ("dims", ctypes.c_int32 * 3),
                ("scale", ctypes.c_double)]


def iso_grid(origin, spacing, dims, scale=0.65) -> IsoGrid:
    g = IsoGrid()
    g.origin[:] = [float(v) for v in origin]
    sp = spacing if hasattr(spacing, "__len__") else (spacing,) * 3
    g.spacing[:] = [float(v) for v in sp]
    g.dims[:] = [int(v) for v in dims]
    g.scale = float(scale)
    return g


def grid_nodes(g: IsoGrid) -> np.ndarray:
    """Node positions (x fastest), shape (nx*ny*nz, 3)."""
    axes = [g.origin[a] + np.arange(g.dims[a]) * g.spacing[a] for a in range(3)]
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1)


def iso_field(scene, pos, rho, g: IsoGrid) -> np.ndarray:
    pos = np.ascontiguousarray(pos, np.float64)
    rho = np.ascontiguousarray(rho if rho is not None else np.ones(pos.shape[0]), np.float64)
    out = np.zeros(int(np.prod(list(g.dims))))
    P = params(scene, n=pos.shape[0])
    lib().orc_iso_field(ctypes.byref(P), _ptr(pos), _ptr(rho), ctypes.byref(g), _ptr(out))
    return out


def mc_table():
    ntri = np.zeros(256, np.uint8)
    tri = np.zeros((256, 30), np.int8)
    lib().orc_mc_table(_ptr(ntri), _ptr(tri))
    return ntri, tri


def marching_cubes(g: IsoGrid, iso, level):
    """(vertices (V, 3) float64, triangles (T, 3) int32)."""
    iso = np.ascontiguousarray(iso, np.float64)
    nv = ctypes.c_int64(0)
    nt = ctypes.c_int64(0)
    lib().orc_marching_cubes(ctypes.byref(g), _ptr(iso), float(level), 0, None, ctypes.byref(nv), 0, None,
                             ctypes.byref(nt))
    vert = np.zeros((max(nv.value, 1), 3))
    tri = np.zeros((max(nt.value, 1), 3), np.int32)
    rc = lib().orc_marching_cubes(ctypes.byref(g), _ptr(iso), float(level), nv.value, _ptr(vert), ctypes.byref(nv),
                                  nt.value, _ptr(tri), ctypes.byref(nt))
    if rc != 0:
        raise RuntimeError("orc_marching_cubes: capacity")
    return vert[:nv.value], tri[:nt.value]


def ref_marching_cubes(g: IsoGrid, iso, level) -> np.ndarray:
    """The reference's polygonize kernel on the same nodes: triangle corners
    (3 per triangle) in cell order, shape (3T, 3)."""
    nodes4 = np.concatenate([grid_nodes(g), np.asarray(iso, np.float64)[:, None]], 1)
    return ref_polygonize(nodes4, g.dims, level)


def ref_polygonize(nodes4, dims, level) -> np.ndarray:
    """polygonize_MarchingCube_Kernel over nodes (x, y, z, value), x fastest:
    triangle corners (3 per triangle) in cell order, shape (3T, 3)."""
    nodes4 = np.ascontiguousarray(nodes4, np.float64)
    cap = 16 * nodes4.shape[0] + 64
    out = np.zeros((cap, 3))
    nv = ctypes.c_int64(0)
    rc = ref_lib().ref_marching_cubes(_ptr(nodes4), int(dims[0]), int(dims[1]), int(dims[2]), float(level), cap,
                                      _ptr(out), ctypes.byref(nv))
    if rc != 0:
        raise RuntimeError("ref_marching_cubes: capacity")
    return out[:nv.value]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_reference=False)
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.orc_lattice.argtypes = [P, ctypes.c_double, P, ctypes.c_double, ctypes.c_uint64, ctypes.c_int32, P]
        L.orc_lattice.restype = None
        L.orc_cell_keys.argtypes = [ctypes.c_int32, P, P, ctypes.c_float, P, P, P]
        L.orc_cell_keys.restype = None
        L.orc_sort_perm.argtypes = [ctypes.c_int32, P, P]
        L.orc_sort_perm.restype = None
        L.orc_neighbors.argtypes = [ctypes.POINTER(OrcParams), P, ctypes.c_int32, P, P]
        L.orc_neighbors.restype = ctypes.c_int64
        L.orc_density.argtypes = [ctypes.POINTER(OrcParams), P, P, P, ctypes.c_int32, ctypes.c_int, P]
        L.orc_density.restype = None
        L.orc_features.argtypes = [ctypes.POINTER(OrcParams), P, P, P, P]
        L.orc_features.restype = None
        L.orc_step.argtypes = [ctypes.POINTER(OrcParams), ctypes.POINTER(OrcState), ctypes.POINTER(OrcStats), P, P, P]
        L.orc_step.restype = ctypes.c_int
        L.orc_presolve.argtypes = [ctypes.POINTER(OrcParams), ctypes.POINTER(OrcState), ctypes.c_int32,
                                   ctypes.POINTER(OrcStats)]
        L.orc_presolve.restype = ctypes.c_int
        L.orc_pci_delta.argtypes = [ctypes.POINTER(OrcParams)]
        L.orc_pci_delta.restype = ctypes.c_double
        L.orc_iso_field.argtypes = [ctypes.POINTER(OrcParams), P, P, ctypes.POINTER(IsoGrid), P]
        L.orc_iso_field.restype = None
        L.orc_mc_table.argtypes = [P, P]
        L.orc_mc_table.restype = None
        L.orc_marching_cubes.argtypes = [ctypes.POINTER(IsoGrid), P, ctypes.c_double, ctypes.c_int64, P, P,
                                         ctypes.c_int64, P, P]
        L.orc_marching_cubes.restype = ctypes.c_int
        L.orc_boundary_psi.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int32, P, P]
        L.orc_boundary_psi.restype = None
        L.orc_pressure_force.argtypes = [ctypes.POINTER(OrcParams), P, P, P, P, P, ctypes.c_int32, P]
        L.orc_pressure_force.restype = None
        L.orc_boundary_reaction.argtypes = [ctypes.POINTER(OrcParams), P, P, ctypes.c_int32, P, P, P]
        L.orc_boundary_reaction.restype = None
        L.orc_collide.argtypes = [ctypes.POINTER(OrcCollider), ctypes.c_int32, P, P, P, ctypes.c_float]
        L.orc_collide.restype = ctypes.c_int32
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_PATH} is not built (make -C oracle ref)")
        L = ctypes.CDLL(REF_PATH)
        P = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_int, P, ctypes.c_float, P]
        L.ref_create.restype = P
        L.ref_destroy.argtypes = [P]
        L.ref_set.argtypes = [P, ctypes.c_char_p, P]
        L.ref_get.argtypes = [P, ctypes.c_char_p, P]
        L.ref_search.argtypes = [P]
        L.ref_neighbors.argtypes = [P, P, P]
        L.ref_density_pci.argtypes = [P]
        L.ref_pcisph_update.argtypes = [P, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_float, P, P]
        L.ref_wcsph_update.argtypes = [P, ctypes.c_float, P, ctypes.c_float, ctypes.c_int, ctypes.c_float, P, P]
        L.ref_dem_update.argtypes = [P, ctypes.c_float, P, ctypes.c_float, ctypes.c_int, ctypes.c_float, P, P]
        L.ref_iso.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, P]
        L.ref_marching_cubes.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int64,
                                         P, P]
        L.ref_collide.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                  ctypes.c_float, P, ctypes.c_int, P, P]
        L.ref_collide.restype = ctypes.c_int
        F = ctypes.c_float
        L.ref_densities_forces.argtypes = [P]
        L.ref_vertex_normals.argtypes = [P, P, ctypes.c_int, F, P]
        L.ref_force_trochoid.argtypes = [ctypes.c_int, P, P, P, F, F, F, F, F, F]
        L.ref_force_constant.argtypes = [ctypes.c_int, P, P, P, F]
        L.ref_mc_grid.argtypes = [P, ctypes.c_double, ctypes.c_double, ctypes.c_double, F, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, P]
        _ref = L
    return _ref


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def lattice(nxyz, spacing, origin, jitter, seed, id0=0) -> np.ndarray:
    n = int(nxyz[0]) * int(nxyz[1]) * int(nxyz[2])
    out = np.empty((n, 3), np.float32)
    nx = np.asarray(nxyz, np.int32)
    org = np.asarray(origin, np.float64)
    lib().orc_lattice(_ptr(nx), float(spacing), _ptr(org), float(jitter), int(seed) & (2**64 - 1), int(id0), _ptr(out))
    return out


def scene_positions(scene) -> np.ndarray:
    return np.concatenate([lattice(b.nxyz, b.spacing, b.origin, b.jitter, b.seed, b.id0) for b in scene.blocks])


def params(scene, *, float_state: bool = False, n: Optional[int] = None) -> OrcParams:
    p = OrcParams()
    p.n = scene.n if n is None else n
    p.box_min[:] = list(scene.box_min)
    p.box_max[:] = list(scene.box_max)
    p.grid_min[:] = list(scene.grid_min)
    p.cell = scene.cell
    p.dims[:] = list(scene.dims)
    p.h, p.mass, p.rho0, p.k = scene.h, scene.mass, scene.rho0, scene.k
    p.mu, p.sigma, p.l = scene.mu, scene.sigma, scene.l
    p.particle_radius, p.dt = scene.particle_radius, scene.dt
    p.gravity[:] = list(scene.gravity)
    p.profile, p.method = scene.profile, scene.method
    p.min_iters, p.max_iters, p.eta = scene.min_iters, scene.max_iters, scene.eta
    p.wall_k, p.wall_c = scene.wall_k, scene.wall_c
    p.float_state = 1 if float_state else 0
    p.warm_start = 1 if scene.warm_start else 0
    p.spacing = scene.spacing
    p.skin = scene.skin
    p.xsph = scene.xsph
    p.dem_spring, p.dem_damping = scene.dem_spring, scene.dem_damping
    p.dem_shear, p.dem_attraction = scene.dem_shear, scene.dem_attraction
    return p


def boundary_psi(scene, bpos) -> np.ndarray:
    """Akinci volumes psi_b (kg) of a boundary sampling."""
    bpos = np.ascontiguousarray(bpos, np.float64)
    psi = np.empty(bpos.shape[0])
    P = params(scene)
    lib().orc_boundary_psi(ctypes.byref(P), bpos.shape[0], _ptr(bpos), _ptr(psi))
    return psi


def boundary_reaction(scene, pos, p, bpos) -> np.ndarray:
    """The fluid's force on each boundary particle (nb, 3)."""
    pos = np.ascontiguousarray(pos, np.float64)
    p = np.ascontiguousarray(p, np.float64)
    bpos = np.ascontiguousarray(bpos, np.float64)
    psi = boundary_psi(scene, bpos)
    out = np.zeros((bpos.shape[0], 3))
    P = params(scene, n=pos.shape[0])
    lib().orc_boundary_reaction(ctypes.byref(P), _ptr(pos), _ptr(p), bpos.shape[0], _ptr(bpos), _ptr(psi), _ptr(out))
    return out


def pci_delta(scene) -> float:
    P = params(scene)
    return lib().orc_pci_delta(ctypes.byref(P))


def cell_keys(scene, pos) -> np.ndarray:
    pos = np.ascontiguousarray(pos, np.float64)
    n = pos.shape[0]
    keys = np.empty(n, np.uint32)
    ncl = ctypes.c_int32(0)
    gmin = np.asarray(scene.grid_min, np.float32)
    dims = np.asarray(scene.dims, np.int32)
    lib().orc_cell_keys(n, _ptr(pos), _ptr(gmin), scene.cell, _ptr(dims), _ptr(keys), ctypes.addressof(ncl))
    return keys


def sort_perm(keys) -> np.ndarray:
    keys = np.ascontiguousarray(keys, np.uint32)
    perm = np.empty(keys.shape[0], np.int32)
    lib().orc_sort_perm(keys.shape[0], _ptr(keys), _ptr(perm))
    return perm


def neighbors(scene, pos, with_lists=True):
    """(counts, lists) at pos; lists is an (n, cap) int32 array padded with -1."""
    pos = np.ascontiguousarray(pos, np.float64)
    P = params(scene, n=pos.shape[0])
    counts = np.empty(pos.shape[0], np.int32)
    lib().orc_neighbors(ctypes.byref(P), _ptr(pos), 0, _ptr(counts), None)
    if not with_lists:
        return counts, None
    cap = max(1, int(counts.max()))
    lists = np.full((pos.shape[0], cap), -1, np.int32)
    lib().orc_neighbors(ctypes.byref(P), _ptr(pos), cap, _ptr(counts), _ptr(lists))
    return counts, lists


def density(scene, pos, counts, lists, clamp) -> np.ndarray:
    pos = np.ascontiguousarray(pos, np.float64)
    P = params(scene, n=pos.shape[0])
    rho = np.empty(pos.shape[0], np.float64)
    lists = np.ascontiguousarray(lists, np.int32)
    lib().orc_density(ctypes.byref(P), _ptr(pos), _ptr(np.ascontiguousarray(counts, np.int32)), _ptr(lists),
                      lists.shape[1], 1 if clamp else 0, _ptr(rho))
    return rho


def features(scene, pos, vel, p_prev, boundary=None) -> np.ndarray:
    """Inputs of the learned warm start at the state (pos, vel, carried
    pressure p_prev), (n, 7) in id order (orc_features; FP64)."""
    pos = np.ascontiguousarray(pos, np.float64)
    vel = np.ascontiguousarray(vel, np.float64)
    p_prev = np.ascontiguousarray(p_prev, np.float64)
    P = params(scene, n=pos.shape[0])
    keep = []
    if boundary is not None:
        bpos = np.ascontiguousarray(boundary, np.float64)
        psi = boundary_psi(scene, bpos)
        keep += [bpos, psi]
        P.n_bnd, P.bnd_pos, P.bnd_psi = bpos.shape[0], bpos.ctypes.data, psi.ctypes.data
    out = np.empty((pos.shape[0], 7), np.float64)
    lib().orc_features(ctypes.byref(P), _ptr(pos), _ptr(vel), _ptr(p_prev), _ptr(out))
    return out


def _bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), kept as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def mlp_forward(w, X, n_in, activation) -> np.ndarray:
    """The warm-start network y(X) on the CPU, FP64 arithmetic on the
    library's BF16 rounding points: inputs, weights and both hidden layers'
    activations rounded to BF16. w: the FP32 parameter vector (W1 [64 x
    n_in], b1, W2 [64 x 64], b2, w3 [64], b3); activation "silu" or "relu".
    Returns (y, h1, h2) with the hidden activations for error bounds."""
    w = _bf16(np.asarray(w, np.float32)).astype(np.float64)
    H = 64
    o = 0
    W1 = w[o:o + H * n_in].reshape(H, n_in); o += H * n_in
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    w3 = w[o:o + H]; o += H
    b3 = w[o]
    # SiLU z sigma(z) written as z/2 (1 + tanh(z/2)), finite for every z
    act = (lambda z: 0.5 * z * (1.0 + np.tanh(0.5 * z))) if activation == "silu" else (lambda z: np.maximum(z, 0.0))
    x = _bf16(np.asarray(X, np.float32)[:, :n_in]).astype(np.float64)
    h1 = _bf16(act(x @ W1.T + b1)).astype(np.float64)
    h2 = _bf16(act(h1 @ W2.T + b2)).astype(np.float64)
    return h2 @ w3 + b3, h1, h2


def learned_pressure(scene, pos, vel, p_prev, w, arch, boundary=None) -> np.ndarray:
    """The learned warm start's initial pressure on the CPU: the FP64
    features (orc_features) through the network (mlp_forward) with the
    library's BF16 rounding points, max(0, y) p_scale. arch 0: 6 inputs,
    SiLU; 1: 7 inputs, ReLU (the library's PSB_MLP_SILU6, PSB_MLP_RELU7).
    boundary: the static boundary particles' positions, if the scene has them."""
    F = features(scene, pos, vel, p_prev, boundary)
    n_in, act = (6, "silu") if arch == 0 else (7, "relu")
    y, _, _ = mlp_forward(w, F.astype(np.float32), n_in, act)
    g = float(np.linalg.norm(np.asarray(scene.gravity, np.float64)))
    p_scale = scene.rho0 * (g if g > 0 else 9.81) * 0.1
    return np.maximum(0.0, y) * p_scale


class OracleSim:
    """FP64 state in particle-id order, stepped by orc_step."""

    def __init__(self, scene, pos, vel=None, vel_half=None, pressure=None, *, float_state=False, boundary=None,
                 colliders=None):
        n = pos.shape[0]
        self.scene = scene
        self.P = params(scene, float_state=float_state, n=n)
        if colliders:                 # collision objects after the box (Colliders or its object list)
            self.coll = colliders if isinstance(colliders, Colliders) else Colliders(colliders)
            self.P.n_coll = self.coll.n
            self.P.coll = ctypes.addressof(self.coll.arr)
        if boundary is not None:      # static boundary particles (config profile)
            self.bnd_pos = np.ascontiguousarray(boundary, np.float64)
            self.bnd_psi = boundary_psi(scene, self.bnd_pos)
            self.P.n_bnd = self.bnd_pos.shape[0]
            self.P.bnd_pos = self.bnd_pos.ctypes.data
            self.P.bnd_psi = self.bnd_psi.ctypes.data
        self.pos = np.ascontiguousarray(pos, np.float64).copy()
        self.vel = np.zeros((n, 3)) if vel is None else np.ascontiguousarray(vel, np.float64).copy()
        self.vel_half = np.zeros((n, 3)) if vel_half is None else np.ascontiguousarray(vel_half, np.float64).copy()
        self.rho = np.zeros(n)
        self.p = np.zeros(n) if pressure is None else np.ascontiguousarray(pressure, np.float64).copy()
        self.rho_x = np.zeros(n)
        self.f_np = np.zeros((n, 3))
        self.nbr = np.zeros(n, np.int32)
        self.stats = OrcStats()

    def append(self, pos, vel=None, vel_half=None):
        """Particles appended at the end (ids n ..), density and pressure 0."""
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        k = pos.shape[0]
        z3 = np.zeros((k, 3))
        vel = z3 if vel is None else np.asarray(vel, np.float64).reshape(-1, 3)
        vel_half = z3 if vel_half is None else np.asarray(vel_half, np.float64).reshape(-1, 3)
        self.pos = np.ascontiguousarray(np.concatenate([self.pos, pos]))
        self.vel = np.ascontiguousarray(np.concatenate([self.vel, vel]))
        self.vel_half = np.ascontiguousarray(np.concatenate([self.vel_half, vel_half]))
        self.rho = np.concatenate([self.rho, np.zeros(k)])
        self.p = np.concatenate([self.p, np.zeros(k)])
        self.rho_x = np.zeros(self.pos.shape[0])
        self.f_np = np.zeros((self.pos.shape[0], 3))
        self.nbr = np.zeros(self.pos.shape[0], np.int32)
        self.P.n = self.pos.shape[0]
        if getattr(self, "ext", None) is not None:
            self.set_external_force(np.concatenate([self.ext, z3]))

    def presolve(self, iters):
        S = OrcState(self.pos.ctypes.data, self.vel.ctypes.data, self.vel_half.ctypes.data,
                     self.rho.ctypes.data, self.p.ctypes.data)
        rc = lib().orc_presolve(ctypes.byref(self.P), ctypes.byref(S), int(iters), ctypes.byref(self.stats))
        if rc != 0:
            raise RuntimeError(f"orc_presolve failed: {rc}")
        return self.stats

    def set_external_force(self, f):
        """DEM: a per-sphere external force (n, 3) for the following steps (None: off)."""
        if f is None:
            self.ext = None
            self.P.dem_ext = None
        else:
            self.ext = np.ascontiguousarray(f, np.float64).reshape(-1, 3)
            self.P.dem_ext = self.ext.ctypes.data

    def set_boundary_motion(self, vel, fext, mass):
        """Config PCISPH: the boundary particles move with the corrector
        (two-way coupling inside the step): their velocities and non-fluid
        forces at the step's start (n_bnd, 3) and their mass; None: static.
        After a step, bnd_pred holds the predicted boundary positions and
        bnd_force the fluid's reaction they were predicted with."""
        if vel is None:
            self.P.bnd_vel = self.P.bnd_fext = self.P.bnd_pred = self.P.bnd_force = None
            return
        nb = self.bnd_pos.shape[0]
        self.bnd_vel = np.ascontiguousarray(vel, np.float64).reshape(nb, 3).copy()
        self.bnd_fext = np.ascontiguousarray(fext, np.float64).reshape(nb, 3).copy()
        self.bnd_pred = np.zeros((nb, 3))
        self.bnd_force = np.zeros((nb, 3))
        self.P.bnd_vel = self.bnd_vel.ctypes.data
        self.P.bnd_fext = self.bnd_fext.ctypes.data
        self.P.bnd_inv_mass = 1.0 / float(mass)
        self.P.bnd_pred = self.bnd_pred.ctypes.data
        self.P.bnd_force = self.bnd_force.ctypes.data

    def step(self):
        S = OrcState(self.pos.ctypes.data, self.vel.ctypes.data, self.vel_half.ctypes.data,
                     self.rho.ctypes.data, self.p.ctypes.data)
        rc = lib().orc_step(ctypes.byref(self.P), ctypes.byref(S), ctypes.byref(self.stats),
                            _ptr(self.rho_x), _ptr(self.f_np), _ptr(self.nbr))
        if rc != 0:
            raise RuntimeError(f"orc_step failed: {rc}")
        return self.stats


def dem_forces(scene, pos, vel):
    """DEM: gravity and contact force (n, 3) on each sphere at (pos, vel),
    the force its next step applies apart from an external one (FP64)."""
    probe = OracleSim(scene, np.array(pos, np.float64), np.array(vel, np.float64), np.array(vel, np.float64))
    probe.step()
    return probe.f_np.copy()


class Coupling:
    """The fluid-DEM coupled step (config C1) on FP64 oracle states, as the
    library's FluidDemCoupling runs it: every sphere one boundary particle
    of the fluid. implicit: the spheres move with the fluid's corrector
    (set_boundary_motion) and then step with the reaction of its last
    prediction; else the staggered exchange (the fluid steps with the
    spheres held, then the spheres step with its reaction)."""

    def __init__(self, fluid_scene, fluid, sphere_scene, spheres, implicit=True):
        self.fs, self.fluid, self.ss, self.spheres, self.implicit = fluid_scene, fluid, sphere_scene, spheres, implicit

    def step(self):
        fl, sp = self.fluid, self.spheres
        fl.bnd_pos[:] = sp.pos
        fl.bnd_psi[:] = boundary_psi(self.fs, fl.bnd_pos)
        if self.implicit:
            fl.set_boundary_motion(sp.vel, dem_forces(self.ss, sp.pos, sp.vel), float(self.ss.mass))
            st = fl.step()
            force = fl.bnd_force.copy()
        else:
            fl.set_boundary_motion(None, None, None)
            st = fl.step()
            force = boundary_reaction(self.fs, fl.pos, fl.p, fl.bnd_pos)
        sp.set_external_force(force)
        sp.step()
        return st, force


def collide(obj, old_pos, pos, vel, dt):
    """One collision object (a Colliders entry tuple) on FP64 copies of
    (pos, vel); returns (pos, vel, hits)."""
    c = Colliders([obj])
    x = np.ascontiguousarray(pos, np.float64).copy()
    v = np.ascontiguousarray(vel, np.float64).copy()
    xo = np.ascontiguousarray(old_pos, np.float64)
    hits = lib().orc_collide(ctypes.byref(c.arr[0]), x.shape[0], _ptr(xo), _ptr(x), _ptr(v), ctypes.c_float(dt))
    return x, v, hits


def ref_collide(obj, old_pos, pos, vel, dt, particle_radius=0.0):
    """The same object through the reference's own kernel on the CPU
    (oracle/_ref); returns (pos, vel)."""
    typ, v, elast, container, faces, terms = obj
    x = np.ascontiguousarray(pos, np.float64).copy()
    u = np.ascontiguousarray(vel, np.float64).copy()
    xo = np.ascontiguousarray(old_pos, np.float64).copy()
    vv = np.zeros(16, np.float32)
    vv[:len(v)] = v
    f = None if faces is None else np.ascontiguousarray(faces, np.float32).reshape(-1, 12)
    t = None if terms is None else np.ascontiguousarray(terms, np.float64).reshape(-1, 6)
    count = f.shape[0] if f is not None else (t.shape[0] if t is not None else 0)
    L = ref_lib()
    rc = L.ref_collide(int(typ), x.shape[0], _ptr(xo), _ptr(x), _ptr(u), ctypes.c_float(dt), ctypes.c_float(elast),
                       int(bool(container)), ctypes.c_float(particle_radius), _ptr(vv), count,
                       None if f is None else _ptr(f), None if t is None else _ptr(t))
    if rc != 0:
        raise RuntimeError(f"ref_collide failed: {rc}")
    return x, u


# ---- emitters (src/Kernel/Emitters/*), restated --------------------------------
# The reference's emitters need its Particle, SimulationData and GL geometry
# classes, so they are restated here rather than compiled: each loop as its
# emitParticles runs it, with its float and double types, and the C
# library's math (Python's math module and numpy's float32 power call it).

_M64 = (1 << 64) - 1


def _splitmix64(x):
    z = (x + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def _uniform(seed, emission, particle, draw):
    k = _splitmix64(seed ^ _splitmix64(((emission << 32) | draw) & _M64) ^ _splitmix64(particle + 1))
    return (k >> 11) * (1.0 / 9007199254740992.0)


def _box(v, rho):
    f32 = np.float32
    cx, cy, cz = (float(f32(t)) for t in v[:3])
    sx, sy, sz = (f32(t) for t in v[3:6])
    wx, wy, wz = (float(f32(t)) for t in v[6:9])
    step = f32(rho) * f32(2)

    def axis(c, sz_):
        out, x = [], f32(c - float(sz_ / f32(2)))
        while float(x) <= c + float(sz_ / f32(2)):
            out.append(x)
            x = f32(x + step)
        return out
    pts = []
    for z in axis(cz, sz):
        for y in axis(cy, sy):
            for x in axis(cx, sx):
                pts.append((f32(float(x) + wx), f32(float(y) + wy), f32(float(z) + wz)))
    return np.array(pts, np.float32).reshape(-1, 3)


def _ring(cx, cz, y, r, dtheta, pts):
    import math
    theta, theta_ap = 0.0, 1.0
    while theta <= 2 * math.pi and theta_ap > 0:
        pts.append((cx + r * math.cos(theta), y, cz + r * math.sin(theta)))
        theta += dtheta
        theta_ap = theta


def _sphere(v, rho):
    import math
    f32 = np.float32
    cx, cy, cz = (float(f32(t)) for t in v[:3])
    R, rho = f32(v[3]), f32(rho)
    RR, rr2 = float(R * R), float(f32(2) * rho * rho)
    pts = []

    def layer(y):
        r = 0.0
        while RR - y * y >= 0 and r <= math.sqrt(RR - y * y):
            _ring(cx, cz, y, r, math.acos(r / math.sqrt(r * r + rr2)), pts)
            r += float(rho)
    y = cy
    while y < cy + float(R):
        layer(y)
        y += float(rho)
    y = cy - float(rho)
    while y >= cy - float(R):
        layer(y)
        y -= float(rho)
    return np.array(pts, np.float64).astype(np.float32).reshape(-1, 3)


def _cylinder(v, rho):
    import math
    f32 = np.float32
    cx, cy, cz = (float(f32(t)) for t in v[:3])
    dy = float(f32(v[4]))
    rb, half, rho = f32(v[6]), float(f32(v[7]) / f32(2)), f32(rho)
    rr = float(rho * rho)
    pts = []
    y, top = cy - dy * half, cy + dy * half
    while y < top:
        r = 0.0
        while r <= float(rb):
            _ring(cx, cz, y, r, math.acos(r / math.sqrt(r * r + rr)), pts)
            r += float(rho)
        y += float(rho)
    return np.array(pts, np.float64).astype(np.float32).reshape(-1, 3)


def _heart():
    vals, x = [], -3.0
    while x <= 3.0:
        vals.append(x)
        x += 0.02
    a = np.array(vals)
    Y, Z = np.meshgrid(a, a, indexing="ij")
    pts = []
    for x in a:
        arg = x * x + 2 * Y * Y + Z * Z - 1
        res = np.power(arg.astype(np.float32), np.float32(3)).astype(np.float64) - x * x * Z * Z * Z
        m = (res >= -0.001) & (res <= 0.001)
        pts.append(np.stack([np.full(m.sum(), x), Y[m], Z[m]], 1))
    return np.concatenate(pts).astype(np.float32)


def emitter_positions(typ, v, particle_radius=0.0, count=0, faces=None, seed=0, emission=0) -> np.ndarray:
    """One emission of an emitter (types as psb_emitter's), float32 (k, 3)."""
    import math
    f32 = np.float32
    if typ == 1:
        return _box(v, particle_radius)
    if typ == 2:
        return _sphere(v, particle_radius)
    if typ == 3:
        return _cylinder(v, particle_radius)
    if typ == 4:
        return _heart()
    if typ == 5:
        out = np.empty((count, 3), np.float32)
        a, b = f32(v[3]), f32(v[4])
        for i in range(count):
            t = _uniform(seed, emission, i, 0) * 6.283185307179586
            cxe, cze = float(a) * math.cos(t), float(b) * math.sin(t)
            x = f32(float(-a / f32(2)) + _uniform(seed, emission, i, 1) * float(a))
            z = f32(float(-b / f32(2)) + _uniform(seed, emission, i, 2) * float(b))
            out[i] = (f32(float(f32(v[0])) + float(x) + cxe / 100), f32(v[1]), f32(float(f32(v[2])) + float(z) + cze / 100))
        return out
    if typ == 6:
        F = np.asarray(faces, np.float32).reshape(-1, 9)
        out = np.empty((count * F.shape[0], 3), np.float32)
        for i in range(out.shape[0]):
            w = [f32(_uniform(seed, emission, i, d) * 0.5) for d in range(3)]
            s_ = float(w[0] + w[1] + w[2])
            face = F[i // count].astype(np.float64)
            for k in range(3):
                out[i, k] = f32((float(w[0]) * face[k] + float(w[1]) * face[3 + k] + float(w[2]) * face[6 + k]) / s_)
        return out
    raise ValueError(typ)


def ref_force_constant(accum, mass, direction, amplitude):
    """evaluate_ForceExt_Constante (ForceExt.cu:24-34) on a copy of accum."""
    acc = np.ascontiguousarray(accum, np.float64).copy()
    d = np.asarray(direction, np.float32)
    ref_lib().ref_force_constant(len(mass), _ptr(acc), _ptr(np.ascontiguousarray(mass, np.float64)), _ptr(d),
                                 np.float32(amplitude))
    return acc


def ref_force_trochoid(pos, accum, mass, A, k, theta, w, phi, t):
    """evaluate_ForceExt_Trochoide (ForceExt.cu:37-52) on a copy of accum."""
    acc = np.ascontiguousarray(accum, np.float64).copy()
    ref_lib().ref_force_trochoid(len(mass), _ptr(np.ascontiguousarray(pos, np.float64)), _ptr(acc),
                                 _ptr(np.ascontiguousarray(mass, np.float64)), A, k, theta, w, phi, t)
    return acc


def ref_mc_grid(centre, l, w, d, cell, dims):
    """createGrid_MarchingCube_CUDA's node centres, (nodes, 4) with value 0."""
    nx, ny, nz = (int(v) for v in dims)
    out = np.zeros((nx * ny * nz, 4), np.float64)
    c = np.asarray(centre, np.float64)
    ref_lib().ref_mc_grid(_ptr(c), l, w, d, np.float32(cell), nx, ny, nz, _ptr(out))
    return out


def refcuda_available() -> bool:
    return os.path.exists(REFCUDA_PATH)


_refcuda = None


def refcuda_lib():
    """The reference's own CUDA path (oracle/_ref/libpsbref_cuda.so)."""
    global _refcuda
    if _refcuda is None:
        if not refcuda_available():
            raise FileNotFoundError(f"{REFCUDA_PATH} is not built (make -C oracle refcuda)")
        L = ctypes.CDLL(REFCUDA_PATH)
        P, F = ctypes.c_void_p, ctypes.c_float
        L.rc_create.argtypes = [ctypes.c_int, P, F, P]
        L.rc_create.restype = P
        L.rc_destroy.argtypes = [P]
        L.rc_set.argtypes = [P, ctypes.c_char_p, P]
        L.rc_get.argtypes = [P, ctypes.c_char_p, P]
        L.rc_neighbors.argtypes = [P, P]
        L.rc_error.argtypes = [P]
        L.rc_error.restype = ctypes.c_char_p
        L.rc_pcisph_update.argtypes = [P, F, ctypes.c_double, F, P, P, ctypes.POINTER(F)]
        L.rc_wcsph_update.argtypes = [P, F, P, F, F, P, P, ctypes.POINTER(F)]
        _refcuda = L
    return _refcuda


class RefCudaSim:
    """The reference's kernels and its PCISPH launcher compiled for the GPU,
    on the reference's device layouts (AoS double), behind our guards: a
    step that would write past the reference's arrays is refused."""

    def __init__(self, scene, pos, vel=None, vel_half=None):
        L = refcuda_lib()
        n = pos.shape[0]
        self.n, self.scene = n, scene
        gmin = np.asarray(scene.grid_min, np.float32)
        dims = np.asarray(scene.dims, np.int32)
        self.h = L.rc_create(n, _ptr(gmin), scene.cell, _ptr(dims))
        if not self.h:
            raise RuntimeError("rc_create failed")
        z3 = np.zeros((n, 3))
        p = np.ascontiguousarray(pos, np.float64)
        v = z3 if vel is None else np.ascontiguousarray(vel, np.float64)
        vh = z3 if vel_half is None else np.ascontiguousarray(vel_half, np.float64)
        for name, arr in (("pos", p), ("pos_old", p), ("r_pos", p), ("r_pos_old", p), ("vel", v), ("vel_old", v),
                          ("vel_ap", vh), ("vel_av", vh), ("r_vel_ap", vh), ("r_vel_av", vh)):
            self.set(name, arr)
        ones = np.ones(n)
        for name, val in (("mass", scene.mass), ("radius", scene.h), ("rho0", scene.rho0), ("k", scene.k),
                          ("mu", scene.mu), ("sigma", scene.sigma), ("l", scene.l)):
            self.set(name, ones * val)
        self.box = (np.asarray(scene.box_min, np.float32), np.asarray(scene.box_max, np.float32))

    def __del__(self):
        if getattr(self, "h", None):
            refcuda_lib().rc_destroy(self.h)
            self.h = None

    def set(self, name, arr):
        arr = np.ascontiguousarray(arr, np.float64)
        if refcuda_lib().rc_set(self.h, name.encode(), _ptr(arr)) != 0:
            raise KeyError(name)

    def get(self, name, width):
        out = np.empty((self.n, width) if width > 1 else self.n, np.float64)
        if refcuda_lib().rc_get(self.h, name.encode(), _ptr(out)) != 0:
            raise KeyError(name)
        return out

    def neighbors(self):
        c = np.empty(self.n, np.int32)
        refcuda_lib().rc_neighbors(self.h, _ptr(c))
        return c

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {rc} ({refcuda_lib().rc_error(self.h).decode()})")

    def pcisph_update(self, threshold=10.0) -> float:
        """PCI_SPHSystem::update through the reference's pci_SPH_update; returns
        the reference's device milliseconds of the step."""
        ms = ctypes.c_float()
        s = self.scene
        self._check(refcuda_lib().rc_pcisph_update(self.h, s.dt, threshold, s.particle_radius, _ptr(self.box[0]),
                                                   _ptr(self.box[1]), ctypes.byref(ms)), "rc_pcisph_update")
        return ms.value

    def wcsph_update(self) -> float:
        ms = ctypes.c_float()
        s = self.scene
        g = np.asarray([0.0, -1.0, 0.0], np.float32)
        self._check(refcuda_lib().rc_wcsph_update(self.h, s.dt, _ptr(g), np.float32(9.81), s.particle_radius,
                                                  _ptr(self.box[0]), _ptr(self.box[1]), ctypes.byref(ms)),
                    "rc_wcsph_update")
        return ms.value


class RefSim:
    """The reference's kernels on the CPU, AoS double state (oracle/_ref)."""

    def __init__(self, scene, pos, vel=None, vel_half=None):
        L = ref_lib()
        n = pos.shape[0]
        self.n = n
        self.scene = scene
        gmin = np.asarray(scene.grid_min, np.float32)
        dims = np.asarray(scene.dims, np.int32)
        self.h = L.ref_create(n, _ptr(gmin), scene.cell, _ptr(dims))
        if not self.h:
            raise RuntimeError("ref_create failed")
        z3 = np.zeros((n, 3))
        p = np.ascontiguousarray(pos, np.float64)
        v = z3 if vel is None else np.ascontiguousarray(vel, np.float64)
        vh = z3 if vel_half is None else np.ascontiguousarray(vel_half, np.float64)
        # State as _initialize leaves it, with the restore buffers filled
        # (the reference leaves some unset: PciSphSystem.cpp:93,127-130).
        for name, arr in (("pos", p), ("pos_old", p), ("r_pos", p), ("r_pos_old", p), ("vel", v), ("vel_old", v),
                          ("vel_ap", vh), ("vel_av", vh), ("r_vel_ap", vh), ("r_vel_av", vh)):
            self.set(name, arr)
        ones = np.ones(n)
        for name, val in (("mass", scene.mass), ("radius", scene.h), ("rho0", scene.rho0), ("k", scene.k),
                          ("mu", scene.mu), ("sigma", scene.sigma), ("threshold", scene.l), ("l", scene.l)):
            self.set(name, ones * val)

    def __del__(self):
        if getattr(self, "h", None):
            ref_lib().ref_destroy(self.h)
            self.h = None

    def set(self, name, arr):
        arr = np.ascontiguousarray(arr, np.float64)
        if ref_lib().ref_set(self.h, name.encode(), _ptr(arr)) != 0:
            raise KeyError(name)

    def get(self, name, width):
        out = np.empty((self.n, width) if width > 1 else self.n, np.float64)
        if ref_lib().ref_get(self.h, name.encode(), _ptr(out)) != 0:
            raise KeyError(name)
        return out

    def search(self):
        rc = ref_lib().ref_search(self.h)
        if rc != 0:
            raise RuntimeError(f"ref_search: {rc}")
        counts = np.empty(self.n, np.int32)
        ref_lib().ref_neighbors(self.h, _ptr(counts), None)
        return counts

    def density_pci(self):
        ref_lib().ref_density_pci(self.h)
        return self.get("density", 1)

    def pcisph_update(self, iters=3, collide=True):
        s = self.scene
        bmin = np.asarray(s.box_min, np.float32)
        bmax = np.asarray(s.box_max, np.float32)
        rc = ref_lib().ref_pcisph_update(self.h, s.dt, iters, 1 if collide else 0, s.particle_radius, _ptr(bmin), _ptr(bmax))
        if rc != 0:
            raise RuntimeError(f"ref_pcisph_update: {rc}")

    def iso(self, g: IsoGrid) -> np.ndarray:
        """evaluateIso_Kernel over the nodes of g, at the current positions."""
        nodes = np.ascontiguousarray(grid_nodes(g))
        out = np.zeros(nodes.shape[0])
        rc = ref_lib().ref_iso(self.h, _ptr(nodes), int(g.dims[0]), int(g.dims[1]), int(g.dims[2]), float(g.scale),
                               _ptr(out))
        if rc != 0:
            raise RuntimeError(f"ref_iso: {rc}")
        return out

    def dem_update(self, collide=True):
        """CudaSystem::update (CudaSystem.cpp:207-224) on the state, the
        step's start state serving as the old buffers (pos_old = pos,
        vel_old = vel), with the scene's uniform contact coefficients."""
        s = self.scene
        ones = np.ones(self.n)
        for name, val in (("spring", s.dem_spring), ("damping", s.dem_damping), ("shear", s.dem_shear),
                          ("attraction", s.dem_attraction)):
            self.set(name, ones * val)
        self.set("pos_old", self.get("pos", 3))
        self.set("vel_old", self.get("vel", 3))
        bmin = np.asarray(s.box_min, np.float32)
        bmax = np.asarray(s.box_max, np.float32)
        g = np.asarray(s.gravity, np.float64)
        amp = float(np.linalg.norm(g))
        gdir = (g / amp if amp > 0 else g).astype(np.float32)
        rc = ref_lib().ref_dem_update(self.h, s.dt, _ptr(gdir), np.float32(amp), 1 if collide else 0,
                                      s.particle_radius, _ptr(bmin), _ptr(bmax))
        if rc != 0:
            raise RuntimeError(f"ref_dem_update: {rc}")

    def densities_forces(self):
        """evaluate_densities_forces (SphSystem.cu:27-43) at the current
        positions: density, pressure, f_press, f_visc, f_surf, normals, f_accum."""
        rc = ref_lib().ref_densities_forces(self.h)
        if rc != 0:
            raise RuntimeError(f"ref_densities_forces: {rc}")
        return {k: self.get(k, w) for k, w in (("density", 1), ("pressure", 1), ("f_press", 3), ("f_visc", 3),
                                                ("f_surf", 3), ("normals", 3), ("f_accum", 3))}

    def vertex_normals(self, verts, scale=1.0):
        """computeNormales_Vertex_CUDA at the vertices (n, 3), with the
        current densities."""
        verts = np.ascontiguousarray(verts, np.float64)
        out = np.zeros_like(verts)
        rc = ref_lib().ref_vertex_normals(self.h, _ptr(verts), verts.shape[0], np.float32(scale), _ptr(out))
        if rc != 0:
            raise RuntimeError(f"ref_vertex_normals: {rc}")
        return out

    def wcsph_update(self, collide=True):
        s = self.scene
        bmin = np.asarray(s.box_min, np.float32)
        bmax = np.asarray(s.box_max, np.float32)
        g = np.asarray([0.0, -1.0, 0.0], np.float32)
        rc = ref_lib().ref_wcsph_update(self.h, s.dt, _ptr(g), np.float32(9.81), 1 if collide else 0,
                                        s.particle_radius, _ptr(bmin), _ptr(bmax))
        if rc != 0:
            raise RuntimeError(f"ref_wcsph_update: {rc}")
