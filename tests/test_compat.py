"""The reference-signature launchers (include/psb_compat.h) on the GPU,
called as the reference's system classes call them: device buffers in the
reference's AoS double3 layout, UniformGrid and partVoisine by the
reference's definitions.

  * createGrid / storeParticles / searchNeighbooring: the same neighbour
    sets as the reference's kernels run on the host (slot order inside a
    cell follows atomics there as here, so sets are compared);
  * integrateSPHSystem, interpolateSPHVelocities, integrateSystem,
    collisionSystem_Box_CUDA, interactionSystem: the reference's formulas
    restated in numpy, within a few ulps (FMA contraction on the GPU);
  * pci_SPH_update: against the reference's own pci_SPH_update on the host,
    at the parity suite's tolerances (positions 4 ulps of FP32 + 1e-5 of the
    displacement, velocities 3e-5, density 1e-5, pressure 2e-5 of the max).
"""
import ctypes

import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from psb_project_b200 import runtime as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

F3 = ctypes.c_float * 3


class UniformGrid(ctypes.Structure):
    _fields_ = [("Min", F3), ("Max", F3), ("sizeCell", ctypes.c_float), ("l", ctypes.c_double),
                ("h", ctypes.c_double), ("d", ctypes.c_double), ("indexParticles", ctypes.c_void_p),
                ("nbParticles", ctypes.c_void_p), ("m_dPos", ctypes.c_void_p), ("m_hPos", ctypes.c_void_p),
                ("m_dIsoVal", ctypes.c_void_p), ("m_hIsoVal", ctypes.c_void_p), ("m_dIsoNorm", ctypes.c_void_p),
                ("m_hIsoNorm", ctypes.c_void_p), ("nbCellsX", ctypes.c_int), ("nbCellsY", ctypes.c_int),
                ("nbCellsZ", ctypes.c_int)]


class PartVoisine(ctypes.Structure):
    _fields_ = [("nbVoisines", ctypes.c_void_p), ("listeVoisine", ctypes.c_void_p)]


class Vec3(ctypes.Structure):
    _fields_ = [("e", ctypes.c_double * 3)]


def L():
    lib = R.lib()
    D, I, V = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    lib.createGrid.argtypes = [D, D, D, D, D, D, ctypes.c_float, ctypes.POINTER(UniformGrid)]
    lib._finalizeGrid.argtypes = [ctypes.POINTER(UniformGrid)]
    lib.reinitCells.argtypes = [ctypes.POINTER(UniformGrid)]
    lib.storeParticles.argtypes = [ctypes.POINTER(UniformGrid), V, ctypes.c_uint]
    lib.searchNeighbooring.argtypes = [V, V, ctypes.POINTER(UniformGrid), D, PartVoisine, ctypes.c_uint]
    lib.integrateSPHSystem.argtypes = [V, V, V, V, V, V, D, I]
    lib.interpolateSPHVelocities.argtypes = [V, V, V, V, I]
    lib.integrateSystem.argtypes = [V, V, V, V, V, V, D, I, I]
    lib.interactionSystem.argtypes = [V, V, V, V, V, V, V, V, PartVoisine, I]
    # Vector3 by value reaches the callee through a hidden pointer (its copy
    # constructor is user-provided): a C caller passes the pointer
    PV3 = ctypes.POINTER(Vec3)
    lib.collisionSystem_Box_CUDA.argtypes = [V, V, V, ctypes.c_float, ctypes.c_float, I, PV3, PV3, ctypes.c_bool,
                                             ctypes.c_float]
    lib.pci_SPH_update.argtypes = [V] * 19 + [D, PartVoisine, V, V, V, V, V, ctypes.c_float, ctypes.c_uint]
    for f in ("createGrid", "_finalizeGrid", "reinitCells", "storeParticles", "searchNeighbooring",
              "integrateSPHSystem", "interpolateSPHVelocities", "integrateSystem", "interactionSystem",
              "collisionSystem_Box_CUDA", "pci_SPH_update"):
        getattr(lib, f).restype = None
    return lib


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_grid_and_neighbour_lists_match_reference():
    lib = L()
    sc = P.ref_scene(seed=4, jitter=2e-3)
    pos = oracle.scene_positions(sc).astype(np.float64)
    n = pos.shape[0]
    g = UniformGrid()
    # the reference's PCISPH grid: createGrid(0, 0, 0, 1, 1, 1, h) (PciSphSystem.cpp:143)
    lib.createGrid(0.0, 0.0, 0.0, 1.0, 1.0, 1.0, np.float32(sc.h), ctypes.byref(g))
    d_pos, d_rad = dev(pos), dev(np.full(n, sc.h))
    nb, lst = dev(np.zeros(n), torch.int32), dev(np.zeros(n * 200), torch.int32)
    lib.reinitCells(ctypes.byref(g))
    lib.storeParticles(ctypes.byref(g), ptr(d_pos), n)
    lib.searchNeighbooring(ptr(d_pos), ptr(d_rad), ctypes.byref(g), 1.0, PartVoisine(nb.data_ptr(), lst.data_ptr()), n)
    counts, lists = host(nb), host(lst).reshape(n, 200)
    ref = oracle.RefSim(sc.replace(grid_min=(-0.5, -0.5, -0.5), dims=(g.nbCellsX, g.nbCellsY, g.nbCellsZ),
                                   cell=float(np.float32(sc.h))), pos)
    want = ref.search()
    assert np.array_equal(counts, want)
    wl = np.zeros((n, 200), np.int32)
    oracle.ref_lib().ref_neighbors(ref.h, oracle._ptr(np.zeros(n, np.int32)), oracle._ptr(wl))
    for i in range(n):
        assert sorted(lists[i, :counts[i]]) == sorted(wl[i, :counts[i]])
    lib._finalizeGrid(ctypes.byref(g))


def test_elementwise_launchers():
    lib = L()
    rng = np.random.default_rng(5)
    n = 1000
    x, v, vh, f = (rng.normal(0, 1, (n, 3)) for _ in range(4))
    rho, m = rng.uniform(900, 1100, n), rng.uniform(0.5, 2.0, n)
    dt = 1e-3
    dtf = float(np.float32(dt))
    tol = 4 * np.finfo(np.float64).eps
    # integrateSPHSystem: v- = v+, v+ += F/rho dt, x_old = x, x += v+ dt
    d = {k: dev(a) for k, a in dict(vav=np.zeros((n, 3)), vap=vh, xold=np.zeros((n, 3)), x=x, f=f, rho=rho).items()}
    lib.integrateSPHSystem(ptr(d["vav"]), ptr(d["vap"]), ptr(d["xold"]), ptr(d["x"]), ptr(d["f"]), ptr(d["rho"]), dt, n)
    vap = vh + (f * (1.0 / rho)[:, None]) * dtf
    assert np.allclose(host(d["vap"]), vap, rtol=tol, atol=0)
    assert np.array_equal(host(d["vav"]), vh) and np.array_equal(host(d["xold"]), x)
    assert np.allclose(host(d["x"]), x + vap * dtf, rtol=tol, atol=1e-15)
    # interpolateSPHVelocities
    d2 = {k: dev(a) for k, a in dict(vav=v, vap=vh, vold=np.zeros((n, 3)), vel=f).items()}
    lib.interpolateSPHVelocities(ptr(d2["vav"]), ptr(d2["vap"]), ptr(d2["vold"]), ptr(d2["vel"]), n)
    assert np.array_equal(host(d2["vold"]), f) and np.array_equal(host(d2["vel"]), (v + vh) * 0.5)
    # integrateSystem (integrateEuler on the new buffers)
    d3 = {k: dev(a) for k, a in dict(x=x, v=v, f=f, m=m).items()}
    lib.integrateSystem(None, ptr(d3["x"]), None, ptr(d3["v"]), ptr(d3["f"]), ptr(d3["m"]), dt, 0, n)
    assert np.allclose(host(d3["v"]), v + (f * (1.0 / m)[:, None]) * dtf, rtol=tol, atol=1e-15)
    assert np.allclose(host(d3["x"]), x + v * dtf, rtol=tol, atol=1e-15)
    # collisionSystem_Box_CUDA on a unit box, r = 0.1
    bx = rng.uniform(-0.2, 1.2, (n, 3))
    d4 = {k: dev(a) for k, a in dict(x=bx, v=v).items()}
    lo, hi = Vec3((ctypes.c_double * 3)(0, 0, 0)), Vec3((ctypes.c_double * 3)(1, 1, 1))
    lib.collisionSystem_Box_CUDA(ptr(d4["x"]), None, ptr(d4["v"]), 0.1, dtf, n, ctypes.byref(lo), ctypes.byref(hi),
                                 True, 0.0)
    xw, vw = bx.copy(), v.copy()
    r = np.float32(0.1)
    for i in range(n):
        pI, nI = xw[i].copy(), np.zeros(3)
        for a in range(3):
            if xw[i, a] >= np.float32(1) - r:
                pI[a], nI[a] = np.float32(1) - r, -1.0
        for a in range(3):
            if xw[i, a] <= np.float32(0) + r:
                pI[a], nI[a] = np.float32(0) + r, 1.0
        ln = np.linalg.norm(nI)
        if ln > 0:
            nI = nI / ln
            xw[i] = pI
            vw[i] = vw[i] - np.dot(vw[i], nI) * nI
    assert np.allclose(host(d4["x"]), xw, rtol=0, atol=1e-15)
    assert np.allclose(host(d4["v"]), vw, rtol=1e-14, atol=1e-15)


def test_interaction_system_spring_forces():
    lib = L()
    sc = P.dem_block((6, 6, 6), 0.02, (0.1, 0.1, 0.1), (0.5, 0.5, 0.5), 0.01, profile=P.PROFILE_REF, spring=20.0,
                     h=0.025, jitter=2e-3, seed=2)
    pos = oracle.scene_positions(sc).astype(np.float64)
    n = pos.shape[0]
    counts, lists = oracle.neighbors(sc, pos)
    nb, lst = np.zeros(n, np.int32), np.zeros((n, 200), np.int32)
    for i in range(n):
        nb[i] = counts[i]
        lst[i, :counts[i]] = lists[i, :counts[i]]
    d_nb, d_lst = dev(nb, torch.int32), dev(lst.ravel(), torch.int32)
    d_x, d_f = dev(pos), dev(np.zeros((n, 3)))
    d_r, d_k = dev(np.full(n, sc.h)), dev(np.full(n, 20.0))
    lib.interactionSystem(ptr(d_x), None, ptr(d_f), ptr(d_r), ptr(d_k), None, None, None,
                          PartVoisine(d_nb.data_ptr(), d_lst.data_ptr()), n)
    want = np.zeros((n, 3))
    R2 = float(np.float32(sc.h + sc.h))
    for a in range(n):
        for b in lst[a, :nb[a]]:
            rel = pos[b] - pos[a]
            dist = np.sqrt((rel[0] ** 2 + rel[1] ** 2) + rel[2] ** 2)
            if dist > 0 and dist < np.float32(R2 * 2):
                want[a] += (-20.0 * (R2 - dist)) * (rel * (1.0 / dist))
    assert np.allclose(host(d_f), want, rtol=1e-12, atol=1e-12)


def test_pci_sph_update_matches_reference():
    lib = L()
    sc = P.ref_scene(seed=6, jitter=1e-4)
    pos = P.scene_positions(sc).astype(np.float64)
    n = pos.shape[0]
    rng = np.random.default_rng(2)
    vel = rng.normal(0, 0.05, (n, 3)).astype(np.float32).astype(np.float64)
    ref = oracle.RefSim(sc, pos, vel, vel)
    ref.pcisph_update(collide=False)
    z3, z1 = np.zeros((n, 3)), np.zeros(n)
    b = {k: dev(a) for k, a in dict(old=z3, pos=pos, vel=vel, vav=z3, vap=vel, rho=z1, p=z1, err=z1).items()}
    prm = {k: dev(np.full(n, v)) for k, v in dict(m=sc.mass, h=sc.h, rho0=sc.rho0, k=sc.k, mu=sc.mu, l=sc.l,
                                                  sigma=sc.sigma).items()}
    scratch = [dev(z3) for _ in range(9)]      # restore_* x4, normales, force* x4: the caller's buffers
    pv = PartVoisine(None, None)
    args = [ptr(b["old"]), ptr(b["pos"]), ptr(b["vel"]), ptr(b["vav"]), ptr(b["vap"])] + \
           [ptr(t) for t in scratch[:4]] + \
           [ptr(prm["m"]), ptr(prm["h"]), ptr(b["rho"]), ptr(prm["rho0"]), ptr(b["err"]), ptr(b["p"]),
            ptr(prm["k"]), ptr(prm["mu"]), ptr(prm["l"]), ptr(prm["sigma"]), sc.l, pv] + \
           [ptr(t) for t in scratch[4:]] + [float(np.float32(sc.dt)), n]
    lib.pci_SPH_update(*args)
    out_pos, out_vap = host(b["pos"]), host(b["vap"])
    disp = np.max(np.abs(ref.get("pos", 3) - pos))
    ulp = np.spacing(np.float32(np.max(np.abs(pos))))
    assert np.max(np.abs(out_pos - ref.get("pos", 3))) <= 4 * float(ulp) + 1e-5 * disp
    rel = lambda a, w: np.max(np.abs(a - w)) / np.max(np.abs(w))
    assert rel(out_vap, ref.get("vel_ap", 3)) <= 3e-5
    assert np.array_equal(host(b["vav"]), vel) and np.array_equal(host(b["old"]), pos)
    assert np.max(np.abs(host(b["rho"]) - ref.get("density", 1)) / ref.get("density", 1)) <= 1e-5
    assert rel(host(b["p"]), ref.get("pressure", 1)) <= 2e-5
