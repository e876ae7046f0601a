"""Batched scenes (psb_create_batch) and CUDA-graph stepping.

A batch steps independent scenes together, one launch per sweep over all of
them, with each scene's own grid, walls and convergence test. The known
answer is the single-scene path: every scene of a batch must end in exactly
the state (bit for bit) and with exactly the corrector iteration counts it
has when stepped alone, because it takes the same passes over the same data
in the same order. Graph stepping (the whole step one cudaGraphLaunch, the
corrector a conditional while node) must equal eager stepping bit for bit.

CPU tests: the C3 scene generator, and the batch checks psb_create_batch
makes before it touches a device.
"""
import ctypes

import numpy as np
import pytest

import psb_project_b200 as P
from psb_project_b200.runtime import EINVAL, lib
from psb_project_b200.scene import PsbScene


def small_batch(n=5, warm_start=P.WARM_ZERO, seed=11):
    return P.batch_scenes(n_scenes=n, seed=seed, n_range=(300, 2500), side=(0.3, 0.5), warm_start=warm_start,
                          dt=5e-4)


def test_c3_generator():
    sc = P.batch_scenes()
    assert len(sc) == 64
    ns = np.array([s.n for s in sc])
    assert ns.min() >= 3000 and ns.max() <= 140000
    assert 1.5e6 < ns.sum() < 3.5e6
    for s in sc:
        assert all(1.0 <= b <= 2.0 for b in s.box_max)
        nx, ny, nz = s.blocks[0].nxyz
        frac = ny * s.blocks[0].spacing / s.box_max[1]
        assert 0.39 <= frac <= 0.71
        assert nx * s.blocks[0].spacing < s.box_max[0] and nz * s.blocks[0].spacing < s.box_max[2]
        assert s.warm_start == P.WARM_LEARNED and s.method == P.PCISPH and s.profile == P.PROFILE_CONFIG
    # seeded: the same draw every time
    assert [s.n for s in P.batch_scenes()] == list(ns)
    # shared constants (a batch's requirement)
    for s in sc[1:]:
        assert (s.h, s.mass, s.dt, s.cell, s.particle_radius, s.xsph) == \
               (sc[0].h, sc[0].mass, sc[0].dt, sc[0].cell, sc[0].particle_radius, sc[0].xsph)


def _create(scenes):
    arr = (PsbScene * len(scenes))(*[s.to_c() for s in scenes])
    h = ctypes.c_void_p()
    return lib().psb_create_batch(arr, len(scenes), ctypes.byref(h))


def test_batch_rejects_mismatched_scenes():
    sc = small_batch(3)
    assert _create([sc[0], sc[1].replace(dt=1e-3)]) == EINVAL
    assert _create([sc[0], sc[1].replace(h=0.021)]) == EINVAL
    assert _create([sc[0], sc[1].replace(eta=0.02)]) == EINVAL
    assert _create([sc[0].replace(method=P.WCSPH), sc[1].replace(method=P.WCSPH)]) == EINVAL
    assert _create([s.replace(profile=P.PROFILE_REF) for s in sc]) == EINVAL
    assert _create([]) == EINVAL


def run_single(sc, steps, weights=None, presolve=0):
    with P.Simulation(sc) as sim:
        if weights is not None:
            sim.mlp_set_weights(weights)
        sim.upload(P.scene_positions(sc))
        if presolve:
            sim.presolve(presolve)
        iters = []
        for _ in range(steps):
            sim.step(1)
            iters.append(sim.stats().iters)
        return sim.download(), iters


def run_batch(scenes, steps, weights=None, presolve=0, graph=False, corrector=P.CORRECTOR_LAUNCHES):
    with P.BatchSimulation(scenes) as b:
        if weights is not None:
            b.mlp_set_weights(weights)
        b.set_graph(graph)
        b.set_corrector(corrector)
        b.upload(P.batch_positions(scenes))
        if presolve:
            b.presolve(presolve)
        iters = []
        for _ in range(steps):
            b.step(1)
            iters.append(b.batch_stats()["iters"].copy())
        return b.download(), np.array(iters), b.split, b.batch_stats()


@pytest.mark.gpu
@pytest.mark.parametrize("warm", ["zero", "learned"])
def test_batch_equals_scenes_alone(warm):
    mode = P.WARM_ZERO if warm == "zero" else P.WARM_LEARNED
    scenes = small_batch(4, warm_start=mode)
    w = P.mlp_init_weights(3) if warm == "learned" else None
    steps = 12
    out, iters, split, st = run_batch(scenes, steps, w, presolve=16)
    for s, sc in enumerate(scenes):
        ref, ref_iters = run_single(sc, steps, w, presolve=16)
        for key in ("pos", "vel", "vel_half", "pressure", "density"):
            got = split(out[key])[s]
            assert np.array_equal(got, ref[key]), (s, key, np.max(np.abs(got - ref[key])))
        assert list(iters[:, s]) == ref_iters, (s, list(iters[:, s]), ref_iters)
        assert st["iters_total"][s] == sum(ref_iters)
    # the scenes really differed in work
    assert iters.max() >= 3


@pytest.mark.gpu
def test_graph_equals_eager():
    scenes = small_batch(6, warm_start=P.WARM_LEARNED, seed=12)
    w = P.mlp_init_weights(5)
    steps = 10
    eager, it_e, _, st_e = run_batch(scenes, steps, w, presolve=8, graph=False)
    graph, it_g, _, st_g = run_batch(scenes, steps, w, presolve=8, graph=True)
    for key in ("pos", "vel", "vel_half", "pressure", "density"):
        assert np.array_equal(eager[key], graph[key]), key
    assert np.array_equal(it_e, it_g)
    assert np.array_equal(st_e["iters_total"], st_g["iters_total"])
    assert np.array_equal(st_e["err_final"], st_g["err_final"])


@pytest.mark.gpu
def test_batch_of_one_equals_single_and_retires_scenes():
    sc = small_batch(1, warm_start=P.WARM_ZERO, seed=13)[0]
    out, iters, split, st = run_batch([sc], 8, presolve=4, graph=True)
    ref, ref_iters = run_single(sc, 8, presolve=4)
    assert np.array_equal(out["pos"], ref["pos"]) and list(iters[:, 0]) == ref_iters
    assert st["converged"][0] == 1 and st["err_final"][0] <= sc.eta


@pytest.mark.gpu
def test_batch_max_iters_and_noconv():
    # eta unreachable in 3 passes: every scene stops at max_iters, unconverged
    scenes = [s.replace(eta=1e-9, min_iters=1, max_iters=3) for s in small_batch(3, seed=14)]
    with P.BatchSimulation(scenes) as b:
        b.set_graph(True)
        b.upload(P.batch_positions(scenes))
        rc = b.step(3)
        st = b.batch_stats()
    assert rc == P.runtime.ENOCONV
    assert list(st["iters"]) == [3, 3, 3] and list(st["converged"]) == [0, 0, 0]
    assert list(st["unconverged_steps"]) == [3, 3, 3]
    ref, ref_iters = run_single(scenes[1], 3)
    assert ref_iters == [3, 3, 3]


@pytest.mark.gpu
def test_graph_after_reupload_equals_eager():
    # the step right after an upload also runs as a graph (its reset node
    # clears the previous set's cells); restoring a downloaded state and
    # stepping must give the same result both ways
    scenes = small_batch(3, warm_start=P.WARM_ZERO, seed=15)
    res = []
    for graph in (False, True):
        with P.BatchSimulation(scenes) as b:
            b.set_graph(graph)
            b.upload(P.batch_positions(scenes))
            b.step(3)
            snap = b.download()
            for _ in range(2):
                b.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])
                b.step(2)
            res.append((b.download(), b.batch_stats()["iters_total"]))
    for key in ("pos", "vel", "pressure"):
        assert np.array_equal(res[0][0][key], res[1][0][key]), key
    assert np.array_equal(res[0][1], res[1][1])


def run_single_graph(sc, steps, weights, presolve, graph, corrector=P.CORRECTOR_LAUNCHES):
    with P.Simulation(sc) as sim:
        if weights is not None:
            sim.mlp_set_weights(weights)
        sim.set_graph(graph)
        sim.set_corrector(corrector)
        sim.upload(P.scene_positions(sc))
        if presolve:
            sim.presolve(presolve)
        its, errs = [], []
        for _ in range(steps):
            sim.step(1)
            st = sim.stats()
            its.append(st.iters)
            errs.append([st.err[k] for k in range(st.iters + 1)])
        out = sim.download()
        out["iters_total"] = sim.stats().iters_total
        return out, its, errs


@pytest.mark.gpu
@pytest.mark.parametrize("warm", ["zero", "learned"])
def test_single_scene_graph_equals_eager(warm):
    """A config-profile PCISPH scene stepped as one CUDA graph per step
    (the corrector a device-side while node) gives the kernel-by-kernel
    result bit for bit, with the same corrections and error history."""
    mode = P.WARM_ZERO if warm == "zero" else P.WARM_LEARNED
    sc = small_batch(1, warm_start=mode, seed=21)[0]
    w = P.mlp_init_weights(7) if warm == "learned" else None
    eager, it_e, err_e = run_single_graph(sc, 12, w, 8, graph=False)
    graph, it_g, err_g = run_single_graph(sc, 12, w, 8, graph=True)
    for key in ("pos", "vel", "vel_half", "pressure", "density"):
        assert np.array_equal(eager[key], graph[key]), key
    assert it_e == it_g and err_e == err_g
    assert eager["iters_total"] == graph["iters_total"] == sum(it_e)
    assert max(it_e) >= 3


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_persistent_corrector_equals_launches(graph):
    """The corrector loop as one cooperative launch (grid-wide barriers for
    the kernel boundaries) gives the three-kernels-per-pass loop's batch bit
    for bit: same corrections per scene, same error history, same state;
    stepped eagerly and captured in the step's graph."""
    # eta 0.1% from p = 0 with min_iters 1: the scenes need different numbers
    # of corrections (the oracle takes 4 to 9 on the first step), so they
    # retire at different passes
    scenes = [s.replace(eta=1e-3, min_iters=1) for s in small_batch(6, warm_start=P.WARM_ZERO, seed=31)]
    ref, it_r, _, st_r = run_batch(scenes, 10, None, presolve=8, graph=graph)
    got, it_p, _, st_p = run_batch(scenes, 10, None, presolve=8, graph=graph, corrector=P.CORRECTOR_PERSISTENT)
    for key in ("pos", "vel", "vel_half", "pressure", "density"):
        assert np.array_equal(ref[key], got[key]), key
    assert np.array_equal(it_r, it_p)
    assert np.array_equal(st_r["iters_total"], st_p["iters_total"])
    assert np.array_equal(st_r["err_final"], st_p["err_final"])
    assert any(len(set(row)) >= 2 for row in it_r)           # scenes retired at different passes


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_single_scene_persistent_corrector_equals_launches(graph):
    sc = small_batch(1, warm_start=P.WARM_ZERO, seed=32)[0]
    ref, it_r, err_r = run_single_graph(sc, 10, None, 8, graph=graph)
    got, it_p, err_p = run_single_graph(sc, 10, None, 8, graph=graph, corrector=P.CORRECTOR_PERSISTENT)
    for key in ("pos", "vel", "vel_half", "pressure", "density"):
        assert np.array_equal(ref[key], got[key]), key
    assert it_r == it_p and err_r == err_p
    assert ref["iters_total"] == got["iters_total"] == sum(it_r)


@pytest.mark.gpu
def test_persistent_corrector_max_iters_and_modes():
    # eta unreachable in 3 passes: every scene stops at max_iters, as the launches do
    scenes = [s.replace(eta=1e-9, min_iters=1, max_iters=3) for s in small_batch(3, seed=33)]
    with P.BatchSimulation(scenes) as b:
        b.set_corrector(P.CORRECTOR_PERSISTENT)
        b.upload(P.batch_positions(scenes))
        rc = b.step(3)
        st = b.batch_stats()
        with pytest.raises(P.runtime.PsbError):
            b.set_corrector(7)
    assert rc == P.runtime.ENOCONV
    assert list(st["iters"]) == [3, 3, 3] and list(st["converged"]) == [0, 0, 0]
    assert list(st["unconverged_steps"]) == [3, 3, 3]
    ref = P.ref_scene()
    with P.Simulation(ref) as sim:                # the reference profile keeps its host loop
        with pytest.raises(P.runtime.PsbError):
            sim.set_corrector(P.CORRECTOR_PERSISTENT)
