"""The reference's own CUDA path on the GPU (oracle/_ref/libpsbref_cuda.so:
its kernel files and its pci_SPH_update launcher compiled unchanged for
sm_100a, behind guards that refuse a step that would write past its
arrays), pinned against the same kernels run as host code (oracle/_ref/
libpsbref.so). Both are FP64; the GPU contracts multiply-adds and fills its
cells in atomic order (so each neighbour list is a permutation of the
host's), which leaves differences of ~1e-15 per operation: 1e-9 of each
field's max over three steps. Neighbour counts are exact.

It is the baseline the bench's reference-cuda arm times; the product never
loads it."""
import numpy as np
import pytest

import oracle
import psb_project_b200 as P

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.refcuda_available() and oracle.ref_available()),
                                 reason="oracle/_ref not built")]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.mark.parametrize("method", [P.PCISPH, P.WCSPH])
def test_reference_cuda_matches_reference_on_host(method):
    sc = P.ref_scene(method=method, nxyz=(10, 14, 8), box=(0.25, 0.3, 0.2), seed=5)
    pos = oracle.scene_positions(sc).astype(np.float64)
    gpu = oracle.RefCudaSim(sc, pos)
    cpu = oracle.RefSim(sc, pos)
    for _ in range(3):
        counts = cpu.search()          # the lists of the step's start positions
        ms = gpu.pcisph_update() if method == P.PCISPH else gpu.wcsph_update()
        cpu.pcisph_update() if method == P.PCISPH else cpu.wcsph_update()
        assert ms > 0
        assert np.array_equal(gpu.neighbors(), counts)
        for name, w in (("pos", 3), ("vel", 3), ("vel_ap", 3), ("density", 1), ("pressure", 1)):
            assert rel(gpu.get(name, w), cpu.get(name, w)) <= 1e-9, name


def test_reference_cuda_refuses_a_crowded_cell():
    """65 particles in one cell: the guard refuses the step (the reference's
    storeParticles would write past the cell's 64 slots) and nothing runs."""
    sc = P.ref_scene(method=P.PCISPH)
    pos = oracle.scene_positions(sc).astype(np.float64)
    pos[:65] = pos[0] + np.random.default_rng(0).uniform(0, 1e-4, (65, 3))
    gpu = oracle.RefCudaSim(sc, pos)
    with pytest.raises(RuntimeError, match="64"):
        gpu.pcisph_update()
    assert np.array_equal(gpu.get("pos", 3), pos)


def test_reference_cuda_refuses_a_particle_outside_the_grid():
    sc = P.ref_scene(method=P.PCISPH)
    pos = oracle.scene_positions(sc).astype(np.float64)
    pos[3] = (-10.0, 0.1, 0.1)
    gpu = oracle.RefCudaSim(sc, pos)
    with pytest.raises(RuntimeError, match="grid"):
        gpu.pcisph_update()
