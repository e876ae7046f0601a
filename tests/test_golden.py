"""The oracle against golden fixtures generated from the reference's own
kernels run on the CPU (tests/golden/make_golden.py). These pin the oracle
even where the reference tree and oracle/_ref are absent."""
import os

import numpy as np
import pytest

import oracle
import psb_project_b200 as P
from tests.golden.make_golden import CASES

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_fixture(name):
    g = np.load(os.path.join(HERE, f"{name}.npz"))
    kw = CASES[name]
    sc = P.ref_scene(method=P.PCISPH, **kw)
    pos = oracle.scene_positions(sc).astype(np.float64)
    assert np.array_equal(pos, g["pos0"]), "scene generator drifted from the fixture"
    counts, lists = oracle.neighbors(sc, pos)
    assert np.array_equal(counts, g["nbr"])
    rho = oracle.density(sc, pos, counts, lists, clamp=False)
    assert rel(rho, g["rho_x"]) < 1e-12
    for method, tag in ((P.PCISPH, "pci"), (P.WCSPH, "wc")):
        sc = P.ref_scene(method=method, **kw)
        sim = oracle.OracleSim(sc, pos)
        for _ in range(3):
            sim.step()
        assert rel(sim.pos, g[f"{tag}_pos"]) < 1e-12
        assert rel(sim.vel, g[f"{tag}_vel"]) < 1e-10
        assert rel(sim.vel_half, g[f"{tag}_vel_ap"]) < 1e-10
        assert rel(sim.rho, g[f"{tag}_density"]) < 1e-12
        assert rel(sim.p, g[f"{tag}_pressure"]) < 1e-10
