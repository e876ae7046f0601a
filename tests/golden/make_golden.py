"""Generates the golden fixtures in this directory from the reference's own
kernels, run on the CPU (oracle/_ref, built from the reference sources by
oracle/Makefile). Run it where the reference tree exists:

    python tests/golden/make_golden.py

Each fixture holds a small seeded scene (reference-compatible physics), the
neighbour counts the reference's searchNeighbooring_Kernel produced, its
compute_Density_PCI densities, and its state after three
PCI_SPHSystem::update and three SPHSystem::update steps. The oracle must
reproduce them (tests/test_golden.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import psb_project_b200 as P  # noqa: E402

CASES = {
    "ref_small": dict(nxyz=(12, 10, 8), spacing=0.01, box=(0.3, 0.3, 0.3), h=0.02, dt=5e-4, seed=7),
    "ref_tall": dict(nxyz=(6, 20, 6), spacing=0.01, box=(0.2, 0.4, 0.2), h=0.02, dt=1e-3, seed=3),
}


def make(name, kw):
    out = {}
    for method, tag in ((P.PCISPH, "pci"), (P.WCSPH, "wc")):
        sc = P.ref_scene(method=method, **kw)
        pos = oracle.scene_positions(sc).astype(np.float64)
        ref = oracle.RefSim(sc, pos)
        if tag == "pci":
            out["pos0"] = pos
            out["nbr"] = ref.search()
            out["rho_x"] = ref.density_pci()
            ref = oracle.RefSim(sc, pos)
        for _ in range(3):
            ref.pcisph_update() if tag == "pci" else ref.wcsph_update()
        for f, w in (("pos", 3), ("vel", 3), ("vel_ap", 3), ("density", 1), ("pressure", 1)):
            out[f"{tag}_{f}"] = ref.get(f, w)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if not oracle.ref_available():
        oracle.build(with_reference=True)
    for name, kw in CASES.items():
        make(name, kw)
