"""Autotuner (psb_autotune / psb_tune_set): launch configurations per size
bucket.

The known answer: every candidate computes the same result bit for bit.
One thread still handles one particle and sums its list in the same
order; the row-tile schedule of the neighbour build accepts the same
candidates in the same slot order as the per-thread walk; the fused
schedule computes the density at x (and the network's inputs) with the
separate pass's pair arithmetic in the same order. So a scene stepped under
any configuration -- block sizes 128/256/512, any neighbour schedule -- must
end in exactly the default's state, in both physics profiles and in a
batch (where the fused schedule runs as the per-thread walk). The tuner itself must leave the state
untouched and store its choice for the bucket.
"""
import numpy as np
import pytest

import psb_project_b200 as P
from psb_project_b200.runtime import FIELD_NBR_COUNT, FIELD_SORTED_ID, PsbTune, Simulation

CONFIGS = [
    dict(nbr_block=128, nbr_schedule=1, density_block=128, init_block=128, pci_density_block=128, force_block=128,
         xsph_block=128),
    dict(nbr_block=512, nbr_schedule=1, density_block=512, init_block=512, pci_density_block=512, force_block=512,
         xsph_block=512),
    dict(nbr_block=256, nbr_schedule=1),
    dict(nbr_block=512, nbr_schedule=0, density_block=128, force_block=512),
    dict(nbr_block=128, nbr_schedule=2),
    dict(nbr_block=512, nbr_schedule=2, density_block=128, force_block=128),
]


def test_bucket():
    assert Simulation.size_bucket(1) == 0 and Simulation.size_bucket(1024) == 10
    assert Simulation.size_bucket(1048575) == 19 and Simulation.size_bucket(1048576) == 20
    assert PsbTune.KERNELS[0] == "build_nbr"


def run(sc, steps, tune=None, weights=None):
    with P.Simulation(sc) as sim:
        if weights is not None:
            sim.mlp_set_weights(weights)
        if tune is not None:
            sim.tune_set(Simulation.size_bucket(sc.n), **tune)
        sim.upload(P.scene_positions(sc))
        if sc.method == P.PCISPH and sc.profile == P.PROFILE_CONFIG:
            sim.presolve(8)
        for _ in range(steps):
            sim.step(1)
        out = sim.download()
        out["nbr"] = sim.read_field(FIELD_NBR_COUNT)
        out["order"] = sim.read_field(FIELD_SORTED_ID)
        return out


def same(a, b):
    for k in ("pos", "vel", "vel_half", "density", "pressure", "nbr", "order"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", range(len(CONFIGS)))
def test_configs_bit_identical_config_profile(cfg):
    sc = P.dam_break((14, 12, 10), 0.01, (0.4, 0.4, 0.3), 0.02, dt=5e-4, seed=21).replace(warm_start=P.WARM_LEARNED)
    w = P.mlp_init_weights(2)
    same(run(sc, 6, None, w), run(sc, 6, CONFIGS[cfg], w))


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [0, 1, 4])
def test_configs_bit_identical_reference_profile(cfg):
    sc = P.ref_scene(seed=22, jitter=2e-3)
    same(run(sc, 4), run(sc, 4, CONFIGS[cfg]))


@pytest.mark.gpu
def test_configs_bit_identical_batch():
    scenes = P.batch_scenes(n_scenes=4, seed=23, n_range=(300, 2500), side=(0.3, 0.5), dt=5e-4)
    w = P.mlp_init_weights(4)
    outs = []
    for tune in (None, CONFIGS[1], CONFIGS[5]):
        with P.BatchSimulation(scenes) as b:
            b.mlp_set_weights(w)
            b.set_graph(True)
            if tune is not None:
                b.tune_set(Simulation.size_bucket(b.first[-1]), **tune)
            b.upload(P.batch_positions(scenes))
            b.step(5)
            outs.append((b.download(), b.batch_stats()["iters_total"]))
    for o in outs[1:]:
        for k in ("pos", "vel", "pressure"):
            assert np.array_equal(outs[0][0][k], o[0][k]), k
        assert np.array_equal(outs[0][1], o[1])


@pytest.mark.gpu
def test_autotune_keeps_state_and_stores_choice():
    sc = P.dam_break((16, 14, 12), 0.01, (0.5, 0.4, 0.4), 0.02, dt=5e-4, seed=24).replace(warm_start=P.WARM_LEARNED)
    w = P.mlp_init_weights(1)
    ref = run(sc, 6, None, w)
    with P.Simulation(sc) as sim:
        sim.mlp_set_weights(w)
        sim.upload(P.scene_positions(sc))
        sim.presolve(8)
        sim.step(3)
        before = sim.download()
        t = sim.autotune(trials=2)
        after = sim.download()
        for k in ("pos", "vel", "vel_half", "density", "pressure"):
            assert np.array_equal(before[k], after[k]), k
        assert t["bucket"] == Simulation.size_bucket(sc.n)
        for k in ("nbr_block", "density_block", "init_block", "pci_density_block", "force_block", "xsph_block"):
            assert t[k] in (128, 256, 512), (k, t[k])
        assert t["nbr_schedule"] in (0, 1, 2)
        assert all(t["ms"][k] > 0 and t["ms"][k] <= t["ms_default"][k] for k in t["ms"])
        assert sim.tune_get(t["bucket"])["force_block"] == t["force_block"]
        sim.step(3)
        got = sim.download()
    for k in ("pos", "vel", "pressure"):
        assert np.array_equal(got[k], ref[k]), k


@pytest.mark.gpu
def test_tune_cache_round_trip(tmp_path):
    sc = P.dam_break((10, 10, 8), 0.01, (0.3, 0.3, 0.3), 0.02, dt=5e-4, seed=25)
    path = str(tmp_path / "tune.json")
    b = Simulation.size_bucket(sc.n)
    with P.Simulation(sc) as a:
        a.tune_set(b, **CONFIGS[3])
        a.tune_set(b + 3, **CONFIGS[0])
        a.save_tune(path)
    with P.Simulation(sc) as c:
        assert c.load_tune(path) == 2
        for bucket, cfg in ((b, CONFIGS[3]), (b + 3, CONFIGS[0])):
            got = c.tune_get(bucket)
            for k in Simulation.TUNE_FIELDS:
                assert got[k] == cfg.get(k, 0), (bucket, k)
