"""psb_upload's copies overlap the next step's grid and neighbour build.

psb_upload copies the positions on the context's stream and the
velocities, half-step velocities and pressures on a copy stream of its own;
a step taken straight after it waits for those only where it gathers them
into sorted order, after its neighbour build. Every other entry point waits
for them first.

At 1,048,576 particles from pinned host memory the 28 MB of the copy stream
outlast the grid, sort and neighbour build, so a missing wait would read
half-copied arrays. Checked here, bit for bit against the same calls with
the upload joined before the step:
  * steps straight after an upload, kernel by kernel and as CUDA graphs
    (a graph carries an event wait node that must wait for the upload made
    before each of its launches, including a graph captured earlier);
  * a download, a field read, a stream switch, a pressure pre-solve and an
    emission straight after an upload.
"""
import numpy as np
import pytest

import psb_project_b200 as P
from psb_project_b200 import runtime as R

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def pinned(a):
    out = torch.empty(np.shape(a), dtype=torch.float32, pin_memory=True).numpy()
    out[...] = a
    return out


@pytest.fixture(scope="module")
def inputs():
    sc = P.config_scene("C2").replace(warm_start=P.WARM_PREVIOUS)
    n = sc.n
    rng = np.random.default_rng(5)
    arrays = {
        "pos": pinned(P.scene_positions(sc)),
        "vel": pinned(rng.normal(0.0, 0.05, (n, 3))),
        "vel_half": pinned(rng.normal(0.0, 0.05, (n, 3))),
        "pressure": pinned(rng.uniform(0.0, 500.0, n)),
        "zero3": pinned(np.zeros((n, 3))),
        "zero1": pinned(np.zeros(n)),
    }
    return sc, arrays


def run_steps(sc, a, graph, join, rounds=3):
    outs = []
    with P.Simulation(sc) as sim:
        sim.set_graph(graph)
        # an earlier upload and step: buffers in use, and a sort for the graphs to follow
        sim.upload(a["pos"], a["zero3"], a["zero3"], a["zero1"])
        sim.step(1)
        for _ in range(rounds):
            sim.upload(a["pos"], a["vel"], a["vel_half"], a["pressure"])
            if join:
                sim.download()          # joins the copies before the step
            sim.step(1)
            outs.append(sim.download())
    return outs


def assert_same(outs, refs):
    for o, r in zip(outs, refs):
        for k in ("pos", "vel", "vel_half", "density", "pressure"):
            np.testing.assert_array_equal(o[k], r[k], err_msg=k)


def test_step_after_upload_kernel_by_kernel(inputs):
    sc, a = inputs
    assert_same(run_steps(sc, a, graph=False, join=False), run_steps(sc, a, graph=False, join=True))


def test_step_after_upload_as_graph(inputs):
    sc, a = inputs
    # graph and kernel-by-kernel steps are bit-identical, so either joined run is the reference
    assert_same(run_steps(sc, a, graph=True, join=False), run_steps(sc, a, graph=False, join=True))


def test_entry_points_see_the_upload(inputs):
    sc, a = inputs
    with P.Simulation(sc) as sim:
        sim.upload(a["pos"], a["zero3"], a["zero3"], a["zero1"])
        sim.step(1)
        sim.upload(a["pos"], a["vel"], a["vel_half"], a["pressure"])
        out = sim.download()
        for k in ("pos", "vel", "vel_half", "pressure"):
            np.testing.assert_array_equal(out[k], a[k], err_msg=k)
        sim.upload(a["pos"], a["vel_half"], a["vel"], a["zero1"])
        np.testing.assert_array_equal(sim.read_field(R.FIELD_VEL), a["vel_half"])
        np.testing.assert_array_equal(sim.read_field(R.FIELD_PRESSURE), a["zero1"])


def test_stream_switch_after_upload(inputs):
    sc, a = inputs
    ref = run_steps(sc, a, graph=False, join=True, rounds=1)
    with P.Simulation(sc) as sim:
        sim.upload(a["pos"], a["zero3"], a["zero3"], a["zero1"])
        sim.step(1)
        sim.upload(a["pos"], a["vel"], a["vel_half"], a["pressure"])
        s = torch.cuda.Stream()
        sim.set_stream(s.cuda_stream)
        sim.step(1)
        out = sim.download()
        sim.set_stream(0)
    assert_same([out], ref)


def test_presolve_and_emission_after_upload(inputs):
    """psb_presolve and psb_emit wait for the copies before they touch the state."""
    sc, a = inputs
    k = 4096
    # a block of the lattice moved into the empty half of the box
    extra = {"pos": a["pos"][:k] + np.float32([2.0, 0.0, 0.0]), "vel": a["vel"][:k]}

    def run(join):
        with P.Simulation(sc.replace(n=sc.n + k)) as sim:       # capacity for the emitted block
            sim.upload(a["pos"], a["zero3"], a["zero3"], a["zero1"])
            sim.step(1)
            sim.upload(a["pos"], a["vel"], a["vel_half"], a["pressure"])
            if join:
                sim.download()
            sim.presolve(2)
            p = sim.read_field(R.FIELD_PRESSURE)
            sim.upload(a["pos"], a["vel"], a["vel_half"], a["pressure"])
            if join:
                sim.download()
            sim.emit(extra["pos"], extra["vel"])
            sim.step(1)
            return p, sim.download()

    p_a, out_a = run(False)
    p_b, out_b = run(True)
    np.testing.assert_array_equal(p_a, p_b)
    assert_same([out_a], [out_b])
