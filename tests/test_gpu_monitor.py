"""The state monitor (the reference's -logp option) through the C ABI: the file
eb_open_monitor writes while eb_run advances equals, byte for byte, the file the
reference writes for the same network and inputs (kept with the golden fixtures):
a line at every delivery into a monitored neuron, then after each step the lines
of the neurons that spiked and of every monitored neuron."""
import pytest

from tests._cases import build_case, load_golden_text
from tests.golden.make_golden import LOG_CASES

pytestmark = pytest.mark.gpu


def monitored_run(tmp_path, name, chunks, chunk_steps=0, **kw):
    from edlut_b200.simulation import Simulation
    net, t, c, nsteps, _ = build_case(name)
    sim = Simulation.from_description(net, **kw)
    sim.inject_spikes(t, c)
    path = str(tmp_path / (name + ".logp"))
    sim.open_monitor(path, chunk_steps=chunk_steps)
    done = 0
    for n in chunks(nsteps):
        sim.run(n)
        done += n
    assert done == nsteps
    sim.close_monitor()
    sim.close()
    return open(path, "rb").read()


@pytest.mark.parametrize("kernel", ["default", "block_per_neuron"])
@pytest.mark.parametrize("persistent", [False, True], ids=["graphs", "persistent"])
@pytest.mark.parametrize("name", LOG_CASES)
def test_monitor_file_matches_the_reference_file(tmp_path, name, persistent, kernel):
    got = monitored_run(tmp_path, name, lambda n: [n], persistent=persistent,
                        wide_indegree=0 if kernel == "block_per_neuron" else None)
    want = load_golden_text(name, ".logp")
    if got != want:
        g, w = got.decode().splitlines(), want.decode().splitlines()
        first = next((i for i, (a, b) in enumerate(zip(g, w)) if a != b), min(len(g), len(w)))
        raise AssertionError("line %d differs (%d vs %d lines):\n%s\n%s" % (
            first, len(g), len(w), g[first] if first < len(g) else "<end>", w[first] if first < len(w) else "<end>"))


@pytest.mark.parametrize("name", LOG_CASES[:1])
def test_monitor_file_is_independent_of_runs_and_chunks(tmp_path, name):
    """Uneven eb_run calls, chunks shorter than a run and plain launches write the
    same file."""
    want = load_golden_text(name, ".logp")
    got = monitored_run(tmp_path, name, lambda n: [1, 7, 50, n - 58], chunk_steps=13)
    assert got == want
    got = monitored_run(tmp_path, name, lambda n: [n // 3, n - n // 3], chunk_steps=8, graph_steps=1)
    assert got == want


def test_monitor_refuses_async_runs_and_stops_at_close(tmp_path):
    from edlut_b200.simulation import Simulation
    from edlut_b200._lib import EdlutError
    net, t, c, nsteps, _ = build_case(LOG_CASES[0])
    sim = Simulation.from_description(net)
    sim.inject_spikes(t, c)
    path = str(tmp_path / "m.logp")
    sim.open_monitor(path)
    with pytest.raises(EdlutError):
        sim.run_async(5)
    sim.run(5)
    sim.close_monitor()
    size = len(open(path, "rb").read())
    assert size > 0
    sim.run(5)  # no longer monitored
    sim.run_async(5)
    sim.sync()
    assert len(open(path, "rb").read()) == size
    # the file holds the first 5 steps of the reference's file
    want = load_golden_text(LOG_CASES[0], ".logp").decode().splitlines(keepends=True)
    assert "".join(want).startswith(open(path).read())
    sim.close()


def test_monitor_off_for_unflagged_populations(tmp_path):
    """Populations without the log flag write nothing; the file still opens."""
    from edlut_b200.simulation import Simulation
    net, t, c, nsteps, _ = build_case(LOG_CASES[0])
    for layer in net.layers:
        layer.log = 0
    sim = Simulation.from_description(net)
    sim.inject_spikes(t, c)
    path = str(tmp_path / "m.logp")
    sim.open_monitor(path)
    sim.run(20)
    sim.close_monitor()
    assert open(path, "rb").read() == b""
    sim.close()
