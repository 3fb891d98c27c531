"""Serving (continuous batching) on the GPU: every request's result equals
the same search run alone, bit for bit, whatever else shares its launches;
admission waits for device memory; cancellation and declines.

Results are compared on the full history (best fitness, mean fitness, best
wrong count and nodes, best row per history entry) and the whole final
ranked population (fitness, wrong, nodes, rows): exact equality, the
tolerance of every parity test of this engine."""
import pytest

from gagp_b200 import task as T, workloads as W

pytestmark = pytest.mark.gpu

# (population, cases, generations, seed): uneven populations, case counts
# and lengths, so that searches join and finish at different steps
SHAPES = [(256, 16, 4, 11), (512, 40, 6, 12), (1024, 100, 5, 13), (300, 64, 8, 14), (768, 23, 3, 15),
          (640, 129, 7, 16)]


def _tasks():
    cache = {}
    return [T.from_files(W.poly4(population=p, generations=g, seed=s, cases=c, max_nodes=40), cache)
            for p, c, g, s in SHAPES]


@pytest.fixture(scope="module")
def alone():
    from gagp_b200 import build
    from gagp_b200.engine import Engine
    build.build()
    with Engine(0) as engine:
        out = []
        for lt in _tasks():
            s = engine.admit(lt)
            s.run()
            out.append(s.result())
            s.close()
        return out


def _drain(server, tickets, limit=500):
    finished = {}
    for _ in range(limit):
        running, queued, _done = server.step()
        for i, t in tickets.items():
            if i not in finished and server.poll(t) == 2:
                finished[i] = server.result(t)
        if not running and not queued:
            break
    return finished


@pytest.mark.parametrize("rounds_per_step", [1, 5])
def test_results_in_the_mix_equal_alone(alone, rounds_per_step):
    from gagp_b200.engine import Engine, Server
    tasks = _tasks()
    with Engine(0) as engine, Server(engine, rounds_per_step=rounds_per_step) as server:
        tickets = {}
        # arrivals spread over the first steps: later requests join running ones
        arrivals = {0: [0, 1], 1: [2], 3: [3, 4], 4: [5]}
        for step in range(6):
            for i in arrivals.get(step, []):
                tickets[i] = server.submit(tasks[i])
            server.step()
        finished = _drain(server, tickets)
    assert sorted(finished) == list(range(len(SHAPES)))
    for i, result in finished.items():
        assert result == alone[i], i


def test_admission_waits_for_memory(alone):
    from gagp_b200.engine import Engine, Server
    tasks = _tasks()
    sizes = [Engine.search_bytes(lt) for lt in tasks]
    budget = sorted(sizes)[-1] + sorted(sizes)[-2]  # the two largest fit together
    with Engine(0) as engine, Server(engine, memory_budget=budget) as server:
        tickets = {i: server.submit(lt) for i, lt in enumerate(tasks)}
        finished, waited = {}, False
        for _ in range(500):
            running, queued, _ = server.step()
            states = {i: server.poll(t) for i, t in tickets.items() if i not in finished}
            held = sum(sizes[i] for i, st in states.items() if st == 1)
            assert held <= budget
            waited |= queued > 0
            for i, st in states.items():
                if st == 2:
                    finished[i] = server.result(tickets[i])
            if not running and not queued:
                break
    assert waited  # some request had to wait for memory
    assert sorted(finished) == list(range(len(SHAPES)))
    for i, result in finished.items():
        assert result == alone[i], i


def test_cancel_and_decline():
    from gagp_b200.engine import Engine, EngineError, Server
    tasks = _tasks()
    with Engine(0) as engine, Server(engine, max_active=1) as server:
        first, second = server.submit(tasks[0]), server.submit(tasks[1])
        server.step()
        assert server.poll(first) == 1 and server.poll(second) == 0
        server.cancel(second)  # queued
        server.cancel(first)   # running
        running, queued, _ = server.step()
        assert (running, queued) == (0, 0)
        generational = _tasks()[2]
        generational.settings.steady_state = False
        with pytest.raises(EngineError) as err:
            server.submit(generational)
        assert err.value.status == 1  # GAGP_DECLINED


def test_list_requests_equal_alone():
    """List programs through the server: a request owns copies of every
    table and case array it was submitted with (the traversal table and the
    IntList values included), so it runs the same search whenever the server
    admits it."""
    from gagp_b200 import build
    from gagp_b200.engine import Engine, Server
    build.build()
    shapes = [(128, 12, 3, 21), (200, 20, 4, 22), (96, 16, 3, 23)]
    make = lambda p, c, g, s: T.from_files(W.list_threshold(population=p, generations=g, seed=s, cases=c))  # noqa: E731
    with Engine(0) as engine:
        alone = []
        for shape in shapes:
            s = engine.admit(make(*shape))
            s.run()
            alone.append(s.result())
            s.close()
        with Server(engine, max_active=1, rounds_per_step=3) as server:
            # the tasks' own buffers go away after submit; later admissions
            # read the server's copies
            tickets = {i: server.submit(make(*shape)) for i, shape in enumerate(shapes)}
            finished = _drain(server, tickets)
    assert sorted(finished) == list(range(len(shapes)))
    for i, result in finished.items():
        assert result == alone[i], i


def test_statement_and_region_requests_equal_alone():
    """Statement programs and bounded regions through the server: each
    request's tables (the bounded-region plans of the region table
    included) are the server's copies, and the region kernel's workspace is
    sized at admission, so a request runs the same search as alone."""
    from gagp_b200 import build
    from gagp_b200.engine import Engine, Server
    build.build()
    makers = [lambda: T.from_files(W.list_statements(population=128, generations=4, seed=31, cases=16)),
              lambda: T.from_files(W.grid_paths(population=160, generations=5, seed=32, cases=30)),
              lambda: T.from_files(W.grid_paths(population=96, generations=4, seed=33, cases=20, ambiguous=True))]
    with Engine(0) as engine:
        alone = []
        for make in makers:
            s = engine.admit(make())
            s.run()
            alone.append(s.result())
            s.close()
        with Server(engine, max_active=2, rounds_per_step=2) as server:
            tickets = {i: server.submit(make()) for i, make in enumerate(makers)}
            finished = _drain(server, tickets)
    assert sorted(finished) == list(range(len(makers)))
    for i, result in finished.items():
        assert result == alone[i], i
