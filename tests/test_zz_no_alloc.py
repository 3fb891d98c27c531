"""The no-allocation row evaluator against the allocating one (GPU).

gagp_b200_evaluate_rows_static serves callers that may not allocate device
memory (a host application whose own allocator owns the device memory, or a
latency-critical scoring loop that cannot pay for an allocation per call):
its buffers live in one static device array.  Two calls in a row must each equal gagp_b200_evaluate_rows exactly
(fitness and wrong counts are integers here), which also shows the shared
array carries nothing over from the previous call; an oversized request is
rejected before any device work.  Collected last so that a failure here
leaves every other test already run."""
import numpy as np
import pytest

from gagp_b200 import abi, task as T, workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


def _rows_for(tmp_path, seed, cases, population):
    files = W.poly4(population=population, generations=2, seed=seed, cases=cases)
    lt = T.load(files.write(str(tmp_path / str(seed))), str(tmp_path / str(seed) / "search.json"))
    rows = oracle.initial_population(abi.GrammarBlob(lt.tables), lt.settings)
    return lt, rows


def test_static_evaluation_matches_allocating_evaluation_twice(tmp_path):
    from gagp_b200 import build
    from gagp_b200.engine import Engine, evaluate_rows_static
    build.build()
    first = _rows_for(tmp_path, 21, 256, 1024)
    second = _rows_for(tmp_path, 22, 40, 300)  # fewer cases and rows: stale scratch would show
    with Engine(0) as engine:
        for lt, rows in (first, second):
            want_f, want_w = engine.evaluate_rows(lt, rows)
            got_f, got_w = evaluate_rows_static(lt, rows)
            assert np.array_equal(got_f, want_f)
            assert np.array_equal(got_w, want_w)


def test_static_evaluation_on_a_caller_stream(tmp_path):
    """The stream argument: the call runs on a stream the caller created
    (a non-default, non-blocking one), twice in a row, with the same
    results as the allocating evaluator."""
    import torch
    from gagp_b200.engine import Engine, evaluate_rows_static
    lt, rows = _rows_for(tmp_path, 24, 130, 700)
    stream = torch.cuda.Stream(device=0)
    with Engine(0) as engine:
        want_f, want_w = engine.evaluate_rows(lt, rows)
    for _ in range(2):
        got_f, got_w = evaluate_rows_static(lt, rows, stream=stream.cuda_stream)
        assert np.array_equal(got_f, want_f)
        assert np.array_equal(got_w, want_w)


def test_static_evaluation_rejects_oversized_requests(tmp_path):
    from gagp_b200.engine import EngineError, evaluate_rows_static
    lt, rows = _rows_for(tmp_path, 23, 100, 16384)
    big = abi.RowsBuffer(16384 * 4, rows.stride)
    for k in range(4):
        big.node_counts[k * 16384:(k + 1) * 16384] = rows.node_counts
        big.origins[k * 16384:(k + 1) * 16384] = rows.origins
        big.constant_counts[k * 16384:(k + 1) * 16384] = rows.constant_counts
        big.constants[k * 16384:(k + 1) * 16384] = rows.constants
    with pytest.raises(EngineError) as err:
        evaluate_rows_static(lt, big)
    assert "static scratch" in str(err.value)
