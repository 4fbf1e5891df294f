"""The continuous-batching loop: every request's result is the same when it
is served alone (one request per launch) and when it is coalesced with
others into one segmented launch, overlapped on several streams.

All three request kinds are exact here: sort_by_key and inclusive_scan are
integer work (bit-exact), and reduce_by_key sums runs of f32 integers below
2^16 (runs far shorter than 256 items on these seeded inputs), whose sums
stay below 2^24 and are therefore exact in f32 in any association order."""
import numpy as np
import pytest

from tests.gpu_util import executor, gpu

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


def _host(ex, d):
    return {k: ex.to_host(v) for k, v in d.items()}


def _expected(r, inputs):
    """Host answer of a request from its (host) inputs."""
    from massively_b200 import serving as S
    if r.kind == S.SORT:
        order = np.argsort(inputs["keys"], kind="stable")
        return {"keys": inputs["keys"][order], "values": inputs["values"][order]}
    if r.kind == S.SCAN:
        return {"y": np.cumsum(inputs["x"], dtype=np.uint64).astype(np.uint32)}
    k, v = inputs["keys"], inputs["values"].astype(np.float64)
    heads = np.flatnonzero(np.concatenate([[True], k[1:] != k[:-1]]))
    return {"keys": k[heads], "values": np.add.reduceat(v, heads).astype(np.float32)}


@pytest.mark.parametrize("small_n,streams", [(1 << 14, 4), (1 << 16, 2), (1 << 12, 1)])
def test_same_alone_and_in_the_mix(ex, small_n, streams):
    from massively_b200 import serving as S
    trace = S.make_trace(rate=1e6, duration=1.0, lo_log2=8, hi_log2=17, seed=7,
                         max_requests=90)
    assert {r.kind for r in trace} == {S.SORT, S.SCAN, S.RBK}
    st = S.serve(ex, trace, small_n=small_n, max_batch=16, streams=streams, keep_outputs=True)
    assert st.requests == len(trace) and st.launches < len(trace)
    for r in trace:
        mixed = _host(ex, r.outputs)
        S.materialize_inputs(ex, r)
        inputs = _host(ex, r.inputs)
        S.run_single(ex, r)
        alone = _host(ex, r.outputs)
        want = _expected(r, inputs)
        assert mixed.keys() == alone.keys() == want.keys()
        for key in want:
            np.testing.assert_array_equal(alone[key], want[key], err_msg=f"{r.kind} {r.n} {key}")
            np.testing.assert_array_equal(mixed[key], alone[key], err_msg=f"{r.kind} {r.n} {key}")
        r.inputs, r.outputs = {}, {}


def test_reduce_by_key_segmented_breaks_runs_at_segments(ex):
    """Equal keys on both sides of a segment start form two runs."""
    from massively_b200 import op, vector
    keys = np.array([1, 1, 1, 2, 2, 2, 2, 3, 3, 3], np.uint32)
    vals = np.arange(10, dtype=np.float32)
    off = np.array([0, 2, 2, 5, 10], np.uint32)  # an empty segment too
    k, v = vector.reduce_by_key_segmented(ex, ex.to_device(keys), ex.to_device(vals), op.Equal,
                                          np.float32(0), op.Add, ex.to_device(off))
    np.testing.assert_array_equal(ex.to_host(k), [1, 1, 2, 2, 3])
    np.testing.assert_array_equal(ex.to_host(v), [1, 2, 7, 11, 24])


def test_serving_stats_and_plain_dispatch(ex):
    from massively_b200 import serving as S
    trace = S.make_trace(rate=5e4, duration=1.0, lo_log2=10, hi_log2=16, seed=3,
                         max_requests=40)
    st = S.plain_dispatch(ex, trace)
    assert st.requests == len(trace) and st.launches == len(trace)
    assert 0 < st.p50_ms <= st.p99_ms
    assert all(r.done >= r.arrival for r in trace)


def test_coalesced_reduce_by_key_irregular_runs(ex):
    """A coalesced reduce_by_key launch splits its outputs per request from
    the device: runs of any length, runs that continue across a request
    boundary (split there), and requests of one row."""
    from massively_b200 import serving as S
    rng = np.random.default_rng(11)
    sizes = [1, 37, 1000, 5, 4096, 1, 777]
    reqs = [S.Request(i, S.RBK, n, 0.0, i) for i, n in enumerate(sizes)]
    total = sum(sizes)
    runs = rng.integers(1, 60, size=total)
    keys = np.repeat(np.arange(len(runs), dtype=np.uint32) % 5, runs)[:total]
    vals = rng.integers(0, 1 << 16, size=total).astype(np.float32)  # run sums stay exact
    batch = {"keys": ex.to_device(keys), "values": ex.to_device(vals)}
    finish = S.run_coalesced(ex, reqs, batch)
    assert finish is not None
    ex.sync()
    finish()
    off = np.concatenate([[0], np.cumsum(sizes)])
    for i, r in enumerate(reqs):
        inputs = {"keys": keys[off[i]:off[i + 1]], "values": vals[off[i]:off[i + 1]]}
        want = _expected(r, inputs)
        got = _host(ex, r.outputs)
        for key in want:
            np.testing.assert_array_equal(got[key], want[key], err_msg=f"request {i} {key}")
