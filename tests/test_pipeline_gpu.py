"""The group-by chain (copy_where -> sort -> reduce_by_key -> set_intersection)
over device counts, run eagerly and as a captured CUDA graph, against numpy.

Values are small integers held as f32, so every per-key sum is exact in any
association order and all outputs compare bit-exactly."""
import numpy as np
import pytest

from tests.gpu_util import executor, gpu

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


def _inputs(n, seed, nkeys=1 << 12):
    rng = np.random.default_rng(seed)
    ranks = np.arange(1, nkeys + 1, dtype=np.float64)
    p = ranks ** -1.1
    keys = rng.choice(nkeys, size=n, p=p / p.sum()).astype(np.uint32) * np.uint32(2654435761 % 2**32)
    values = rng.integers(-1000, 1000, n).astype(np.float32)
    flag = (rng.random(n) < 0.3).astype(np.uint32)
    other = np.sort(rng.choice(keys, size=min(n, 1 << 10))).astype(np.uint32)
    return keys, values, flag, other


def _expected(keys, values, flag, other):
    m = flag != 0
    k, v = keys[m], values[m]
    o = np.argsort(k, kind="stable")
    k, v = k[o], v[o]
    uniq, idx, cnt = np.unique(k, return_index=True, return_counts=True)
    if len(k) == 0:
        return {"keys": uniq, "sum": np.empty(0, np.float32), "count": cnt.astype(np.uint32),
                "min": np.empty(0, np.float32), "common": uniq}
    return {"keys": uniq, "sum": np.add.reduceat(v.astype(np.float64), idx).astype(np.float32),
            "count": cnt.astype(np.uint32), "min": np.minimum.reduceat(v, idx),
            "common": np.intersect1d(uniq, other)}


def _check(ex, out, want):
    for name, w in want.items():
        np.testing.assert_array_equal(ex.to_host(out[name]), w, err_msg=name)


@pytest.mark.parametrize("n", [1, 4097, 1 << 20])
def test_group_by_eager(ex, n):
    from massively_b200 import pipeline
    k, v, f, o = _inputs(n, seed=n)
    out = pipeline.group_by(ex, ex.to_device(k), ex.to_device(v), ex.to_device(f),
                            ex.to_device(o))
    _check(ex, out, _expected(k, v, f, o))


def test_group_by_nothing_kept(ex):
    from massively_b200 import pipeline
    k, v, f, o = _inputs(5000, seed=1)
    f[:] = 0
    out = pipeline.group_by(ex, ex.to_device(k), ex.to_device(v), ex.to_device(f),
                            ex.to_device(o))
    _check(ex, out, _expected(k, v, f, o))


def test_group_by_captured_graph_replays(ex):
    """One capture, replayed on three different inputs copied into the
    captured buffers: every replay matches numpy."""
    import torch

    from massively_b200 import pipeline
    n = 1 << 18
    k, v, f, o = _inputs(n, seed=11)
    dk, dv, df, do = (ex.to_device(a) for a in (k, v, f, o))
    cap = pipeline.Captured(ex, lambda e: pipeline.group_by(e, dk, dv, df, do))
    for seed in (11, 12, 13):
        k, v, f, o = _inputs(n, seed=seed)
        for dst, src in ((dk, k), (dv, v), (df, f), (do, o)):
            dst.tensor.copy_(ex.to_device(src).tensor)
        torch.cuda.synchronize()
        cap.replay()
        torch.cuda.synchronize()
        _check(ex, cap.outputs, _expected(k, v, f, o))


def test_run_host_batches_overlapped(ex):
    # Five batches of host pairs streamed through the radix sort with the
    # copies overlapped; every batch's result matches the oracle, including
    # when two batches share an output array (the later one lands last).
    import torch
    from massively_b200 import pipeline, vector
    from oracle import oracle as orc
    from tests.gpu_util import seeded
    n = 300_007
    pin = lambda a: torch.from_numpy(a.view(np.uint8)).pin_memory().numpy().view(a.dtype)
    batches, want = [], []
    for seed in range(5):
        k = seeded(np.uint32, n, 40 + seed) % np.uint32(1 << (8 + 4 * seed))
        v = seeded(np.uint32, n, 50 + seed)
        batches.append((pin(k), pin(v)))
        want.append(v[orc.radix_perm([k])])
    outs = [pin(np.zeros(n, np.uint32)) for _ in range(5)]
    fn = lambda e, dk, dv: vector.radix_sort_pairs(e, dk, dv)[1]
    pipeline.run_host_batches(ex, fn, batches, outs)
    for o, w in zip(outs, want):
        np.testing.assert_array_equal(o, w)
    shared = [outs[0], outs[1], outs[0], outs[1], outs[0]]
    pipeline.run_host_batches(ex, fn, batches, shared)
    np.testing.assert_array_equal(outs[0], want[4])
    np.testing.assert_array_equal(outs[1], want[3])
    with pytest.raises(ValueError):
        pipeline.run_host_batches(ex, fn, [batches[0], (batches[0][0][:10], batches[0][1][:10])],
                                  outs[:2])
