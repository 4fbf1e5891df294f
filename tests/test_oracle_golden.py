"""Pins the CPU oracle to massively's own known answers (CPU only).

Every vector in tests/golden/known_answers.py comes from a massively test or
doctest; the oracle must reproduce each one before any GPU result is judged
against it.
"""
import numpy as np
import pytest

from tests.golden import known_answers as K


def test_scan_known_answers(orc):
    for case in K.SCAN:
        if case["kind"] == "inclusive":
            got = orc.inclusive_scan(case["x"], case["op"])
        else:
            got = orc.exclusive_scan(case["x"], case["op"], case["init"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])


def test_scan_boundary_probes(orc):
    ones = np.ones(K.SCAN_ONES["n"], np.uint32)
    inc = orc.inclusive_scan(ones, "add")
    for i, v in K.SCAN_ONES["probes"].items():
        assert inc[i] == v
    exc = orc.exclusive_scan(ones, "add", K.SCAN_EXCL_ONES["init"])
    for i in K.SCAN_EXCL_ONES["probes"]:
        assert exc[i] == K.SCAN_EXCL_ONES["init"] + i
    tl = orc.exclusive_scan(np.ones(K.SCAN_TAKE_LEFT["n"], np.uint32), "take_left",
                            K.SCAN_TAKE_LEFT["init"])
    assert (tl == K.SCAN_TAKE_LEFT["want"]).all()


def test_reduce_known_answers(orc):
    for case in K.REDUCE:
        assert orc.reduce(case["x"], case["op"], case["init"]) == case["want"], case["src"]


def test_selection_known_answers(orc):
    for case in K.SELECT:
        fn = orc.copy_where if case["kind"] == "copy_where" else orc.remove_where
        np.testing.assert_array_equal(fn(case["x"], case["stencil"]), case["want"],
                                      err_msg=case["src"])
    rows = K.COPY_WHERE_ROWS
    got = orc.copy_where(rows["cols"], rows["stencil"])
    for g, w in zip(got, rows["want"]):
        np.testing.assert_array_equal(g, w)
    sp = K.STENCIL_POSITIONS
    np.testing.assert_array_equal(orc.inclusive_scan(orc.flags(sp["stencil"], "is_true"), "add"),
                                  sp["want"])
    for case in K.PARTITION:
        out, b = orc.partition(case["x"], case["pred"])
        assert b == case["boundary"], case["src"]
        np.testing.assert_array_equal(out, case["want"], err_msg=case["src"])


def test_gather_scatter_known_answers(orc):
    for case in K.GATHER:
        got = orc.gather(case["values"], case["idx"], case["stencil"], case["out"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])
    for case in K.SCATTER:
        got = orc.scatter(case["values"], case["idx"], case["out"], case["stencil"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])


def test_replace_transform_where_known_answers(orc):
    for case in K.REPLACE_WHERE:
        got = orc.replace_where(case["value"], case["stencil"], case["out"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])
    for case in K.TRANSFORM_WHERE:
        got = orc.transform_where(case["x"], case["op"], case["stencil"], case["out"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])


def test_ordering_known_answers(orc):
    for case in K.SORT:
        np.testing.assert_array_equal(orc.sort(case["x"]), case["want"], err_msg=case["src"])
    for case in K.SORT_BY_KEY:
        _, v = orc.sort_by_key(case["keys"], case["values"])
        np.testing.assert_array_equal(v, case["want"], err_msg=case["src"])
    for case in K.RADIX:
        got = orc.radix_sort_by_key(case["keys"], case["values"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])
    for case in K.RADIX_INTEGER_EXTREMES + K.RADIX_FLOAT_TOTAL_ORDER:
        np.testing.assert_array_equal(orc.radix_perm([case["keys"]]), case["want"],
                                      err_msg=case["src"])
    c = K.RADIX_COMPOUND
    np.testing.assert_array_equal(orc.radix_perm(c["keys"]), c["want"], err_msg=c["src"])
    n = K.RADIX_513["n"]
    keys = ((np.arange(n) * 37) % 11).astype(np.uint32)
    got = orc.radix_sort_by_key([keys], np.arange(n, dtype=np.uint32))
    np.testing.assert_array_equal(got, np.argsort(keys, kind="stable"))


def test_by_key_known_answers(orc):
    for case in K.BY_KEY:
        if case["kind"] == "reduce":
            k, v = orc.reduce_by_key(case["keys"], case["values"], "add", case["init"])
            np.testing.assert_array_equal(k, case["want_keys"])
            np.testing.assert_array_equal(v, case["want"])
            k2, v2 = orc.reduce_by_key_literal_u32(case["keys"], case["values"], "add",
                                                   case["init"])
            np.testing.assert_array_equal(k2, k)
            np.testing.assert_array_equal(v2, v)
        else:
            got = orc.scan_by_key(case["keys"], case["values"], "add",
                                  exclusive=case["kind"] == "exclusive", init=case["init"])
            np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])
    s = K.BY_KEY_SEVEN
    n = s["n"]
    keys = np.where(np.arange(n) < 300, 1, 2).astype(np.uint32)
    cols = [np.full(n, c, np.uint32) for c in range(1, 8)]
    inc = [orc.scan_by_key(keys, col, "add") for col in cols]
    assert (inc[0][299], inc[0][300], inc[0][599]) == (300, 1, 300)
    assert (inc[6][299], inc[6][300], inc[6][599]) == (2100, 7, 2100)
    exc = orc.scan_by_key(keys, cols[0], "add", exclusive=True, init=s["inits"][0])
    assert (exc[0], exc[1], exc[300], exc[301]) == (10, 11, 10, 11)
    k, vals = orc.reduce_by_key(keys, cols, ["add"] * 7, s["inits"])
    np.testing.assert_array_equal(k, [1, 2])
    np.testing.assert_array_equal(vals[0], [310, 310])
    np.testing.assert_array_equal(vals[6], [2170, 2170])


def test_merge_and_set_known_answers(orc):
    for case in K.MERGE:
        np.testing.assert_array_equal(orc.merge(case["left"], case["right"]), case["want"])
    m = K.MERGE_BY_KEY
    _, v = orc.merge_by_key(m["lk"], m["lv"], m["rk"], m["rv"])
    np.testing.assert_array_equal(v, m["want"])
    for case in K.SETS:
        np.testing.assert_array_equal(orc.set_union(case["left"], case["right"]), case["union"])
        np.testing.assert_array_equal(orc.set_intersection(case["left"], case["right"]),
                                      case["intersection"])
        np.testing.assert_array_equal(orc.set_difference(case["left"], case["right"]),
                                      case["difference"])
    for case in K.UNIQUE:
        np.testing.assert_array_equal(orc.unique(case["x"]), case["want"])


def test_bounds_known_answers(orc):
    for case in K.BOUNDS:
        np.testing.assert_array_equal(orc.lower_bound(case["source"], case["values"]),
                                      case["lower"], err_msg=case["src"])
        np.testing.assert_array_equal(orc.upper_bound(case["source"], case["values"]),
                                      case["upper"], err_msg=case["src"])
    # numpy's searchsorted is the same partition point for `<`
    rng = np.random.default_rng(3)
    src = np.sort(rng.integers(0, 50, 1000).astype(np.uint32))
    vals = rng.integers(0, 60, 500).astype(np.uint32)
    np.testing.assert_array_equal(orc.lower_bound(src, vals), np.searchsorted(src, vals, "left"))
    np.testing.assert_array_equal(orc.upper_bound(src, vals), np.searchsorted(src, vals, "right"))


def _call_predicate(mod, case):
    fn = getattr(mod, case["fn"])
    return fn(case["a"], case["b"], case["arg"]) if "b" in case else fn(case["a"], case["arg"])


def test_predicate_known_answers(orc):
    for case in K.PREDICATES:
        assert _call_predicate(orc, case) == case["want"], case["src"]


def test_predicate_edges(orc):
    u = np.uint32
    # mismatch: equal prefix but different lengths -> the shorter length
    assert orc.mismatch(np.array([1, 2], u), np.array([1, 2, 3], u)) == 2
    assert orc.mismatch(np.array([1, 2], u), np.array([1, 2], u)) is None
    assert orc.equal(np.array([1, 2], u), np.array([1, 2, 3], u)) is False
    assert orc.lexicographical_compare(np.array([1, 2], u), np.array([1, 2, 3], u)) is True
    assert orc.lexicographical_compare(np.array([1, 2, 3], u), np.array([1, 2], u)) is False
    assert orc.is_sorted_until(np.array([], u)) == 0
    assert orc.min_element(np.array([], u)) is None
    assert orc.minmax_element(np.array([], u)) is None
    # minmax keeps the LAST minimum and the FIRST maximum
    assert orc.minmax_element(np.array([2, 1, 5, 1, 5], u)) == (3, 2)
    assert orc.min_element(np.array([2, 1, 5, 1, 5], u)) == 1
    assert orc.max_element(np.array([2, 1, 5, 1, 5], u)) == 2
    # NaN under `<`: at index 0 it is the first minimum / maximum; elsewhere
    # never taken; minmax's minimum restarts after the last NaN
    nan = np.float32("nan")
    f = np.float32
    assert orc.min_element(np.array([nan, -1, -2], f)) == 0
    assert orc.max_element(np.array([1, nan, 3], f)) == 2
    assert orc.minmax_element(np.array([0, -5, nan, 3, 4], f)) == (3, 4)
    assert orc.minmax_element(np.array([0, -5, nan], f)) == (2, 0)
    # numpy agrees on NaN-free input
    rng = np.random.default_rng(11)
    x = rng.integers(0, 100, 5000).astype(np.int32)
    assert orc.min_element(x) == int(np.argmin(x))
    assert orc.max_element(x) == int(np.argmax(x))
    assert orc.minmax_element(x)[0] == int(np.flatnonzero(x == x.min())[-1])
    assert orc.find_if(x, "is_negative") is None
    assert orc.count_if(x, "is_odd") == int((x % 2 == 1).sum())


def test_scatter_reduce_known_answers(orc):
    for case in K.SCATTER_REDUCE:
        for v, init, out, want in zip(case["values"], case["init"], case["output"], case["want"]):
            got = orc.scatter_reduce(v, case["indices"], init, case["op"], out)
            np.testing.assert_array_equal(got, want, err_msg=case["src"])
    # a non-identity init is folded in once per destination that received a
    # proposal; untouched destinations keep their value
    got = orc.scatter_reduce(np.array([1, 2, 3], np.int32), np.array([0, 0, 2], np.uint32), 100,
                             "add", np.array([5, 6, 7], np.int32))
    np.testing.assert_array_equal(got, [108, 6, 110])
    got = orc.scatter_reduce(np.array([4, 9], np.uint8), np.array([1, 1], np.uint32), 255, "min",
                             np.array([7, 7], np.uint8))
    np.testing.assert_array_equal(got, [7, 4])


def test_seg_query_known_answers(orc):
    for case in K.SEG_QUERIES:
        np.testing.assert_array_equal(orc.seg_query(case["x"], case["offsets"], case["query"],
                                                    case["op"]), case["want"], err_msg=case["src"])


def test_seg_take_known_answers(orc):
    for case in K.SEG_TAKE:
        v, off = orc.seg_transform(case["x"], case["offsets"], "take", case["k"])
        np.testing.assert_array_equal(v, case["values"], err_msg=case["src"])
        np.testing.assert_array_equal(off, case["new_offsets"], err_msg=case["src"])
    # unique compares with the last kept item; reverse and adjacent_difference
    x = np.array([1, 1, 2, 2, 2, 3, 9, 9], np.uint32)
    off = np.array([0, 3, 3, 8], np.uint32)
    v, o = orc.seg_transform(x, off, "unique")
    np.testing.assert_array_equal(v, [1, 2, 2, 3, 9])
    np.testing.assert_array_equal(o, [0, 2, 2, 5])
    v, _ = orc.seg_transform(x, off, "reverse")
    np.testing.assert_array_equal(v, [2, 1, 1, 9, 9, 3, 2, 2])
    v, _ = orc.seg_transform(x.astype(np.int32), off, "adjacent_difference", "add")
    np.testing.assert_array_equal(v, [1, 2, 3, 2, 4, 5, 12, 18])


def test_seg_known_answers(orc):
    for case in K.SEG:
        if case["kind"] == "reduce":
            got = orc.seg_reduce(case["x"], case["offsets"], case["op"], case["init"])
        else:
            got = orc.seg_exclusive_scan(case["x"], case["offsets"], case["op"], case["init"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])
    for case in K.SEGMENTATION:
        off = np.concatenate([[0], np.cumsum(case["lengths"], dtype=np.uint64)]).astype(np.uint32)
        np.testing.assert_array_equal(off, case["offsets"])
        assert orc.validate_offsets(off) == off[-1]
    for bad in K.INVALID_OFFSETS["cases"]:
        assert orc.validate_offsets(bad) is None


def test_rng_streams_are_pcg(orc):
    # random.rs:12-22: the hash and seed key of the host restatement.
    x = 12345
    state = (x * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    assert orc.pcg_hash32(x) == ((word >> 22) ^ word)
    a = orc.uniform_u32(10, 20, 123, 64)
    assert ((a >= 10) & (a <= 20)).all()
    np.testing.assert_array_equal(a, orc.uniform_u32(10, 20, 123, 64))
    assert not np.array_equal(a, orc.uniform_u32(10, 20, 124, 64))
    # random_uses_generic_taken_and_tracks_nested_slice_offsets (random.rs tests)
    full = orc.uniform_u32(10, 20, 123, 16)
    np.testing.assert_array_equal(orc.uniform_u32(10, 20, 123, 4, offset=5), full[5:9])
    assert not np.array_equal(orc.uniform_u32(0, 0xFFFFFFFF, 7, 64),
                              orc.uniform_u32(0, 0xFFFFFFFF, 7 | (1 << 32), 64))
    assert (orc.uniform_u32(4, 4, 1, 8) == 4).all()
    u = orc.uniform_u64(1000, 2000, 777, 32)
    assert ((u >= 1000) & (u <= 2000)).all()
    z = orc.normal_f32(0, 1 << 16)
    assert np.isfinite(z).all() and abs(z.mean()) < 0.02 and abs(z.std() - 1) < 0.02


@pytest.mark.parametrize("n", K.ORACLE_LENGTHS)
def test_oracle_agrees_with_numpy(orc, n):
    # Independent cross-check of the oracle loops on the boundary lengths.
    x = orc.uniform_u32(0, 0xFFFFFFFF, n + 1, n)
    np.testing.assert_array_equal(orc.inclusive_scan(x, "add"),
                                  np.cumsum(x, dtype=np.uint64).astype(np.uint32))
    assert orc.reduce(x.astype(np.uint64), "add", 0) == int(x.astype(np.uint64).sum())
    keys = x % 13
    np.testing.assert_array_equal(orc.sort_perm(keys), np.argsort(keys, kind="stable"))
    st = orc.flags(x, "is_even")
    np.testing.assert_array_equal(orc.copy_where(x, st), x[st.astype(bool)])


@pytest.mark.parametrize("dtype", [np.uint32, np.int32, np.float32, np.uint64, np.int64,
                                   np.float64])
@pytest.mark.parametrize("n,threads", [(0, 4), (1, 3), (1000, 7), (100_003, 8)])
def test_parallel_stable_order_equals_the_sequential_oracle(orc, dtype, n, threads):
    """radix_perm_par (the full-size checks' stable order on all host
    cores) gives the sequential oracle's permutation, ties and signed zeros
    included."""
    dt = np.dtype(dtype)
    if dt.kind == "f":
        x = (orc.normal_f32(7, n) * 3).round().astype(dt)  # many ties, -0.0 and +0.0
    else:
        x = orc.uniform_u32(0, 50, 7, n).astype(dt) - (25 if dt.kind == "i" else 0)
    np.testing.assert_array_equal(orc.radix_perm_par(x, threads), orc.radix_perm([x]))
