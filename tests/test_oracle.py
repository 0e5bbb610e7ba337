"""The CPU oracle restatement is pinned against the reference's own code
(oracle/_ref, built from the reference sources) and against the order rules of
thrust::sort / CUB 2.8.2 that the reference's sort path inherits."""
import numpy as np
import pytest

INT_TYPES = [np.uint32, np.int32, np.uint64, np.int64]
ALL_TYPES = INT_TYPES + [np.float32, np.float64]


def rand(dt, n, seed):
    rng = np.random.default_rng(seed)
    dt = np.dtype(dt)
    if dt.kind == "f":
        return (rng.standard_normal(n) * 1e3).astype(dt)
    bits = rng.integers(0, 2 ** 63, n, dtype=np.uint64) * 2 + rng.integers(0, 2, n, dtype=np.uint64)
    return bits.astype(np.uint32 if dt.itemsize == 4 else np.uint64).view(dt)


@pytest.mark.parametrize("dt", ALL_TYPES)
@pytest.mark.parametrize("n", [0, 1, 2, 3, 255, 256, 257, 10000])
def test_sort_matches_numpy_on_nan_free_keys(orc, dt, n):
    a = rand(dt, n, n)
    assert np.array_equal(orc.sort(a), np.sort(a, kind="stable"))


@pytest.mark.parametrize("dt", ALL_TYPES)
def test_sort_matches_reference_gnu_parallel_sort(orc, dt):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    a = rand(dt, 300001, 5)
    b = a.copy()
    orc.ref_gnu_parallel_sort(b, 4)  # src/sort_benchmark.cu:103-108
    assert orc.sort(a).tobytes() == b.tobytes()


@pytest.mark.parametrize("dt,ut", [(np.float32, np.uint32), (np.float64, np.uint64)])
def test_float_order_nan_and_signed_zero(orc, dt, ut):
    bits_of = lambda x: np.array([x], dtype=dt).view(ut)[0]
    sign = ut(1) << ut(np.dtype(ut).itemsize * 8 - 1)
    qnan = bits_of(np.nan)
    vals = np.array([1.0, -0.0, np.inf, 0.0, -np.inf, -2.0, -0.0, 0.0, 3.0], dtype=dt)
    extra = np.array([qnan, qnan | sign, qnan | ut(5), (qnan | ut(7)) | sign], dtype=ut).view(dt)
    a = np.concatenate([vals, extra])
    out = orc.sort(a).view(ut)
    # negative-sign NaNs first (larger payload first: the whole key is inverted), then -inf
    assert list(out[:2]) == [(qnan | ut(7)) | sign, qnan | sign]
    assert out[2] == bits_of(-np.inf)
    # zeros: -0.0, +0.0, -0.0, +0.0 exactly in input order (equal keys, stable)
    zeros = out[(out == sign) | (out == ut(0))]
    assert list(zeros) == [sign, ut(0), sign, ut(0)]
    # +inf then positive NaNs by payload
    assert list(out[-3:]) == [bits_of(np.inf), qnan, qnan | ut(5)]


@pytest.mark.parametrize("dt", ALL_TYPES)
def test_merge_is_stable_first_range_first(orc, dt):
    a = np.sort(rand(dt, 5000, 1) % 50 if np.dtype(dt).kind != "f" else np.round(rand(dt, 5000, 1)))
    b = np.sort(rand(dt, 3001, 2) % 50 if np.dtype(dt).kind != "f" else np.round(rand(dt, 3001, 2)))
    out = orc.merge(a, b)
    ref = np.concatenate([a, b])
    order = np.argsort(ref, kind="stable")
    assert np.array_equal(out, ref[order])


def test_merge_signed_zero_ties_take_first_range(orc):
    a = np.array([-0.0, 1.0], dtype=np.float32)
    b = np.array([0.0, 0.5], dtype=np.float32)
    out = orc.merge(a, b)
    assert np.signbit(out[0]) and not np.signbit(out[1])


def brute_pivot(orc, parts, psize, g):
    half = g // 2
    L = parts[: half * psize]
    R = parts[half * psize:]
    keyL, keyR = orc.order_keys(L), orc.order_keys(R)
    N = half * psize
    best = 0
    for p in range(1, N + 1):
        if keyL[N - p] > keyR[p - 1]:
            best = p
    return best


@pytest.mark.parametrize("g", [2, 4, 8])
@pytest.mark.parametrize("seed", range(6))
def test_find_pivot_matches_definition(orc, g, seed):
    psize = 37
    parts = np.concatenate([np.sort(rand(np.uint32, psize, seed * 10 + i) % 200) for i in range(g)])
    # the pivot of the top-level step is over the two sorted halves
    half = g // 2
    parts = np.concatenate([np.sort(parts[: half * psize]), np.sort(parts[half * psize:])])
    assert orc.find_pivot(parts, psize, g) == brute_pivot(orc, parts, psize, g)


@pytest.mark.parametrize("dt", ALL_TYPES)
@pytest.mark.parametrize("g", [1, 2, 4, 8])
@pytest.mark.parametrize("n", [1, 2, 7, 8, 1000, 4099, 65536])
def test_tanasic_restatement_sorts(orc, dt, g, n):
    a = rand(dt, n, n + g)
    if np.dtype(dt).kind != "f":
        a = a % 997 if np.dtype(dt).kind == "u" else a  # many duplicates for unsigned
    assert np.array_equal(orc.tanasic_sort(a, g), orc.sort(a))


def test_tanasic_filler_defect_is_reproduced(orc):
    # With g not dividing n the reference pads with numeric_limits<T>::max()
    # (src/tanasic_sort.cuh:255-259). For floats that is FLT_MAX, which sorts
    # before +inf, so the copy-back keeps a filler and drops one +inf.
    a = np.array([np.inf, 1.0, 2.0, 3.0, 4.0], dtype=np.float32)  # n=5, g=2 -> 1 filler
    out = orc.tanasic_sort(a, 2)
    assert out[-1] == np.finfo(np.float32).max
    assert np.count_nonzero(np.isinf(out)) == 0
    assert np.array_equal(orc.tanasic_sort(a, 1), np.sort(a))


@pytest.mark.parametrize("dt", INT_TYPES)
@pytest.mark.parametrize("k", [2, 8, 32, 64])
def test_kway_merge_matches_reference_multiway_merge(orc, dt, k):
    rng = np.random.default_rng(k)
    lens = rng.multinomial(200000, rng.dirichlet(np.ones(k)))
    runs = [np.sort(rand(dt, int(L), i)) for i, L in enumerate(lens)]
    out = orc.kway_merge(runs)
    assert np.array_equal(out, np.sort(np.concatenate(runs)))
    if orc.ref_available():
        ref, _ = orc.ref_multiway_merge(runs, 4)
        assert out.tobytes() == ref.tobytes()


def test_kway_merge_stable_by_run_index(orc):
    runs = [np.array([-0.0, 1.0], np.float32), np.array([0.0], np.float32), np.array([-0.0], np.float32)]
    out = orc.kway_merge(runs)
    assert list(np.signbit(out[:3])) == [True, False, True]


def test_segmented_sort(orc):
    a = rand(np.uint32, 1000, 3)
    offs = np.array([0, 0, 1, 10, 500, 1000], dtype=np.uint64)
    out = orc.segmented_sort(a, offs)
    for s in range(len(offs) - 1):
        b, e = int(offs[s]), int(offs[s + 1])
        assert np.array_equal(out[b:e], np.sort(a[b:e]))


def test_oracle_libraries_are_built_from_their_current_sources():
    """A stale oracle library would be called with another signature: each one must be at least as new as its
    recipe's source (rebuild with __graft_entry__.build())."""
    import os
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")
    for lib, src in (("_build/liboracle.so", "oracle.cpp"), ("_ref/libref.so", "ref_wrap.cu")):
        lp, sp = os.path.join(here, lib), os.path.join(here, src)
        if os.path.exists(lp):
            assert os.path.getmtime(lp) >= os.path.getmtime(sp), f"oracle/{lib} is older than oracle/{src}"
