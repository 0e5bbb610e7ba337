"""Onesweep variant table (tile shape x ranking mode per key width and size
class): set/get, tuning-file save/load round trips and error handling. Host
only: the table lives in the library and needs no GPU."""
import pytest


@pytest.fixture
def saved_table(mgs, tmp_path):
    """Restores the process's table after the test."""
    path = tmp_path / "before.tune"
    mgs.tune_save(str(path))
    yield tmp_path
    mgs.tune_load(str(path))


def test_set_then_get_per_size_class(mgs, saved_table):
    mgs.tune_set("u32", 0, 1, 2)
    mgs.tune_set("u32", 5, 6, 3)
    mgs.tune_set("f64", 2, 0, 2)
    assert mgs.tune_get("u32", 1000) == (1, 2)          # class 0: n < 2^16
    assert mgs.tune_get("i32", (1 << 16) - 1) == (1, 2)  # same width, same class
    assert mgs.tune_get("f32", 1 << 30) == (6, 3)        # class 5
    assert mgs.tune_get("u64", 3 << 18) == (0, 2)        # 8-byte keys, class 2: n < 2^20


def test_save_load_round_trip(mgs, saved_table):
    path = str(saved_table / "t.tune")
    mgs.tune_set("u32", 3, 2, 3)
    mgs.tune_save(path)
    mgs.tune_set("u32", 3, 4, 2)
    assert mgs.tune_get("u32", 3 << 20) == (4, 2)
    mgs.tune_load(path)
    assert mgs.tune_get("u32", 3 << 20) == (2, 3)
    lines = [l for l in open(path) if l.strip() and not l.startswith("#")]
    assert len(lines) == 12 and all(len(l.split()) == 4 for l in lines)


def test_invalid_entries_are_rejected(mgs, saved_table):
    for args in [("u32", 6, 5, 3), ("u32", -1, 5, 3), ("u32", 0, 7, 3), ("u32", 0, 5, 1)]:
        with pytest.raises(mgs.MgsError):
            mgs.tune_set(*args)
    bad = saved_table / "bad.tune"
    bad.write_text("# comment\n4 1 3 2\n4 1 9 9\nnot a line\n")
    with pytest.raises(mgs.MgsError):
        mgs.tune_load(str(bad))
    assert mgs.tune_get("u32", 3 << 16) == (3, 2)  # the valid line was applied
    with pytest.raises(mgs.MgsError):
        mgs.tune_load(str(saved_table / "missing.tune"))
