"""Autotune cache files (host logic only: no GPU is touched by save, load,
clear or size)."""
import pytest

import perf_libs_sparse_b200 as pls

GOOD = """plsparse_b200_tune_cache 1 2
cc100-sm148 1000 1000 5000 00000000deadbeef 1 0 1 32 256 0 3
0 0 0 4 0.0125 1
1 32 256 0 0.0100 0.93
2 0 0 1024 0.0150 1
cc100-sm148 64 80 300 0123456789abcdef 0 1 0 0 0 8 1
0 0 0 8 0.003 1
"""


@pytest.fixture(autouse=True)
def empty_cache():
    pls.tune_cache_clear()
    yield
    pls.tune_cache_clear()


def test_load_save_round_trip(tmp_path):
    src = tmp_path / "a.cache"
    src.write_text(GOOD)
    pls.tune_cache_load(src)
    assert pls.tune_cache_size() == 2
    out = tmp_path / "b.cache"
    pls.tune_cache_save(out)
    pls.tune_cache_clear()
    assert pls.tune_cache_size() == 0
    pls.tune_cache_load(out)
    assert pls.tune_cache_size() == 2
    again = tmp_path / "c.cache"
    pls.tune_cache_save(again)
    assert again.read_text() == out.read_text()
    # loading the same entries again replaces them
    pls.tune_cache_load(src)
    assert pls.tune_cache_size() == 2


@pytest.mark.parametrize("bad", [
    "not_a_cache 1 0\n",
    "plsparse_b200_tune_cache 2 0\n",                         # other version
    GOOD.replace("0 0 0 8 0.003 1\n", ""),                    # cut short
    GOOD.replace("1 32 256 0 0.0100", "1 24 256 0 0.0100"),   # C not 8/16/32
    GOOD.replace("1 32 256 0 0.0100", "1 32 100 0 0.0100"),   # sigma not a multiple of C
    GOOD.replace("0 1 0 0 0 8 1", "0 1 7 0 0 8 1"),            # unknown kind
])
def test_malformed_file_changes_nothing(tmp_path, bad):
    ok = tmp_path / "ok.cache"
    ok.write_text(GOOD)
    pls.tune_cache_load(ok)
    f = tmp_path / "bad.cache"
    f.write_text(bad)
    with pytest.raises(pls.PerflibsError) as e:
        pls.tune_cache_load(f)
    assert e.value.status == pls.STATUS_INPUT_PARAMETER_ERROR
    assert pls.tune_cache_size() == 2


def test_missing_file(tmp_path):
    with pytest.raises(pls.PerflibsError):
        pls.tune_cache_load(tmp_path / "absent.cache")
    assert pls.tune_cache_size() == 0
