"""The pass-shape autotuner: every line-pairs-per-block choice of the Y pass
gives the same bits, so tuned and untuned engines step identically; tuning
fills the table, which is written to the cache file and read back."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(ib, prob, nsteps=4):
    st = ib.configs.seed_vorticity(ib.State(prob))
    s = ib.create_solver(st)
    for _ in range(nsteps):
        s.advance_()
    s.getstate()
    return st.Gamma.copy(), st.q.copy(), s.total_force().copy()


@pytest.mark.parametrize("n,L", [(128, 4), (96, 3)])
def test_every_block_shape_gives_the_same_bits(ib, monkeypatch, n, L):
    prob = ib.configs.small_cylinder(n, L)
    monkeypatch.delenv("IBPM_TUNE", raising=False)
    monkeypatch.delenv("IBPM_TUNE_FORCE_NG", raising=False)
    ref = _run(ib, prob)
    for ng in ("1", "2", "4", "8"):
        monkeypatch.setenv("IBPM_TUNE_FORCE_NG", ng)
        got = _run(ib, prob)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b), ng


def test_tuning_fills_the_table_and_the_cache(ib, monkeypatch, tmp_path):
    abi = importlib.import_module(ib.__name__ + "._abi")
    cache = tmp_path / "tune.txt"
    monkeypatch.delenv("IBPM_TUNE_FORCE_NG", raising=False)
    monkeypatch.setenv("IBPM_TUNE_CACHE", str(cache))
    monkeypatch.setenv("IBPM_TUNE", "1")
    prob = ib.configs.small_cylinder(256, 3)
    tuned = _run(ib, prob)
    table = abi.tune_table()
    keys = [k for k in table if "ypass M=256 fp64" in k]
    assert keys and all(v in (1, 2, 4, 8) for v in table.values())
    lines = cache.read_text().splitlines()
    assert {line.rsplit(" ", 1)[0] for line in lines} >= set(keys)
    # untuned (the fixed rule) gives the same bits
    monkeypatch.setenv("IBPM_TUNE", "0")
    monkeypatch.setenv("IBPM_TUNE_FORCE_NG", "2")
    plain = _run(ib, prob)
    for a, b in zip(tuned, plain):
        assert np.array_equal(a, b)
    # a cache file written by another process is read at first use
    other = tmp_path / "other.txt"
    other.write_text("".join(f"{k} 8\n" for k in keys))
    monkeypatch.delenv("IBPM_TUNE_FORCE_NG")
    monkeypatch.setenv("IBPM_TUNE_CACHE", str(other))
    again = _run(ib, prob)
    assert all(abi.tune_table()[k] == 8 for k in keys)
    for a, b in zip(tuned, again):
        assert np.array_equal(a, b)
