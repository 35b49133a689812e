"""Survivor-set parity of the depth-16 / primes-to-2^17 profile (W = 31#,
88-bit roots): the engine's survivors on 64+ seeded 2^14-tile windows equal
the oracle's committed survivor sets (tests/golden/cc16_windows.json, 300+
survivors in total), swept on the plain lattice and on the extended lattice,
through the plain entry point and through one batched launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def as_set(arr):
    a = np.asarray(arr.cpu().numpy() if hasattr(arr, "cpu") else arr)
    if a.dtype.names:
        a = a.view(np.uint32).reshape(len(a), -1)
    a = a.astype(np.int64) & 0xFFFFFFFF
    return sorted(map(tuple, a[:, :3].tolist()))


@pytest.fixture(scope="module")
def fixture(golden):
    g = golden("cc16_windows.json")
    assert len(g["windows"]) >= 64 and g["total_survivors"] >= 300
    return g


@pytest.fixture(scope="module")
def eng(ccs):
    e = ccs.Engine(**ccs.config_cc16_scale())
    yield e
    e.close()


@pytest.mark.parametrize("lattice", ["plain", "extended"])
def test_windows_match_oracle(eng, fixture, lattice):
    eng.set_tuning(ext_min_words=0xFFFFFFFF if lattice == "plain" else 1)
    total = 0
    for w in fixture["windows"]:
        ts, n = int(w["tile_start"]), w["n_tiles"]
        assert eng.plan_range(ts, n)["extended"] == (lattice == "extended")
        got = as_set(eng.filter_range(ts, n, cap=1 << 16))
        want = sorted(map(tuple, w["survivors"]))
        assert got == want, (lattice, ts)
        total += len(got)
    assert total == fixture["total_survivors"]
    eng.set_tuning(ext_min_words=256)


def test_windows_match_oracle_batched(ccs, eng, fixture):
    """All windows as the ranges of one batched launch."""
    ranges = [(int(w["tile_start"]), w["n_tiles"], 0, 88) for w in fixture["windows"]]
    b = ccs.Batch([eng], len(ranges), surv_cap=1 << 16, chain_cap=1 << 14)
    try:
        res, surv, _ = b.run(ranges)
    finally:
        b.close()
    rid = surv["_pad"].astype(np.int64)
    for i, w in enumerate(fixture["windows"]):
        assert as_set(surv[rid == i]) == sorted(map(tuple, w["survivors"])), i
        assert res[i]["n_survivors"] == len(w["survivors"])
