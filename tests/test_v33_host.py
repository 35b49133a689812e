"""The oracle's restatement of the reference CPU engine's proving path
(CCS_PRIME_V33: root test strong PRP to 2, 3, 5; Baillie-PSW predecessors;
screened Fermat links) equals the reference engine itself, run through its
own functions (tests/golden/v33_native.json, made by make_golden.py)."""
import random

import pytest


def test_oracle_prove_equals_reference_native_path(ob, golden):
    g = golden("v33_native.json")
    n_rec = 0
    for run in g["runs"]:
        lat = ob.Lattice(lattice_len=run["target"], depth=run["target"],
                         stages=[(ob.L2_PRIMES, 0), (ob.EXT_PRIMES, 0), (ob.LINE_PRIMES, 1)])
        ts = int(run["tile_start"])
        surv = lat.filter_range(ts, run["n_tiles"])
        assert sorted(map(tuple, surv[:, :3].tolist())) == sorted(tuple(x[:3]) for x in run["survivors"])
        for b, k, t, code, root_hex, is_root in run["survivors"]:
            n = lat.reconstruct(ts, b, k, t)
            rec, isp = ob.prove_v33(n, run["bits"], run["target"])
            assert code != -2                      # no prefilter skip at these widths
            if code <= 0:
                assert rec is None and isp == (code > 0), (n, code)
            else:
                assert isp and rec == (code, int(root_hex, 16), bool(is_root)), (n, code, rec)
                n_rec += 1
    assert n_rec > 50


def test_oracle_walk_equals_reference_screened_walk(ob, golden):
    """Includes the reference's screen quirk: a link that is itself a screen
    prime counts as composite (root 89 -> length 1; GMP's walk gives 6)."""
    walks = golden("v33_native.json")["walks"]
    assert len(walks) > 500
    for s, length in walks:
        assert ob.chain_from_v33(int(s)) == length, s
    assert dict(walks)["89"] == 1


def test_native_tests_equal_reference(ob):
    r33 = ob.ref33()
    if r33 is None:
        pytest.skip("reference harness not built")
    rnd = random.Random(33)
    nums = [rnd.getrandbits(b) | 1 for b in (8, 20, 40, 61, 64, 89, 110, 126) for _ in range(60)]
    nums += [2047, 3277, 4033, 4681, 8321, 25326001, 3215031751, 341, 561, 1105, 1729, 7, 9, 5, 3]
    for n in nums:
        lo, hi = n & (2**64 - 1), n >> 64
        assert ob.oracle().orc_chain_from_v33(ob.int_to_words(n), 4, 0, 127) == \
            r33.ref33_follow_native(lo, hi, 0), n
