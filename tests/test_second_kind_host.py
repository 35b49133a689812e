"""Second-kind chains (p -> 2p - 1, the reference's v13b) on the CPU: the
oracle's lattice, forbidden sets and prover semantics are pinned to the
reference's own v13b code (built into oracle/_ref) and to GMP, and the
engine's host-side lattice description equals the oracle's."""
import os

import numpy as np
import pytest

REF13B = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libref13b.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF13B), reason="reference not built")


@needs_ref
def test_oracle_lattice_equals_v13b_builders(ob):
    r13b = ob.ref13b()
    for L in (18, 16, 14):
        lat = ob.Lattice(lattice_len=L, depth=L, kind_=2)
        n13 = r13b.ref13_setup(L, L)
        assert n13 == min(lat.n_bases, 64)     # v13b keeps v13's MAX_BASES = 64
        for b in range(n13):
            assert r13b.ref13_base(b) == lat.base(b)
            assert r13b.ref13_tkm6(b) == lat.tkm6(b)
            for m in range(6):
                n = r13b.ref13_bucket_size(b, m)
                o = np.zeros(max(n, 1), dtype=np.uint32)
                r13b.ref13_bucket(b, m, o)
                assert np.array_equal(o[:n], lat.bucket(b, m))
        for i, q in enumerate(ob.L2_PRIMES):
            for d in range(1, L + 1):
                m = r13b.ref13_l2_mask(i, d)
                assert sorted(x for x in range(64) if m >> x & 1) == ob.forbidden(q, d, 0, kind_=2)
        for i, q in enumerate(ob.LINE_PRIMES):
            kills = sorted(r for r in range(q) if r13b.ref13_line_kill(i, r))
            assert kills == ob.forbidden(q, L, 1, kind_=2)


def test_second_kind_members_are_1_mod_6(ob):
    lat = ob.Lattice(kind_=2)
    ts = (1 << 60) // (20677 * 1616615) + 77
    for b, k, t, _ in lat.filter_range(ts, 40)[:200]:
        assert lat.reconstruct(ts, int(b), int(k), int(t)) % 6 == 1


def test_known_second_kind_chains(ob, golden):
    for row in golden("second_kind.json")["chains"]:
        n = int(row["root"])
        assert row["forward"] == row["selftest_len"]
        assert ob.chain_from(n, ob.PRIME_BPSW, kind_=2) == row["forward"]
        assert ob.chain_from(n, ob.PRIME_MR, kind_=2) == row["forward"]


def test_oracle_prover_matches_v13b_prover(ob, golden, ccs):
    """The oracle's CPU-prover semantics for the second kind reproduce the
    output lines of the v13b GMP prover pool on the same survivors."""
    for run in golden("second_kind.json")["prover"]:
        L = run["target"]
        lat = ob.Lattice(lattice_len=L, depth=L, kind_=2)
        ts = int(run["tile_start"])
        lines, primes = [], 0
        for b, k, t, _ in run["survivors"]:
            n = lat.reconstruct(ts, b, k, t)
            res, isp = ob.prove_n(n, run["bits"], mode=1, kind_=2)
            primes += isp
            if res is not None:
                ln, root, is_root = res
                lines.append(ccs.format_chain_line(ln, root, L, is_root))
        assert primes == run["primes"]
        assert sorted(lines) == run["lines"]


def test_engine_description_second_kind(ob, ccs):
    info, bases = ccs.describe(kind=ccs.KIND_SECOND)
    lat = ob.Lattice(kind_=2)
    assert list(bases) == lat.bases()
    assert info["n_lines"] == 123552 and info["candidates_per_tile"] == 20592
    with pytest.raises(ccs.CCSError):
        ccs.describe(kind=3)
