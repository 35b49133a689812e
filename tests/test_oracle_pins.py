"""Pins the oracle (CPU restatement, oracle/ccs_oracle.c) against the
reference: its own self-test vectors, golden fixtures produced by the
reference's GMP code, and -- where oracle/_ref was built -- the reference
engines called in-process."""
import os
import subprocess

import numpy as np
import pytest


def test_reference_lattice_counts(ob):
    # v13 --test prints 36 bases, 123,552 wheel positions, 20,592 candidates/tile
    lat = ob.Lattice()
    assert lat.n_bases == 36
    assert lat.candidates_per_tile() == 20592
    total = sum(len(lat.bucket(b, m)) for b in range(36) for m in range(6))
    assert total == 123552


def test_mod6_buckets_give_5_mod_6(ob):
    # v13:2663-2708: every bucket-selected candidate has n % 6 == 5
    lat = ob.Lattice()
    M, WP = lat.M, lat.WP
    for tile in range(60):
        for b in range(lat.n_bases):
            bucket = (lat.tkm6(b) + 6 - tile % 6) % 6
            for k in lat.bucket(b, bucket)[:5]:
                assert ((tile * WP + int(k)) * M + lat.base(b)) % 6 == 5


def test_cc17_base_reachable(ob):
    # v13:2740-2771
    lat = ob.Lattice()
    assert 2759832934171386593519 % lat.M in lat.bases()


def test_q7_roots_decompose(ob, golden):
    # v13:2807-2910: 109-bit q7-immunized roots land in a base with base % 7 == 6
    # and their k offset sits in the bucket the tile selects
    lat = ob.Lattice()
    bases = lat.bases()
    for hx in golden("known_roots.json")["q7_roots"]:
        n = int(hx, 16)
        base = n % lat.M
        assert base in bases and base % 7 == 6
        k = (n - base) // lat.M
        tile, koff = divmod(k, lat.WP)
        b = bases.index(base)
        assert koff in set(int(x) for x in lat.bucket(b, (lat.tkm6(b) + 6 - tile % 6) % 6))


def test_forbidden_residues_definition(ob):
    for q in (37, 61, 97, 101, 863, 1021, 16411, 131071):
        for L in (1, 8, 16, 18):
            for lo in (0, 1):
                f = ob.forbidden(q, L, lo)
                want = set()
                for i in range(lo, min(L, q)):
                    want.add((pow(pow(2, i, q), -1, q) - 1) % q)
                assert f == sorted(want)
                # every forbidden residue makes some chain member divisible by q
                for r in f:
                    assert any((pow(2, i) * (r + 1) - 1) % q == 0 for i in range(lo, min(L, q)))


def _v33_tile_range(bits, prefix, bases, M, WP):
    """tiles v33's sequential prefix sweep visits (v33:2994-3061, 1741-1793)"""
    pbits = len(prefix) - 2
    pv = int(prefix[2:], 2)
    shift = bits - pbits
    cmin, cmax = pv << shift, ((pv + 1) << shift) - 1
    cmin, cmax = max(cmin, 1 << (bits - 1)), min(cmax, (1 << bits) - 1)
    kmin = -(-(cmin - max(bases)) // M) if cmin > max(bases) else 0
    kmax = (cmax - min(bases)) // M
    return kmin // WP, -(-kmax // WP)


def test_oracle_matches_v33_counters(ob, golden):
    """Candidates, stage pass counts and survivors equal the reference CPU
    engine's own counters on sequential prefix ranges."""
    for run in golden("v33_counts.json")["runs"]:
        L = run["target"]
        line = ob.LINE_PRIMES
        lat = ob.Lattice(lattice_len=L, depth=L,
                         stages=[(ob.L2_PRIMES, 0), (ob.EXT_PRIMES, 0), (line, 1)])
        t0, t1 = _v33_tile_range(run["bits"], run["prefix"], lat.bases(), lat.M, lat.WP)
        _, n, cnt = lat.filter_range(t0, t1 - t0, counters=True)
        assert cnt[0] == run["candidates"]
        assert cnt[1] == run["pass_l2"]
        assert cnt[2] == run["pass_ext"]
        assert n == run["survivors"]


def test_bpsw_and_mr_match_gmp(ob, golden):
    cases = golden("gmp_primality.json")["cases"]
    assert len(cases) > 500
    for s, g in cases:
        n = int(s)
        assert ob.is_prime_bpsw(n) == (g > 0), n
        assert ob.is_prime_mr(n) == (g > 0), n


def test_powmod_vectors(ob):
    # v33:2620-2679
    assert ob.powmod(2, 13, 97) == 44
    assert ob.powmod(3, 50, 1000000007) == pow(3, 50, 1000000007)
    import random
    r = random.Random(7)
    for _ in range(200):
        m = r.getrandbits(r.randint(2, 190)) | 1
        b, e = r.getrandbits(190) % m, r.getrandbits(r.randint(1, 190))
        assert ob.powmod(b, e, m) == pow(b, e, m)


def test_carmichael_rejected(ob):
    # v33:2681-2708
    for c in (561, 1105, 1729, 2821):
        assert not ob.is_prime_mr(c) and not ob.is_prime_bpsw(c)
    for p in (1000000007, 998244353, 999999999989, 18446744073709551557):
        assert ob.is_prime_mr(p) and ob.is_prime_bpsw(p)


def test_known_chain_vectors(ob, golden):
    # v13:2089-2101, v33:2401 (CC13), v33:2735 (135-bit CC15)
    want = {"2": 5, "89": 6, "1122659": 7, "19099919": 8, "85864769": 9, "26089808579": 10,
            "665043081119": 11, "554688278429": 12, "4090932431513069": 13,
            "95405042230542329": 14, "2759832934171386593519": 17}
    for row in golden("known_roots.json")["chains"]:
        n = int(row["root"])
        got = ob.chain_from(n, ob.PRIME_BPSW)
        assert got == row["forward"]
        assert ob.chain_from(n, ob.PRIME_MR) == row["forward"]
        if row["root"] in want:
            assert got == want[row["root"]]


def test_nonroot_backward_walk(ob):
    # v13:2213-2304: position-5 member of the CC17 walks back to the root
    root = 2759832934171386593519
    m = root
    for _ in range(5):
        m = 2 * m + 1
    (ln, r, is_root), isp = ob.prove_n(m, m.bit_length(), mode=1)
    assert isp and not is_root and r == root and ln == 17


def test_data_sample_chains(ob, golden):
    rows = golden("cc10_sample.json")["roots"]
    assert len(rows) == 1000
    for row in rows[::10]:
        n = int(row["root"], 16)
        assert row["forward"] >= 10
        assert ob.chain_from(n, ob.PRIME_BPSW) == row["forward"]


def test_walk_roots_golden(ob, golden):
    rows = golden("walk_roots.json")["roots"]
    for row in rows[::4]:
        assert ob.chain_from(int(row["n"]), ob.PRIME_BPSW) == row["forward"]


def test_oracle_prover_matches_reference_prover(ob, golden, ccs):
    """Oracle CPU-prover semantics reproduce the reference GMP prover pool's
    output lines (v13:2030-2033) on the same survivors."""
    for run in golden("v13_prover.json")["runs"]:
        L = run["target"]
        lat = ob.Lattice(lattice_len=L, depth=L)
        ts = int(run["tile_start"])
        lines = []
        primes = 0
        for b, k, t, _ in run["survivors"]:
            n = lat.reconstruct(ts, b, k, t)
            res, isp = ob.prove_n(n, run["bits"], mode=1)
            primes += isp
            if res is None:
                continue
            ln, root, is_root = res
            lines.append(ccs.format_chain_line(ln, root, L, is_root))
        assert primes == run["primes"]
        assert sorted(lines) == run["lines"]


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libref33.so")), reason="reference not built")
def test_oracle_lattice_equals_reference_builders(ob):
    r33 = ob.ref33()
    r13 = ob.ref13()
    for L in (18, 16, 14):
        lat = ob.Lattice(lattice_len=L, depth=L)
        n33 = r33.ref33_setup(L, 17)
        assert n33 == lat.n_bases
        for b in range(lat.n_bases):
            assert r33.ref33_base(b) == lat.base(b)
            assert r33.ref33_tkm6(b) == lat.tkm6(b)
            for m in range(6):
                n = r33.ref33_bucket_size(b, m)
                o = np.zeros(max(n, 1), dtype=np.uint32)
                r33.ref33_bucket(b, m, o)
                assert np.array_equal(o[:n], lat.bucket(b, m))
        n13 = r13.ref13_setup(L, L)
        assert n13 == min(lat.n_bases, 64)     # v13 caps at MAX_BASES = 64
        for b in range(n13):
            assert r13.ref13_base(b) == lat.base(b)
        # L2 masks, ext bytes and line kills equal the oracle's forbidden sets
        for i, q in enumerate(ob.L2_PRIMES):
            for d in range(1, L + 1):
                m = r13.ref13_l2_mask(i, d)
                assert sorted(x for x in range(64) if m >> x & 1) == ob.forbidden(q, d, 0)
        for i, q in enumerate(ob.LINE_PRIMES):
            kills = sorted(r for r in range(q) if r13.ref13_line_kill(i, r))
            assert kills == ob.forbidden(q, L, 1)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "cc_gmp_v33")), reason="reference not built")
def test_reference_engine_selftest_passes():
    exe = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "cc_gmp_v33")
    out = subprocess.run([exe, "--test"], capture_output=True, text=True, timeout=120).stdout
    assert "19 passed, 0 failed" in out
