"""Fingerprint-pool Q iteration (the reference's v16 engine), host side and
oracle pins, on the CPU: pool-file parsing, sieve lists, Q windows, the
oracle's forbidden residues against the reference's own function (where
oracle/_ref was built) and against the definition p_j = 2^(E+j) Q D_V - 1,
the oracle's Q sieve against a brute-force evaluation, and the oracle's
prove on chains with known lengths."""
import os
import random

import pytest

REF16 = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                     "libref16.so")
# fingerprint shapes of the kind the reference's pools hold (2*3*5 floor and
# small-prime factors of p + 1)
SHAPES = ["2*3*5*11*13*19", "2*3^2*5*11*13*19", "2*3*5*7*11*13*19", "2*3*5^2*11*13*19",
          "2*3*5*11*13*17*19", "2*3*5*11*13*19*29", "2*3^3*5*7*11*13*19*23"]


def test_pool_file_format(ccs):
    text = """# a comment line
2*3*5*11*13*19  # freq=271525 bits=16.31

2*3^2*5*11*13*19
  2*3*5*5*11*13*19   # repeated factor
"""
    pool = ccs.pool_from_text(text)
    assert [p[1] for p in pool] == [2 * 3 * 5 * 11 * 13 * 19, 2 * 9 * 5 * 11 * 13 * 19,
                                    2 * 3 * 25 * 11 * 13 * 19]
    assert pool[1][2] == {2: 1, 3: 2, 5: 1, 11: 1, 13: 1, 19: 1}
    prim = ccs.parse_pool_specs("41#/31/37/41, 7#")
    assert prim[0][1] == 2 * 3 * 5 * 7 * 11 * 13 * 17 * 19 * 23 * 29 and prim[1][1] == 210
    for bad in ("2*4*5", "2*3^0", "2*3^17", "x*3", "41#/43"):
        with pytest.raises(ValueError):
            ccs.parse_pool_spec(bad)


def test_sieve_lists(ccs):
    k1 = ccs.qiter_sieve_primes(ext=False)
    assert k1[0] == 7 and k1[-1] == 503 and len(k1) == 93           # "7..503 (93)"
    full = ccs.qiter_sieve_primes()
    assert full[93:] == list(ccs.V16_EXT_PRIMES) and full[-1] == 1009 and len(full) == 166
    assert ccs.qiter_sieve_primes(sieve_max=211, ext=False)[-1] == 211


def test_q_window_bounds(ccs):
    r = random.Random(3)
    for _ in range(200):
        D = ccs.parse_pool_spec(r.choice(SHAPES))[1]
        E = r.choice([0, 0, 1, 5])
        b1 = r.randint(60, 110)
        b2 = r.randint(b1, 127)
        qmin, qmax = ccs.q_window(D, E, b1, b2)
        p = lambda Q: Q * D * 2 ** E - 1
        assert p(qmin).bit_length() >= b1 and p(qmin - 1).bit_length() < b1
        assert p(qmax).bit_length() <= b2 and p(qmax + 1).bit_length() > b2


def test_forbidden_residues_definition(ob, ccs):
    """Q = r is forbidden for q exactly when q divides some p_j, j < depth."""
    r = random.Random(5)
    for _ in range(300):
        D = ccs.parse_pool_spec(r.choice(SHAPES))[1]
        q = r.choice(ccs.qiter_sieve_primes())
        E, depth = r.choice([0, 0, 2, 7]), r.randint(1, 24)
        got = ob.qiter_forbidden(q, D, E, depth)
        want = sorted(Q for Q in range(q)
                      if any(((Q * D) << (E + j)) % q == 1 for j in range(depth)))
        assert sorted(got) == want, (q, D, E, depth)
        assert (D % q == 0) == (got == [])


@pytest.mark.skipif(not os.path.exists(REF16), reason="reference harness not built")
def test_forbidden_residues_match_reference(ob, ccs):
    import numpy as np
    ref = ob.ref16()
    r = random.Random(7)
    out = np.zeros(64, dtype=np.uint32)
    for _ in range(500):
        D = ccs.parse_pool_spec(r.choice(SHAPES))[1] * r.choice([1, 1, 7, 23, 29 * 31])
        q = r.choice(ccs.qiter_sieve_primes())
        E, depth = r.choice([0, 1, 3]), r.randint(1, 24)
        n = ref.ref16_forbidden(q, D & (2**64 - 1), D >> 64, E, depth, out, 64)
        want = [] if n < 0 else [int(x) for x in out[:n]]
        assert ob.qiter_forbidden(q, D, E, depth) == want, (q, D, E, depth)


def test_oracle_sieve_brute_force(ob, ccs):
    r = random.Random(11)
    primes = ccs.qiter_sieve_primes(sieve_max=61, ext=False)
    for _ in range(6):
        D = ccs.parse_pool_spec(r.choice(SHAPES))[1]
        E, depth = r.choice([0, 3]), r.choice([4, 6])
        qb = r.randint(1, 1 << 100)
        n = r.randint(1, 20000)
        got = ob.qiter_filter_seg(qb, n, D, E, depth, primes)
        want = [o for o in range(n)
                if not any((((qb + o) * D << (E + j)) - 1) % q == 0 for j in range(depth) for q in primes)]
        assert got == want


def test_oracle_prove_known_chains(ob, golden):
    """Known chain roots written as p + 1 = Q * D (D = 2 * 3 * 5 * the odd
    part's small factors when they divide) prove to their known lengths,
    forward and in reverse order at the target."""
    for ch in golden("known_roots.json")["chains"]:
        p = int(ch["root"])
        want = ch["full"]
        if p < 1000 or ch["full_root"] != ch["root"]:
            continue
        D = 1
        for q in (2, 3, 5, 7, 11, 13):
            if (p + 1) % (D * q) == 0:
                D *= q
        Q = (p + 1) // D
        res, isp = ob.qiter_prove(Q, D, 0, target=want, reverse=False)
        assert isp and res is not None and res[0] == want and res[1] == p and res[2]
        res, _ = ob.qiter_prove(Q, D, 0, target=want, reverse=True)
        assert res is not None and res[0] == want
        res, _ = ob.qiter_prove(Q, D, 0, target=want + 1, reverse=True)
        assert res is None                    # position target - 1 is composite


def test_random_segments_reproducible(ccs):
    class FakeQIter(ccs.QIter):
        def __init__(self, dv):
            self.dv, self.exp_start = dv, 0
    pool = [ccs.parse_pool_spec(s)[1] for s in SHAPES]
    f = FakeQIter(pool)
    a = f.random_segments(50, 1 << 24, 90, 107, seed=9)
    b = f.random_segments(50, 1 << 24, 90, 107, seed=9)
    assert a == b and a != f.random_segments(50, 1 << 24, 90, 107, seed=10)
    wins = f.windows(90, 107)
    for qb, n, v in a:
        assert wins[v][0] <= qb and qb + n - 1 <= wins[v][1] and n == 1 << 24
    assert [v for _, _, v in a[:len(pool)]] == list(range(len(pool)))


def test_hit_line_format(ccs):
    line = ccs.format_hit_line("exp_d", 12, 12345, 0x1F, fp=[3, 5], pool=["2*3*5"])
    assert line == "HIT seed=exp_d len=12 fp={3,5} pool=[2*3*5] A=12345 p_0=0x1f"
