"""Fingerprint-pool Q iteration on the GPU: the bit-sliced Q sweep equals
the oracle's per-Q sieve and the reference's own v16_q_iter_kernel (where
oracle/_ref was built); the device prove of q-iteration survivors equals the
oracle's restatement of the reference's CPU prove worker."""
import os
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF16 = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                     "libref16.so")
SHAPES = ["2*3*5*11*13*19", "2*3^2*5*11*13*19", "2*3*5*7*11*13*19", "2*3*5^2*11*13*19",
          "2*3*5*11*13*17*19", "2*3*5*11*13*19*29", "2*3^3*5*7*11*13*19*23", "2*3*5*7*11*13*17*19*23*29"]


def _pool(ccs):
    return [ccs.parse_pool_spec(s) for s in SHAPES]


def _set(t):
    a = np.asarray(t.cpu().numpy()).astype(np.int64) & 0xFFFFFFFF
    return sorted(map(tuple, a[:, :3].tolist()))


@pytest.mark.parametrize("E,depth,sieve_max,ext", [(0, 8, 61, False), (0, 12, 211, False),
                                                   (3, 10, 503, True), (0, 21, 503, False)])
def test_filter_matches_oracle(ccs, ob, E, depth, sieve_max, ext):
    pool = _pool(ccs)
    primes = ccs.qiter_sieve_primes(sieve_max=sieve_max, ext=ext)
    qi = ccs.QIter(pool, target=depth, depth=depth, exp_start=E, primes=primes)
    r = random.Random(depth * 31 + E)
    # depth 21 over 7..503 leaves ~1.5e-6 of the Q: one long segment gives it survivors
    sizes = [1, 63, 64, 65, 1000, 4095 * 64 + 17, 262144, 262145, 700001, 30_000_000 if depth > 12 else 0]
    segs = []
    for n in sizes:
        v = r.randrange(len(pool))
        qb = r.choice([r.randint(1, 1 << 40), (1 << 64) - r.randint(1, 5000), r.randint(1 << 90, 1 << 100)])
        segs.append((qb, n, v))
    got = _set(qi.filter(segs, cap=1 << 22))
    want = []
    for s, (qb, n, v) in enumerate(segs):
        want += [(o, s, v) for o in ob.qiter_filter_seg(qb, n, pool[v][1], E, depth, primes)]
    assert got == sorted(want) and (len(want) > 0 or depth > 12)
    qi.close()


def test_filter_empty_and_overflow(ccs):
    pool = _pool(ccs)
    qi = ccs.QIter(pool, target=6, depth=6, primes=ccs.qiter_sieve_primes(sieve_max=61, ext=False))
    assert qi.filter([]).shape[0] == 0
    assert qi.filter([(12345, 0, 0)]).shape[0] == 0
    segs = [(1 << 50, 100000, 1)]
    full = qi.filter(segs)
    assert full.shape[0] > 50
    with pytest.raises(ccs.CCSError) as e:
        qi.filter(segs, cap=7)
    assert e.value.status == ccs.OVERFLOW and str(full.shape[0]) in str(e.value)
    with pytest.raises(ccs.CCSError):
        qi.filter([(1, 10, len(pool))])                     # variant out of range
    qi.close()


def test_forbidden_counts(ccs, ob):
    pool = _pool(ccs)
    primes = ccs.qiter_sieve_primes()
    qi = ccs.QIter(pool, target=21, depth=21, exp_start=1, primes=primes)
    for v in range(len(pool)):
        want = [len(ob.qiter_forbidden(q, pool[v][1], 1, 21)) for q in primes]
        assert qi.forbidden_counts(v) == want
    qi.close()


@pytest.mark.skipif(not os.path.exists(REF16), reason="reference harness not built")
@pytest.mark.parametrize("depth", [12, 21])
def test_filter_matches_reference_kernel(ccs, ob, depth):
    """The same survivor offsets as the reference's v16_q_iter_kernel over
    one variant's 2^22-Q launch, for every shape of the test pool, at its
    production sieve (7..503)."""
    ref = ob.ref16()
    pool = _pool(ccs)
    primes = ccs.qiter_sieve_primes(ext=False)
    qi = ccs.QIter(pool, target=depth, depth=depth, primes=primes)
    pr = np.asarray(primes, dtype=np.uint32)
    r = random.Random(depth)
    n_q = 1 << 22
    for v, (_, D, _) in enumerate(pool):
        qmin, qmax = ccs.q_window(D, 0, 90, 107)
        qb = r.randint(qmin, qmax - n_q)
        out = np.zeros(1 << 20, dtype=np.uint32)
        cnt = ref.ref16_qiter_filter(pr, len(pr), D & (2**64 - 1), D >> 64, 0, depth,
                                     qb & (2**64 - 1), qb >> 64, n_q, out, len(out))
        want = sorted(int(x) for x in out[:cnt])
        got = sorted(o for o, _, _ in _set(qi.filter([(qb, n_q, v)])))
        assert got == want, (v, depth)
    qi.close()


@pytest.mark.parametrize("reverse,mode", [(True, "ROOTS"), (False, "ROOTS"), (False, "FULL")])
def test_prove_matches_oracle(ccs, ob, reverse, mode):
    """Chain records and prime counts of q-iteration survivors equal the
    oracle's: p_0 = Q D_V 2^E - 1, reverse gate at position target - 1,
    BPSW, root check, forward walk."""
    pool = _pool(ccs)
    target, depth, E = 6, 6, 1
    primes = ccs.qiter_sieve_primes(sieve_max=131, ext=False)
    qi = ccs.QIter(pool, target=target, depth=depth, exp_start=E, primes=primes, reverse=reverse,
                   prove_mode=getattr(ccs, "PROVE_" + mode))
    r = random.Random(17 + reverse)
    segs = []
    for v, (_, D, _) in enumerate(pool):
        qmin, qmax = ccs.q_window(D, E, 70, 96)
        segs.append((r.randint(qmin, qmax - 400000), 400000, v))
    surv = qi.filter(segs)
    assert surv.shape[0] > 500
    chains, primes_ = qi.prove(segs, surv, cap=1 << 18)
    got = sorted((int(c[1]), int(c[0]), int(c[3]), sum(int(x & 0xFFFFFFFF) << (32 * i) for i, x in
                                                        enumerate(c[4:10])), int(c[10]) & 1)
                 for c in chains.cpu().numpy().astype(np.int64))
    want, n_prime = [], 0
    for off, s, v in _set(surv):
        qb, _, _ = segs[s]
        res, isp = ob.qiter_prove(qb + off, pool[v][1], E, target, reverse=reverse,
                                  mode=0 if mode == "ROOTS" else 1)
        n_prime += isp
        if res is not None:
            want.append((s, off, res[0], res[1], int(res[2])))
    assert primes_ == n_prime
    assert got == sorted(want) and len(want) > 10
    flags = chains.cpu().numpy()[:, 10]
    lens = chains.cpu().numpy()[:, 3]
    assert (((flags & 2) != 0) == (lens >= target)).all()
    # below 256 survivors the one-thread-per-survivor kernel proves them:
    # the same records for the same survivors
    part = surv[:200]
    keys = set((int(o), int(sg)) for o, sg in part.cpu().numpy()[:, :2].astype(np.int64))
    c2, p2 = qi.prove(segs, part)
    got2 = sorted((int(c[1]), int(c[0]), int(c[3]), sum(int(x & 0xFFFFFFFF) << (32 * i) for i, x in
                                                         enumerate(c[4:10])), int(c[10]) & 1)
                  for c in c2.cpu().numpy().astype(np.int64))
    assert got2 == sorted(w for w in want if (w[1], w[0]) in keys)
    qi.close()


def test_prove_rejects_wide_segments(ccs):
    pool = _pool(ccs)
    qi = ccs.QIter(pool, target=8, depth=8)
    import torch
    surv = torch.zeros((1, 4), dtype=torch.int32, device="cuda")
    with pytest.raises(ccs.CCSError):
        qi.prove([((1 << 128) - 1000, 10, len(SHAPES) - 1)], surv)   # p_0 above 2^160
    with pytest.raises(ValueError):
        qi.prove([(1 << 150, 10, 0)], surv)                  # Q beyond 128 bits
    qi.close()


def test_pipelined_run_equals_sequential(ccs):
    """QIter.run (prove of step i beside the filter of step i + 1, two
    threads and streams) gives the totals and HIT lines of plain
    filter-then-prove calls, step by step."""
    pool = _pool(ccs)
    qi = ccs.QIter(pool, target=8, depth=8, primes=ccs.qiter_sieve_primes(sieve_max=131, ext=False))
    plan = [qi.random_segments(16, 1 << 18, 64, 80, seed=s, start_variant=s) for s in range(6)]
    tot, lines = qi.run(plan, min_report_len=4, dedup_p0=False)
    want_lines, n_s, n_c, n_p = [], 0, 0, 0
    for segs in plan:
        s_ = qi.filter(segs)
        c_, p_ = qi.prove(segs, s_, cap=1 << 18)
        n_s += s_.shape[0]
        n_c += c_.shape[0]
        n_p += p_
        want_lines += qi.hit_lines(segs, c_, min_report_len=4)
    assert (tot["steps"], tot["survivors"], tot["chains"], tot["primes"]) == (6, n_s, n_c, n_p)
    assert tot["q"] == 6 * 16 * (1 << 18)
    assert lines == sorted(want_lines) and len(lines) > 0 and n_s > 1000
    # the same plan twice with --dedup-p0: the second sighting of every p_0
    # is a HIT-DUP line
    _, lines2 = qi.run(plan + plan, min_report_len=4)
    dups = [l for l in lines2 if l.startswith("HIT-DUP")]
    assert len(dups) == len(lines) and len(lines2) == 2 * len(lines)
    qi.close()
