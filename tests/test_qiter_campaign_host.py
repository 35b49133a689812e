"""Q-iteration campaign shell on the CPU: the reference's Q walkers
(round-robin variants, sequential cursors, random starts, per-variant choice
by window width) and its q-iter checkpoint file, read and written both ways
through the reference's own save/load functions where oracle/_ref was
built."""
import os

import numpy as np
import pytest

REF16 = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                     "libref16.so")
SHAPES = ["2*3*5*11*13*19", "2*3^2*5*11*13*19", "2*3*5*7*11*13*19", "2*3*5*7*11*13*17*19*23*29*31*37"]


@pytest.fixture
def fake(ccs):
    class FakeQIter(ccs.QIter):
        def __init__(self, pool, target=21, depth=21, exp_start=0, seed_name="exp_d"):
            self.dv = [p[1] for p in pool]
            self.names = [p[0] for p in pool]
            self.target, self.depth, self.exp_start, self.seed_name = target, depth, exp_start, seed_name

        def run(self, plan, min_report_len=8, **kw):
            q = sum(n for segs in plan for _, n, _ in segs)
            return {"steps": len(plan), "q": q, "survivors": 0, "chains": 0, "primes": 0}, []
    return FakeQIter


def _pool(ccs):
    return [ccs.parse_pool_spec(s) for s in SHAPES]


def test_sequential_walkers_cover_windows(ccs, fake):
    qi = fake(_pool(ccs))
    # bits 40..41: windows of at most ~2^25 Q (the widest D_V leaves none)
    c = ccs.QCampaign(qi, bits_min=40, bits_max=41, q_order="sequential", q_chunk=1 << 20, chunks_per_step=7)
    assert sum(b - a + 1 for a, b in c.win if a <= b) < 1 << 27
    seen = {v: [] for v in range(len(SHAPES))}
    while True:
        segs = c.next_step()
        if segs is None:
            break
        for qb, n, v in segs:
            seen[v].append((qb, n))
    for v, (qmn, qmx) in enumerate(c.win):
        runs = seen[v]
        if qmn > qmx:
            assert runs == []
            continue
        assert runs[0][0] == qmn and runs[-1][0] + runs[-1][1] - 1 == qmx
        assert all(runs[i][0] + runs[i][1] == runs[i + 1][0] for i in range(len(runs) - 1))


def test_exhaustive_band_mode_picks_per_variant(ccs, fake):
    qi = fake(_pool(ccs))
    c = ccs.QCampaign(qi, bits_min=90, bits_max=107, q_band_mode="exhaustive", exhaustive_max_q_bits=70)
    for (qmn, qmx), rnd in zip(c.win, c.random):
        assert rnd == ((qmx - qmn + 1).bit_length() > 70)
    assert any(c.random) and not all(c.random)


def test_checkpoint_round_trip_and_identity(ccs, fake, tmp_path):
    qi = fake(_pool(ccs))
    path = str(tmp_path / "ck.txt")
    c = ccs.QCampaign(qi, bits_min=70, bits_max=72, q_order="sequential", q_chunk=1 << 16,
                      chunks_per_step=5, checkpoint_path=path)
    c.run(max_steps=3)
    text = open(path).read()
    assert text.startswith("version=v16.0.3-drained-cursor\nmode=q-iter\n") and "v_cursor_drained[" in text
    c2 = ccs.QCampaign(qi, bits_min=70, bits_max=72, q_order="sequential", q_chunk=1 << 16,
                       checkpoint_path=path, resume=True)
    assert c2.cursor == c.cursor
    with pytest.raises(ValueError):
        ccs.QCampaign(fake(_pool(ccs), seed_name="other"), bits_min=70, bits_max=72, q_order="sequential",
                      checkpoint_path=path, resume=True)
    with pytest.raises(ValueError):
        ccs.QCampaign(qi, bits_min=70, bits_max=73, q_order="sequential", checkpoint_path=path, resume=True)


def _ref_args(c, path):
    gl = np.asarray(c.gpu_list, dtype=np.uint32)
    im = np.asarray(c.immune, dtype=np.uint32)
    pool = ",".join(str(d) for d in c.qi.dv).encode()
    return [path.encode(), c.qi.target, c.qi.depth, c.bits_min, c.bits_max, c.qi.seed_name.encode(), im,
            len(im), c.qi.exp_start, c.sieve_max, gl, len(gl), 1 if c.q_order == "random" else 0, c.seed,
            c.q_chunk, 1 if c.q_band_mode == "exhaustive" else 0, c.xbits, pool, len(c.qi.dv)]


@pytest.mark.skipif(not os.path.exists(REF16), reason="reference harness not built")
def test_checkpoint_matches_reference_both_ways(ccs, fake, ob, tmp_path):
    ref = ob.ref16()
    qi = fake(_pool(ccs))
    c = ccs.QCampaign(qi, bits_min=70, bits_max=72, q_order="sequential", q_chunk=1 << 16, chunks_per_step=6)
    c.run(max_steps=2)
    ours = str(tmp_path / "ours.txt")
    c.save(ours)
    n = len(qi.dv)
    lo = np.array([x & (2**64 - 1) for x in c.cursor], dtype=np.uint64)
    hi = np.array([x >> 64 for x in c.cursor], dtype=np.uint64)
    # the reference reads our file and finds our cursors
    rl, rh = np.zeros(n, dtype=np.uint64), np.zeros(n, dtype=np.uint64)
    qmin = [a for a, _ in c.win]
    for v in range(n):
        rl[v], rh[v] = qmin[v] & (2**64 - 1), qmin[v] >> 64
    assert ref.ref16_ckpt_load(*_ref_args(c, ours), rl, rh) == 0
    assert (rl == lo).all() and (rh == hi).all()
    # the reference writes the same file (line for line) and we read it
    theirs = str(tmp_path / "theirs.txt")
    ql = np.array([a & (2**64 - 1) for a in qmin], dtype=np.uint64)
    qh = np.array([a >> 64 for a in qmin], dtype=np.uint64)
    assert ref.ref16_ckpt_save(*_ref_args(c, theirs), lo, hi, ql, qh) == 0
    assert open(theirs).read() == open(ours).read()
    c2 = ccs.QCampaign(qi, bits_min=70, bits_max=72, q_order="sequential", q_chunk=1 << 16,
                       checkpoint_path=theirs, resume=True)
    assert c2.cursor == c.cursor
    # a changed identity is refused by both
    other = fake(_pool(ccs), seed_name="other")
    c3 = ccs.QCampaign(other, bits_min=70, bits_max=72, q_order="sequential", q_chunk=1 << 16)
    assert ref.ref16_ckpt_load(*_ref_args(c3, ours), rl, rh) == -1
