"""Batched (persistent, graph-replayed) execution gives each range exactly
the survivors and chains of a plain per-range call."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_equals_plain(ccs):
    engines = [ccs.Engine(target=18, bits=64), ccs.Engine(target=16, depth=16, bits=64),
               ccs.Engine(target=14, depth=14, bits=64)]
    batch = ccs.Batch(engines, max_ranges=64, surv_cap=1 << 20, chain_cap=1 << 18)
    r = random.Random(3)
    ranges = []
    for i in range(24):
        p = i % 3
        ts = (1 << 63) // (20677 * 1616615) + r.randint(0, 10**6)
        ranges.append((ts, r.choice([0, 1, 5, 40, 300, 1200]), p, 64))
    for rep in range(2):                     # the second run replays the graph
        res, surv, chains = batch.run(ranges)
        surv_by = {}
        for rec in surv:
            surv_by.setdefault(int(rec["_pad"]), []).append(
                (int(rec["base_idx"]), int(rec["k_offset"]), int(rec["tile_idx"])))
        for i, (ts, n, p, bits) in enumerate(ranges):
            plain = engines[p].filter_range(ts, n, cap=1 << 18)
            want = sorted(map(tuple, (plain.cpu().numpy()[:, :3].astype(np.int64) & 0xFFFFFFFF).tolist()))
            assert sorted(surv_by.get(i, [])) == want
            assert res[i]["n_survivors"] == len(want)
            pch, pprimes = engines[p].prove(plain, ts)
            assert res[i]["n_chains"] == pch.shape[0]
            assert res[i]["n_primes"] == pprimes
            assert res[i]["candidates"] >= n * engines[p].candidates_per_tile - engines[p].info["n_lines"]
    batch.close()
    for e in engines:
        e.close()


def test_batch_tuning_keeps_results(ccs):
    """Every batch block shape and unit length gives the same per-range
    survivor sets; the batch autotuner leaves one of them set."""
    engines = [ccs.Engine(target=16, depth=16, bits=64), ccs.Engine(target=18, bits=64)]
    batch = ccs.Batch(engines, max_ranges=32, surv_cap=1 << 20, chain_cap=1 << 18)
    r = random.Random(17)
    ranges = [((1 << 63) // (20677 * 1616615) + r.randint(0, 10**7), r.choice([3, 70, 900, 20000]), i % 2, 64)
              for i in range(16)]

    def sets():
        res, surv, _ = batch.run(ranges)
        by = {}
        for rec in surv:
            by.setdefault(int(rec["_pad"]), []).append(
                (int(rec["base_idx"]), int(rec["k_offset"]), int(rec["tile_idx"])))
        return [sorted(by.get(i, [])) for i in range(len(ranges))], [x["n_primes"] for x in res]

    want = sets()
    for bt, uw in [(128, 0), (256, 2), (128, 4096), (256, 1024)]:
        batch.set_tuning(block_threads=bt, unit_words=uw)
        assert batch.tuning()["block_threads"] == bt
        assert sets() == want
    chosen, points = batch.autotune(ranges)
    assert 5 + 2 <= len(points) <= 5 + 8 and chosen == batch.tuning()
    assert sets() == want
    batch.close()
    for e in engines:
        e.close()


def test_two_batches_in_flight_equal_run(ccs):
    """ccs_batch_launch / ccs_batch_wait: two batches over the same engines
    launched back to back (the second launched before the first is waited
    for) give the same records as blocking runs; a batch refuses a second
    launch while one is in flight."""
    engines = [ccs.Engine(target=16, depth=16, bits=64), ccs.Engine(target=18, bits=64)]
    b0 = ccs.Batch(engines, max_ranges=16, surv_cap=1 << 18, chain_cap=1 << 16)
    b1 = ccs.Batch(engines, max_ranges=16, surv_cap=1 << 18, chain_cap=1 << 16)
    r = random.Random(29)
    ra = [((1 << 63) // (20677 * 1616615) + r.randint(0, 10**7), r.choice([5, 300, 4000]), i % 2, 64)
          for i in range(8)]
    rb = [((1 << 62) // (20677 * 1616615) + r.randint(0, 10**7), r.choice([7, 900, 3000]), i % 2, 64)
          for i in range(8)]

    def key(out):
        res, surv, ch = out
        return ([(x["n_survivors"], x["n_chains"], x["n_primes"]) for x in res],
                sorted(map(tuple, surv.view(np.uint32).reshape(-1, 4).tolist())),
                sorted(map(tuple, ch.view(np.uint32).reshape(-1, 12)[:, :11].tolist())))
    want_a, want_b = key(b0.run(ra)), key(b1.run(rb))
    for _ in range(2):
        b0.launch(ra)
        b1.launch(rb)
        with pytest.raises(ccs.CCSError) as e:
            b0.launch(ra)
        assert e.value.status == ccs.ERR_BUSY
        got_a = key(b0.wait())
        got_b = key(b1.wait())
        assert got_a == want_a and got_b == want_b
    b0.close()
    b1.close()
    for e in engines:
        e.close()
