"""Project autotuner and the tuning knobs it turns: every tuning gives the
same survivors (oracle parity after a table rebuild, unchanged sets after a
full autotune), and table rebuilds are refused while a batch holds the
engine."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def as_set(arr):
    a = np.asarray(arr.cpu().numpy() if hasattr(arr, "cpu") else arr).astype(np.int64) & 0xFFFFFFFF
    return sorted(map(tuple, a[:, :3].tolist()))


@pytest.mark.parametrize("split,table,threads", [(512, 7, 256), (1024, 22, 128), (2048, 7, 256), (1024, 7, 128)])
def test_stage_split_rebuild_matches_oracle(ccs, ob, split, table, threads):
    eng = ccs.Engine()
    eng.set_tuning(split_prime=split, table_primes=table, block_threads=threads)
    t = eng.tuning()
    assert (t["split_prime"], t["table_primes"], t["block_threads"]) == (split, table, threads)
    lat = ob.Lattice()
    r = random.Random(split + table)
    for n in (1, 7, 300, 2000):
        ts = r.randint(1 << 44, 1 << 60)
        for ext in (1, 0xFFFFFFFF):
            eng.set_tuning(ext_min_words=ext)
            assert as_set(eng.filter_range(ts, n, cap=1 << 18)) == as_set(lat.filter_range(ts, n)), (ts, n, ext)
    eng.close()


def test_autotune_keeps_results(ccs):
    cfg = ccs.config_cc16_scale()
    eng = ccs.Engine(**cfg)
    ts = (1 << 87) // (1616615 * 20677) + 424242
    before = as_set(eng.filter_range(ts, 600_000, cap=1 << 18))
    chosen, points = eng.autotune(ts, 1 << 20)
    assert points and all(ms > 0 for _, _, ms in points)
    assert chosen == eng.tuning()
    assert chosen["block_threads"] in (128, 256) and chosen["unit_words"] >= 128
    after = as_set(eng.filter_range(ts, 600_000, cap=1 << 18))
    assert before == after and len(before) > 10
    eng.close()


def test_table_rebuild_refused_while_batched(ccs):
    eng = ccs.Engine(target=16, depth=16)
    batch = ccs.Batch([eng], 4)
    with pytest.raises(ccs.CCSError) as e:
        eng.set_tuning(split_prime=512)
    assert e.value.status == ccs.ERR_BUSY
    eng.set_tuning(unit_words=512)              # no rebuild: allowed
    batch.close()
    eng.set_tuning(split_prime=512)
    assert eng.tuning()["split_prime"] == 512
    eng.close()
