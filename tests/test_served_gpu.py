"""Served path: requests that arrive while others run share ticks on the
GPU (two ticks in flight, on alternating batch executors), and each
request's survivors and chains equal a plain filter + prove of the same
range alone."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def surv_set(a):
    return sorted(map(tuple, np.asarray(a[["base_idx", "k_offset", "tile_idx"]].tolist())))


def chain_set(a):
    return sorted((int(r["base_idx"]), int(r["k_offset"]), int(r["tile_idx"]), int(r["chain_len"]),
                   tuple(int(x) for x in r["root"])) for r in a)


def chain_rows(t):
    a = t.cpu().numpy().astype(np.int64) & 0xFFFFFFFF
    return sorted((int(r[0]), int(r[1]), int(r[2]), int(r[3]), tuple(int(x) for x in r[4:10])) for r in a)


def test_served_results_equal_alone_and_in_the_mix(ccs):
    engines = [ccs.Engine(**ccs.config_depth_profile(d)) for d in (14, 16, 18)]
    for e in engines:
        e.bits = 64
    ranges = ccs.mixed_ranges(engines, 40, seed=5, min_log2=20, max_log2=31, width_lo=62, width_hi=66)
    srv = ccs.Server(engines, max_active=8, chunk_tiles=3000)
    ids = []
    for i, (ts, nt, p, bits) in enumerate(ranges):
        ids.append(srv.submit(ts, nt, p, bits))
        if i % 7 == 3:
            time.sleep(0.002)          # arrivals while earlier requests run
        if i == 20:                    # executor re-tuned between ticks
            srv.set_batch_tuning(block_threads=128, unit_words=2048)
    mixed = {}
    for rid in ids:
        srv.wait(rid)
        st, res, surv, chains = srv.poll(rid)
        assert st == ccs.OK
        mixed[rid] = (res, surv_set(surv), chain_set(chains))
    stats = srv.stats()
    assert stats["completed"] == len(ranges) and stats["ticks"] < len(ranges) * 10
    # overlap: some request took part in a tick together with others
    assert any(v[0]["ticks"] > 1 for v in mixed.values())
    # alone: one request on an otherwise idle server, and a plain run
    for rid, (ts, nt, p, bits) in list(zip(ids, ranges))[:12]:
        r2 = srv.submit(ts, nt, p, bits)
        srv.wait(r2)
        st, res2, s2, c2 = srv.poll(r2)
        assert (surv_set(s2), chain_set(c2)) == mixed[rid][1:]
        eng = engines[p]
        eng_bits = eng.bits
        plain = eng.filter_range(ts, nt, cap=1 << 18)
        want = sorted(map(tuple, (plain.cpu().numpy()[:, :3].astype(np.int64) & 0xFFFFFFFF).tolist()))
        assert mixed[rid][1] == want
        assert res2["n_survivors"] == len(want)
        # chains equal a plain prove of the plain survivors
        eng.set_bits(bits)
        pch, pprimes = eng.prove(plain, ts)
        assert mixed[rid][2] == chain_rows(pch)
        assert mixed[rid][0]["n_primes"] == pprimes
    # device-byte admission: reserved while running, released at the end
    now, peak = srv.memory()
    assert now == 0 and peak > 0
    srv.close()
    for e in engines:
        e.close()


def test_cancel_and_unknown_ids(ccs):
    eng = ccs.Engine(**ccs.config_depth_profile(16))
    srv = ccs.Server([eng], max_active=1, chunk_tiles=1000)
    ts = (1 << 87) // (1616615 * 20677)
    a = srv.submit(ts, 200000, 0, 88)
    b = srv.submit(ts + 10**7, 5000, 0, 88)
    srv.cancel(b)
    srv.wait(a)
    st, res, _, _ = srv.poll(a)
    assert st == ccs.OK and res["candidates"] > 0
    srv.wait(b)
    st, res, _, _ = srv.poll(b)
    assert st == ccs.ERR_CANCELLED
    with pytest.raises(ccs.CCSError):
        srv.cancel(987654321)
    srv.close()
    eng.close()
