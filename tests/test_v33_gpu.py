"""CCS_PRIME_V33 on the GPU: the engine with the reference CPU engine's own
lattice, filter stages and tests gives, for every survivor of seeded ranges,
the record the reference engine's native proving path gives
(tests/golden/v33_native.json, made from its own functions), through the
staged prove, the per-survivor prove and the batched path; the walk of given
numbers equals its screened walk."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def engine(ccs, run):
    return ccs.Engine(target=run["target"], depth=run["target"], bits=run["bits"],
                      stages=ccs.reference_cpu_stages(), primality=ccs.PRIME_V33,
                      prove_mode=ccs.PROVE_FULL)


def want_records(run):
    rec = {}
    for b, k, t, code, root_hex, is_root in run["survivors"]:
        if code > 0:
            rec[(b, k, t)] = (code, int(root_hex, 16), bool(is_root))
    primes = sum(1 for x in run["survivors"] if x[3] > 0 or x[3] == -2)
    return rec, primes


def got_records(chains):
    a = chains.cpu().numpy().astype(np.int64) & 0xFFFFFFFF
    out = {}
    for r in a:
        root = sum(int(r[4 + w]) << (32 * w) for w in range(6))
        out[(int(r[0]), int(r[1]), int(r[2]))] = (int(r[3]), root, bool(r[10] & 1))
    return out


def test_v33_prove_equals_reference(ccs, golden):
    for run in golden("v33_native.json")["runs"]:
        eng = engine(ccs, run)
        ts = int(run["tile_start"])
        surv = eng.filter_range(ts, run["n_tiles"], cap=1 << 18)
        a = surv.cpu().numpy().astype(np.int64) & 0xFFFFFFFF
        assert sorted(map(tuple, a[:, :3].tolist())) == sorted(tuple(x[:3]) for x in run["survivors"])
        want, want_primes = want_records(run)
        # all survivors at once (staged prove from 256 on), then in slices of
        # 100 (one thread per survivor)
        chains, primes = eng.prove(surv, ts, cap=1 << 16)
        assert got_records(chains) == want and primes == want_primes, run["target"]
        got, tot = {}, 0
        for i in range(0, surv.shape[0], 100):
            c, p = eng.prove(surv[i:i + 100].contiguous(), ts, cap=1 << 16)
            got.update(got_records(c))
            tot += p
        assert got == want and tot == want_primes
        eng.close()


def test_v33_batched_equals_reference(ccs, golden):
    """Every run as one range of one batched launch (one profile per run)."""
    runs = golden("v33_native.json")["runs"]
    engs = [engine(ccs, r) for r in runs]
    b = ccs.Batch(engs, len(runs), surv_cap=1 << 18, chain_cap=1 << 16)
    res, surv, chains = b.run([(int(r["tile_start"]), r["n_tiles"], i, r["bits"]) for i, r in enumerate(runs)])
    b.close()
    rid = surv["_pad"].astype(np.int64)
    crid = rid[chains["survivor"].astype(np.int64)]
    raw = chains.view(np.uint32).reshape(-1, 12)
    for i, run in enumerate(runs):
        want, want_primes = want_records(run)
        got = {}
        for r in raw[crid == i].astype(np.int64):
            root = sum(int(r[4 + w]) << (32 * w) for w in range(6))
            got[(int(r[0]), int(r[1]), int(r[2]))] = (int(r[3]), root, bool(r[10] & 1))
        assert got == want and res[i]["n_primes"] == want_primes
    for e in engs:
        e.close()


def test_v33_walk_equals_reference(ccs, golden):
    walks = golden("v33_native.json")["walks"]
    eng = ccs.Engine(target=8, depth=8, bits=61, stages=ccs.reference_cpu_stages(),
                     primality=ccs.PRIME_V33, prove_mode=ccs.PROVE_FULL)
    nums = [int(s) for s, _ in walks]
    got = eng.walk_numbers(nums, limbs=6)
    assert [int(x) for x in got] == [ln for _, ln in walks]
    assert dict(walks)["89"] == 1
    eng.close()


def test_v33_is_a_first_kind_full_prove(ccs):
    with pytest.raises(ccs.CCSError):
        ccs.Engine(target=8, primality=ccs.PRIME_V33, prove_mode=ccs.PROVE_ROOTS)
    with pytest.raises(ccs.CCSError):
        ccs.Engine(target=8, primality=ccs.PRIME_V33, kind=2)
