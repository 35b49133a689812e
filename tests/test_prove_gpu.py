"""Prove / chain-walk parity on the GPU against GMP-derived golden fixtures,
the oracle's restatement of both reference prove paths, and (where built)
the reference K2 kernel itself."""
import os
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF13 = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                     "libref13.so")


@pytest.fixture(scope="module")
def eng_bpsw(ccs):
    e = ccs.Engine(primality=ccs.PRIME_BPSW, prove_mode=ccs.PROVE_FULL)
    yield e
    e.close()


@pytest.fixture(scope="module")
def eng_mr(ccs):
    e = ccs.Engine(primality=ccs.PRIME_MR, prove_mode=ccs.PROVE_ROOTS)
    yield e
    e.close()


def test_known_roots(eng_bpsw, eng_mr, golden):
    rows = golden("known_roots.json")["chains"]
    nums = [int(r["root"]) for r in rows]
    want = [r["forward"] for r in rows]
    assert list(eng_bpsw.walk_numbers(nums)) == want
    assert list(eng_mr.walk_numbers(nums)) == want


def test_primality_matches_gmp(eng_bpsw, eng_mr, golden):
    cases = golden("gmp_primality.json")["cases"]
    nums = [int(s) for s, _ in cases]
    is_p = [g > 0 for _, g in cases]
    for eng in (eng_bpsw, eng_mr):
        got = eng.walk_numbers(nums)
        assert [bool(x > 0) for x in got] == is_p


def test_data_sample_chain_lengths(eng_bpsw, eng_mr, golden):
    rows = golden("cc10_sample.json")["roots"]
    nums = [int(r["root"], 16) for r in rows]
    want = [r["forward"] for r in rows]
    assert list(eng_bpsw.walk_numbers(nums)) == want
    assert list(eng_mr.walk_numbers(nums)) == want


def test_walk_roots_golden(eng_bpsw, golden):
    rows = golden("walk_roots.json")["roots"]
    got = eng_bpsw.walk_numbers([int(r["n"]) for r in rows])
    assert list(got) == [r["forward"] for r in rows]


def test_walk_matches_oracle_random(eng_bpsw, eng_mr, ob):
    r = random.Random(11)
    nums = [r.getrandbits(r.randint(60, 127)) | 1 for _ in range(300)]
    # plant chains: 2^k-smooth-free odd numbers around known chain members
    nums += [2759832934171386593519 * 2 + 1, 95405042230542329 * 4 + 3]
    assert list(eng_bpsw.walk_numbers(nums)) == [ob.chain_from(n, ob.PRIME_BPSW) for n in nums]
    assert list(eng_mr.walk_numbers(nums)) == [ob.chain_from(n, ob.PRIME_MR) for n in nums]


def _lines(ccs, chains, target):
    out = []
    for rec in np.asarray(chains.cpu().numpy()).astype(np.int64) & 0xFFFFFFFF:
        root = sum(int(rec[4 + i]) << (32 * i) for i in range(6))
        out.append(ccs.format_chain_line(int(rec[3]), root, target, bool(rec[10] & 1)))
    return sorted(out)


def test_prove_matches_reference_cpu_prover(ccs, golden):
    """Chain records reproduce the reference GMP prover pool's output lines
    (prove_survivors_mt, v13:1967-2068) on the same survivors."""
    import torch
    for run in golden("v13_prover.json")["runs"]:
        eng = ccs.Engine(target=run["target"], bits=run["bits"])
        surv = torch.tensor(np.array(run["survivors"], dtype=np.int64).astype(np.uint32).view(np.int32),
                            device="cuda").reshape(-1, 4)
        chains, primes = eng.prove(surv, int(run["tile_start"]))
        assert primes == run["primes"]
        assert _lines(ccs, chains, run["target"]) == run["lines"]
        eng.close()


def test_prove_roots_mode_matches_oracle(ccs, ob, eng_mr):
    """K2 semantics (roots only, 132-prime trial division, 20-witness MR)."""
    lat = ob.Lattice()
    eng = ccs.Engine(bits=61, primality=ccs.PRIME_MR, prove_mode=ccs.PROVE_ROOTS)
    ts = (1 << 60) // (20677 * 1616615) + 999
    surv = eng.filter_range(ts, 800)
    chains, primes = eng.prove(surv, ts)
    want = []
    nprime = 0
    for b, k, t, _ in np.asarray(surv.cpu().numpy()).astype(np.int64):
        n = lat.reconstruct(ts, b, k, t)
        res, isp = ob.prove_n(n, 61, mode=0, primality=ob.PRIME_MR)
        nprime += isp
        if res is not None:
            want.append(ccs.format_chain_line(res[0], res[1], 18, res[2]))
    assert primes == nprime
    assert _lines(ccs, chains, 18) == sorted(want)
    eng.close()


def test_search_range_host_path(ccs, ob):
    """Host-buffer boundary: same survivors and chains as the device path."""
    eng = ccs.Engine(bits=64)
    ts = (1 << 63) // (20677 * 1616615) + 31337
    surv, chains, primes = eng.search_range_host(ts, 500)
    dev = eng.filter_range(ts, 500)
    assert sorted(map(tuple, surv[["base_idx", "k_offset", "tile_idx"]].tolist())) == \
        sorted(map(tuple, (dev.cpu().numpy()[:, :3].astype(np.int64) & 0xFFFFFFFF).tolist()))
    lat = ob.Lattice()
    want = 0
    for rec in surv:
        n = lat.reconstruct(ts, int(rec["base_idx"]), int(rec["k_offset"]), int(rec["tile_idx"]))
        res, _ = ob.prove_n(n, 64, mode=1)
        want += res is not None
    assert len(chains) == want
    eng.close()


@pytest.mark.skipif(not os.path.exists(REF13), reason="reference harness not built")
def test_roots_mode_matches_reference_k2(ccs, ob):
    """Same ChainResult set as the reference cc18_prove_kernel on the
    reference kernel's own survivors (bits 61: no 2^128 wrap)."""
    r13 = ob.ref13()
    r13.ref13_setup(18, 18)
    r13.ref13_upload(18, 61)
    import ctypes as C
    import torch
    eng = ccs.Engine(bits=61, primality=ccs.PRIME_MR, prove_mode=ccs.PROVE_ROOTS)
    ts = (1 << 60) // (20677 * 1616615) + 4321
    cap = 1 << 20
    out = np.zeros(4 * cap, dtype=np.uint32)
    cnt = r13.ref13_filter(ts & (2**64 - 1), ts >> 64, 2000, 12, out, cap)
    res = np.zeros(4 * 65536, dtype=np.uint32)
    pr = C.c_uint(0)
    nres = r13.ref13_prove_gpu(ts & (2**64 - 1), ts >> 64, res, 65536, C.byref(pr))
    ref = sorted(map(tuple, res[: 4 * nres].reshape(-1, 4).astype(np.int64).tolist()))
    surv = torch.tensor(out[: 4 * cnt].view(np.int32), device="cuda").reshape(-1, 4)
    chains, primes = eng.prove(surv, ts)
    got = sorted(map(tuple, (chains.cpu().numpy()[:, :4].astype(np.int64) & 0xFFFFFFFF).tolist()))
    assert got == ref
    assert primes == pr.value
    eng.close()


def test_walk_rounds_across_chunks(ccs, ob, eng_bpsw):
    """1.7e7 numbers (two walk chunks of 2^24): 40,000 distinct 80..110-bit
    odd numbers repeated 425 times give 425 identical length vectors, equal
    to the oracle's on a seeded sample."""
    import torch
    r = random.Random(2024)
    distinct = []
    for _ in range(40000):
        b = r.randint(80, 110)
        distinct.append(r.getrandbits(b) | (1 << (b - 1)) | 1)
    arr = np.zeros((len(distinct), 4), dtype=np.uint32)
    for i, v in enumerate(distinct):
        for w in range(4):
            arr[i, w] = (v >> (32 * w)) & 0xFFFFFFFF
    base = torch.from_numpy(arr.view(np.int32)).cuda()
    nums = base.repeat(425, 1).contiguous()
    lengths = torch.full((nums.shape[0],), -1, dtype=torch.int32, device="cuda")
    eng_bpsw.walk_numbers_dev(nums, 4, lengths)
    L = lengths.cpu().numpy().reshape(425, -1)
    assert (L == L[0]).all()
    for i in r.sample(range(len(distinct)), 300):
        assert L[0, i] == ob.chain_from(distinct[i], ob.PRIME_BPSW), distinct[i]


REF15 = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                     "libref15.so")


@pytest.mark.skipif(not os.path.exists(REF15), reason="reference harness not built")
@pytest.mark.parametrize("reverse", [False, True])
def test_matches_reference_v15_filter_and_prove_order(ccs, ob, reverse):
    """The reference v15 engine (the throughput kernel): its K1 survivor set
    equals ours, and its K2 in forward and in reverse order (--prove-order,
    chain position target - 1 tested first) gives our ChainResult set and
    prime count (bits 61, target 18: no 2^128 wrap)."""
    import ctypes as C
    import torch
    r15 = ob.ref15()
    r15.ref15_setup(18, 18)
    r15.ref15_upload(18, 61, 18, 0 if reverse else 1)
    eng = ccs.Engine(bits=61, primality=ccs.PRIME_MR, prove_mode=ccs.PROVE_ROOTS, reverse_prove=reverse)
    rr = random.Random(15 + reverse)
    for n_tiles in (1, 700, 3000):
        ts = (1 << 60) // (20677 * 1616615) + rr.randint(0, 10**6)
        cap = 1 << 20
        out = np.zeros(4 * cap, dtype=np.uint32)
        cnt = r15.ref15_filter(ts & (2**64 - 1), ts >> 64, n_tiles, 12, out, cap)
        ref_surv = sorted(map(tuple, out[: 4 * cnt].reshape(-1, 4)[:, :3].astype(np.int64).tolist()))
        ours = eng.filter_range(ts, n_tiles, cap=cap)
        assert sorted(map(tuple, (ours.cpu().numpy()[:, :3].astype(np.int64) & 0xFFFFFFFF).tolist())) == ref_surv
        res = np.zeros(4 * 65536, dtype=np.uint32)
        pr = C.c_uint(0)
        nres = r15.ref15_prove_gpu(ts & (2**64 - 1), ts >> 64, res, 65536, C.byref(pr))
        ref = sorted(map(tuple, res[: 4 * nres].reshape(-1, 4).astype(np.int64).tolist()))
        surv = torch.tensor(out[: 4 * cnt].view(np.int32), device="cuda").reshape(-1, 4)
        chains, primes = eng.prove(surv, ts)
        got = sorted(map(tuple, (chains.cpu().numpy()[:, :4].astype(np.int64) & 0xFFFFFFFF).tolist()))
        assert got == ref, (reverse, n_tiles)
        assert primes == pr.value
    eng.close()


@pytest.mark.parametrize("cfg", [
    dict(bits=89, primality="MR", prove_mode="ROOTS"),
    dict(bits=89, primality="BPSW", prove_mode="FULL"),
    dict(bits=61, primality="MR", prove_mode="ROOTS", reverse_prove=True),
    dict(bits=70, primality="BPSW", prove_mode="ROOTS", reverse_prove=True),
    dict(bits=80, primality="BPSW", prove_mode="FULL", kind=2),
])
def test_staged_prove_equals_per_survivor_prove(ccs, cfg):
    """ccs_prove runs a breadth-first staged prove from 256 survivors up and
    the one-thread-per-survivor kernel below that: the whole survivor set in
    one call must give the records of the same set proved in slices of 200
    (survivor index shifted by the slice start), and the same prime count."""
    import torch
    kw = dict(cfg)
    kw["primality"] = getattr(ccs, "PRIME_" + kw["primality"])
    kw["prove_mode"] = getattr(ccs, "PROVE_" + kw["prove_mode"])
    eng = ccs.Engine(**kw)
    info = eng.info
    lo, hi = ccs.bit_tile_range(cfg["bits"], eng.bases(), info["lattice_m"], info["wheel_period"])
    r = random.Random(cfg["bits"] * 7 + cfg.get("kind", 1))
    ts = r.randint(lo, max(lo, hi - 40000))
    surv = eng.filter_range(ts, min(20000, hi - ts), cap=1 << 20)
    assert surv.shape[0] >= 600
    whole, p_whole = eng.prove(surv, ts, cap=1 << 18)
    parts, p_parts = [], 0
    for s0 in range(0, surv.shape[0], 200):
        c, p = eng.prove(surv[s0:s0 + 200], ts, cap=1 << 16)
        c = c.clone()
        c[:, 11] += s0
        parts.append(c)
        p_parts += p
    parts = torch.cat(parts)
    key = lambda t: sorted(map(tuple, (t.cpu().numpy().astype(np.int64) & 0xFFFFFFFF).tolist()))
    assert p_whole == p_parts
    assert key(whole) == key(parts) and whole.shape[0] > 0
    eng.close()


def test_birth_certificates_replace_predecessor_tests(ccs, ob):
    """A prime n == 1 (mod q) for a screen prime q has a predecessor divisible
    by q (v34:70-77): the staged prove marks it a root without testing the
    predecessor.  Records still equal the oracle's full predecessor tests;
    every prime n is either certified or has its predecessor tested."""
    lat = ob.Lattice()
    eng = ccs.Engine(bits=61)
    ts = (1 << 60) // (20677 * 1616615) + 4321
    surv = eng.filter_range(ts, 3000)
    assert surv.shape[0] >= 256                       # staged path
    eng.prove_stats(reset=True)
    chains, primes = eng.prove(surv, ts)
    st = eng.prove_stats(reset=True)
    assert st["survivors"] == surv.shape[0] and st["primes"] == primes
    assert st["predecessor_tests"] + st["certified_roots"] == primes
    assert st["certified_roots"] > 0.2 * primes
    want = []
    for b, k, t, _ in np.asarray(surv.cpu().numpy()).astype(np.int64):
        res, _ = ob.prove_n(lat.reconstruct(ts, b, k, t), 61, mode=1)
        if res is not None:
            want.append(ccs.format_chain_line(res[0], res[1], 18, res[2]))
    assert _lines(ccs, chains, 18) == sorted(want)
    eng.close()
