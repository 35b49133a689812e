"""Second-kind chains (p -> 2p - 1) on the GPU: survivor sets equal the
oracle's and the reference v13b kernel's own, chain records equal the v13b
K2's and the v13b CPU prover's lines, and chain walks equal GMP's."""
import ctypes as C
import os
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF13B = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                      "libref13b.so")


def as_set(arr):
    a = np.asarray(arr.cpu().numpy() if hasattr(arr, "cpu") else arr).astype(np.int64) & 0xFFFFFFFF
    return sorted(map(tuple, a[:, :3].tolist()))


@pytest.mark.parametrize("profile", ["reference", "cc16"])
def test_filter_matches_oracle(ccs, ob, profile):
    if profile == "reference":
        cfg, lat = {}, ob.Lattice(kind_=2)
    else:
        cfg = ccs.config_cc16_scale()
        lat = ob.Lattice(lattice_len=16, depth=16, stages=cfg["stages"], kind_=2)
    eng = ccs.Engine(kind=ccs.KIND_SECOND, **cfg)
    r = random.Random(len(profile))
    for ext in (0xFFFFFFFF, 1):
        eng.set_tuning(ext_min_words=ext)
        for n in (1, 7, 300) if profile == "cc16" else (1, 7, 300, 1500):
            ts = r.randint(1 << 40, 1 << 60)
            assert as_set(eng.filter_range(ts, n, cap=1 << 20)) == as_set(lat.filter_range(ts, n)), (ts, n, ext)
    eng.close()


@pytest.mark.skipif(not os.path.exists(REF13B), reason="reference harness not built")
def test_matches_reference_v13b_kernels(ccs, ob):
    """Bit-identical survivor sets versus v13b's cc18_filter_kernel and the
    same ChainResult records and prime count as its cc18_prove_kernel."""
    import torch
    r13b = ob.ref13b()
    r13b.ref13_setup(18, 18)
    r13b.ref13_upload(18, 61)
    eng = ccs.Engine(kind=ccs.KIND_SECOND, bits=61, primality=ccs.PRIME_MR, prove_mode=ccs.PROVE_ROOTS)
    r = random.Random(13)
    for n in (1, 97, 2000, 16384):
        ts = (1 << 60) // (20677 * 1616615) + r.randint(0, 10**6)
        cap = 1 << 20
        out = np.zeros(4 * cap, dtype=np.uint32)
        cnt = r13b.ref13_filter(ts & (2**64 - 1), ts >> 64, n, 12, out, cap)
        ref = as_set(out[: 4 * cnt].reshape(-1, 4))
        assert as_set(eng.filter_range(ts, n, cap=cap)) == ref, n
        res = np.zeros(4 * 65536, dtype=np.uint32)
        pr = C.c_uint(0)
        nres = r13b.ref13_prove_gpu(ts & (2**64 - 1), ts >> 64, res, 65536, C.byref(pr))
        want = sorted(map(tuple, res[: 4 * nres].reshape(-1, 4).astype(np.int64).tolist()))
        surv = torch.tensor(out[: 4 * cnt].view(np.int32), device="cuda").reshape(-1, 4)
        chains, primes = eng.prove(surv, ts)
        got = sorted(map(tuple, (chains.cpu().numpy()[:, :4].astype(np.int64) & 0xFFFFFFFF).tolist()))
        assert got == want and primes == pr.value, n
    eng.close()


def test_prove_matches_v13b_cpu_prover(ccs, golden):
    import torch
    for run in golden("second_kind.json")["prover"]:
        eng = ccs.Engine(kind=ccs.KIND_SECOND, target=run["target"], bits=run["bits"])
        surv = torch.tensor(np.array(run["survivors"], dtype=np.int64).astype(np.uint32).view(np.int32),
                            device="cuda").reshape(-1, 4)
        chains, primes = eng.prove(surv, int(run["tile_start"]))
        lines = []
        for rec in np.asarray(chains.cpu().numpy()).astype(np.int64) & 0xFFFFFFFF:
            root = sum(int(rec[4 + i]) << (32 * i) for i in range(6))
            lines.append(ccs.format_chain_line(int(rec[3]), root, run["target"], bool(rec[10] & 1)))
        assert primes == run["primes"]
        assert sorted(lines) == run["lines"]
        eng.close()


def test_second_kind_walks(ccs, ob, golden):
    rows = golden("second_kind.json")["chains"]
    nums = [int(r["root"]) for r in rows]
    want = [r["forward"] for r in rows]
    r = random.Random(2)
    extra = [r.getrandbits(r.randint(40, 120)) | 1 for _ in range(400)]
    for primality in (ccs.PRIME_BPSW, ccs.PRIME_MR):
        eng = ccs.Engine(kind=ccs.KIND_SECOND, primality=primality)
        assert list(eng.walk_numbers(nums)) == want
        assert list(eng.walk_numbers(extra)) == [ob.chain_from(n, primality, kind_=2) for n in extra]
        eng.close()
