"""Generates the committed golden fixtures under tests/golden/ from the
reference itself (run in the container that holds the reference tree):

  * known_roots.json   -- the reference self-test vectors (v13:2089-2101,
                          v33:2401, v33:2735) with chain lengths from GMP's
                          mpz_probab_prime_p walk of the CPU prover
                          (v13:1870-1881) and from v33's screened walker
  * cc10_sample.json   -- roots from the reference data sample
                          (data/sample/cc10plus_roots_sample_1000.txt) with
                          their GMP chain lengths
  * gmp_primality.json -- GMP 6.3.0 mpz_probab_prime_p(n, 1) verdicts on
                          seeded primes, composites, base-2 strong
                          pseudoprimes and Carmichael numbers
  * v33_counts.json    -- survivor / stage counters of the reference CPU
                          engine (cc_gmp_v33 --sieve-only) on seeded
                          sequential prefix ranges
  * v13_prover.json    -- output lines of the reference CPU GMP prover pool
                          (prove_survivors_mt) on survivors of seeded ranges
  * walk_roots.json    -- seeded 80..110-bit odd roots with GMP forward chain
                          lengths (the prove-batch workload)

  * second_kind.json   -- the same for second-kind chains (v13b): self-test
                          vectors with GMP 2p - 1 walks and the v13b CPU
                          prover's output lines
  * v33_native.json    -- the reference CPU engine's own proving path (root
                          test, root check, backward / screened forward walks)
                          on every survivor of seeded ranges of its lattice,
                          and its screened walk of seeded numbers
  * cc16_windows.json  -- the oracle's survivor sets on 64+ seeded windows of
                          the depth-16 / primes-to-2^17 profile (W = 31#,
                          88-bit roots) holding at least 300 survivors in
                          total; no reference engine takes stage primes up to
                          2^17, so these pin the GPU filter to the oracle,
                          whose per-candidate test is itself pinned to the
                          reference's counters and kernels at 37..863

Usage: python tests/golden/make_golden.py [--second-kind | --cc16-windows | --v33-native]
(the reference fixtures need oracle/_ref built by `make -C oracle` and the
reference tree in $CCS_REFERENCE_DIR).
"""
import json
import os
import random
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_bind as ob  # noqa: E402



def reference_dir():
    """The reference tree: $CCS_REFERENCE_DIR, else a directory named
    `reference` beside this repository."""
    d = os.environ.get("CCS_REFERENCE_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "..", "reference")
    d = os.path.abspath(d)
    if not os.path.isdir(os.path.join(d, "src")):
        sys.exit(f"reference tree not found at {d}: set CCS_REFERENCE_DIR")
    return d


def dump_compact(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, separators=(",", ":"))
    print("wrote", name)


def dump(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, indent=1)
    print("wrote", name)


def main():
    r33 = ob.ref33()
    r13 = ob.ref13()
    assert r33 is not None and r13 is not None, "build oracle/_ref first (make -C oracle)"

    # ---- known roots -----------------------------------------------------
    vecs = ["2", "89", "1122659", "19099919", "85864769", "26089808579", "665043081119",
            "554688278429", "4090932431513069", "95405042230542329", "2759832934171386593519",
            str(int("3d3aa382c918303b5470bad", 16)), str(int("5062b474874cd337fe0f061aaef7c442d1", 16))]
    known = []
    for v in vecs:
        n = int(v)
        buf = C_buf()
        full = r33.ref33_full_chain(hex(n)[2:].encode(), buf)
        fwd = r33.ref_gmp_forward_chain(hex(n)[2:].encode())
        scr = r33.ref33_forward_chain(hex(n)[2:].encode())
        known.append({"root": v, "forward": fwd, "v33_screened": scr, "full": full,
                      "full_root": str(int(buf.value, 16))})
    q7 = ["0x140ECDB88F050428006DE301E959", "0x1F4FFB48D6888D03552C06F4F1ED",
          "0x1FEC88EDDD75548569E35D0B2871", "0x1FB44BE8961B14B6BCA70B0059B1"]
    dump("known_roots.json", {"source": "v13:2089-2101, v33:2401, v33:2735, v13:2816-2821",
                              "chains": known, "q7_roots": q7})

    # ---- data sample -----------------------------------------------------
    rows = []
    with open(os.path.join(reference_dir(), "data/sample/cc10plus_roots_sample_1000.txt")) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[1].startswith("0x"):
                rows.append((parts[0], parts[1]))
    sample = []
    for tag, hx in rows:
        n = int(hx, 16)
        fwd = r33.ref_gmp_forward_chain(hx[2:].encode())
        sample.append({"tag": tag, "root": hx, "forward": fwd})
    dump("cc10_sample.json", {"source": "data/sample/cc10plus_roots_sample_1000.txt",
                              "roots": sample})

    # ---- GMP primality ---------------------------------------------------
    rnd = random.Random(20261203)
    nums = set()
    for bits in (8, 16, 31, 32, 33, 63, 64, 65, 80, 89, 96, 110, 127, 128, 129, 150, 180):
        for _ in range(40):
            nums.add(rnd.getrandbits(bits) | (1 << (bits - 1)) | 1)
    # primes by search
    for bits in (40, 64, 89, 110, 128, 160, 190):
        found = 0
        while found < 25:
            n = rnd.getrandbits(bits) | (1 << (bits - 1)) | 1
            if r33.ref33_gmp_probab_prime(hex(n)[2:].encode(), 25) > 0:
                nums.add(n)
                found += 1
    # strong pseudoprimes to base 2, Carmichael numbers, Wieferich squares
    spsp2 = [2047, 3277, 4033, 4681, 8321, 15841, 29341, 42799, 49141, 52633, 65281, 74665,
             80581, 85489, 88357, 90751, 3215031751, 2152302898747, 3474749660383,
             341550071728321, 3825123056546413051]
    carm = [561, 1105, 1729, 2465, 2821, 6601, 8911, 10585, 15841, 29341, 41041, 46657, 52633]
    for v in spsp2 + carm + [1093 ** 2, 3511 ** 2, 1093 * 3511, 2, 3, 5, 7, 9, 15, 25, 49, 97 * 97]:
        nums.add(v)
    nums.add(18446744073709551557)  # largest 64-bit prime
    prim = []
    for n in sorted(nums):
        prim.append([str(n), r33.ref33_gmp_probab_prime(hex(n)[2:].encode(), 1)])
    dump("gmp_primality.json", {"source": "GMP 6.3.0 mpz_probab_prime_p(n, 1) via oracle/_ref",
                                "cases": prim})

    # ---- v33 sieve-only counts on sequential prefix ranges ----------------
    counts = []
    for (bits, target, pbits, seed) in [(89, 18, 47, 1), (89, 18, 47, 2), (89, 18, 46, 3),
                                        (61, 18, 21, 4), (100, 18, 58, 5), (89, 16, 47, 6),
                                        (89, 14, 48, 7)]:
        rr = random.Random(seed)
        prefix = (1 << (pbits - 1)) | rr.getrandbits(pbits - 1)
        pstr = "0b" + bin(prefix)[2:]
        out = subprocess.run([os.path.join(ob.REF_DIR, "cc_gmp_v33"), "--sieve-only", "--prefix", pstr,
                              "--sequential", "--bits", str(bits), "--target", str(target),
                              "--threads", "1"], capture_output=True, text=True).stdout
        wc = int(re.search(r"Wheel candidates \(L1\):\s+(\d+)", out).group(1))
        l2 = int(re.search(r"Passed L2 bitmask:\s+(\d+)", out).group(1))
        ext = int(re.search(r"Passed ext L2 \(OPT-7\):\s+(\d+)", out).group(1))
        lp = int(re.search(r"Line-sieve \(OPT-17\):\s+(\d+) passed", out).group(1))
        counts.append({"bits": bits, "target": target, "prefix": pstr, "candidates": wc,
                       "pass_l2": l2, "pass_ext": ext, "survivors": lp})
    dump("v33_counts.json", {"source": "cc_gmp_v33 --sieve-only --sequential (v33:1690-1960)",
                             "runs": counts})

    # ---- v13 CPU prover on oracle survivors --------------------------------
    prover = []
    for (target, bits, ts, nt) in [(18, 61, (1 << 60) // (20677 * 1616615) + 12345, 600),
                                   (18, 64, (1 << 63) // (20677 * 1616615) + 777, 400),
                                   (16, 61, (1 << 60) // (20677 * 1616615) + 4242, 300)]:
        r13.ref13_setup(target, target)
        lat = ob.Lattice(lattice_len=target, depth=target)
        surv = lat.filter_range(ts, nt)
        lat13_n = r13.ref13_num_bases()
        if target < 18:
            # v13 caps the base list at MAX_BASES = 64 (v13:966): keep the
            # survivors its CPU prover can address
            surv = surv[surv[:, 0] < lat13_n]
        s = np.ascontiguousarray(surv.astype(np.uint32))
        path = tempfile.mktemp(suffix=".txt")
        import ctypes as C
        pr, ch = C.c_ulonglong(0), C.c_ulonglong(0)
        r13.ref13_prove_cpu(s.reshape(-1), len(s), ts & (2**64 - 1), ts >> 64, target, bits,
                            path.encode(), C.byref(pr), C.byref(ch))
        lines = [ln.strip() for ln in open(path) if ln.strip()]
        os.unlink(path)
        prover.append({"target": target, "depth": target, "bits": bits, "tile_start": str(ts),
                       "n_tiles": nt, "n_survivors": int(len(surv)), "primes": pr.value,
                       "chains": ch.value, "lines": sorted(lines),
                       "survivors": surv.astype(np.int64).tolist()})
    dump("v13_prover.json", {"source": "prove_survivors_mt (v13:1967-2068) via oracle/_ref",
                             "runs": prover})

    # ---- walk roots (prove-batch workload) ---------------------------------
    # odd roots drawn from seeded 80..110-bit tile windows of the 31# lattice at
    # depth 16, pre-filtered by primes 37..1021 at chain positions 0..15 (the
    # first filter stage of the prove-batch configuration)
    rw = random.Random(424242)
    lat = ob.Lattice(lattice_len=16, depth=16, stages=[(ob.primes_between(37, 1024), 0)])
    M, WP = lat.M, lat.WP
    bases = lat.bases()
    walks = []
    while len(walks) < 400:
        bits = rw.randint(80, 110)
        lo = (1 << (bits - 1)) // (M * WP)
        hi = (1 << bits) // (M * WP)
        ts = rw.randint(lo, hi - 20)
        surv = lat.filter_range(ts, 6)
        for b, k, t, _ in surv[:4]:
            n = ((ts + int(t)) * WP + int(k)) * M + bases[int(b)]
            walks.append({"n": str(n), "forward": r33.ref_gmp_forward_chain(hex(n)[2:].encode())})
    dump("walk_roots.json", {"source": "GMP mpz_probab_prime_p(., 1) forward walk (v13:1870-1881)",
                             "roots": walks})


def second_kind():
    """second_kind.json: the reference v13b self-test vectors (read from its
    source, v13b:2095-2112) and seeded survivors of its filter, with GMP
    2p - 1 walk lengths (the v13b CPU prover's loop), plus the v13b CPU
    prover's output lines on survivors of seeded ranges."""
    r33 = ob.ref33()
    r13b = ob.ref13b()
    assert r33 is not None and r13b is not None, "build oracle/_ref first (make -C oracle)"
    src = open(os.path.join(reference_dir(), "src/cuda/cc18_filter_cuda_CpC_v13b.cu")).read()
    table = src[src.index("Known second-kind Cunningham chain test vectors"):]
    table = table[:table.index("};")]
    vecs = re.findall(r'\{\s*"(\d+)",\s*(\d+),', table)
    known = [{"root": v, "selftest_len": int(n), "forward": r33.ref_gmp_forward_chain2(hex(int(v))[2:].encode())}
             for v, n in vecs]
    prover = []
    import ctypes as C
    for (target, bits, ts, nt) in [(18, 61, (1 << 60) // (20677 * 1616615) + 5151, 600),
                                   (16, 64, (1 << 63) // (20677 * 1616615) + 99, 300)]:
        r13b.ref13_setup(target, target)
        lat = ob.Lattice(lattice_len=target, depth=target, kind_=2)
        surv = lat.filter_range(ts, nt)
        if target < 18:
            surv = surv[surv[:, 0] < r13b.ref13_num_bases()]
        s_ = np.ascontiguousarray(surv.astype(np.uint32))
        path = tempfile.mktemp(suffix=".txt")
        pr, ch = C.c_ulonglong(0), C.c_ulonglong(0)
        r13b.ref13_prove_cpu(s_.reshape(-1), len(s_), ts & (2**64 - 1), ts >> 64, target, bits,
                             path.encode(), C.byref(pr), C.byref(ch))
        lines = [ln.strip() for ln in open(path) if ln.strip()]
        os.unlink(path)
        prover.append({"target": target, "bits": bits, "tile_start": str(ts), "n_tiles": nt,
                       "primes": pr.value, "chains": ch.value, "lines": sorted(lines),
                       "survivors": surv.astype(np.int64).tolist()})
    dump("second_kind.json", {"source": "v13b self-test vectors (v13b:2095-2112), GMP 2p-1 walks; "
                                        "prove_survivors_mt of v13b via oracle/_ref",
                              "chains": known, "prover": prover})


def v33_native():
    """v33_native.json: the reference CPU engine's native proving path
    (worker_sequential, v33:2112-2215) on every survivor of seeded ranges of
    its own lattice (W = 31#, stages 37..61 / 67..97 at positions 0..L-1,
    101..863 at 1..line_depth), and its screened walk (follow_chain_first,
    v33:1512-1577) of the self-test vectors, the data-sample roots, the
    walk-batch roots and small numbers near the screen primes."""
    r33 = ob.ref33()
    assert r33 is not None, "build oracle/_ref first (make -C oracle)"
    runs = []
    # (about 2,500 / 670 / 150 / 0.1 survivors per tile at targets 10 / 11 / 12 / 18)
    for (target, line_depth, bits, seed, n_tiles) in [(10, 9, 61, 1, 1), (11, 10, 64, 2, 2),
                                                       (12, 11, 72, 3, 8), (18, 17, 89, 4, 4000)]:
        r33.ref33_setup(target, line_depth)
        lat = ob.Lattice(lattice_len=target, depth=target,
                         stages=[(ob.L2_PRIMES, 0), (ob.EXT_PRIMES, 0), (ob.LINE_PRIMES, 1)])
        M, WP = lat.M, lat.WP
        bases = lat.bases()
        rr = random.Random(seed)
        lo = (1 << (bits - 1)) // (M * WP) + 1
        hi = (1 << bits) // (M * WP) - n_tiles - 1
        ts = rr.randint(lo, hi)
        surv = lat.filter_range(ts, n_tiles)
        out = []
        for b, k, t, _ in surv:
            n = ((ts + int(t)) * WP + int(k)) * M + bases[int(b)]
            code, root, is_root = ob.ref33_prove_native(r33, n, 1)
            out.append([int(b), int(k), int(t), code, format(root, "x"), int(is_root)])
        runs.append({"target": target, "line_depth": line_depth, "bits": bits, "tile_start": str(ts),
                     "n_tiles": n_tiles, "survivors": out})
        print(f"target {target} bits {bits}: {len(out)} survivors, "
              f"{sum(1 for x in out if x[3] > 0 or x[3] == -2)} primes", flush=True)
    r33.ref33_setup(18, 17)
    walks = []
    known = json.load(open(os.path.join(HERE, "known_roots.json")))["chains"]
    nums = [int(c["root"]) for c in known]
    nums += [int(x["root"], 16) for x in json.load(open(os.path.join(HERE, "cc10_sample.json")))["roots"]][:300]
    nums += [int(x["n"]) for x in json.load(open(os.path.join(HERE, "walk_roots.json")))["roots"]][:300]
    nums += [89, 179, 359, 719, 1439, 2879, 5, 11, 23, 47, 67, 137, 863, 1727]
    for n in nums:
        if n >= 1 << 127:
            continue
        walks.append([str(n), r33.ref33_follow_native(n & (2**64 - 1), n >> 64, 0)])
    dump_compact("v33_native.json", {
        "source": "cc_gmp_v33 native proving path (v33:2112-2215) and follow_chain_first "
                  "(v33:1512-1577) via oracle/_ref/libref33.so; codes: -1 trial division, "
                  "0 root test failed, -2 skipped by the prefilter (log threshold 1), "
                  "else the chain length of the root",
        "runs": runs, "walks": walks})


CC16_WINDOW_TILES = 16384


def _cc16_window(args):
    """Oracle survivors of one window (runs in a spawned worker)."""
    ts, n = args
    lat = ob.Lattice(lattice_len=16, depth=16, stages=cc16_stages())
    surv = lat.filter_range(ts, n)
    return sorted(map(tuple, surv[:, :3].astype(np.int64).tolist()))


def cc16_stages():
    """Stage primes 37..2^10 / 2^10..2^14 / 2^14..2^17 at chain positions 0..15."""
    return [(ob.primes_between(37, 1 << 10), 0), (ob.primes_between(1 << 10, 1 << 14), 0),
            (ob.primes_between(1 << 14, 1 << 17), 0)]


def cc16_windows(min_windows=64, min_survivors=300):
    """cc16_windows.json: seeded 2^14-tile windows spread over the 88-bit tile
    range of the depth-16 profile, filtered by the oracle on every core, until
    at least min_windows windows and min_survivors survivors are collected."""
    import multiprocessing as mp
    lat = ob.Lattice(lattice_len=16, depth=16, stages=cc16_stages())
    M, WP = lat.M, lat.WP
    bases = lat.bases()
    t_lo = -(-((1 << 87) - max(bases)) // (M * WP))
    t_hi = ((1 << 88) - 1) // (M * WP) - CC16_WINDOW_TILES
    rw = random.Random(16172026)
    windows, total = [], 0
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        while len(windows) < min_windows or total < min_survivors:
            batch = [(rw.randint(t_lo, t_hi), CC16_WINDOW_TILES) for _ in range(16)]
            for (ts, n), surv in zip(batch, pool.map(_cc16_window, batch)):
                windows.append({"tile_start": str(ts), "n_tiles": n, "survivors": surv})
                total += len(surv)
            print(f"{len(windows)} windows, {total} survivors", flush=True)
    dump("cc16_windows.json", {
        "source": "oracle orc_filter_range (per-candidate restatement of v13:1551-1714 / "
                  "v33:1795-1960) on the depth-16 profile",
        "profile": {"target": 16, "depth": 16, "bits": 88, "crt": ob.CRT_PRIMES,
                    "wheel": ob.WHEEL_PRIMES,
                    "stages": "primes 37..2^10 / 2^10..2^14 / 2^14..2^17, positions 0..15"},
        "candidates_per_tile": 73008, "total_survivors": total, "windows": windows})


def C_buf():
    import ctypes as C
    return C.create_string_buffer(256)


if __name__ == "__main__":
    if "--cc16-windows" in sys.argv:
        cc16_windows()
    elif "--v33-native" in sys.argv:
        v33_native()
    elif "--second-kind" in sys.argv:
        second_kind()
    else:
        main()
        second_kind()
