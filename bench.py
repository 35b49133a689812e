"""Benchmark: candidates/s of the filter + prove hot path on B200.

Workload (one GPU): the CC18-style GPU filter scale -- lattice W = 31#,
depth 16, stage primes 37..2^10 / 2^10..2^14 / 2^14..2^17 at chain positions
0..15, roots of 88 bits starting at a seed-drawn tile, 1e13 candidates in
total.  One step filters 2^24 tiles (1.22e12 candidates) and proves every
survivor (BPSW, backward + forward walk).  Candidates are admissible lattice
points, the reference's own unit (tiles x candidates per tile).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank sweeps its own lane of tiles (weak scaling); the
timed region is bracketed by a barrier and synchronize on both sides and the
reported time is the max over ranks.  `--impl reference` times the
reference's own CPU engine (cc_gmp_v33 built from the reference sources into
oracle/_ref) on this host's cores over a bounded sample of the same lattice.
"""
import argparse
import importlib
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "candidates/s filtered + MR proofs/s on 1 B200, served vs plain; p50/p99 latency"
WORKLOAD = ("cc16-scale GPU filter: W=31#, depth 16, stage primes 37..2^10/2^10..2^14/2^14..2^17 "
            "at positions 0..15, 88-bit roots, 1e13 candidates (8 steps of 2^24 tiles)")
SEED = 20261203
TILES_PER_STEP = 1 << 24
BITS = 88


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_model():
    """lscpu model name of this host (the CPU baselines' hardware)."""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        m = re.search(r"Model name:\s*(.+)", out)
        return m.group(1).strip() if m else None
    except (OSError, subprocess.SubprocessError):
        return None


def v33_sample(bits, target, seconds_goal=15.0):
    """Runs the reference CPU engine (sieve only) on a sequential prefix range
    sized for about seconds_goal on this host.  Returns the parsed figures."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cc_gmp_v33")
    if not os.path.exists(exe):
        return None
    cores = os.cpu_count() or 1
    # v33 sieve-only runs ~50M candidates/s per core at depth 16-18
    want = max(2e8, 5e7 * cores * seconds_goal)
    tiles = want / 73008.0
    span = tiles * 20677 * 1616615                     # n-range covered by the tiles
    pbits = max(2, int(round(bits - (span.bit_length() if isinstance(span, int) else
                                     __import__("math").log2(span)))))
    prefix = "0b1" + format(SEED & ((1 << (pbits - 1)) - 1), f"0{pbits - 1}b")
    t0 = time.time()
    r = subprocess.run([exe, "--sieve-only", "--prefix", prefix, "--sequential", "--bits", str(bits),
                        "--target", str(target), "--threads", str(cores)],
                       capture_output=True, text=True, timeout=600)
    wall = time.time() - t0
    out = r.stdout
    wc = int(re.search(r"Wheel candidates \(L1\):\s+(\d+)", out).group(1))
    secs = float(re.search(r"Time: ([\d.]+) seconds", out).group(1))
    return {"candidates": wc, "seconds": secs, "wall": wall, "cores": cores, "prefix": prefix,
            "rate": wc / max(secs, 1e-9)}


def reference_qiter(segs_per_step=32):
    """The reference's own v16_q_iter_kernel (through oracle/_ref/libref16.so,
    launched as its dispatch loop launches it) on the first 32 chunks of the
    q-iteration section's first timed step; its sieve on the GPU is 7..503
    (the 509..1009 primes run on its CPU prove workers)."""
    import ctypes as C
    import importlib
    import numpy as np
    path = os.path.join(ROOT, "oracle", "_ref", "libref16.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libref16.so not built"}
    lib = C.CDLL(path)
    u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
    lib.ref16_qiter_time.restype = C.c_float
    lib.ref16_qiter_time.argtypes = [u32p, C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_int, C.c_int,
                                     C.c_ulonglong, C.c_ulonglong, C.c_uint, C.c_int, C.POINTER(C.c_uint)]
    ccs = importlib.import_module("cunningham-chain-search_b200")

    class _Plan(ccs.QIter):                   # windows and chunk draws only, no device state
        def __init__(self, pool):
            self.dv, self.exp_start = [p[1] for p in pool], 0

    pool = ccs.synthetic_pool(QITER_CFG["pool"], SEED + 61)
    segs = qiter_plan(ccs, _Plan(pool), 2, 256)[1][:segs_per_step]
    primes = np.asarray(ccs.qiter_sieve_primes(ext=False), dtype=np.uint32)
    ms = 0.0
    n = 0
    reps = 4
    for qb, nq, v in segs:
        D = pool[v][1]
        c = C.c_uint(0)
        ms += lib.ref16_qiter_time(primes, len(primes), D & (2**64 - 1), D >> 64, 0, QITER_CFG["depth"],
                                   qb & (2**64 - 1), qb >> 64, nq, reps, C.byref(c))
        n += reps * nq
    return {"qv_per_s_filter": n / (ms * 1e-3), "ms": ms, "chunks": len(segs), "reps": reps,
            "sieve": "7..503 on the GPU (its kernel's list)", "unit": "(Q, variant) pairs/s"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    s = v33_sample(BITS, 16)
    if s is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cc_gmp_v33 not built"}))
        return 0
    rates = [s["rate"]]
    for _ in range(max(0, min(args.steps, 2) - 1)):
        rates.append(v33_sample(BITS, 16)["rate"])
    v = statistics.median(rates)
    sample = (f"cc_gmp_v33 --sieve-only --sequential --prefix {s['prefix']} --bits {BITS} --target 16 "
              f"--threads {s['cores']}: {s['candidates']} candidates in {s['seconds']:.1f} s "
              f"(its own stage primes 37..863 on the same W=31# depth-16 lattice)")
    line = {"metric": METRIC, "value": v, "unit": "candidates/s", "impl": "reference",
            "n_gpus": ws, "steps": len(rates), "warmup": 0, "ms_per_step": 1e3 * s["seconds"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "bits": BITS, "target": 16},
            "cpu_baseline": {"value": v, "unit": "candidates/s", "cores": s["cores"],
                             "cpu_model": cpu_model(), "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "candidates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if not args.headline_only:
        try:
            line["qiter_reference_kernel"] = reference_qiter()
        except Exception as ex:
            line["qiter_reference_kernel"] = {"error": repr(ex)}
    print(json.dumps(line))
    return 0


def _gmp_walk_worker(hexes):
    """Reference GMP chain walk (v13:1870-1881 via oracle/_ref) on a list of
    hex numbers; runs in a spawned process."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref33.so"))
    lib.ref_gmp_forward_chain.argtypes = [ctypes.c_char_p]
    return [lib.ref_gmp_forward_chain(h.encode()) for h in hexes]


def gmp_walk_baseline(roots, seconds_goal=10.0):
    """Proofs/s of the reference GMP prover walk on all host cores over a
    bounded sample (the first n) of the prove-batch roots.  Returns the
    baseline dict and the GMP chain lengths of the sample, in order."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref33.so")):
        return None, None
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    hexes = [format(int(n), "x") for n in roots]
    # calibrate on one core
    t0 = time.time()
    _gmp_walk_worker(hexes[:200])
    per = (time.time() - t0) / 200
    n = int(min(len(hexes), max(cores * 200, seconds_goal * cores / max(per, 1e-7))))
    step = -(-n // cores)
    chunks = [hexes[i:min(n, i + step)] for i in range(0, n, step)]
    with ctx.Pool(cores) as pool:
        t0 = time.time()
        res = pool.map(_gmp_walk_worker, chunks)
        dt = time.time() - t0
    lengths = [x for part in res for x in part]
    return ({"value": n / dt, "unit": "roots/s", "cores": cores, "kind": "reference",
             "cpu_model": cpu_model(),
             "sample": f"{n} prove-batch roots walked with GMP mpz_probab_prime_p(.,1) "
                       f"(the reference CPU prover's walk, v13:1870-1881) in {dt:.1f} s"},
            lengths)


def section_prove(ccs, torch, eng, dev, local, n_unique=65536, copies=256, cpu=True):
    """Prove batch: 2^24 roots of 80..110 bits pre-filtered by every prime
    < 2^17 at chain positions 0..15 (survivors of the cc16 filter at seeded
    widths), walked p -> 2p+1 until the first composite (BPSW)."""
    import random
    r = random.Random(SEED + 3)
    info = eng.info
    bases = eng.bases()
    M, WP = info["lattice_m"], info["wheel_period"]
    roots = []
    t_gen = time.time()
    out = torch.empty((1 << 20, 4), dtype=torch.int32, device=dev)
    while len(roots) < n_unique:
        bits = r.randint(80, 110)
        t0, t1 = ccs.bit_tile_range(bits, bases, M, WP)
        ts = r.randint(t0, t1 - (1 << 22) - 1)
        surv = eng.filter_range(ts, 1 << 22, out=out).cpu().numpy().astype("int64") & 0xFFFFFFFF
        for b, k, t, _ in surv:
            n = ((ts + int(t)) * WP + int(k)) * M + bases[int(b)]
            if n.bit_length() == bits:
                roots.append(n)
    roots = roots[:n_unique]
    t_gen = time.time() - t_gen
    import numpy as np
    arr = np.zeros((n_unique, 4), dtype=np.uint32)
    for i, v in enumerate(roots):
        for w in range(4):
            arr[i, w] = (v >> (32 * w)) & 0xFFFFFFFF
    uniq = torch.from_numpy(arr.view(np.int32)).to(dev)
    nums = uniq.repeat(copies, 1).contiguous()
    total = nums.shape[0]
    lengths = torch.zeros(total, dtype=torch.int32, device=dev)
    # warm-up over the whole batch: the walk's work lists (32 bytes per
    # number in each of four lists) are reserved here, outside the timing
    eng.walk_numbers_dev(nums, 4, lengths)
    torch.cuda.synchronize()
    eng.walk_word_products(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    eng.walk_numbers_dev(nums, 4, lengths)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    mm, words = eng.walk_word_products(reset=True)
    L = lengths[:n_unique].cpu().numpy()
    tests = int(((L + 1).clip(max=64)).sum()) * copies           # numbers tested
    primes = int(L.sum()) * copies
    imad = ccs.measure_imad_peak(local)
    # IMAD ops: one lo/hi pair per 32x32-bit word product, counted on the device
    ops_per_mm = 2.0 * words / max(mm, 1)
    achieved = 2.0 * words / (ms * 1e-3) / 1e12
    cpu, gmp_len = gmp_walk_baseline(roots[:20000]) if cpu else (None, None)
    walk_mm = None
    if gmp_len is not None:
        walk_mm = {"compared": len(gmp_len),
                   "mismatches": int(sum(int(a) != int(b) for a, b in zip(L[:len(gmp_len)], gmp_len)))}
    return {"workload": f"{total} roots (= {copies} x {n_unique} distinct), 80..110-bit, pre-filtered "
                        "by all primes < 2^17 at positions 0..15, BPSW walk",
            "roots_per_s": total / (ms * 1e-3), "primality_tests_per_s": tests / (ms * 1e-3),
            "prime_verdicts_per_s": primes / (ms * 1e-3), "modmuls_per_s": mm / (ms * 1e-3),
            "ms": ms, "mean_chain_len": float(L.mean()), "max_chain_len": int(L.max()),
            "root_generation_s": t_gen,
            "roofline": {"bound": "imad", "achieved": achieved, "peak": imad, "unit": "TOPS",
                         "frac": achieved / imad,
                         "work": f"{ops_per_mm:.1f} IMAD ops per Montgomery product (2 per word product, "
                                 "2NL^2+NL word products per CIOS product)",
                         "peak_source": "measured: ccs_measure_imad_peak"},
            "cpu_baseline": cpu, "walk_vs_gmp": walk_mm}


def autotune_engines(ccs, engines, seed, probe_log2=34):
    """Project autotuner on every depth profile (before any batch holds the
    engines): a probe of 2^probe_log2 candidates, the longest range of the
    mixed workloads, at a seeded 88-bit start; the lattice threshold is
    searched on its prefixes down to 1/64 of it."""
    import random
    r = random.Random(seed)
    out = []
    t0 = time.time()
    for e in engines:
        info = e.info
        nt = max(1024, (1 << probe_log2) // info["candidates_per_tile"])
        lo, hi = ccs.bit_tile_range(88, e.bases(), info["lattice_m"], info["wheel_period"])
        chosen, pts = e.autotune(r.randint(lo, hi - nt - 1), nt)
        out.append({"depth": info["depth"], "chosen": chosen, "points": len(pts)})
    return {"seconds": time.time() - t0, "engines": out}


def _ref_gpu_lib(name):
    """The reference's own engine harness (built from its sources into
    oracle/_ref by oracle/Makefile) with its batch timer bound, or None."""
    import ctypes as C
    path = os.path.join(ROOT, "oracle", "_ref", f"lib{name}.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    fn = getattr(lib, f"{name}_time_batches")
    fn.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_uint, C.c_int, C.c_int, C.c_int,
                   C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_ulonglong)]
    return lib


def reference_gpu_batches(name, target, depth, plan, tiles, batch_tiles, blocks_per_sm, prove_forward):
    """The reference's cc18_filter_kernel (K1) and cc18_prove_kernel (K2) on
    the same tiles, launched as its main loop launches them: batches of
    batch_tiles (its --batch), SMs x blocks_per_sm blocks of 256 (its
    --blocks-per-sm), K2 over the fixed 2^20-survivor grid; device time of
    each kernel from CUDA events."""
    import ctypes as C
    lib = _ref_gpu_lib(name)
    if lib is None:
        return None
    getattr(lib, f"{name}_setup")(target, depth)
    if name == "ref15":
        lib.ref15_upload(depth, plan[0][0], target, prove_forward)
    else:
        lib.ref13_upload(depth, plan[0][0])
    set_bits = getattr(lib, f"{name}_set_bits")
    timer = getattr(lib, f"{name}_time_batches")
    k1 = k2 = 0.0
    tot = [0, 0, 0]
    nb = tiles // batch_tiles
    for i, (bits, ts) in enumerate(plan):
        set_bits(bits)
        a, b = C.c_float(0), C.c_float(0)
        cnt = (C.c_ulonglong * 3)()
        timer(ts & (2**64 - 1), ts >> 64, batch_tiles, 1 if i == 0 else nb, blocks_per_sm, 1,
              C.byref(a), C.byref(b), cnt)
        if i == 0:
            continue                                   # warm-up batch
        k1 += a.value
        k2 += b.value
        for j in range(3):
            tot[j] += cnt[j]
    return {"k1_ms": k1, "k2_ms": k2, "survivors": tot[0], "chains": tot[1], "primes": tot[2],
            "batch_tiles": batch_tiles, "blocks_per_sm": blocks_per_sm}


def section_reference_runs(ccs, torch, dev, local, tiles=1 << 22, steps=4):
    """The reference's own GPU run configurations, on this engine and on the
    reference's own kernels over the same tiles: v13 defaults (target =
    depth = 18, 89-bit roots, K2 roots-only prove with the v13 witnesses,
    12 blocks/SM) and the v15 CC19 configuration (target = depth = 19, 88-107
    bit shells, reverse prove order, --batch 524288, 16 blocks/SM); filter +
    prove per 2^22 tiles, device-timed.  Survivor, chain and prime counts of
    the two engines are compared tile for tile."""
    import random
    out = {}
    for name, ref, kw, bits_list, ref_bps in [
            ("v13_defaults_cc18", "ref13", dict(target=18, bits=89), [89], 12),
            ("v15_cc19_reverse", "ref15", dict(target=19, depth=19, reverse_prove=True),
             list(range(88, 108)), 16)]:
        eng = ccs.Engine(device=local, primality=ccs.PRIME_MR, prove_mode=ccs.PROVE_ROOTS, **kw)
        info = eng.info
        bases = eng.bases()
        r = random.Random(SEED + 41)
        stream = torch.cuda.Stream(device=dev)
        surv = torch.empty((1 << 22, 4), dtype=torch.int32, device=dev)
        chains = torch.empty((1 << 18, 12), dtype=torch.int32, device=dev)
        plan = []
        for i in range(steps + 1):
            bits = bits_list[i % len(bits_list)]
            lo, hi = ccs.bit_tile_range(bits, bases, info["lattice_m"], info["wheel_period"])
            plan.append((bits, r.randint(lo, hi - tiles - 1)))
        ms = f_ms = 0.0
        n_s = n_c = n_p = 0
        for i, (bits, ts) in enumerate(plan):
            eng.set_bits(bits)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            torch.cuda.synchronize()
            e0.record(stream)
            s_ = eng.filter_range(ts, tiles, out=surv, stream=stream)
            e1.record(stream)
            c_, p_ = eng.prove(s_, ts, out=chains, stream=stream)
            e2.record(stream)
            torch.cuda.synchronize()
            if i == 0:
                continue                                   # warm-up batch
            ms += e0.elapsed_time(e2)
            f_ms += e0.elapsed_time(e1)
            n_s += s_.shape[0]
            n_c += c_.shape[0]
            n_p += p_
        eng.close()
        cand = steps * tiles * info["candidates_per_tile"]
        res = {"candidates_per_s": cand / (ms * 1e-3), "filter_candidates_per_s": cand / (f_ms * 1e-3),
               "survivors": n_s, "chains": n_c, "primes": n_p, "ms": ms, "filter_ms": f_ms,
               "tiles_per_batch": tiles, "batches": steps,
               "candidates_per_tile": info["candidates_per_tile"]}
        try:
            rg = reference_gpu_batches(ref, kw["target"], kw.get("depth", kw["target"]), plan, tiles,
                                       524288, ref_bps, 0 if kw.get("reverse_prove") else 1)
        except Exception as ex:
            rg = {"error": repr(ex)}
        if rg and "k1_ms" in rg:
            rg["k1_candidates_per_s"] = cand / (rg["k1_ms"] * 1e-3)
            rg["k1k2_candidates_per_s"] = cand / ((rg["k1_ms"] + rg["k2_ms"]) * 1e-3)
            rg["ours_over_ref_k1"] = res["filter_candidates_per_s"] / rg["k1_candidates_per_s"]
            rg["ours_over_ref_k1k2"] = res["candidates_per_s"] / rg["k1k2_candidates_per_s"]
            rg["count_mismatches"] = {"survivors": abs(rg["survivors"] - n_s),
                                      "chains": abs(rg["chains"] - n_c),
                                      "primes": abs(rg["primes"] - n_p)}
        res["reference_kernels"] = rg
        out[name] = res
    return out


QITER_CFG = dict(target=21, depth=21, bits_min=90, bits_max=107, chunk=1 << 24, pool=4248)


def qiter_plan(ccs, qi, steps, segs_per_step):
    return [qi.random_segments(segs_per_step, QITER_CFG["chunk"], QITER_CFG["bits_min"],
                               QITER_CFG["bits_max"], seed=SEED + 71 + i, start_variant=i * segs_per_step)
            for i in range(steps)]


def v33_prefix_range(bits, prefix_value, prefix_bits, bases, M, WP):
    """The candidates cc_gmp_v33 --prefix P --sequential --bits B visits
    (v33:2994-3061, 1783-1793, 2108-2114): k = tile WP + k_offset in
    [k_min, k_max) and n in [n_min, n_max], over the tiles [t0, t1)."""
    shift = bits - prefix_bits
    n_min = max(prefix_value << shift, 1 << (bits - 1))
    n_max = min(((prefix_value + 1) << shift) - 1, (1 << bits) - 1)
    k_min = -(-(n_min - max(bases)) // M) if n_min > max(bases) else 0
    k_max = (n_max - min(bases)) // M
    return k_min // WP, -(-k_max // WP), k_min, k_max, n_min, n_max


def v33_prove_run(bits, target, prefix_bits, seed, threads, log_threshold=6):
    """cc_gmp_v33 (the reference CPU engine, filter + prove) on a sequential
    prefix range; returns its figures and its chain lines as (len, root,
    is_root)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cc_gmp_v33")
    if not os.path.exists(exe):
        return None
    pv = (1 << (prefix_bits - 1)) | (seed & ((1 << (prefix_bits - 1)) - 1))
    prefix = "0b" + format(pv, "b")
    r = subprocess.run([exe, "--prefix", prefix, "--sequential", "--bits", str(bits), "--target", str(target),
                        "--line-depth", str(target - 1), "--log", str(log_threshold), "--threads", str(threads)],
                       capture_output=True, text=True, timeout=900)
    out = r.stdout
    lines = [(int(m.group(1)), int(m.group(2), 16), True)
             for m in re.finditer(r"\*\*\* CC(\d+)a FOUND! 0x([0-9a-fA-F]+)", out)]
    lines += [(int(m.group(1)), int(m.group(2), 16), False)
              for m in re.finditer(r"\[NON-ROOT\] CC(\d+)a elem, root: 0x([0-9a-fA-F]+)", out)]
    return {"prefix": prefix, "prefix_value": pv, "prefix_bits": prefix_bits,
            "candidates": int(re.search(r"Wheel candidates \(L1\):\s+(\d+)", out).group(1)),
            "primes": int(re.search(r"Primes found:\s+(\d+)", out).group(1)),
            "seconds": float(re.search(r"Time: ([\d.]+) seconds", out).group(1)),
            "lines": sorted(lines)}


def section_cpu_method(ccs, torch, dev, local, seconds_goal=8.0):
    """BASELINE's CPU-method configuration and the reference CPU engine
    beside it.

    GPU: lattice W = 23#, depth 8, filter primes 29..1021 at positions 0..7,
    a seed-drawn 60-bit block offset (88-bit n), 1e9 candidates; every
    survivor proved with the reference CPU engine's own tests
    (CCS_PRIME_V33, full prove: true roots and lengths), chains >= 6
    counted.  CPU: cc_gmp_v33 --target 8 --line-depth 7 --log 6 on all host
    cores over a sequential prefix range of 61-bit n, sized for about
    seconds_goal, on its own lattice (W = 31#, stages 37..61 / 67..97 /
    101..863); the engine then runs the same lattice, stages, tests and
    range, and its prime count and chain lines (>= 6) are compared with the
    reference's output."""
    import random
    import numpy as np
    cores = os.cpu_count() or 1
    r = random.Random(SEED + 81)
    # ---- GPU, config 1 ----
    cfg = ccs.config_cpu_method()
    probe = ccs.Engine(device=local, **cfg)
    info = probe.info
    cpt = info["candidates_per_tile"]
    probe.close()
    j0 = r.getrandbits(59) | (1 << 59)                 # 60-bit block offset
    ts = 6 * j0
    tiles = -(-10**9 // cpt)
    n0 = ts * info["wheel_period"] * info["lattice_m"]
    bits = n0.bit_length()
    cfg["bits"] = bits
    eng = ccs.Engine(device=local, primality=ccs.PRIME_V33, prove_mode=ccs.PROVE_FULL, **cfg)
    stream = torch.cuda.Stream(device=dev)
    surv = torch.empty((1 << 23, 4), dtype=torch.int32, device=dev)
    chains = torch.empty((1 << 22, 12), dtype=torch.int32, device=dev)
    best = None
    for rep in range(3):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(stream)
        s_ = eng.filter_range(ts, tiles, out=surv, stream=stream)
        e1.record(stream)
        c_, p_ = eng.prove(s_, ts, out=chains, stream=stream)
        e2.record(stream)
        torch.cuda.synchronize()
        t = (e0.elapsed_time(e2), e0.elapsed_time(e1), s_.shape[0], c_.shape[0], p_)
        if rep > 0 and (best is None or t[0] < best[0]):
            best = t
    lens = chains[:best[3]].cpu().numpy()[:, 3] if best[3] else np.zeros(0)
    eng.close()
    cand = tiles * cpt
    gpu = {"workload": f"W = 23#, depth 8, primes 29..1021 at positions 0..7, {bits}-bit n from a "
                       f"seed-drawn 60-bit block offset, {cand} candidates",
           "candidates_per_s": cand / (best[0] * 1e-3), "filter_candidates_per_s": cand / (best[1] * 1e-3),
           "ms": best[0], "survivors": best[2], "primes": best[4],
           "proofs_per_s": best[4] / (best[0] * 1e-3),
           "chains_ge6": int((lens >= 6).sum()), "predicate": "CCS_PRIME_V33 (the reference CPU engine's)"}
    # ---- reference CPU engine, and the engine on its range ----
    out = {"gpu_config1": gpu}
    ref_bits, target = 61, 8
    e_ref = ccs.Engine(device=local, target=target, depth=target, bits=ref_bits,
                       stages=ccs.reference_cpu_stages(), primality=ccs.PRIME_V33,
                       prove_mode=ccs.PROVE_FULL)
    rinfo = e_ref.info
    bases = e_ref.bases()
    M, WP = rinfo["lattice_m"], rinfo["wheel_period"]
    # about 1.5e6 candidates per second per core at target 8 with its prove
    # (2.37e7 measured on 16 cores): size the range
    want = 1.5e6 * cores * seconds_goal
    pbits = 2
    while pbits < ref_bits - 1:
        t0_, t1_ = v33_prefix_range(ref_bits, 1 << (pbits - 1), pbits, bases, M, WP)[:2]
        if (t1_ - t0_) * rinfo["candidates_per_tile"] <= want:
            break
        pbits += 1
    ref = v33_prove_run(ref_bits, target, pbits, SEED + 83, cores)
    if ref is None:
        out["reference_cpu"] = {"unavailable": "oracle/_ref/cc_gmp_v33 not built"}
        e_ref.close()
        return out
    t0, t1, k_min, k_max, n_min, n_max = v33_prefix_range(ref_bits, ref["prefix_value"], ref["prefix_bits"],
                                                         bases, M, WP)
    n_t = t1 - t0
    s_ = e_ref.filter_range(t0, n_t, cap=1 << 26)
    c_, p_ = e_ref.prove(s_, t0, cap=1 << 24)
    e_ref.close()
    a = c_.cpu().numpy().astype(np.int64) & 0xFFFFFFFF
    ours, primes_in = [], 0
    for rec in a:
        k = (t0 + int(rec[2])) * WP + int(rec[1])
        n = k * M + bases[int(rec[0])]
        if not (k_min <= k < k_max and n_min <= n <= n_max):
            continue
        primes_in += 1
        if rec[3] >= 6:
            root = sum(int(rec[4 + w]) << (32 * w) for w in range(6))
            ours.append((int(rec[3]), root, bool(rec[10] & 1)))
    ours.sort()
    out["reference_cpu"] = {
        "value": ref["candidates"] / ref["seconds"], "unit": "candidates/s", "cores": cores,
        "cpu_model": cpu_model(), "kind": "reference",
        "sample": (f"cc_gmp_v33 --prefix {ref['prefix']} --sequential --bits {ref_bits} --target {target} "
                   f"--line-depth {target - 1} --log 6 --threads {cores}: {ref['candidates']} candidates, "
                   f"{ref['primes']} primes, {len(ref['lines'])} chain lines in {ref['seconds']:.1f} s"),
        "proofs_per_s": ref["primes"] / ref["seconds"]}
    out["parity_vs_reference_cpu"] = {
        "tiles": n_t, "engine_candidates": n_t * rinfo["candidates_per_tile"],
        "reference_candidates": ref["candidates"], "engine_primes": primes_in,
        "reference_primes": ref["primes"], "chain_lines_ge6": len(ref["lines"]),
        "chain_lines_equal": ours == ref["lines"],
        "lines_only_in_reference": len(set(ref["lines"]) - set(ours)),
        "lines_only_in_engine": len(set(ours) - set(ref["lines"]))}
    return out


def section_qiter(ccs, torch, dev, local, steps=8, segs_per_step=256):
    """Fingerprint-pool Q iteration as the reference's v16 production run
    (--immune-prime 5 --target 21 --depth 21 --sieve-max 503 --bits-min 90
    --bits-max 107 --q-order random, extended sieve 509..1009 on): a seeded
    4248-variant synthetic pool, 256 random 2^24-Q chunks per step
    round-robin over the variants, filter then prove, device-timed on one
    stream; e2e = QIter.run on host segment lists (packing beside the
    filter, proves of groups of steps beside later filters, HIT lines),
    timed on the host."""
    pool = ccs.synthetic_pool(QITER_CFG["pool"], SEED + 61)
    qi = ccs.QIter(pool, target=QITER_CFG["target"], depth=QITER_CFG["depth"], device=local)
    plan = [qi.pack(p) for p in qiter_plan(ccs, qi, steps + 1, segs_per_step)]
    stream = torch.cuda.Stream(device=dev)
    surv = torch.empty((1 << 22, 4), dtype=torch.int32, device=dev)
    chains = torch.empty((1 << 16, 12), dtype=torch.int32, device=dev)
    f_ms = p_ms = 0.0
    n_s = n_c = n_p = 0
    for i, segs in enumerate(plan):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        s_ = qi.filter(segs, out=surv, stream=stream)
        ev[1].record(stream)
        c_, p_ = qi.prove(segs, s_, out=chains, stream=stream)
        ev[2].record(stream)
        torch.cuda.synchronize()
        if i == 0:
            continue                                       # warm-up step
        f_ms += ev[0].elapsed_time(ev[1])
        p_ms += ev[1].elapsed_time(ev[2])
        n_s += s_.shape[0]
        n_c += c_.shape[0]
        n_p += p_
    qv = steps * segs_per_step * QITER_CFG["chunk"]
    raw = qiter_plan(ccs, qi, steps + 1, segs_per_step)
    qi.run(raw[:1], min_report_len=10)                     # warm-up: buffers, prove thread
    torch.cuda.synchronize()
    t0 = time.time()
    tot, hits = qi.run(raw[1:], min_report_len=10)
    e2e_s = time.time() - t0
    assert tot["survivors"] == n_s and tot["chains"] == n_c
    qi.close()
    return {"workload": f"{QITER_CFG['pool']}-variant seeded pool, target = depth = 21, sieve 7..1009, "
                        f"bits 90..107, {steps} steps x {segs_per_step} chunks of 2^24 Q",
            "qv_per_s_filter": qv / (f_ms * 1e-3), "qv_per_s_filter_prove": qv / ((f_ms + p_ms) * 1e-3),
            "qv_per_s_e2e": qv / e2e_s, "filter_ms": f_ms, "prove_ms": p_ms, "survivors": n_s,
            "chains": n_c, "primes": n_p, "hit_lines_len10": len(hits),
            "unit": "(Q, variant) pairs/s, the reference's G(Q,V)/s x 1e9"}


def record_set(rec, words):
    """Sorted tuples of the first `words` 32-bit words of survivor (16-byte)
    or chain (48-byte) records: a numpy structured array, an int32 tensor or
    an ndarray.  Survivors compare on 3 words (base, k, tile), chains on 11
    (ChainResult words, root limbs, flags; not the survivor index)."""
    import numpy as np
    if hasattr(rec, "cpu"):
        rec = rec.cpu().numpy()
    a = np.ascontiguousarray(rec)
    if len(a) == 0:
        return []
    a = a.view(np.uint32).reshape(len(a), -1)[:, :words].astype(np.int64)
    return sorted(map(tuple, a.tolist()))


def batched_rerun(ccs, eng, starts, sets, tiles, bits):
    """Re-runs ranges already filtered and proved by the plain path through
    one ccs_batch_run and counts the ranges whose survivor set, chain set or
    prime count differ."""
    import numpy as np
    batch = ccs.Batch([eng], len(starts), surv_cap=1 << 21, chain_cap=1 << 18)
    try:
        res, bs, bc = batch.run([(t, tiles, 0, bits) for t in starts])
    finally:
        batch.close()
    rid = bs["_pad"].astype(np.int64)
    crid = rid[bc["survivor"].astype(np.int64)] if len(bc) else np.zeros(0, dtype=np.int64)
    bad = 0
    for i, (sv, ch, p) in enumerate(sets):
        same = (record_set(bs[rid == i], 3) == record_set(sv, 3)
                and record_set(bc[crid == i], 11) == record_set(ch, 11)
                and res[i]["n_primes"] == p)
        bad += not same
    return {"ranges": len(starts), "tiles_per_range": tiles,
            "survivors": int(sum(r["n_survivors"] for r in res)),
            "chains": int(sum(r["n_chains"] for r in res)),
            "ranges_differing": int(bad)}


def section_batched(ccs, engines, n_ranges=4096):
    """Uneven ranges: one batched graph replay versus per-range plain calls."""
    ranges = ccs.mixed_ranges(engines, n_ranges, SEED + 11)
    batch = ccs.Batch(engines, n_ranges, surv_cap=1 << 22, chain_cap=1 << 20)
    # batch autotuner on a separately drawn sample of the same distribution
    t_tune = time.time()
    chosen, pts = batch.autotune(ccs.mixed_ranges(engines, min(512, n_ranges), SEED + 13))
    tune = {"chosen": chosen, "points": len(pts), "seconds": time.time() - t_tune}
    batch.run(ranges[:32], want_records=False)
    t0 = time.time()
    res, surv, ch = batch.run(ranges)
    tb = time.time() - t0
    dev_ms = batch.last_ms()
    cand = sum(x["candidates"] for x in res)
    nsurv = sum(x["n_survivors"] for x in res)
    nprimes = sum(x["n_primes"] for x in res)
    batch.close()
    t0 = time.time()
    psurv = pprimes = 0
    for ts, nt, p, bits in ranges:
        e = engines[p]
        e.set_bits(bits)
        s = e.filter_range(ts, nt, cap=1 << 20)
        c, pr = e.prove(s, ts)
        psurv += s.shape[0]
        pprimes += pr
    tp = time.time() - t0
    return {"workload": f"{n_ranges} ranges, log-uniform 2^20..2^34 candidates, depth 14..19, "
                        "width 64..110 bits",
            "candidates": cand, "batched_candidates_per_s": cand / tb,
            "batched_device_ms": dev_ms, "plain_candidates_per_s": cand / tp,
            "speedup": tp / tb, "survivors": nsurv, "plain_survivors": psurv,
            "primes": nprimes, "plain_primes": pprimes,
            "batched_proofs_per_s": nprimes / tb, "plain_proofs_per_s": pprimes / tp,
            "batch_autotune": tune}, chosen


def section_served(ccs, engines, n_req=2048, lam=2000.0, batch_tuning=None):
    """Poisson arrivals of uneven range requests: continuous-batching server
    versus a plain first-come-first-served loop; p50/p99 request latency."""
    import random
    import numpy as np
    ranges = ccs.mixed_ranges(engines, n_req, SEED + 23)
    rr = random.Random(SEED + 29)
    arr = []
    t = 0.0
    for _ in range(n_req):
        t += rr.expovariate(lam)
        arr.append(t)
    cand_total = 0

    # served
    srv = ccs.Server(engines, max_active=256, chunk_tiles=1 << 19, mem_cap_bytes=120 << 30)
    if batch_tuning:
        srv.set_batch_tuning(**batch_tuning)
    ids = [None] * n_req
    base = time.monotonic() + 0.05

    def submitter():
        for i, (ts, nt, p, bits) in enumerate(ranges):
            d = base + arr[i] - time.monotonic()
            if d > 0:
                time.sleep(d)
            ids[i] = srv.submit(ts, nt, p, bits)
    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    # backlog when the last request arrived: queued (not admitted) requests
    # and admitted ones not yet done
    st_last = srv.stats()
    backlog = {"pending": st_last["pending"],
               "admitted_not_done": st_last["admitted"] - st_last["completed"] - st_last["cancelled"]}
    lat = []
    waits = []
    first, last = 1e30, 0
    served_sets = []
    for rid in ids:
        srv.wait(rid)
        st, res, sv, ch = srv.poll(rid, surv_cap=1 << 16, chain_cap=1 << 14)
        served_sets.append((record_set(sv, 3), record_set(ch, 11)))
        lat.append(res["done_s"] - res["submit_s"])
        waits.append(res["admit_s"] - res["submit_s"])
        first = min(first, res["submit_s"])
        last = max(last, res["done_s"])
        cand_total += res["candidates"]
    stats = srv.stats()
    mem_now, mem_peak = srv.memory()
    srv.close()
    served = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
              "admission_wait_p50_s": float(np.percentile(waits, 50)),
              "admission_wait_p99_s": float(np.percentile(waits, 99)),
              "candidates_per_s": cand_total / (last - first), "makespan_s": last - first,
              "ticks": stats["ticks"], "backlog_at_last_arrival": backlog,
              "device_bytes_reserved_peak": mem_peak}

    # plain: one request at a time in arrival order
    lat_p = []
    plain_sets = []
    base = time.monotonic() + 0.05
    t_first = base + arr[0]
    for i, (ts, nt, p, bits) in enumerate(ranges):
        d = base + arr[i] - time.monotonic()
        if d > 0:
            time.sleep(d)
        e = engines[p]
        e.set_bits(bits)
        s = e.filter_range(ts, nt, cap=1 << 20)
        c, _ = e.prove(s, ts, cap=1 << 14)
        lat_p.append(time.monotonic() - (base + arr[i]))
        plain_sets.append((s.cpu(), c.cpu()))
    t_last = time.monotonic()
    mism = sum(served_sets[i] != (record_set(a, 3), record_set(b, 11))
               for i, (a, b) in enumerate(plain_sets))
    plain = {"p50_s": float(np.percentile(lat_p, 50)), "p99_s": float(np.percentile(lat_p, 99)),
             "candidates_per_s": cand_total / (t_last - t_first), "makespan_s": t_last - t_first}
    return {"workload": f"{n_req} requests, Poisson arrivals {lam:.0f}/s, log-uniform 2^20..2^34 "
                        "candidates, depth 14..19, width 64..110 bits, admission cap 120 GB",
            "offered_candidates_per_s": cand_total / arr[-1], "served": served, "plain": plain,
            "requests_differing_from_plain": int(mism)}


SWEEP_PROFILE = os.path.join(ROOT, "profiles", "sweep_kernel_cc16_4M_tiles.md")


def profile_figures(path):
    """Per-unit figures of an ncu summary under profiles/: the line starting
    with `bench-figures:` holds a JSON object."""
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("bench-figures:"):
                    return json.loads(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def sweep_roofline(ccs, device, plan, candidates, ms, clk, int_peak, ref_ops_per_candidate):
    """Roofline of the dominant kernel (sweep_kernel) for one headline launch.

    The kernel is bound by instruction issue: every SM sub-partition issues
    at most one warp instruction per cycle, so the peak is SMs x 4 x the SM
    clock sampled during the timed region.  Achieved = warp instructions of
    the launch / its CUDA-event duration, with warp instructions per
    candidate from the ncu summary of the same kernel and profile
    (smsp__inst_executed.sum on a smaller launch of the current code).
    traffic = that summary's DRAM bytes per work unit x the launch's units.
    The reference's per-candidate test costs 4 x E[tests] INT32 operations;
    candidates/s x that over the measured INT32 peak is reported separately
    as the algorithmic gain over the reference's test, not as a roofline."""
    import torch
    fig = profile_figures(SWEEP_PROFILE) or {}
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz")
    out = {"bound": "issue", "unit": "warp instructions/s",
           "kernel": "sweep_kernel", "launch_ms": ms, "candidates_per_launch": candidates,
           "plan": plan, "peak_source": f"{sms} SMs x 4 issue slots x median sampled SM clock "
                                        f"({mhz} MHz)",
           "figures_source": os.path.relpath(SWEEP_PROFILE, ROOT)}
    ipc = fig.get("warp_inst_per_candidate")
    if mhz and ipc:
        peak = sms * 4 * mhz * 1e6
        ach = ipc * candidates / (ms * 1e-3)
        out.update({"achieved": ach, "peak": peak, "frac": ach / peak,
                    "warp_inst_per_candidate": ipc})
    else:
        out.update({"achieved": None, "peak": None, "frac": None})
    bpu = fig.get("dram_bytes_per_unit")
    out["traffic"] = bpu * plan["units"] if bpu else None
    out["algorithmic_gain_vs_reference_test"] = {
        "ops_per_candidate": ref_ops_per_candidate,
        "tops_equivalent": candidates * ref_ops_per_candidate / (ms * 1e-3) / 1e12,
        "int32_peak_tops": int_peak,
        "ratio": candidates * ref_ops_per_candidate / (ms * 1e-3) / 1e12 / int_peak,
        "note": "4 x E[tests] INT32 ops per candidate is the reference's per-candidate test; "
                "the bit-sliced sweep does far fewer operations per candidate"}
    return out


def run_ours(args):
    ws, rank, local = dist_env()
    import torch
    ccs = importlib.import_module("cunningham-chain-search_b200")
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    cfg = ccs.config_cc16_scale()
    eng = ccs.Engine(device=local, **cfg)
    TILES = args.tiles_per_step
    info = eng.info
    tune_report = None
    if not args.no_autotune:
        # project autotuner on a probe away from the timed tiles
        bases0 = eng.bases()
        lo0, hi0 = ccs.bit_tile_range(BITS, bases0, info["lattice_m"], info["wheel_period"])
        t_tune = time.time()
        # a probe as long as one step, so the unit length is tuned for it
        chosen, pts = eng.autotune(lo0 + 1000, TILES)
        tune_report = {"probe_tiles": TILES, "points": len(pts), "seconds": time.time() - t_tune}
    if args.unit_words:
        eng.set_tuning(unit_words=args.unit_words)
    if args.ext_min_words:
        eng.set_tuning(ext_min_words=args.ext_min_words)
    cpt = info["candidates_per_tile"]
    bases = eng.bases()
    t_lo, t_hi = ccs.bit_tile_range(BITS, bases, info["lattice_m"], info["wheel_period"])
    import random
    rnd = random.Random(SEED)
    total_tiles = (args.warmup + args.steps + 8) * TILES
    start = rnd.randint(t_lo, t_hi - total_tiles * max(ws, 1) - 1)
    lane0, _ = ccs.lane_range(start, start + total_tiles * ws, ws, rank)

    stream = torch.cuda.Stream(device=dev)
    surv_buf = torch.empty((1 << 20, 4), dtype=torch.int32, device=dev)
    chain_buf = torch.empty((1 << 16, 12), dtype=torch.int32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2

    def step(ts):
        surv = eng.filter_range(ts, TILES, out=surv_buf, stream=stream)
        chains, primes = eng.prove(surv, ts, out=chain_buf, stream=stream)
        return surv.shape[0], chains.shape[0], primes

    # warm-up
    ts = lane0
    for _ in range(args.warmup):
        step(ts)
        ts += TILES
    torch.cuda.synchronize()
    if pg:
        pg.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches0 = eng.launches()
    eng.prove_stats(reset=True)
    n_surv = n_chain = n_prime = 0
    torch.cuda.synchronize()
    t_wall = time.time()
    step_starts, step_sets = [], []
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()                      # L2 flush between timed steps (not timed)
        ev[i][0].record(stream)
        s, c, p = step(ts)
        ev[i][1].record(stream)
        n_surv += s
        n_chain += c
        n_prime += p
        # this step's records, kept for the batched re-run (after the events)
        step_starts.append(ts)
        step_sets.append((surv_buf[:s].cpu(), chain_buf[:c].cpu(), p))
        ts += TILES
    torch.cuda.synchronize()
    t_wall = time.time() - t_wall
    step_ms = [a.elapsed_time(b) for a, b in ev]
    launches = eng.launches() - launches0
    pstats = eng.prove_stats(reset=True)
    clk = clocks.stop()
    ms_total = sum(step_ms)
    if pg:
        t = torch.tensor([ms_total], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_total = float(t.item())
        pg.barrier()
    cand_step = TILES * cpt
    value = ws * args.steps * cand_step / (ms_total * 1e-3)

    # dominant kernel: time one filter launch alone on its stream
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    eng.filter_range(ts, TILES, out=surv_buf, stream=stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    filt_ms = ev0.elapsed_time(ev1)
    int_peak = ccs.measure_int32_peak(local)
    E = info["expected_tests"]
    plan = eng.plan_range(ts, TILES)
    roofline = sweep_roofline(ccs, local, plan, cand_step, filt_ms, clk, int_peak, 4.0 * E)

    # end to end through the host-buffer C-ABI call (copies inside), after
    # one untimed call that sizes the call's own device scratch
    e2e_steps = max(1, min(args.steps, 3))
    eng.search_range_host(ts, TILES, surv_cap=1 << 20, chain_cap=1 << 16)
    ts += TILES
    torch.cuda.synchronize()
    t0 = time.time()
    h2d = d2h = 0
    for _ in range(e2e_steps):
        surv, chains, primes = eng.search_range_host(ts, TILES, surv_cap=1 << 20,
                                                     chain_cap=1 << 16)
        h2d += 80 + 16 + 16 + 64                       # range, prefix, header, prove descriptors
        d2h += 16 * len(surv) + 48 * len(chains) + 16  # records + counters
        ts += TILES
    e2e_s = time.time() - t0
    e2e_value = ws * e2e_steps * cand_step / e2e_s

    # the timed tiles again through the batched executor (one persistent
    # launch over all steps' ranges): survivor and chain sets must be equal
    headline_mm = None
    if not args.headline_only:
        try:
            headline_mm = batched_rerun(ccs, eng, step_starts, step_sets, TILES, BITS)
        except Exception as ex:
            headline_mm = {"error": repr(ex)}

    # the CPU baseline and the sections after the headline run at N = 1 only:
    # a multi-GPU run reports the headline (the other ranks would wait in the
    # final barrier while rank 0 ran them)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        s = v33_sample(BITS, 16)
        if s:
            cpu = {"value": s["rate"], "unit": "candidates/s", "cores": s["cores"], "kind": "reference",
                   "cpu_model": cpu_model(),
                   "sample": (f"cc_gmp_v33 --sieve-only --sequential --prefix {s['prefix']} --bits {BITS} "
                              f"--target 16 --threads {s['cores']}: {s['candidates']} candidates in "
                              f"{s['seconds']:.1f} s (reference stage primes 37..863 on the same "
                              f"W=31# depth-16 lattice)")}
    extra = {}
    if rank == 0 and ws == 1 and not args.headline_only:
        try:
            extra["prove"] = section_prove(ccs, torch, eng, dev, local)
        except Exception as ex:                       # report, keep the headline
            extra["prove"] = {"error": repr(ex)}
        try:
            extra["reference_runs"] = section_reference_runs(ccs, torch, dev, local)
        except Exception as ex:
            extra["reference_runs"] = {"error": repr(ex)}
        try:
            extra["qiter"] = section_qiter(ccs, torch, dev, local)
        except Exception as ex:
            extra["qiter"] = {"error": repr(ex)}
        try:
            extra["cpu_method"] = section_cpu_method(ccs, torch, dev, local)
        except Exception as ex:
            extra["cpu_method"] = {"error": repr(ex)}
        depth_engines = [ccs.Engine(device=local, **ccs.config_depth_profile(d)) for d in range(14, 20)]
        if not args.no_autotune:
            try:
                extra["autotune_depth_profiles"] = autotune_engines(ccs, depth_engines, SEED + 5)
            except Exception as ex:
                extra["autotune_depth_profiles"] = {"error": repr(ex)}
        btune = None
        try:
            extra["batched"], btune = section_batched(ccs, depth_engines, args.batch_ranges)
        except Exception as ex:
            extra["batched"] = {"error": repr(ex)}
        try:
            extra["served"] = section_served(ccs, depth_engines, args.served_requests, batch_tuning=btune)
        except Exception as ex:
            extra["served"] = {"error": repr(ex)}
        for e in depth_engines:
            e.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "candidates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "tiles_per_step": TILES,
                       "candidates_per_step": cand_step, "bits": BITS, "seed": SEED,
                       "start_tile": start, "l2": "flushed (512 MB write) between timed steps",
                       "parallelism": f"lanes{ws}", "tuning": eng.tuning(), "autotune": tune_report},
            "survivors": n_surv, "chains": n_chain, "primes": n_prime,
            "survivor_rate": n_surv / (args.steps * cand_step),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "candidates/s", "h2d_bytes_per_step": h2d // e2e_steps,
                    "d2h_bytes_per_step": d2h // e2e_steps},
            "gpu_launches": launches,
            "prove_stats": pstats,
            "wall_s_timed": t_wall,
        }
        line.update(extra)
        mm = {"headline_batched": headline_mm}
        pv = extra.get("prove", {})
        mm["walk_vs_gmp"] = pv.get("walk_vs_gmp") if isinstance(pv, dict) else None
        sv = extra.get("served", {})
        mm["served_vs_plain"] = sv.get("requests_differing_from_plain") if isinstance(sv, dict) else None
        rr = extra.get("reference_runs", {})
        mm["reference_kernels"] = {k: (v.get("reference_kernels") or {}).get("count_mismatches")
                                   for k, v in rr.items() if isinstance(v, dict)} if isinstance(rr, dict) else None
        cm = extra.get("cpu_method", {})
        par = cm.get("parity_vs_reference_cpu") if isinstance(cm, dict) else None
        mm["cpu_method_vs_reference_cpu"] = (
            {"chain_lines": par["lines_only_in_reference"] + par["lines_only_in_engine"],
             "primes": abs(par["engine_primes"] - par["reference_primes"]),
             "candidates": abs(par["engine_candidates"] - par["reference_candidates"])} if par else None)
        line["mismatches"] = mm
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    eng.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tiles-per-step", type=int, default=TILES_PER_STEP,
                    help="tiles per step (smaller values: profiling cases)")
    ap.add_argument("--unit-words", type=int, default=0, help="sweep work-unit length (0: tuned)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the engine's default tuning")
    ap.add_argument("--ext-min-words", type=lambda v: int(v, 0), default=0,
                    help="extended-lattice threshold in 64-position words (0: engine default, "
                         "0xFFFFFFFF: plain lattice only)")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the prove-batch, batched and served sections")
    ap.add_argument("--batch-ranges", type=int, default=4096)
    ap.add_argument("--served-requests", type=int, default=2048)
    ap.add_argument("--only", choices=["qiter", "prove"], default=None,
                    help="run one section alone and print its JSON (profiling cases)")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warmup raised to 3")
        args.warmup = 3
    if args.only == "qiter":
        import importlib
        import torch
        ccs = importlib.import_module("cunningham-chain-search_b200")
        if args.impl == "reference":
            print(json.dumps(reference_qiter()))
        else:
            print(json.dumps(section_qiter(ccs, torch, torch.device("cuda:0"), 0, steps=args.steps)))
        return 0
    if args.only == "prove":
        import importlib
        import torch
        ccs = importlib.import_module("cunningham-chain-search_b200")
        eng = ccs.Engine(device=0, **ccs.config_cc16_scale())
        print(json.dumps(section_prove(ccs, torch, eng, torch.device("cuda:0"), 0, cpu=not args.no_cpu_baseline)))
        eng.close()
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
