"""Search campaign over the engine: the host side of the reference's main loop
(v13:3575-4151) -- pick the next batch of tiles (sequential or seeded random,
over a bit range, a binary prefix and a lane), filter and prove it on the
GPU, append the reference's output lines, and keep a resumable checkpoint.

Kept alike on purpose so campaigns can move between the two engines:
  * the checkpoint file is the reference's (v13:540-664): a version line
    "CC18_CUDA_v10" then key=value lines (bits, target, depth, coverage,
    prefix, prefix_lanes, prefix_lane_id, tile_hi/tile_lo in hex, totals,
    best_chain), written to "<path>.tmp" and renamed; loading rejects a file
    whose bits, target, depth, prefix or lane differ;
  * output lines are "[TARGET ][NON-ROOT ]CC<len> 0x<HEX> <bits>" for chains of
    at least the log threshold or the target (v13:1890, 2030-2033);
  * random mode draws batch starts with Marsaglia's xorshift64 (shifts 13, 7,
    17), the generator of the reference's rng_next (v13:707-722).

One difference: the reference mixes the clock into the generator between
batches so that GPUs started with the same seed diverge (v13:3737-3740).
Here a seeded campaign is reproducible, and GPUs are kept apart by giving
each its own lane.
"""
import os

from . import (bit_tile_range, format_chain_line, lane_range, parse_prefix, prefix_tile_range,
               chain_root_int)

CHECKPOINT_MARKER = "CC18_CUDA_v10"
_M64 = (1 << 64) - 1


class XorShift64:
    """Marsaglia xorshift64 with shifts (13, 7, 17); a zero seed becomes 1."""

    def __init__(self, seed):
        self.state = (seed & _M64) or 1

    def next(self):
        x = self.state
        x ^= (x << 13) & _M64
        x ^= x >> 7
        x ^= (x << 17) & _M64
        self.state = x
        return x

    def next128(self):
        hi = self.next()
        return (hi << 64) | self.next()


def checkpoint_save(path, bits, target, depth, tile, totals, prefix=None, lanes=0, lane_id=0):
    """Writes the checkpoint atomically (temporary file, then rename).
    totals: dict with tiles, primes, chains, best."""
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(CHECKPOINT_MARKER + "\n")
        f.write(f"bits={bits}\n")
        f.write(f"target={target}\n")
        f.write(f"depth={depth}\n")
        f.write("coverage=full\n")
        f.write(f"prefix={prefix if prefix else 'none'}\n")
        f.write(f"prefix_lanes={lanes}\n")
        f.write(f"prefix_lane_id={lane_id}\n")
        f.write(f"tile_hi={tile >> 64:016x}\n")
        f.write(f"tile_lo={tile & _M64:016x}\n")
        f.write(f"total_tiles={totals['tiles']}\n")
        f.write(f"total_primes={totals['primes']}\n")
        f.write(f"total_chains={totals['chains']}\n")
        f.write(f"best_chain={totals['best']}\n")
    os.replace(tmp, path)


def checkpoint_load(path, bits, target, depth, prefix=None, lanes=0, lane_id=0):
    """Reads a checkpoint and checks it belongs to this campaign; returns
    (tile, totals).  Raises ValueError on a foreign or malformed file."""
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    if not lines or not lines[0].startswith(CHECKPOINT_MARKER):
        raise ValueError("checkpoint file has wrong version marker")
    kv = {}
    for ln in lines[1:]:
        if "=" in ln:
            k, v = ln.split("=", 1)
            kv[k] = v
    want = {"bits": str(bits), "target": str(target), "depth": str(depth),
            "prefix": prefix if prefix else "none", "prefix_lanes": str(lanes),
            "prefix_lane_id": str(lane_id)}
    for k, v in want.items():
        if kv.get(k) != v:
            raise ValueError(f"checkpoint {k}={kv.get(k)} does not match current {v}")
    tile = (int(kv.get("tile_hi", "0"), 16) << 64) | int(kv.get("tile_lo", "0"), 16)
    totals = {"tiles": int(kv.get("total_tiles", 0)), "primes": int(kv.get("total_primes", 0)),
              "chains": int(kv.get("total_chains", 0)), "best": int(kv.get("best_chain", 0))}
    return tile, totals


class Campaign:
    """One search campaign on one engine.

    mode "sequential" walks the (prefix / lane) tile range from its start, or
    from `start`; mode "random" draws each batch start uniformly from the
    range with a seeded generator.  `run` returns the totals; output lines go
    to `out_path` (appended, like the reference's --output) and to
    `self.lines`."""

    def __init__(self, engine, bits=None, prefix=None, lanes=1, lane_id=0, mode="sequential",
                 seed=1, start=None, batch_tiles=1 << 20, log_threshold=8, out_path=None,
                 checkpoint_path=None, checkpoint_every=1, resume=False):
        if mode not in ("sequential", "random"):
            raise ValueError("mode must be 'sequential' or 'random'")
        self.eng = engine
        info = engine.info
        self.target, self.depth = info["target"], info["depth"]
        self.bits = bits or info["bits"]
        engine.set_bits(self.bits)
        bases = engine.bases()
        M, WP = info["lattice_m"], info["wheel_period"]
        if prefix:
            pv, pb = parse_prefix(prefix)
            t_lo, t_hi = prefix_tile_range(self.bits, pv, pb, bases, M, WP)
        else:
            t_lo, t_hi = bit_tile_range(self.bits, bases, M, WP)
        self.tile_min, self.tile_max = lane_range(t_lo, t_hi, lanes, lane_id) if lanes > 1 else (t_lo, t_hi)
        self.prefix, self.lanes, self.lane_id = prefix, lanes if lanes > 1 else 0, lane_id
        self.mode = mode
        self.rng = XorShift64(seed)
        self.batch_tiles = int(batch_tiles)
        self.log_threshold = log_threshold
        self.out_path = out_path
        self.ck_path = checkpoint_path
        self.ck_every = max(1, int(checkpoint_every))
        self.lines = []
        self.totals = {"tiles": 0, "primes": 0, "chains": 0, "best": 0}
        self.tile = self.tile_min if start is None else int(start)
        if resume and checkpoint_path and os.path.exists(checkpoint_path):
            self.tile, self.totals = checkpoint_load(checkpoint_path, self.bits, self.target, self.depth,
                                                     prefix, self.lanes, lane_id)

    def _save(self):
        if self.ck_path:
            checkpoint_save(self.ck_path, self.bits, self.target, self.depth, self.tile, self.totals,
                            self.prefix, self.lanes, self.lane_id)

    def next_batch(self):
        """(tile_start, n_tiles) of the next batch, or None when a sequential
        campaign has covered its range."""
        if self.mode == "random":
            span = self.tile_max - self.tile_min
            r = span - self.batch_tiles if span > self.batch_tiles else 1
            ts = self.tile_min + self.rng.next128() % r
        else:
            ts = self.tile
        n = min(self.batch_tiles, self.tile_max - ts)
        return (ts, n) if n > 0 else None

    def run(self, max_batches=None):
        done = 0
        out = open(self.out_path, "a") if self.out_path else None
        try:
            while max_batches is None or done < max_batches:
                nb = self.next_batch()
                if nb is None:
                    break
                ts, n = nb
                surv, chains, primes = self.eng.search_range_host(ts, n, surv_cap=1 << 22, chain_cap=1 << 18)
                batch_lines = []
                for rec in chains:
                    cl = int(rec["chain_len"])
                    self.totals["best"] = max(self.totals["best"], cl)
                    if cl >= self.log_threshold or cl >= self.target:
                        batch_lines.append(format_chain_line(cl, chain_root_int(rec), self.target,
                                                             bool(rec["flags"] & 1)))
                # records arrive in device order; a sorted batch makes the file reproducible
                batch_lines.sort()
                self.lines.extend(batch_lines)
                if out and batch_lines:
                    out.write("".join(line + "\n" for line in batch_lines))
                    out.flush()
                self.totals["tiles"] += n
                self.totals["primes"] += int(primes)
                self.totals["chains"] += len(chains)
                if self.mode == "sequential":
                    self.tile = ts + n
                done += 1
                if done % self.ck_every == 0:
                    self._save()
            self._save()
        finally:
            if out:
                out.close()
        return dict(self.totals)
