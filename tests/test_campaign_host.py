"""Campaign shell on the CPU: the batch generator and the checkpoint file are
pinned to the reference's own code (v13 rng_next, checkpoint_save and
checkpoint_load, run through oracle/_ref), and the batch planner is checked
for sequential coverage and seeded random draws."""
import ctypes as C
import importlib
import os

import pytest

camp = importlib.import_module("cunningham-chain-search_b200.campaign")

_u64p = C.POINTER(C.c_ulonglong)


def _ref(ob):
    r = ob.ref13()
    if r is None:
        pytest.skip("reference harness not built")
    r.ref13_rng.argtypes = [C.c_ulonglong, C.c_int, _u64p]
    r.ref13_checkpoint_save.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_int,
                                        C.c_ulonglong, C.c_ulonglong, C.c_ulonglong, C.c_ulonglong,
                                        C.c_ulonglong, C.c_int]
    r.ref13_checkpoint_load.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_int,
                                        _u64p]
    return r


@pytest.mark.parametrize("seed", [1, 0, 12345, (1 << 63) + 5, 0x9E3779B97F4A7C15])
def test_generator_matches_reference(ob, seed):
    r = _ref(ob)
    out = (C.c_ulonglong * 200)()
    r.ref13_rng(seed, 200, out)
    g = camp.XorShift64(seed)
    assert [g.next() for _ in range(200)] == list(out)


def test_checkpoint_files_are_interchangeable(ob, tmp_path):
    r = _ref(ob)
    tile = (0x1234 << 64) | 0xDEADBEEFCAFEF00D
    totals = {"tiles": 123456789, "primes": 4242, "chains": 17, "best": 11}
    ours = str(tmp_path / "ours.ck")
    camp.checkpoint_save(ours, 89, 18, 18, tile, totals, prefix="0b1011", lanes=4, lane_id=2)
    out = (C.c_ulonglong * 6)()
    assert r.ref13_checkpoint_load(ours.encode(), 89, 18, 18, b"0b1011", 4, 2, out) == 0
    assert ((out[0] << 64) | out[1], out[2], out[3], out[4], out[5]) == \
        (tile, totals["tiles"], totals["primes"], totals["chains"], totals["best"])
    # the reference refuses our file for another campaign, like we do
    assert r.ref13_checkpoint_load(ours.encode(), 89, 18, 16, b"0b1011", 4, 2, out) != 0
    with pytest.raises(ValueError):
        camp.checkpoint_load(ours, 89, 18, 18, prefix="0b1011", lanes=4, lane_id=3)
    theirs = str(tmp_path / "theirs.ck")
    assert r.ref13_checkpoint_save(theirs.encode(), 64, 16, 16, b"none", 0, 0, 7, 99, 5, 6, 7, 9) == 0
    t2, tot2 = camp.checkpoint_load(theirs, 64, 16, 16)
    assert t2 == (7 << 64) | 99 and tot2 == {"tiles": 5, "primes": 6, "chains": 7, "best": 9}
    with pytest.raises(ValueError):
        camp.checkpoint_load(theirs, 65, 16, 16)
    with open(theirs) as f:
        assert f.readline().strip() == camp.CHECKPOINT_MARKER


class _HostOnlyEngine:
    """Enough of an Engine for the batch planner (ccs_describe needs no GPU)."""

    def __init__(self, ccs):
        self._info, self._bases = ccs.describe()
        self.bits = None

    @property
    def info(self):
        return self._info

    def bases(self):
        return self._bases

    def set_bits(self, b):
        self.bits = b


def test_batch_planner(ccs):
    eng = _HostOnlyEngine(ccs)
    c = camp.Campaign(eng, bits=64, lanes=3, lane_id=1, batch_tiles=1000)
    lo, hi = c.tile_min, c.tile_max
    t_lo, t_hi = ccs.bit_tile_range(64, eng.bases(), eng.info["lattice_m"], eng.info["wheel_period"])
    assert (lo, hi) == ccs.lane_range(t_lo, t_hi, 3, 1) and eng.bits == 64
    ts, n = c.next_batch()
    assert ts == lo and n == min(1000, hi - lo)
    c.tile = hi - 10
    assert c.next_batch() == (hi - 10, 10)
    c.tile = hi
    assert c.next_batch() is None
    r1 = camp.Campaign(eng, bits=64, mode="random", seed=77, batch_tiles=1000)
    r2 = camp.Campaign(eng, bits=64, mode="random", seed=77, batch_tiles=1000)
    draws = [r1.next_batch() for _ in range(50)]
    assert draws == [r2.next_batch() for _ in range(50)]
    assert all(r1.tile_min <= ts and ts + n <= r1.tile_max for ts, n in draws)
    assert len(set(draws)) == 50
