"""Campaign shell on the GPU: a campaign interrupted and resumed from its
checkpoint writes exactly the output of an uninterrupted one, and its lines
are the reference-format lines of the engine's chains for the same tiles."""
import importlib

import pytest

pytestmark = pytest.mark.gpu

camp = importlib.import_module("cunningham-chain-search_b200.campaign")


def test_resume_equals_uninterrupted(ccs, tmp_path):
    eng = ccs.Engine(bits=64)
    kw = dict(bits=64, batch_tiles=4000, log_threshold=3)
    whole = camp.Campaign(eng, out_path=str(tmp_path / "whole.txt"),
                          checkpoint_path=str(tmp_path / "whole.ck"), **kw)
    tot_whole = whole.run(max_batches=4)
    first = camp.Campaign(eng, out_path=str(tmp_path / "split.txt"),
                          checkpoint_path=str(tmp_path / "split.ck"), **kw)
    first.run(max_batches=2)
    second = camp.Campaign(eng, out_path=str(tmp_path / "split.txt"),
                           checkpoint_path=str(tmp_path / "split.ck"), resume=True, **kw)
    assert second.tile == first.tile_min + 2 * 4000
    tot_split = second.run(max_batches=2)
    assert tot_split == tot_whole and tot_whole["tiles"] == 16000 and tot_whole["chains"] > 0
    assert open(tmp_path / "split.txt").read() == open(tmp_path / "whole.txt").read()
    assert camp.checkpoint_load(str(tmp_path / "split.ck"), 64, 18, 18)[0] == whole.tile

    # the lines are the engine's chains over the same tiles, in reference format
    want = []
    for b in range(4):
        ts = whole.tile_min + 4000 * b
        _, chains, _ = eng.search_range_host(ts, 4000, surv_cap=1 << 22, chain_cap=1 << 18)
        for rec in chains:
            cl = int(rec["chain_len"])
            if cl >= 3:
                want.append(ccs.format_chain_line(cl, ccs.chain_root_int(rec), 18, bool(rec["flags"] & 1)))
    assert sorted(whole.lines) == sorted(want) and len(want) > 0
    eng.close()


def test_random_campaign_is_reproducible(ccs):
    eng = ccs.Engine(bits=64)
    a = camp.Campaign(eng, bits=64, mode="random", seed=99, batch_tiles=2000, log_threshold=3)
    b = camp.Campaign(eng, bits=64, mode="random", seed=99, batch_tiles=2000, log_threshold=3)
    assert a.run(max_batches=3) == b.run(max_batches=3)
    assert sorted(a.lines) == sorted(b.lines)
    eng.close()
