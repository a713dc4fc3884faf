"""The batch dispatcher on CPU: rounds of checkouts over one process and over
two gloo ranks (the reference's stand-in work unit), which must leave the
scene in the same state for the same total batch and seed."""

import json
import os
import socket

import numpy as np
import pytest

from forcepho_b200 import dispatcher as D
from forcepho_b200 import superscene as SS

GOLD = os.path.join(os.path.dirname(__file__), "golden", "superscene_golden.json")


def _scene(seed=21, target=150):
    with open(GOLD) as f:
        g = json.load(f)
    bands = g["bands"]
    cat = np.zeros(len(g["catalog"]["ra"]), dtype=SS.sourcecat_dtype(bands=bands))
    for k in cat.dtype.names:
        cat[k] = g["catalog"][k]
    return SS.SuperScene(sourcecat=cat, bands=bands, maxactive_per_patch=15, target_niter=target,
                         maxactive_fraction=0.5, rng=np.random.default_rng(seed))


def _checked_work(tasks):
    # regions worked together never share an active source
    ids = [set(t["active"]["source_index"].tolist()) for t in tasks]
    for i in range(len(ids)):
        for j in range(i):
            assert not (ids[i] & ids[j])
    return D.dummy_work(tasks)


def test_single_process_rounds_finish_the_scene():
    sc = _scene()
    rounds = D.run(sc, _checked_work, batch_per_rank=6, max_rounds=400)
    assert not sc.undone, "scene not finished in %d rounds" % len(rounds)
    assert sc.n_active == 0 and np.all(sc.sourcecat["is_active"] == 0) and np.all(sc.sourcecat["is_valid"] == 1)
    assert np.all(sc.sourcecat["n_iter"] >= 150) and np.all(sc.sourcecat["n_iter"] % 75 == 0)
    assert all(1 <= r["tasks"] <= 6 for r in rounds)
    # every task was logged once, in order
    assert sc.patchlog == [str(i) for i in range(sum(r["tasks"] for r in rounds))]


def test_checkout_batch_respects_sparsity():
    sc = _scene()
    sc.maxactive_fraction = 0.05
    tasks = D.checkout_batch(sc, 100)
    assert 0 < len(tasks) < 100
    assert not sc.sparse
    assert [t["taskid"] for t in tasks] == list(range(len(tasks)))
    assert all(t["cov"].shape[0] == len(t["active"]) * len(sc.parameter_columns) for t in tasks)


def test_work_must_answer_every_task():
    sc = _scene()
    with pytest.raises(RuntimeError, match="results"):
        D.run(sc, lambda tasks: [], batch_per_rank=2, max_rounds=1)


def _worker(rank, world, port, outdir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        sc = _scene() if rank == 0 else None
        seen = []

        def work(tasks):
            seen.extend(t["taskid"] for t in tasks)
            return _checked_work(tasks)

        rounds = D.run(sc, work, batch_per_rank=3, rank=rank, world=world, max_rounds=400)
        np.save(os.path.join(outdir, "seen%d.npy" % rank), np.array(seen, dtype=np.int64))
        if rank == 0:
            np.save(os.path.join(outdir, "n_iter.npy"), sc.sourcecat["n_iter"])
            with open(os.path.join(outdir, "rounds.json"), "w") as f:
                json.dump(rounds, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_ranks_match_one_process(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    sc = _scene()
    want = D.run(sc, _checked_work, batch_per_rank=6, max_rounds=400)
    np.testing.assert_array_equal(np.load(tmp_path / "n_iter.npy"), sc.sourcecat["n_iter"])
    with open(tmp_path / "rounds.json") as f:
        rounds = json.load(f)
    assert [r["tasks"] for r in rounds] == [r["tasks"] for r in want]
    s0, s1 = np.load(tmp_path / "seen0.npy"), np.load(tmp_path / "seen1.npy")
    assert len(s0) and len(s1)                                   # both ranks worked
    assert sorted(np.concatenate([s0, s1]).tolist()) == list(range(sum(r["tasks"] for r in want)))


def test_empty_scene_and_bad_sampling_arguments():
    cat = np.zeros(0, dtype=SS.sourcecat_dtype(bands=["B0"]))
    sc = SS.SuperScene(sourcecat=cat, bands=["B0"])
    assert not sc.sparse and D.checkout_batch(sc, 4) == []
    assert D.run(sc, D.dummy_work, batch_per_rank=2) == []
    with pytest.raises(ValueError):
        D.hmc_work(lambda: None, ["B0"], n_draws=0)


def _failing_worker(rank, world, port, outdir):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    sc = _scene() if rank == 0 else None

    def work(tasks):
        if rank == 1:
            raise RuntimeError("work failed on rank 1")
        return _checked_work(tasks)

    try:
        D.run(sc, work, batch_per_rank=2, rank=rank, world=world, max_rounds=3)
        outcome = "finished"
    except Exception as e:                      # noqa: BLE001 -- recorded for the test
        outcome = "%s: %s" % (type(e).__name__, str(e)[:200])
    with open(os.path.join(outdir, "outcome%d.txt" % rank), "w") as f:
        f.write(outcome)
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_a_failing_rank_ends_the_run_on_every_rank(tmp_path):
    """A work unit that raises on one rank: that rank leaves the round, and
    rank 0 gets an error from the round's gather (the peer is gone, or the
    process group's 10 s timeout runs out) instead of waiting for ever."""
    import torch.multiprocessing as mp
    mp.spawn(_failing_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    out0 = (tmp_path / "outcome0.txt").read_text()
    out1 = (tmp_path / "outcome1.txt").read_text()
    assert out1.startswith("RuntimeError: work failed on rank 1")
    assert out0 != "finished", out0


def test_checkout_stops_when_every_source_is_taken():
    """Three isolated sources in a scene that stays sparse: three regions of
    one active source each, then nothing is left to seed a region, and
    checkout ends quietly instead of failing on zero seed weights."""
    bands = ["B0"]
    for cls in (SS.SuperScene, SS.LinkedSuperScene):
        cat = np.zeros(3, dtype=SS.sourcecat_dtype(bands=bands))
        cat["ra"] = 53.1 + np.array([0.0, 0.01, 0.02])          # 36 arcsec apart
        cat["dec"] = -27.8
        cat["rhalf"], cat["roi"], cat["q"], cat["sersic"], cat["B0"] = 0.1, 0.3, 0.8, 2.0, 1.0
        sc = cls(sourcecat=cat, bands=bands, maxactive_per_patch=15, maxactive_fraction=2.0,
                 rng=np.random.default_rng(3))
        tasks = D.checkout_batch(sc, 10, ntry=50)
        assert len(tasks) == 3 and sc.sparse
        assert not np.any(sc.sourcecat["is_valid"]) and sc.seed_weight().sum() == 0
        assert sc.checkout_region()[1] is None
        assert D.checkout_batch(sc, 5) == []
