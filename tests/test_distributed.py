"""The multi-process patch farm on CPU: two gloo ranks, each evaluating its
share of the patches (with the CPU oracle standing in for the GPU evaluator),
gathered to rank 0 and compared with a single-process evaluation."""

import os
import socket

import numpy as np

from forcepho_b200.distributed import balance


def test_balance_deterministic_and_complete():
    w = [5, 1, 9, 9, 3, 7, 2, 2, 8]
    parts = balance(w, 3)
    assert sorted(sum(parts, [])) == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert parts == balance(w, 3)
    assert balance(w, 1) == [list(range(len(w)))]


def _patch(i):
    from forcepho_b200 import synthetic as S
    return S.config_multiband(seed=100 + i, n_sources=2, n_bands=2, exp_per_band=1, size=24)


def _oracle_evaluator(patches):
    from oracle import oracle as O

    def run(props):
        return [O.evaluate(p, pr, precision="f32", nthreads=1)[:2] for p, pr in zip(patches, props)]
    return run


def _worker(rank, world, port, n, outdir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from forcepho_b200.distributed import PatchFarm
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        weights = [_patch(i).n_pairs() for i in range(n)]
        farm = PatchFarm(_patch, weights, rank, world, evaluator=_oracle_evaluator)
        props = {i: _patch(i).scene.get_proposal() for i in range(n)}
        res = farm.evaluate_and_gather(props)
        if rank == 0:
            chi = np.array([r[0].sum() for r in res])
            np.save(os.path.join(outdir, "chi.npy"), chi)
            np.save(os.path.join(outdir, "idx.npy"), np.array(farm.indices))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_rank_farm_matches_single_process(tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    n = 5
    mp.spawn(_worker, args=(2, _free_port(), n, str(tmp_path)), nprocs=2, join=True)
    chi = np.load(tmp_path / "chi.npy")
    want = np.array([O.evaluate(_patch(i), _patch(i).scene.get_proposal(), precision="f32",
                                nthreads=1)[0].sum() for i in range(n)])
    np.testing.assert_array_equal(chi, want)
    assert 0 < len(np.load(tmp_path / "idx.npy")) < n     # rank 0 held only its share
