"""Photon-range sharding across ranks (the N-GPU weak-scaling layout of bench.py),
exercised with world_size 2 on the gloo backend: each rank transports its own
photon range with the oracle and the ranks all-reduce their tallies; the sum
equals one run over the whole range, because photon i draws stream (seed, i)
wherever it runs."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from luminis_mc_b200 import workloads as W


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, out):
    import sys
    sys.path[:0] = [os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                 "luminis-mc_b200")]
    from luminis_mc_b200 import workloads as W2
    from oracle import pyoracle as O2
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    spec = W2.bilayer_rgd_mie(n, 2024)
    share = n // world
    res = O2.Oracle(spec).run(share, 2024, begin=rank * share, rng="philox_u24")
    for i, t in enumerate(res.tallies):
        x = torch.from_numpy(t.copy())
        dist.all_reduce(x)
        if rank == 0:
            np.save(os.path.join(out, f"sensor{i}.npy"), x.numpy())
    h = torch.tensor(res.hits.astype(np.int64))
    dist.all_reduce(h)
    if rank == 0:
        np.save(os.path.join(out, "hits.npy"), h.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_photon_ranges_reduce_to_the_single_run(tmp_path):
    from oracle import pyoracle as O
    n = 1200
    mp.start_processes(_worker, args=(2, _free_port(), n, str(tmp_path)), nprocs=2,
                       start_method="spawn")
    whole = O.Oracle(W.bilayer_rgd_mie(n, 2024)).run(n, 2024, rng="philox_u24")
    for i, t in enumerate(whole.tallies):
        np.testing.assert_allclose(np.load(tmp_path / f"sensor{i}.npy"), t, rtol=1e-12,
                                   atol=1e-12 * np.abs(t).max())
    np.testing.assert_array_equal(np.load(tmp_path / "hits.npy"), whole.hits.astype(np.int64))
