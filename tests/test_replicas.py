"""The multi-GPU form of the benchmark runs independent replicas (the solver
does not shard): each rank times its own reconstruction and the job reports
the max time over ranks and the summed throughput.  Checked here with two
gloo ranks on the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [100.0 + 50.0 * rank, 200.0 - 10.0 * rank]   # this rank's served and plain times
    got = bench.max_over_ranks(ms, torch.device("cpu"))
    out[rank] = (got, bench.replica_value(got[0], world))
    dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:   # no fork of this multi-threaded process
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
        res = dict(out)
    for rank in range(world):
        got, value = res[rank]
        assert got == [150.0, 200.0]
        assert abs(value - 2 * 1e3 / 150.0) < 1e-9


def test_single_process_is_identity():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.0], torch.device("cpu")) == [3.0, 4.0]
    assert bench.replica_value(250.0, 1) == 4.0
