"""Two ranks (processes) on one GPU step one room split in two slabs whose
fused steps write each other's ghost planes through CUDA IPC mappings; the
ranks meet at a host barrier (gloo) after each step, so no kernel waits for
another.  Traces and field equal the whole-room engine bit for bit."""
import os
import socket
import tempfile

import numpy as np
import pytest

from conftest import bits_equal, first_mismatch
from test_slab_gpu import edge_room, whole

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_path):
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    from spectral_analyzer_b200.slab import distributed_room
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        room = edge_room()
        run = distributed_room(room, rank, world, peer_memory=True)
        run.step(room.n_steps)
        torch.cuda.synchronize()
        tr = run.traces(len(room.receivers))
        P = run.pressure_field()
        if rank == 0:
            np.savez(out_path, traces=tr, P=P)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_processes_peer_stores():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    import torch.multiprocessing as mp
    room = edge_room()
    tr, P = whole(room)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "r.npz")
        mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        with np.load(out) as z:
            got_tr, got_P = z["traces"], z["P"]
    assert bits_equal(got_tr, tr), first_mismatch(got_tr, tr)
    assert bits_equal(got_P, P)
