"""The multi-rank driver of the partitioned single mesh (pdekit_b200.partition.PartitionedRDS)
run as two processes sharing one GPU, with the gloo backend: the interface and norm sums go
through the host, so no kernel of one rank ever waits for the other rank on the device (each
rank's device work completes before its sums). Rank 0 checks the gathered state and the norm
against the single-context solver."""

import os
import socket

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _rank(rank, world, port, case, iters, out):
    import torch
    import torch.distributed as dist

    from pdekit_b200.partition import PartitionedRDS
    from golden_io import load_golden

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob, a, meta = load_golden(os.path.join(GOLDEN, case))
        pr = PartitionedRDS(prob, rank, world)
        pr.set_solution(a["u0"])
        it, norm = pr.iterate(meta["cfl"], iters, check_every=4)
        u = pr.solution_global()
        pr.close()
        if rank == 0:
            np.save(out + ".u.npy", u)
            np.save(out + ".n.npy", norm)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["burgers_p2_b", "euler2d_tri_p3_b"])
def test_two_rank_driver_matches_single_context(case, tmp_path):
    import torch.multiprocessing as mp

    from helpers import rel_err
    from golden_io import load_golden
    from pdekit_b200.rds import PGRDMethodExplicit

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "r0")
    iters = 8
    mp.start_processes(_rank, args=(2, port, case, iters, out), nprocs=2, join=True,
                       start_method="spawn")
    prob, a, meta = load_golden(os.path.join(GOLDEN, case))
    s = PGRDMethodExplicit(prob.physics, prob.scheme, "fp64").configure_mesh_data(prob)
    s.initialize_work_data()
    s.set_solution(a["u0"])
    _, hist = s.iterate(meta["cfl"], iters)
    u1 = s.solution()
    s.close()
    assert rel_err(np.load(out + ".u.npy"), u1) < 1e-12
    np.testing.assert_allclose(np.load(out + ".n.npy"), hist[-1], rtol=1e-11)
