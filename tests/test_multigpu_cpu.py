"""The multi-GPU split of one solve (hhg-solids_b200/shard.py) on CPU: two gloo ranks, each
propagating its k-row slab (with the CPU oracle standing in for its GPU) and summing the partial
currents with one all_reduce, reproduce the full current."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_golden, rel_l2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, name, out_dir):
    import sys

    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.join(here, "..", "hhg-solids_b200"), os.path.join(here, "..", "oracle"), here):
        sys.path.insert(0, p)
    import oracle
    import shard
    from conftest import load_golden

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    meta, param, _, _ = load_golden(name)
    r0, r1 = shard.row_slab(rank, world, param["nr1"])
    n2 = param["nr2"]
    _, J_part = oracle.run(param["path_tb"], param, r0 * n2, r1 * n2)  # this rank's slab
    J = shard.reduce_current(J_part)
    np.save(os.path.join(out_dir, f"J{rank}.npy"), J)
    dist.barrier()
    dist.destroy_process_group()


def test_row_slabs_partition_the_grid():
    import shard

    for n, w in [(8, 2), (9, 2), (200, 8), (150, 7), (4, 4)]:
        slabs = [shard.row_slab(r, w, n) for r in range(w)]
        assert slabs[0][0] == 0 and slabs[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(slabs, slabs[1:]))
        assert max(b - a for a, b in slabs) - min(b - a for a, b in slabs) <= 1
    with pytest.raises(ValueError):
        shard.row_slab(0, 5, 4)


@pytest.mark.parametrize("name", ["haldane_12_pol", "tmd6_8"])
def test_two_gloo_ranks_sum_to_the_full_current(tmp_path, name):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), name, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    meta, param, _, J_ref = load_golden(name)
    J0 = np.load(tmp_path / "J0.npy")
    J1 = np.load(tmp_path / "J1.npy")
    assert np.array_equal(J0, J1)  # every rank holds the total
    for a in range(2):
        assert rel_l2(J0[a], J_ref[a]) < 1e-10
