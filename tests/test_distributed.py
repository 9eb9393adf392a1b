"""Multi-rank shot sharding and gradient reduction, world size 2 on CPU (gloo).
The per-rank compute is the oracle (no GPU here); the test checks that the
sharded, all-reduced gradient equals the single-process gradient of all shots."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from vtib200.distributed import shard


def test_shard_matches_reference_grouping():
    shots = list(range(7))
    parts = [shard(shots, r, 3) for r in range(3)]
    assert parts == [[0, 1, 2], [3, 4], [5, 6]]
    assert sum(parts, []) == shots
    assert shard([1, 2], 2, 3) == []


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    for p in (root / "thesis-source-code_b200", root / "oracle", root / "tests" / "golden"):
        sys.path.insert(0, str(p))
    import torch
    import torch.distributed as dist
    import cases as K
    import oracle as O
    from vtib200 import distributed as D

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = K.case3d("g3_b")
        s = c["s"]
        gold = np.load(root / "tests" / "golden" / "g3_b.npz")
        g = s.geom()

        def local(shots):
            if not shots:
                return torch.zeros(1 + 3 * s.nxyz, dtype=torch.float64), 0.0
            fg = O.gradient3d(g, c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, shots,
                              s.recloc, gold["dobs"])
            mis = float(fg[0])
            fg[0] = 0.0
            return torch.from_numpy(fg), mis

        grad, mis = D.gradient(local, [0, 1])
        if rank == 0:
            np.save(out_path, np.concatenate([[mis], grad.numpy()[1:]]))
    finally:
        dist.destroy_process_group()


def test_two_rank_gradient_equals_single_process(tmp_path):
    import oracle as O
    import cases as K
    from conftest import ROOT, rel_l2

    out = tmp_path / "g.npy"
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(out)), nprocs=2, start_method="spawn",
                       join=True)
    got = np.load(out)
    c = K.case3d("g3_b")
    s = c["s"]
    gold = np.load(ROOT / "tests" / "golden" / "g3_b.npz")
    ref = O.gradient3d(s.geom(), c["cij"], c["padb"], c["randb"], s.wavelet, s.souloc, [0, 1],
                       s.recloc, gold["dobs"])
    assert abs(got[0] - ref[0]) / ref[0] < 1e-12
    assert rel_l2(got[1:], ref[1:]) < 1e-12
