"""Multi-GPU sharding logic on CPU (gloo, world size 2).

CLOUDSC columns are independent (the recurrence is only vertical), so the
multi-GPU form shards NPROMA blocks across ranks with no data-path
collective; only scalars (timings, warning counts) are reduced.  Here two
gloo ranks each run the product's own column code -- the kernels'
cloudsc_body.cuh built for the host (tests/hostemu), the code each GPU rank
runs -- on their contiguous block range [g*N/G, (g+1)*N/G) of a ragged
workload, and the gathered result must equal the single-process run and the
oracle bit for bit; the MAX reduction of step times and the SUM of warning
counts follow the bench's rules.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from openifs_b200 import fields, inputs, shard
from tests import util

NB, NPROMA, CUT = 7, 16, 5  # the last block holds NPROMA - CUT columns


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p, po = util.params()
        b0, b1 = shard.block_range(NB, rank, world)
        arrs = inputs.generate(NB, NPROMA, p, seed=8, blocks=range(b0, b1))
        # this rank's share of NGPTOT: the ragged last block is the last rank's
        ngptot = (b1 - b0) * NPROMA - (CUT if b1 == NB else 0)
        out, nw = util.run_hostemu(p, arrs, NPROMA, b1 - b0, ngptot)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), **{n: out[n] for n in fields.OUTPUT_NAMES})
        t = torch.tensor([float(rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        w = torch.tensor([nw])
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
        np.save(os.path.join(outdir, f"red{rank}.npy"), np.array([t.item(), w.item()]))
    finally:
        dist.destroy_process_group()


def test_block_ranges_partition():
    for n in (1, 7, 2048):
        for g in (1, 2, 3, 8):
            rs = [shard.block_range(n, r, g) for r in range(g)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))


def test_two_rank_gloo_shards_match_single_process(tmp_path, built):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    p, po = util.params()
    arrs = inputs.generate(NB, NPROMA, p, seed=8)
    ngptot = NB * NPROMA - CUT
    single, nw1 = util.run_hostemu(p, arrs, NPROMA, NB, ngptot)
    ref, nw_ref = util.run_oracle(po, arrs, NPROMA, NB, ngptot, libm="plibm")
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(2)]
    for n in fields.OUTPUT_NAMES:
        got = np.concatenate([parts[0][n], parts[1][n]], axis=0)
        assert np.array_equal(util.defined(n, got), util.defined(n, single[n])), n
        a = util.defined(n, util._valid_cols(got, ngptot, NPROMA))
        b = util.defined(n, util._valid_cols(ref[n], ngptot, NPROMA))
        assert np.array_equal(a, b), n
    red = np.load(tmp_path / "red0.npy")
    assert red[0] == 2.0
    assert red[1] == nw1 == nw_ref
