"""Element partitions and their halo exchange, on the host.

For 2 and 3 parts of a periodic tetrahedral mesh: every rank's renumbered
face pairing reaches the same neighbour elements as the global one; after
the row exchange every ghost row holds its owner's values; after the record
exchange every face record an owned element reads through a partition face
holds the owner's record.  Emulated ranks in one process (LocalTransport)
and two gloo ranks in two processes (torch.distributed point-to-point, as
NCCL runs it between GPUs).  The kernels' use of the ghosts is tested on
the GPU (tests/test_gpu_partition.py).
"""

import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch

from cases import make_disc
from mirgecom_b200.partition import (HaloExchange, LocalTransport, PartitionedDiscretization,
                                     partition_elements)

TW = 8


def _global_records(nel, nf, nfp):
    e, f, m, v = np.meshgrid(np.arange(nel), np.arange(nf), np.arange(nfp), np.arange(TW),
                             indexing="ij")
    return (e * 1000.0 + f * 100.0 + m * 10.0 + v).astype(np.float64)


def _check_rank(d, pd, q_loc, trace_loc, recs):
    c = d.connectivity
    nfp = d.nface_nodes
    # ghost rows carry their owners' values
    assert np.array_equal(q_loc, d_q(d)[:, pd.elements, :])
    # renumbered pairing reaches the same neighbours
    lc = pd.connectivity.conn[:pd.nowned].astype(np.int64)
    gc = c.conn[pd.owned].astype(np.int64)
    inter = gc >= 0
    assert np.array_equal(lc >= 0, inter)
    assert np.array_equal(pd.elements[lc[inter] >> 8], gc[inter] >> 8)
    assert np.array_equal(lc[inter] & 255, gc[inter] & 255)
    # every record an owned element reads through an interior face is its
    # neighbour's own record
    e_, f_ = np.nonzero(inter)
    en = lc[e_, f_] >> 8
    fo = c.fslot[lc[e_, f_] & 255, 0].astype(np.int64) // nfp
    got = trace_loc[en, fo]
    want = recs[pd.elements[en], fo]
    assert np.array_equal(got, want)


def d_q(d):
    x = d.geometry.nodes
    return np.stack([np.sin(x[0] + k) * np.cos(2 * x[1]) + x[2] * k for k in range(5)])


@pytest.mark.parametrize("nparts", [2, 3])
def test_local_transport(nparts):
    d, _ = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (1.0,) * 3, True)
    owner = partition_elements(d.nelements, nparts)
    pds = [PartitionedDiscretization(d, r, nparts, owner=owner) for r in range(nparts)]
    q = d_q(d)
    recs = _global_records(d.nelements, d.nfaces, d.nface_nodes)
    tr = LocalTransport(nparts)
    exs = [HaloExchange(pd, tr) for pd in pds]
    qs, traces = [], []
    for pd in pds:
        ql = np.zeros((5, pd.nelements, q.shape[-1]))
        ql[:, :pd.nowned] = q[:, pd.owned]
        qs.append(torch.from_numpy(ql))
        tl = np.full((pd.nelements,) + recs.shape[1:], np.nan)
        tl[:pd.nowned] = recs[pd.owned]
        traces.append(torch.from_numpy(tl))
    hs = [ex.begin_rows([ql]) for ex, ql in zip(exs, qs)]
    for ex, h in zip(exs, hs):
        ex.end(h)
    hs = [ex.begin_records(tl) for ex, tl in zip(exs, traces)]
    for ex, h in zip(exs, hs):
        ex.end(h)
    for pd, ql, tl in zip(pds, qs, traces):
        _check_rank(d, pd, ql.numpy(), tl.numpy(), recs)
    assert sum(pd.nowned for pd in pds) == d.nelements


def test_partition_covers_every_element_once():
    owner = partition_elements(100, 7)
    assert np.array_equal(np.bincount(owner), np.bincount(owner, minlength=7))
    assert owner.min() == 0 and owner.max() == 6
    assert np.all(np.diff(owner) >= 0)


_WORKER = r"""
import os, sys, numpy as np, torch, torch.distributed as dist
sys.path.insert(0, %(root)r); sys.path.insert(0, %(tests)r)
from datetime import timedelta
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
r, n = dist.get_rank(), dist.get_world_size()
from cases import make_disc
from mirgecom_b200.partition import HaloExchange, PartitionedDiscretization
import test_partition as tp
d, _ = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (1.0,) * 3, True)
pd = PartitionedDiscretization(d, r, n)
q = tp.d_q(d)
recs = tp._global_records(d.nelements, d.nfaces, d.nface_nodes)
ql = np.zeros((5, pd.nelements, q.shape[-1])); ql[:, :pd.nowned] = q[:, pd.owned]
tl = np.full((pd.nelements,) + recs.shape[1:], np.nan); tl[:pd.nowned] = recs[pd.owned]
ql, tl = torch.from_numpy(ql), torch.from_numpy(tl)
ex = HaloExchange(pd, "dist")
ex.exchange_rows([ql])
ex.exchange_records(tl)
tp._check_rank(d, pd, ql.numpy(), tl.numpy(), recs)
dist.barrier()
dist.destroy_process_group()
print("rank", r, "ok")
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    here = os.path.dirname(os.path.abspath(__file__))
    code = _WORKER % {"root": os.path.dirname(here), "tests": here}
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=180) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-3000:]
        assert "ok" in o
