"""Slab/column decomposition of one case over several ranks
(turbid_b200/distributed.py): z-slabs in physical space, spectral columns
(whole Chebyshev columns of a range of modes) in spectral space, one
all-to-all between them.

CPU, 2 and 3 gloo ranks (the local plane transforms are the oracle's numpy
transforms): the distributed forward transform equals the whole-case transform
restricted to each rank's modes, exactly (the exchange only moves values); the
backward transform returns each rank's planes of the whole-case round trip;
uneven partitions of planes and modes.
GPU, one rank (this run has one GPU): the library's plane transforms
(tg_dft_forward_planes / tg_dft_backward_planes) through the same path equal
tg_dft_forward_f64 / tg_dft_backward_f64 of the whole field.
"""
import os
import socket

import numpy as np
import pytest
import torch

import turbid_b200 as tb
from oracle import turbid_oracle as O
from turbid_b200.distributed import SlabColumnExchange, SlabColumnTransform, split_range


def test_split_range_covers_evenly():
    for n, parts in ((17, 2), (17, 3), (14620, 8), (5, 5)):
        r = [split_range(n, parts, k) for k in range(parts)]
        assert r[0][0] == 0 and r[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        sizes = [b - a for a, b in r]
        assert max(sizes) - min(sizes) <= 1


def _numpy_planes(g):
    """Local plane transforms of the oracle on CPU tensors (z-slab layout)."""
    def fwd(phys, spec, planes):
        x = phys.reshape(planes, g.ny, g.nx).numpy()
        s = O.dft_forward(g, x[None])                         # (1, nxh, nyc, planes)
        spec.view(planes, g.M).copy_(torch.from_numpy(tb.to_slab(s)[0]))

    def bwd(spec, phys, planes):
        s = tb.from_slab(spec.reshape(1, planes, g.M).numpy(), g.nxh, g.nyc)
        phys.view(planes, g.ny, g.nx).copy_(torch.from_numpy(O.dft_backward(g, s)[0]))
    return fwd, bwd


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nx, ny, nz, dim, q):
    import torch.distributed as dist
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        g = O.Grid(O.CaseConfig(nx=nx, ny=ny, nz=nz))
        fwd, bwd = _numpy_planes(g)
        tr = SlabColumnTransform(nx, ny, nz, dist=dist, plane_forward=fwd, plane_backward=bwd)
        rng = np.random.default_rng(7)
        full = rng.standard_normal((dim, nz, ny, nx))           # every rank draws the same field
        z0, z1 = tr.ex.my_planes
        m0, m1 = tr.ex.my_modes
        cols = tr.forward(torch.from_numpy(full[:, z0:z1].copy()))
        ref = tb.to_slab(O.dft_forward(g, full))                 # (dim, nz, M)
        ok_fwd = np.array_equal(cols.numpy(), ref[:, :, m0:m1])
        back = tr.backward(cols)
        ref_back = O.dft_backward(g, O.dft_forward(g, full))
        ok_bwd = np.array_equal(back.numpy(), ref_back[:, z0:z1])
        # the exchange alone is a permutation: slabs -> columns -> slabs is the identity
        slab = torch.from_numpy(ref[:, z0:z1].copy())
        ok_perm = torch.equal(tr.ex.to_slabs(tr.ex.to_columns(slab)), slab)
        q.put((rank, ok_fwd, ok_bwd, ok_perm, (z1 - z0, m1 - m0)))
        dist.destroy_process_group()
    except Exception as exc:   # reported to the parent
        q.put((rank, repr(exc)))


@pytest.mark.parametrize("world,nx,ny,nz,dim", [(2, 24, 18, 17, 2), (3, 16, 12, 9, 3)])
def test_gloo_ranks_match_the_whole_case_transform(world, nx, ny, nz, dim):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nx, ny, nz, dim, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for r in res:
        assert len(r) == 5, r
        rank, ok_fwd, ok_bwd, ok_perm, shape = r
        assert ok_fwd and ok_bwd and ok_perm, (rank, ok_fwd, ok_bwd, ok_perm)
    assert sum(r[4][0] for r in res) == nz


def test_single_rank_exchange_is_identity():
    ex = SlabColumnExchange(9, 20)
    x = torch.randn(2, 9, 20, dtype=torch.complex128)
    assert torch.equal(ex.to_columns(x), x) and torch.equal(ex.to_slabs(x), x)
    with pytest.raises(ValueError):
        ex.to_columns(x[:, :8])


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [False, True])
def test_gpu_slab_transform_matches_whole_field(cuda, fp32):
    nx, ny, nz, dim = 32, 24, 17, 3
    case = tb.ChannelCase(nx=nx, ny=ny, nz=nz)
    case.set_stream(torch.cuda.current_stream().cuda_stream)
    tr = SlabColumnTransform(nx, ny, nz, case=case)
    dt = torch.float32 if fp32 else torch.float64
    x = torch.randn(dim, nz, ny, nx, dtype=torch.float64, device=cuda).to(dt)
    cols = tr.forward(x)
    ref = torch.zeros((dim, nz, case.M), dtype=torch.complex128, device=cuda)
    case.dft_forward(x.data_ptr(), ref.data_ptr(), dim, fp32=fp32)
    torch.cuda.synchronize()
    assert torch.equal(cols, ref)
    back = tr.backward(cols, dtype=dt)
    ref_back = torch.zeros_like(x)
    case.dft_backward(ref.data_ptr(), ref_back.data_ptr(), dim, fp32=fp32)
    torch.cuda.synchronize()
    assert torch.equal(back, ref_back)
    case.close()
