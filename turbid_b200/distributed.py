"""Slab/column decomposition of one case over several GPUs, one process per
GPU: the exchange that P3DFFT's pencil transforms make between their x-y and
z passes (build/fcomm1.F90:85, build/fcomm2.F90:57; the decomposition is set
up in src/base.cc:228-237), restated for a slab/column layout.

* Physical space: rank r holds the z planes [z0_r, z1_r) of every field
  (a z-slab), all Nx x Ny points of each plane.
* Spectral space: rank r holds the modes [m0_r, m1_r) of the z-slab layout
  (m = iy + Nyc * ix) at every z plane: whole Chebyshev columns, on which the
  z-operators and Helmholtz solves act without communication.
* Forward transform: the x and y passes of the rank's own planes
  (tg_dft_forward_planes), then one all-to-all: each rank sends, for every
  destination, the destination's modes of its planes and receives its own
  modes of every source's planes.  Backward: the reverse exchange, then the
  y and x passes of the rank's planes.

Every block of the exchange is contiguous on both sides (planes are whole on
the sending side, modes are contiguous within a plane), so it is one
torch.distributed.all_to_all_single over NCCL on the GPUs (gloo on the CPU),
landing in the rank's own memory; no peer memory is read by any kernel.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import torch


def split_range(n: int, parts: int, k: int) -> Tuple[int, int]:
    """The k-th of `parts` contiguous, balanced ranges of [0, n) (the first
    n % parts ranges one longer)."""
    base, extra = divmod(n, parts)
    lo = k * base + min(k, extra)
    return lo, lo + base + (1 if k < extra else 0)


class SlabColumnExchange:
    """The all-to-all between z-slabs and spectral columns of one case.

    nz, M: the case's Chebyshev planes and spectral modes; dist: the
    torch.distributed module with an initialised process group (None for a
    single rank).  Tensors are complex128 on the process's device.
    """

    def __init__(self, nz: int, M: int, dist=None, group=None):
        self.nz, self.M = nz, M
        self.dist, self.group = dist, group
        self.world = dist.get_world_size(group) if dist is not None else 1
        self.rank = dist.get_rank(group) if dist is not None else 0
        if nz < self.world or M < self.world:
            raise ValueError("SlabColumnExchange > fewer planes or modes than ranks")
        self.planes: List[Tuple[int, int]] = [split_range(nz, self.world, r) for r in range(self.world)]
        self.modes: List[Tuple[int, int]] = [split_range(M, self.world, r) for r in range(self.world)]

    @property
    def my_planes(self) -> Tuple[int, int]:
        return self.planes[self.rank]

    @property
    def my_modes(self) -> Tuple[int, int]:
        return self.modes[self.rank]

    def _a2a(self, send: torch.Tensor, send_counts: List[int], recv_counts: List[int]) -> torch.Tensor:
        recv = torch.empty(sum(recv_counts), dtype=send.dtype, device=send.device)
        if self.dist is None:
            recv.copy_(send)
            return recv
        # complex values as pairs of doubles (NCCL and gloo move real types)
        self.dist.all_to_all_single(torch.view_as_real(recv).reshape(-1), torch.view_as_real(send).reshape(-1),
                                    [2 * c for c in recv_counts], [2 * c for c in send_counts], group=self.group)
        return recv

    def to_columns(self, slab: torch.Tensor) -> torch.Tensor:
        """(dim, my planes, M) spectral slab -> (dim, nz, my modes) columns."""
        dim, nzl, M = slab.shape
        z0, z1 = self.my_planes
        if nzl != z1 - z0 or M != self.M:
            raise ValueError("SlabColumnExchange.to_columns > slab shape does not match the partition")
        send = torch.cat([slab[:, :, m0:m1].reshape(-1) for m0, m1 in self.modes])
        m0, m1 = self.my_modes
        recv_counts = [dim * (b - a) * (m1 - m0) for a, b in self.planes]
        recv = self._a2a(send, [dim * nzl * (b - a) for a, b in self.modes], recv_counts)
        blocks = torch.split(recv, recv_counts)
        return torch.cat([blk.view(dim, b - a, m1 - m0) for blk, (a, b) in zip(blocks, self.planes)], dim=1)

    def to_slabs(self, cols: torch.Tensor) -> torch.Tensor:
        """(dim, nz, my modes) columns -> (dim, my planes, M) spectral slab."""
        dim, nz, ml = cols.shape
        m0, m1 = self.my_modes
        if nz != self.nz or ml != m1 - m0:
            raise ValueError("SlabColumnExchange.to_slabs > column shape does not match the partition")
        send = torch.cat([cols[:, a:b, :].reshape(-1) for a, b in self.planes])
        z0, z1 = self.my_planes
        recv_counts = [dim * (z1 - z0) * (b - a) for a, b in self.modes]
        recv = self._a2a(send, [dim * (b - a) * ml for a, b in self.planes], recv_counts)
        blocks = torch.split(recv, recv_counts)
        return torch.cat([blk.view(dim, z1 - z0, b - a) for blk, (a, b) in zip(blocks, self.modes)], dim=2)


class SlabColumnTransform:
    """DftForward / DftBackward of a case distributed as z-slabs (physical)
    and spectral columns: local plane transforms plus the exchange.

    plane_forward(phys, spec, planes) / plane_backward(spec, phys, planes):
    the local x-y transforms of `planes` contiguous z planes; by default those
    of the library (tg_dft_forward_planes / tg_dft_backward_planes) through a
    ChannelCase of the same Nx, Ny (its own Nz plays no part).
    """

    def __init__(self, nx: int, ny: int, nz: int, dist=None, group=None, case=None,
                 plane_forward: Optional[Callable] = None, plane_backward: Optional[Callable] = None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nyc = ny // 3 * 2
        self.nxh = nx // 3 * 2 // 2 + 1
        self.M = self.nyc * self.nxh
        self.ex = SlabColumnExchange(nz, self.M, dist, group)
        if plane_forward is None or plane_backward is None:
            if case is None:
                raise ValueError("SlabColumnTransform > a ChannelCase or both plane transforms are needed")
            plane_forward = plane_forward or self._case_forward(case)
            plane_backward = plane_backward or self._case_backward(case)
        self.plane_forward, self.plane_backward = plane_forward, plane_backward

    @staticmethod
    def _case_forward(case):
        def f(phys: torch.Tensor, spec: torch.Tensor, planes: int):
            case.dft_forward_planes(phys.data_ptr(), spec.data_ptr(), planes, fp32=phys.dtype == torch.float32)
        return f

    @staticmethod
    def _case_backward(case):
        def f(spec: torch.Tensor, phys: torch.Tensor, planes: int):
            case.dft_backward_planes(spec.data_ptr(), phys.data_ptr(), planes, fp32=phys.dtype == torch.float32)
        return f

    def forward(self, phys_slab: torch.Tensor) -> torch.Tensor:
        """(dim, my planes, Ny, Nx) real -> (dim, Nz, my modes) complex128."""
        dim, nzl = phys_slab.shape[:2]
        spec = torch.empty((dim, nzl, self.M), dtype=torch.complex128, device=phys_slab.device)
        self.plane_forward(phys_slab.contiguous(), spec, dim * nzl)
        return self.ex.to_columns(spec)

    def backward(self, cols: torch.Tensor, dtype=torch.float64) -> torch.Tensor:
        """(dim, Nz, my modes) complex128 -> (dim, my planes, Ny, Nx) real."""
        slab = self.ex.to_slabs(cols.contiguous())
        dim, nzl = slab.shape[:2]
        phys = torch.empty((dim, nzl, self.ny, self.nx), dtype=dtype, device=cols.device)
        self.plane_backward(slab.contiguous(), phys, dim * nzl)
        return phys
