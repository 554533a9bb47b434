"""Slab decomposition of a box over several GPUs: the host-side exchange logic.

The reference splits the block over an MPI Cartesian topology in x and z (y unsplit for
wall-bounded cases; field.F90:223-276, cartesian_mpi) and, every stage, swaps ng ghost planes of
the five conserved variables with the x and z neighbours (bcswap, base_cpu.F90:1326-1435: face
halos only, interior j and the other direction's interior range, no edges or corners), and sums
the forcing's bulk partials over all ranks (mpi_allreduce, singleideal_cpu.F90:861, 914) and the
time step's inverse time scales with a maximum (:1513).  This module restates that plumbing over
``torch.distributed``: NCCL between GPUs of one node (each message lands in the receiver's own
buffer), gloo on CPU for the tests.  Ranks are ordered as MPI_Cart_create orders them (row-major
over (x_split, y_split, z_split), no reordering).

Scope: this is the decomposition and exchange layer only.  The device stage kernels read the
periodic ghosts of a split direction by index wrapping inside one block and keep the sensor and
div/3 without ghost layers, so running the stage on a slab needs those arrays ghosted and filled
by this exchange; that is not built, and ``bench.py --gpus N`` runs N independent replicas.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Decomposition:
    """One rank's block of an (nxmax, nymax, nzmax) box split (x_split, 1, z_split)."""

    nxmax: int
    nymax: int
    nzmax: int
    x_split: int
    z_split: int
    periodic_x: bool
    periodic_z: bool
    rank: int

    def __post_init__(self):
        if self.nxmax % self.x_split or self.nzmax % self.z_split:
            raise ValueError("nxmax and nzmax must be multiples of x_split and z_split")
        if not 0 <= self.rank < self.x_split * self.z_split:
            raise ValueError("rank outside the topology")

    @property
    def size(self) -> int:
        return self.x_split * self.z_split

    @property
    def coords(self) -> tuple[int, int, int]:
        # MPI_Cart_create with reorder = .false.: the last dimension varies fastest
        return self.rank // self.z_split, 0, self.rank % self.z_split

    @property
    def nx(self) -> int:
        return self.nxmax // self.x_split

    @property
    def ny(self) -> int:
        return self.nymax

    @property
    def nz(self) -> int:
        return self.nzmax // self.z_split

    @property
    def offset(self) -> tuple[int, int, int]:
        """Global index of the block's first interior cell minus one (i = offset + i_local)."""
        cx, _, cz = self.coords
        return cx * self.nx, 0, cz * self.nz

    def rank_of(self, cx: int, cz: int) -> int | None:
        if self.periodic_x:
            cx %= self.x_split
        if self.periodic_z:
            cz %= self.z_split
        if not (0 <= cx < self.x_split and 0 <= cz < self.z_split):
            return None
        return cx * self.z_split + cz

    def neighbours(self) -> dict[str, int | None]:
        """mpi_cart_shift's left/right neighbours in x and z (None at a non-periodic boundary)."""
        cx, _, cz = self.coords
        return {"xl": self.rank_of(cx - 1, cz), "xr": self.rank_of(cx + 1, cz),
                "zl": self.rank_of(cx, cz - 1), "zr": self.rank_of(cx, cz + 1)}


def _shift(dist, send, dst, recv, src, group=None) -> None:
    """One shift of a halo exchange: every rank sends at most one message and receives at most
    one, so the messages match even when both neighbours are the same rank (two blocks in a
    periodic direction) and whatever the backend's tag support."""
    reqs = []
    if recv is not None and src is not None:
        reqs.append(dist.irecv(recv, src=src, group=group))
    if send is not None and dst is not None:
        reqs.append(dist.isend(send, dst=dst, group=group))
    for r in reqs:
        r.wait()


def halo_exchange(w, d: Decomposition, ng: int, dist, group=None) -> None:
    """bcswap of the block's ghosted array w (any leading variable axis, then z, y, x with ng ghost
    layers; a torch tensor on the process's device): ng planes to and from the x neighbours over
    the interior (j, k) range, then the same in z over the interior (i, j) range.  A direction with
    one block in a periodic topology exchanges with itself (a periodic copy); faces without a
    neighbour keep their ghosts (the boundary conditions fill them)."""
    nb = d.neighbours()
    nx, ny, nz = d.nx, d.ny, d.nz
    J = slice(ng, ng + ny)
    K = slice(ng, ng + nz)
    I = slice(ng, ng + nx)
    for axis, (left, right), n in ((-1, (nb["xl"], nb["xr"]), nx), (-3, (nb["zl"], nb["zr"]), nz)):

        def plane(a, b):
            if axis == -1:
                return (Ellipsis, K, J, slice(a, b))
            return (Ellipsis, slice(a, b), J, I)

        lo_int, hi_int = plane(ng, 2 * ng), plane(n, n + ng)      # planes sent left / right
        lo_gh, hi_gh = plane(0, ng), plane(n + ng, n + 2 * ng)    # ghosts filled from left / right
        if left == d.rank and right == d.rank:
            # one block in a periodic direction: the swap is a copy within the block
            lo, hi = w[lo_int].clone(), w[hi_int].clone()
            w[lo_gh] = hi
            w[hi_gh] = lo
            continue
        # shift right: the right interior planes go to the right neighbour's left ghosts
        buf = w[lo_gh].contiguous() if left is not None else None
        _shift(dist, w[hi_int].contiguous() if right is not None else None, right, buf, left, group)
        if buf is not None:
            w[lo_gh] = buf
        # shift left: the left interior planes go to the left neighbour's right ghosts
        buf = w[hi_gh].contiguous() if right is not None else None
        _shift(dist, w[lo_int].contiguous() if left is not None else None, left, buf, right, group)
        if buf is not None:
            w[hi_gh] = buf


def allreduce_sum(partials, dist, group=None):
    """The forcing's bulk sums over all ranks (mpi_allreduce with mpi_sum), in place."""
    dist.all_reduce(partials, op=dist.ReduceOp.SUM, group=group)
    return partials


def allreduce_max(values, dist, group=None):
    """The time step's inverse time scales over all ranks (mpi_allreduce with mpi_max)."""
    dist.all_reduce(values, op=dist.ReduceOp.MAX, group=group)
    return values


def scatter_blocks(w_global, d: Decomposition, ng: int):
    """The block of rank d.rank cut from a global ghosted field (the halos as the global field
    holds them): for tests and for distributing a set-up's initial field."""
    ox, _, oz = d.offset
    return w_global[..., oz:oz + d.nz + 2 * ng, :, ox:ox + d.nx + 2 * ng].clone()
