"""The slab decomposition's exchange layer (streams_b200.slabs) on CPU ranks (gloo): after the
halo exchange every block's face ghosts equal what the single block's periodic swap (bcswap:
face halos over the interior range, no edges or corners) puts at those points of the global
field; faces without a neighbour keep their ghosts; the bulk sums and the time step's maximum
over the ranks equal the single block's."""
import os
import socket

import numpy as np
import pytest


def free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


NG = 3


def global_field(nx, ny, nz, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((5, nz + 2 * NG, ny + 2 * NG, nx + 2 * NG))


def periodic_swap(w, nx, ny, nz, px, pz):
    """The single block's bcswap: x then z, face halos over the interior range."""
    w = w.copy()
    J, K, I = slice(NG, NG + ny), slice(NG, NG + nz), slice(NG, NG + nx)
    if px:
        w[:, K, J, 0:NG] = w[:, K, J, nx:nx + NG]
        w[:, K, J, nx + NG:nx + 2 * NG] = w[:, K, J, NG:2 * NG]
    if pz:
        w[:, 0:NG, J, I] = w[:, nz:nz + NG, J, I]
        w[:, nz + NG:nz + 2 * NG, J, I] = w[:, NG:2 * NG, J, I]
    return w


def face_mask(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(nz + 2 * NG), np.arange(ny + 2 * NG), np.arange(nx + 2 * NG), indexing="ij")
    out = ((i < NG) | (i >= nx + NG)).astype(int) + ((j < NG) | (j >= ny + NG)) + ((k < NG) | (k >= nz + NG))
    return out <= 1


def _rank(rank, world, port, cfg, q):
    import torch
    import torch.distributed as dist
    from streams_b200.slabs import Decomposition, allreduce_max, allreduce_sum, halo_exchange, scatter_blocks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nx, ny, nz, xs, zs, px, pz = cfg
        d = Decomposition(nx, ny, nz, xs, zs, px, pz, rank)
        wg = torch.from_numpy(global_field(nx, ny, nz))
        w = scatter_blocks(wg, d, NG)
        marker = w.clone()
        halo_exchange(w, d, NG, dist)
        ref = scatter_blocks(torch.from_numpy(periodic_swap(wg.numpy(), nx, ny, nz, px, pz)), d, NG)
        m = torch.from_numpy(face_mask(d.nx, d.ny, d.nz))
        ok_faces = bool(torch.equal(w[:, m], ref[:, m]))
        ok_rest = bool(torch.equal(w[:, ~m], marker[:, ~m]))  # edges and corners untouched
        # forcing sums and the time step's maximum over the ranks
        part = w[:, NG:NG + d.nz, NG:NG + d.ny, NG:NG + d.nx].sum(dim=(1, 2, 3)).clone()
        allreduce_sum(part, dist)
        tmax = w[0, NG:NG + d.nz, NG:NG + d.ny, NG:NG + d.nx].max().reshape(1).clone()
        allreduce_max(tmax, dist)
        q.put((rank, ok_faces, ok_rest, part.numpy(), float(tmax)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("cfg,world", [
    ((16, 6, 8, 2, 1, True, True), 2),     # channel: x split in two, periodic
    ((16, 6, 8, 1, 2, True, True), 2),     # z split in two
    ((16, 6, 8, 2, 2, True, True), 4),     # both
    ((16, 6, 8, 2, 1, False, True), 2),    # boundary layer: x open (inflow / outflow ghosts kept)
    ((24, 6, 8, 3, 1, False, True), 3),
], ids=["x2", "z2", "x2z2", "x2_open", "x3_open"])
def test_halo_exchange_matches_the_single_block_swap(cfg, world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, cfg, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nx, ny, nz = cfg[:3]
    wg = global_field(nx, ny, nz)
    total = wg[:, NG:NG + nz, NG:NG + ny, NG:NG + nx].sum(axis=(1, 2, 3))
    tmax = wg[0, NG:NG + nz, NG:NG + ny, NG:NG + nx].max()
    for rank, ok_faces, ok_rest, part, t in res:
        assert ok_faces and ok_rest, rank
        assert np.allclose(part, total, rtol=1e-12, atol=1e-12)
        assert t == tmax


def test_decomposition_follows_mpi_cart_order():
    from streams_b200.slabs import Decomposition
    d = Decomposition(64, 32, 48, 2, 3, True, True, rank=4)
    assert d.coords == (1, 0, 1) and (d.nx, d.ny, d.nz) == (32, 32, 16) and d.offset == (32, 0, 16)
    assert d.neighbours() == {"xl": 1, "xr": 1, "zl": 3, "zr": 5}
    e = Decomposition(64, 32, 48, 2, 3, False, True, rank=0)
    assert e.neighbours()["xl"] is None and e.neighbours()["xr"] == 3 and e.neighbours()["zl"] == 2
    with pytest.raises(ValueError):
        Decomposition(65, 32, 48, 2, 1, True, True, rank=0)
