"""Slab decomposition's exchanges over real process groups (gloo, world size
2, CPU): particle routing, the mesh halo shifts and the distributed rFFT
transposes give what the one-process LocalComm gives, and the distributed
transform with a plain multiplier equals the full numpy transform; a routing
over capacity raises the same error on every rank and leaves the group
usable.  The device kernels (deposit, gather, Green multiplier) are covered on the GPU by
tests/test_gpu_slab.py; here the multiplier is a torch restatement.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _conf():
    import pmpp_b200 as pb
    return pb.Configuration(4.0, (16, 16, 16), 2, a_start=0.1, device="cpu")


def _particles(conf, seed=1):
    rng = np.random.default_rng(seed)
    n = 2000
    nx, ny, nz = conf.mesh_shape
    pmid = rng.integers(0, [nx, ny, nz], size=(n, 3)).astype(np.int16)
    disp = rng.normal(0, 3 * conf.cell_size, size=(n, 3)).astype(np.float32)
    vel = rng.normal(size=(n, 3)).astype(np.float32)
    return torch.from_numpy(pmid), torch.from_numpy(disp), torch.from_numpy(vel)


def _green(slab):
    """torch restatement of the multiplier on rank r's ky slab (continuum Green,
    masks, spectral gradient, post scale 1/cells)."""
    def g(r, spec):
        t = slab.tables(r, spec.device)
        nx, nyl, nzh = spec.shape
        kx, ky, kz = t[:nx], t[nx:nx + nyl], t[nx + nyl:nx + nyl + nzh]
        o = nx + nyl + nzh
        cx, cy, cz = t[o:o + nx], t[o + nx:o + nx + nyl], t[o + nx + nyl:o + nx + nyl + nzh]
        o2 = 2 * o
        mx, my, mz = t[o2:o2 + nx], t[o2 + nx:o2 + nx + nyl], t[o2 + nx + nyl:o2 + nx + nyl + nzh]
        k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
        m = mx[:, None, None] * my[None, :, None] * mz[None, None, :]
        K = torch.where(k2 > 0, -m / torch.where(k2 > 0, k2, torch.ones_like(k2)), torch.zeros_like(k2))
        phi = spec * K / slab.conf.mesh_size
        c = [cx[:, None, None], cy[None, :, None], cz[None, None, :]]
        return torch.stack([1j * cd * phi for cd in c])
    return g


def _work(slab, pmid, disp, vel):
    states = slab.distribute(pmid, disp, vel)
    moved = []
    for s in states:  # move every particle by about a slab so that most change rank
        s.disp = s.disp + torch.tensor([slab.nxl * slab.conf.cell_size * 0.7, 0.0, 0.0])
        moved.append(s)
    states = slab.migrate(moved)
    nx, ny, nz = slab.conf.mesh_shape
    rng = np.random.default_rng(9)
    full = torch.from_numpy(rng.normal(size=(nx, ny, nz)).astype(np.float32))
    srcs = [full[r * slab.nxl:(r + 1) * slab.nxl].clone() for r in slab.comm.local]
    F = slab.spectral_force(srcs, green=_green(slab))
    planes = slab.comm.shift([f[0, 0] for f in F], -1)
    return ([(s.pmid, s.disp, s.vel) for s in states], F, planes)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pmpp_b200.slab import ProcessGroupComm, SlabPM
        conf = _conf()
        slab = SlabPM(conf, ProcessGroupComm())
        states, F, planes = _work(slab, *_particles(conf))
        total = slab.comm.allreduce_sum(rank + 0.5)
        q.put((rank, [tuple(t.numpy() for t in s) for s in states], [f.numpy() for f in F],
               [p.numpy() for p in planes], total))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_process_group_exchanges_match_local_comm():
    from pmpp_b200.slab import LocalComm, SlabPM
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        r, st, F, planes, total = q.get(timeout=240)
        got[r] = (st, F, planes)
        assert total == 2.0  # 0.5 + 1.5 summed over the two ranks
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # LocalComm in this process
    conf = _conf()
    slab = SlabPM(conf, LocalComm(2))
    states, F, planes = _work(slab, *_particles(conf))
    for r in range(2):
        gs, gF, gp = got[r]
        for a, b in zip(gs[0], states[r]):
            np.testing.assert_array_equal(a, b.numpy())
        np.testing.assert_array_equal(gF[0], F[r].numpy())
        np.testing.assert_array_equal(gp[0], planes[r].numpy())
    # the distributed transform equals the full one
    nx, ny, nz = conf.mesh_shape
    rng = np.random.default_rng(9)
    full = rng.normal(size=(nx, ny, nz)).astype(np.float32).astype(np.float64)
    kx, ky, kz = (np.asarray(k, np.float64) for k in conf.kvec)
    m = [np.asarray(v, np.float64) for v in conf.particle_nyquist_masks()]
    k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        K = np.where(k2 > 0, -m[0][:, None, None] * m[1][None, :, None] * m[2][None, None, :] / k2, 0.0)
    phi = np.fft.rfftn(full) * K
    c = [np.asarray(conf._neg_k(k, conf.cell_size), np.float64) for k in conf.kvec]
    ref = np.stack([np.fft.irfftn(1j * cd * phi, s=(nx, ny, nz)) for cd in
                    (c[0][:, None, None], c[1][None, :, None], c[2][None, None, :])])
    got_full = np.concatenate([F[0].numpy(), F[1].numpy()], axis=1)
    assert np.abs(got_full - ref).max() / np.abs(ref).max() < 1e-5
    # routing: every particle kept, each on the rank owning its cell
    total = sum(s[0].shape[0] for s in states)
    assert total == 2000
    for r, s in enumerate(states):
        assert bool(((slab.owner(s[0], s[1])) == r).all())
        keys = slab.cell_key(s[0], s[1])
        assert bool((keys[1:] >= keys[:-1]).all())  # merged in cell-key order


def _rank_capacity(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pmpp_b200.slab import ProcessGroupComm, SlabPM
        conf = _conf()
        slab = SlabPM(conf, ProcessGroupComm(), capacity=600)
        states = slab.distribute(*_particles(conf))
        for s in states:  # most particles move to the other rank
            s.disp = s.disp + torch.tensor([slab.nxl * slab.conf.cell_size * 0.9, 0.0, 0.0])
        try:
            slab.migrate(states)
            q.put((rank, "moved"))
        except RuntimeError as e:
            q.put((rank, str(e)))
        # the group still works after the refusal: no rank was left inside a collective
        q.put((rank, slab.comm.allreduce_sum(1.0)))
    finally:
        dist.destroy_process_group()


def test_process_group_routing_fails_closed_on_every_rank():
    """A capacity below a rank's incoming share makes every rank raise the same
    error before any particle moves, and the process group stays usable."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_capacity, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(4)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    msgs = [m for _, m in got if isinstance(m, str)]
    sums = [m for _, m in got if not isinstance(m, str)]
    assert len(msgs) == 2 and all("capacity" in m for m in msgs) and msgs[0] == msgs[1]
    assert sums == [2.0, 2.0]
