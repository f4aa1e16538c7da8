"""Slab decomposition's exchanges over real process groups (gloo, world size
2, CPU): particle routing, the mesh halo shifts in both directions and the
distributed rFFT transposes (one source to three force slabs, and the
adjoint's three cotangent slabs to one) give what the one-process LocalComm
gives, and the distributed transforms with plain multipliers equal the full
numpy transforms; a routing over capacity raises the same error on every rank
and leaves the group usable.  The device kernels (deposit, gather, Green multiplier) are covered on the GPU by
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


def _green_adjoint(slab, post):
    """torch restatement of the transposed multiplier on rank r's ky slab:
    K * sum_d conj(i c_d) A_d * post (K as in _green)."""
    def g(r, spec3):
        t = slab.tables(r, spec3.device)
        _, nx, nyl, nzh = spec3.shape
        kx, ky, kz = t[:nx], t[nx:nx + nyl], t[nx + nyl:nx + nyl + nzh]
        o = nx + nyl + nzh
        cx, cy, cz = t[o:o + nx], t[o + nx:o + nx + nyl], t[o + nx + nyl:o + nx + nyl + nzh]
        o2 = 2 * o
        mx, my, mz = t[o2:o2 + nx], t[o2 + nx:o2 + nx + nyl], t[o2 + nx + nyl:o2 + nx + nyl + nzh]
        k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
        m = mx[:, None, None] * my[None, :, None] * mz[None, None, :]
        K = torch.where(k2 > 0, -m / torch.where(k2 > 0, k2, torch.ones_like(k2)), torch.zeros_like(k2))
        c = [cx[:, None, None], cy[None, :, None], cz[None, None, :]]
        acc = sum(-1j * cd * spec3[d] for d, cd in enumerate(c))
        return (acc * K * post)[None]
    return g


def _full_fields3(conf):
    nx, ny, nz = conf.mesh_shape
    rng = np.random.default_rng(21)
    return rng.normal(size=(3, nx, ny, nz)).astype(np.float32)


def _work_adjoint(slab):
    full = torch.from_numpy(_full_fields3(slab.conf))
    fields = [full[:, r * slab.nxl:(r + 1) * slab.nxl].clone() for r in slab.comm.local]
    G = slab._spectral(fields, _green_adjoint(slab, 0.25), 1)
    planes = slab.comm.shift([f[:, slab.nxl - 1].clone() for f in fields], 1)
    return G, planes


def _rank_adjoint(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pmpp_b200.slab import ProcessGroupComm, SlabPM
        G, planes = _work_adjoint(SlabPM(_conf(), ProcessGroupComm()))
        q.put((rank, [g.numpy() for g in G], [p.numpy() for p in planes]))
    finally:
        dist.destroy_process_group()


def test_process_group_adjoint_exchanges_match_local_comm():
    """The force adjoint's exchanges: the halo plane sent to the next rank
    (shift +1) and the distributed transform of three cotangent slabs into one
    with the transposed multiplier, over gloo, equal LocalComm's bitwise and
    the full numpy transform irfft(K sum_d conj(i c_d) rfft(A_d)) / 4 within 1e-5."""
    from pmpp_b200.slab import LocalComm, SlabPM
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_adjoint, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        r, G, planes = q.get(timeout=240)
        got[r] = (G, planes)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    conf = _conf()
    slab = SlabPM(conf, LocalComm(2))
    G, planes = _work_adjoint(slab)
    for r in range(2):
        np.testing.assert_array_equal(got[r][0][0], G[r].numpy())
        np.testing.assert_array_equal(got[r][1][0], planes[r].numpy())
    # each rank receives the last plane of the rank before it
    full = _full_fields3(conf)
    for r in range(2):
        src = (r - 1) % 2
        np.testing.assert_array_equal(planes[r].numpy(), full[:, (src + 1) * slab.nxl - 1])
    nx, ny, nz = conf.mesh_shape
    kx, ky, kz = (np.asarray(k, np.float64) for k in conf.kvec)
    m = [np.asarray(v, np.float64) for v in conf.particle_nyquist_masks()]
    k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        K = np.where(k2 > 0, -m[0][:, None, None] * m[1][None, :, None] * m[2][None, None, :] / k2, 0.0)
    c = [np.asarray(conf._neg_k(k, conf.cell_size), np.float64) for k in conf.kvec]
    cs = (c[0][:, None, None], c[1][None, :, None], c[2][None, None, :])
    f64 = full.astype(np.float64)
    spec = sum(-1j * cd * np.fft.rfftn(f64[d]) for d, cd in enumerate(cs))
    ref = np.fft.irfftn(K * spec * 0.25, s=(nx, ny, nz)) * (nx * ny * nz)
    got_full = np.concatenate([G[0][0].numpy(), G[1][0].numpy()], axis=0)
    assert np.abs(got_full - ref).max() / np.abs(ref).max() < 1e-5
