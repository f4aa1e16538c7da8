"""Kick-drift-kick time integration and the hand-written reverse sweep.

Forward (nbody/solver.py:253-273, nbody/integrator.py:689-731): an initial
force, then per macro step the stages of ``symp_splits``.  With the default
splits ((0, .5), (1, .5)) a step is  kick(a_p -> a_m), drift(a_p -> a_n),
force(a_n), kick(a_m -> a_n); the drift is fused into the cell sort and the
closing half-kick into the force gather, so a step is one axpy plus one
fused force call.

Reverse (nbody/solver.py:385-444, integrator.py:781-837): states are rebuilt
algebraically (vel -= acc K, disp -= vel D) and the force at the earlier time
is recomputed.  The force meshes of that recomputation are exactly the ones
the next reverse step's force adjoint needs (same positions), so they are
kept instead of being recomputed a third time: a reverse step costs one
force adjoint plus one forward force.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call, pmfft_active
from .gravity import force, force_vjp, _om32
from .particles import Particles
from .runtime import stream_handle


def _schedule(a_prev, a_next, conf):
    """Stage list of one macro step (integrator.py:760-778)."""
    D = K = 0
    a_disp = a_vel = a_acc = a_prev
    stages = []
    for d, k in conf.symp_splits:
        if d != 0:
            D += d
            a_disp_next = a_prev * (1 - D) + a_next * D
            stages.append(("drift", a_vel, a_disp, a_disp_next, a_acc))
            a_disp = a_disp_next
            a_acc = a_disp
        if k != 0:
            K += k
            a_vel_next = a_prev * (1 - K) + a_next * K
            stages.append(("kick", a_acc, a_vel, a_vel_next))
            a_vel = a_vel_next
    return stages


def _f32(x):
    return float(np.float32(x))


def kick(a_acc, a_prev, a_next, ptcl, cosmo, conf):
    """vel += acc * K (integrator.py:512-538), in place on a copy of vel."""
    vel = ptcl.vel.clone()
    if vel.dtype == torch.float64:
        from . import x64
        x64.axpy(vel, ptcl.acc, cosmo.kick_factor(a_acc, a_prev, a_next))
        return ptcl.replace(vel=vel)
    K = _f32(cosmo.kick_factor(a_acc, a_prev, a_next))
    call("pmb_axpy", vel.data_ptr(), ptcl.acc.data_ptr(), vel.numel(), K, stream_handle(vel.device))
    return ptcl.replace(vel=vel)


def drift(a_vel, a_prev, a_next, ptcl, cosmo, conf):
    """disp += vel * D (integrator.py:202-237)."""
    disp = ptcl.disp.clone()
    if disp.dtype == torch.float64:
        from . import x64
        x64.axpy(disp, ptcl.vel, cosmo.drift_factor(a_vel, a_prev, a_next))
        return ptcl.replace(disp=disp)
    D = _f32(cosmo.drift_factor(a_vel, a_prev, a_next))
    call("pmb_axpy", disp.data_ptr(), ptcl.vel.data_ptr(), disp.numel(), D, stream_handle(disp.device))
    return ptcl.replace(disp=disp)


def force_state(a, ptcl, cosmo, conf, correction=None):
    """Overwrite acc with the PM force (integrator.py:595-617)."""
    acc, _ = force(ptcl.pmid, ptcl.disp, conf, cosmo.Omega_m, a=a, cosmo=cosmo, correction=correction)
    return ptcl.replace(acc=acc)


def integrate(a_prev, a_next, ptcl, cosmo, conf, correction=None):
    """One macro step with the configured splitting (integrator.py:689-731)."""
    for st in _schedule(a_prev, a_next, conf):
        if st[0] == "drift":
            ptcl = drift(st[1], st[2], st[3], ptcl, cosmo, conf)
            ptcl = force_state(st[3], ptcl, cosmo, conf, correction)
        else:
            ptcl = kick(st[1], st[2], st[3], ptcl, cosmo, conf)
    return ptcl


# ---------------------------------------------------------------------------
# Per-operation adjoints (nbody/integrator.py:429-509, 541-582, 620-686,
# 781-837).  The cosmology cotangent is the Omega_m cotangent, a float: the
# time factors depend on the cosmology through the growth tables of Omega_m,
# and the force is linear in Omega_m.  NBodyRun.adjoint runs the same
# operations fused; these are the step-by-step forms.
# ---------------------------------------------------------------------------
def _zeros_like(t, ref):
    return torch.zeros_like(ref) if t is None else t.clone().to(ref.dtype).contiguous()


def kick_adj(a_acc, a_prev, a_next, ptcl, ptcl_cot, cosmo, cosmo_cot, conf):
    """Reverse a kick from the post-kick state (integrator.py:541-582):
    vel_in = vel - acc K, acc_cot += vel_cot K, cosmo_cot += dK/dOmega_m
    sum(vel_cot acc).  Returns (ptcl_in, ptcl_cot_in, cosmo_cot)."""
    K, dK = cosmo.kick_factor(a_acc, a_prev, a_next, with_grad=True)
    vel = ptcl.vel.clone()
    vc = _zeros_like(ptcl_cot.vel, vel)
    ac = _zeros_like(ptcl_cot.acc, vel)
    dot = torch.zeros(1, dtype=torch.float64, device=vel.device)
    if vel.dtype == torch.float64:
        from . import x64
        x64.dot(vc, ptcl.acc, dot, 0)
        x64.axpy(vel, ptcl.acc, -K)
        x64.axpy(ac, vc, K)
        return ptcl.replace(vel=vel), ptcl_cot.replace(vel=vc, acc=ac), float(cosmo_cot) + dK * float(dot.item())
    call("pmb_kick_adj", vel.data_ptr(), ptcl.acc.data_ptr(), vc.data_ptr(), ac.data_ptr(), vel.numel(), _f32(K),
         dot.data_ptr(), stream_handle(vel.device))
    return ptcl.replace(vel=vel), ptcl_cot.replace(vel=vc, acc=ac), float(cosmo_cot) + dK * float(dot.item())


def drift_adj_from_output(a_vel, a_prev, a_next, ptcl, ptcl_cot, cosmo, cosmo_cot, conf):
    """Reverse a drift from the post-drift state (integrator.py:429-509):
    disp_in = disp - vel D, vel_cot += disp_cot D, cosmo_cot += dD/dOmega_m
    sum(disp_cot vel).  Returns (ptcl_in, ptcl_cot_in, cosmo_cot)."""
    D, dD = cosmo.drift_factor(a_vel, a_prev, a_next, with_grad=True)
    disp = ptcl.disp.clone()
    dc = _zeros_like(ptcl_cot.disp, disp)
    vc = _zeros_like(ptcl_cot.vel, disp)
    dot = torch.zeros(1, dtype=torch.float64, device=disp.device)
    if disp.dtype == torch.float64:
        from . import x64
        x64.axpy(disp, ptcl.vel, -D)
        x64.axpy(vc, dc, D)
        x64.dot(dc, ptcl.vel, dot, 0)
        return ptcl.replace(disp=disp), ptcl_cot.replace(disp=dc, vel=vc), float(cosmo_cot) + dD * float(dot.item())
    call("pmb_drift_adj", disp.data_ptr(), ptcl.vel.data_ptr(), dc.data_ptr(), vc.data_ptr(), disp.numel(), _f32(D),
         dot.data_ptr(), stream_handle(disp.device))
    return ptcl.replace(disp=disp), ptcl_cot.replace(disp=dc, vel=vc), float(cosmo_cot) + dD * float(dot.item())


def force_adj(a, ptcl, ptcl_cot, cosmo, conf, correction=None):
    """Pull the acceleration cotangent through one force evaluation
    (integrator.py:620-686): disp_cot += (d acc / d disp)^T acc_cot, acc_cot
    -> 0, and the Omega_m cotangent sum(acc_cot acc) / Omega_m (the force is
    linear in Omega_m).  Returns (ptcl with acc recomputed, ptcl_cot_in,
    Omega_m cotangent, None: the correction's own cotangent is trained through
    pmpp_b200.learned)."""
    acc, F = force(ptcl.pmid, ptcl.disp.clone(), conf, cosmo.Omega_m, a=a, cosmo=cosmo, correction=correction)
    ac = _zeros_like(ptcl_cot.acc, acc)
    dc = _zeros_like(ptcl_cot.disp, acc)
    om_out = []
    force_vjp(ptcl.pmid, ptcl.disp, conf, cosmo.Omega_m, F, ac, dc, a=a, cosmo=cosmo, correction=correction,
              om_out=om_out)
    om_div = float(cosmo.Omega_m) if acc.dtype == torch.float64 else _om32(cosmo.Omega_m)
    om = om_out[0] if om_out else float((ac.double() * acc.double()).sum()) / om_div
    return ptcl.replace(acc=acc), ptcl_cot.replace(disp=dc, acc=torch.zeros_like(ac)), om, None


def integrate_adj(a_prev, a_next, ptcl, ptcl_cot, cosmo, cosmo_cot, conf, correction=None, correction_cot=None):
    """Reverse one macro step (integrator.py:781-837) with the stage adjoints
    above, restoring the incoming acceleration after each force stage.
    Returns (ptcl_in, ptcl_cot_in, cosmo_cot, correction_cot)."""
    for st in reversed(_schedule(a_prev, a_next, conf)):
        if st[0] == "kick":
            ptcl, ptcl_cot, cosmo_cot = kick_adj(st[1], st[2], st[3], ptcl, ptcl_cot, cosmo, cosmo_cot, conf)
            continue
        _, a_vel, a_disp, a_disp_next, a_acc_in = st
        ptcl, ptcl_cot, om, _ = force_adj(a_disp_next, ptcl, ptcl_cot, cosmo, conf, correction)
        cosmo_cot = float(cosmo_cot) + om
        ptcl, ptcl_cot, cosmo_cot = drift_adj_from_output(a_vel, a_disp, a_disp_next, ptcl, ptcl_cot, cosmo,
                                                          cosmo_cot, conf)
        ptcl = force_state(a_acc_in, ptcl, cosmo, conf, correction)
    return ptcl, ptcl_cot, cosmo_cot, correction_cot


class NBodyRun:
    """Fused forward integration that keeps the final force meshes for the adjoint."""

    def __init__(self, conf, cosmo, correction=None, overlap=False):
        self.conf = conf
        self.cosmo = cosmo
        self.correction = correction
        # reverse sweep: run each force recompute on a side stream beside the
        # force adjoint it does not depend on (results are unchanged).  Off by
        # default: at 512^3 / 1024^3 the step went 3.54 -> 4.03 s, the
        # persistent FFT passes (static tile order, one CTA per SM) stalling
        # behind the other stream's CTAs.
        self.overlap = overlap

    def forward(self, ptcl, a_nbody=None):
        conf, cosmo = self.conf, self.cosmo
        if conf.float_dtype == torch.float64:
            from . import x64
            return x64.nbody(ptcl, cosmo, conf, a_nbody, correction=self.correction)
        a = conf.a_nbody if a_nbody is None else np.asarray(a_nbody)
        disp = ptcl.disp.clone()
        vel = ptcl.vel.clone() if ptcl.vel is not None else torch.zeros_like(disp)
        acc = torch.empty_like(disp)
        F = torch.empty((3, ) + conf.mesh_shape, dtype=torch.float32, device=disp.device)
        s = stream_handle(disp.device)
        S = self._src_hat_buffer(disp.device)
        # stage list of the whole run; every force evaluation takes the kicks
        # that directly follow it (a step's closing kick and the next step's
        # opening kick share its acceleration) into its gather
        ops = [("init", )]
        for a_prev, a_next in zip(a[:-1], a[1:]):
            ops.extend(_schedule(a_prev, a_next, conf))
        i = 0
        while i < len(ops):
            st = ops[i]
            if st[0] == "kick":  # a kick with no force evaluation before it
                call("pmb_axpy", vel.data_ptr(), acc.data_ptr(), vel.numel(),
                     _f32(cosmo.kick_factor(st[1], st[2], st[3])), s)
                i += 1
                continue
            ks = []
            while i + 1 + len(ks) < len(ops) and ops[i + 1 + len(ks)][0] == "kick" and len(ks) < 2:
                k = ops[i + 1 + len(ks)]
                ks.append(_f32(cosmo.kick_factor(k[1], k[2], k[3])))
            kick_f = ks[0] if ks else 0.0
            kick2 = ks[1] if len(ks) == 2 else 0.0
            vk = vel if ks else None
            # the acceleration is needed only if a later op reads it before the
            # next force overwrites it (an unfolded kick, or the returned state)
            j = i + 1 + len(ks)
            keep = vk is None or j >= len(ops) or ops[j][0] != "drift"
            if st[0] == "init":
                force(ptcl.pmid, disp, conf, cosmo.Omega_m, a=float(a[0]), cosmo=cosmo, correction=self.correction,
                      force_meshes=F, acc=acc, vel_kick=vk, kick=kick_f, kick2=kick2, src_hat_out=S, keep_acc=keep)
            else:
                D = _f32(cosmo.drift_factor(st[1], st[2], st[3]))
                force(ptcl.pmid, disp, conf, cosmo.Omega_m, a=float(st[3]), cosmo=cosmo, correction=self.correction,
                      force_meshes=F, acc=acc, drift_vel=vel, drift=D, vel_kick=vk, kick=kick_f, kick2=kick2,
                      src_hat_out=S, keep_acc=keep)
            i += 1 + len(ks)
        self.final_meshes = F
        self.final_src_hat = S
        return ptcl.replace(disp=disp, vel=vel, acc=acc)

    def _trainable(self):
        return self.correction is not None and getattr(self.correction, "trainable", False)

    def _src_hat_buffer(self, device):
        """Source-spectrum buffer, only when a trainable correction needs it in the adjoint."""
        if not self._trainable():
            return None
        nx, ny, nz = self.conf.mesh_shape
        return torch.empty((nx, ny, nz // 2 + 1), dtype=torch.complex64, device=device)

    def _force_adjoint(self, pmid, disp, F, S, ac, dc, a, presorted=False, lane="", concurrent=False):
        """Force adjoint; with a trainable correction also its parameter gradient.

        presorted: the force() call with this lane was at exactly these positions."""
        conf, cosmo, corr = self.conf, self.cosmo, self.correction
        if self._trainable():
            from .corrections import radial_table_len
            tc = torch.zeros(radial_table_len(conf), dtype=torch.float64, device=disp.device)
            force_vjp(pmid, disp, conf, cosmo.Omega_m, F, ac, dc, a=a, cosmo=cosmo, correction=corr, src_hat=S,
                      transfer_cot_out=tc, presorted=presorted, sorted_lane=lane, concurrent=concurrent)
            corr.accumulate(a, cosmo, conf, tc)
        else:
            force_vjp(pmid, disp, conf, cosmo.Omega_m, F, ac, dc, a=a, cosmo=cosmo, correction=corr,
                      presorted=presorted, sorted_lane=lane, concurrent=concurrent, om_out=self._om_exact)

    def _require_f32(self):
        if self.conf.float_dtype != torch.float32:
            raise NotImplementedError("the hand-written adjoints exist for the float32 build")

    def adjoint(self, ptcl, ptcl_cot, force_meshes=None, a_nbody=None, src_hat=None):
        """Reverse sweep from the final state.  Returns (ptcl_in, ptcl_in_cot, Omega_m_cot).

        force_meshes must be the force meshes at ptcl's positions (the
        forward pass leaves them in self.final_meshes)."""
        conf, cosmo, corr = self.conf, self.cosmo, self.correction
        a = conf.a_nbody if a_nbody is None else np.asarray(a_nbody)
        if conf.float_dtype == torch.float64:
            from . import x64
            return x64.nbody_adj(ptcl, ptcl_cot, cosmo, conf, a, force_meshes, correction=corr)
        dev = ptcl.disp.device
        s = stream_handle(dev)
        pmid = ptcl.pmid
        disp, vel, acc = ptcl.disp.clone(), ptcl.vel.clone(), ptcl.acc.clone()
        dc = ptcl_cot.disp.clone().float().contiguous()
        vc = (ptcl_cot.vel if ptcl_cot.vel is not None else torch.zeros_like(dc)).clone().float().contiguous()
        ac = (ptcl_cot.acc if ptcl_cot.acc is not None else torch.zeros_like(dc)).clone().float().contiguous()
        F = self.final_meshes if force_meshes is None else force_meshes
        F2 = torch.empty_like(F)
        S = (self.final_src_hat if src_hat is None else src_hat) if self._trainable() else None
        S2 = self._src_hat_buffer(dev)
        # reversed stage list of the whole run, then the initial force evaluation
        ops = []
        for a_prev, a_next in zip(a[:-1][::-1], a[1:][::-1]):
            ops.extend(reversed(_schedule(a_prev, a_next, conf)))
        ops.append(("init", ))
        dots = torch.zeros(2 * len(ops) + 2, dtype=torch.float64, device=dev)
        # forces whose Omega_m cotangent is not sum(acc_cot acc) / Omega_m
        # (the mesh-CNN correction) report it here instead
        self._om_exact = []
        grads = []  # (d factor / d Omega_m, dot slot) pairs, reduced on the host at the end
        force_slots = []
        slot = 0
        om32 = _om32(cosmo.Omega_m)
        n3 = vel.numel()
        # after the first force adjoint every one follows the force recompute at
        # the same positions (the kick adjoints between them move no particle)
        recomputed = False
        zero_pending = False  # acc_cot consumed by a force adjoint, not yet cleared
        force_dot_done = False
        # The recompute at the previous positions needs only vel (after the kick
        # adjoints) and disp; the force adjoint at the current positions reads
        # its sorted records, meshes and cotangents.  With overlap the recompute
        # runs on a side stream beside it, the drift's position half fused into
        # its sort, alternating two sorted-record lanes.
        overlap = (self.overlap and dev.type == "cuda" and not self._trainable()
                   and pmfft_active(*conf.mesh_shape))
        main = torch.cuda.current_stream(dev) if dev.type == "cuda" else None
        side = torch.cuda.Stream(device=dev) if overlap else None
        ev_force = None  # side-stream force that main must see before touching vel / acc
        lane = 0  # lane holding the sorted records of the current positions
        # the cotangent half of a drift adjoint waiting to run inside the next
        # kick adjoints' pass (D, dot slot), or alone before a force adjoint
        drift_pending = None

        def flush_drift():
            nonlocal drift_pending
            if drift_pending is not None:
                call("pmb_drift_cot_adj", vel.data_ptr(), dc.data_ptr(), vc.data_ptr(), disp.numel(), drift_pending[0],
                     dots[drift_pending[1]:].data_ptr(), s)
                drift_pending = None

        i = 0
        while i < len(ops):
            st = ops[i]
            if ev_force is not None:
                main.wait_event(ev_force)
                ev_force = None
            if st[0] == "kick":
                # consecutive kick adjoints share acc: one kernel for up to two,
                # which also forms the force-slot dot of a following force adjoint
                ks = [st] + ([ops[i + 1]] if i + 1 < len(ops) and ops[i + 1][0] == "kick" else [])
                j = i + len(ks)
                force_next = j < len(ops) and ops[j][0] in ("drift", "init")
                Ks = [cosmo.kick_factor(k[1], k[2], k[3], with_grad=True) for k in ks]
                two = len(ks) == 2
                sa = slot
                sb = slot + 1 if two else None
                sf = slot + len(ks) if force_next else None
                slot += len(ks) + (1 if force_next else 0)
                dp = drift_pending
                call("pmb_kick_adj3", vel.data_ptr(), acc.data_ptr(), vc.data_ptr(), ac.data_ptr(), n3,
                     _f32(Ks[0][0]), _f32(Ks[1][0]) if two else 0.0, int(two), int(zero_pending),
                     dots[sa:].data_ptr(), dots[sb:].data_ptr() if two else None,
                     dots[sf:].data_ptr() if force_next else None, dc.data_ptr() if dp else None,
                     dp[0] if dp else 0.0, dots[dp[1]:].data_ptr() if dp else None, s)
                drift_pending = None
                grads.append((Ks[0][1], sa))
                if two:
                    grads.append((Ks[1][1], sb))
                if force_next:
                    force_slots.append(sf)
                    force_dot_done = True
                zero_pending = False
                i = j
                continue
            # force adjoint at the post-drift positions (or the initial evaluation)
            flush_drift()
            if zero_pending:
                ac.zero_()
                zero_pending = False
            if not force_dot_done:
                call("pmb_dot", ac.data_ptr(), acc.data_ptr(), ac.numel(), dots[slot:].data_ptr(), s)
                force_slots.append(slot)
                slot += 1
            force_dot_done = False
            a_force = float(a[0]) if st[0] == "init" else float(st[3])
            ev_ready = None
            if overlap and recomputed:
                ev_ready = main.record_event()  # vel and acc final for this step
            self._force_adjoint(pmid, disp, F, S, ac, dc, a_force, presorted=recomputed, lane=str(lane),
                                concurrent=overlap)
            if overlap and ev_ready is None:
                ev_ready = main.record_event()  # the first adjoint sorted disp itself
            i += 1
            if st[0] == "init":
                ac.zero_()
                continue
            zero_pending = True
            _, a_vel, a_dp, a_dn, a_acc_in = st
            D, dD = cosmo.drift_factor(a_vel, a_dp, a_dn, with_grad=True)
            D32 = _f32(D)
            # recompute the incoming acceleration at disp - D vel (the drift's
            # position half, fused into the sort); keep its meshes for the next
            # force adjoint
            if overlap:
                side.wait_event(ev_ready)
                with torch.cuda.stream(side):
                    force(pmid, disp, conf, cosmo.Omega_m, a=float(a_acc_in), cosmo=cosmo, correction=corr,
                          force_meshes=F2, acc=acc, src_hat_out=S2, drift_vel=vel, drift=-D32,
                          lane=str(1 - lane))
                ev_force = side.record_event()
            # the drift's cotangent half: vel_cot += D disp_cot (after the force
            # adjoint), run inside the next kick adjoints' pass
            drift_pending = (D32, slot)
            grads.append((dD, slot))
            slot += 1
            if not overlap:
                force(pmid, disp, conf, cosmo.Omega_m, a=float(a_acc_in), cosmo=cosmo, correction=corr,
                      force_meshes=F2, acc=acc, src_hat_out=S2, drift_vel=vel, drift=-D32, lane=str(1 - lane))
            lane = 1 - lane
            recomputed = True
            F, F2 = F2, F
            S, S2 = S2, S
        if ev_force is not None:
            main.wait_event(ev_force)
        flush_drift()
        if zero_pending:
            ac.zero_()
        d = dots.cpu().numpy()
        if self._om_exact:
            om_cot = sum(g * d[k] for g, k in grads) + sum(self._om_exact)
        else:
            om_cot = sum(g * d[k] for g, k in grads) + sum(d[k] for k in force_slots) / om32
        return (ptcl.replace(disp=disp, vel=vel, acc=acc), Particles(conf, pmid, dc, vc, ac), float(om_cot))


def nbody_low_memory(ptcl, cosmo, conf, reverse=False, correction=None):
    """Forward-only KDK run with the streamed force (nbody/solver.py:559-602,
    nbody_low_memory): each force holds one real mesh instead of three, the
    drift is fused into the force's cell sort and nothing is kept for an
    adjoint.  Rejects reverse integration and force corrections, as the
    reference does."""
    if reverse:
        raise ValueError("nbody_low_memory does not support reverse integration.")
    if correction is not None:
        raise ValueError("nbody_low_memory does not support force corrections.")
    if conf.float_dtype != torch.float32:
        raise ValueError("nbody_low_memory runs the float32 path")
    from .gravity import force_streamed
    a = conf.a_nbody
    dev = ptcl.disp.device
    s = stream_handle(dev)
    disp = ptcl.disp.clone()
    vel = ptcl.vel.clone() if ptcl.vel is not None else torch.zeros_like(disp)
    acc = force_streamed(ptcl.pmid, disp, conf, cosmo.Omega_m)
    for a_prev, a_next in zip(a[:-1], a[1:]):
        stages = _schedule(a_prev, a_next, conf)
        i = 0
        while i < len(stages):
            st = stages[i]
            if st[0] == "kick":
                call("pmb_axpy", vel.data_ptr(), acc.data_ptr(), vel.numel(),
                     _f32(cosmo.kick_factor(st[1], st[2], st[3])), s)
            else:
                # drift fused into the streamed force's sort
                D = _f32(cosmo.drift_factor(st[1], st[2], st[3]))
                force_streamed(ptcl.pmid, disp, conf, cosmo.Omega_m, acc=acc, drift_vel=vel, drift=D)
            i += 1
    return ptcl.replace(disp=disp, vel=vel, acc=acc)


def nbody(ptcl, cosmo, conf, reverse=False, correction=None):
    """Advance particles through conf.a_nbody (nbody/solver.py:605-642)."""
    a = conf.a_nbody[::-1] if reverse else conf.a_nbody
    return NBodyRun(conf, cosmo, correction).forward(ptcl, a)


def nbody_scheduled(ptcl, cosmo, confs, reverse=False, correction=None):
    """Run through several configuration segments in turn, each with its own
    schedule, passing the particles on (nbody_static_halo_scheduled,
    nbody/solver.py:645-679); reverse runs the segments, and each schedule,
    backwards."""
    for c in (confs[::-1] if reverse else confs):
        ptcl = nbody(ptcl, cosmo, c, reverse=reverse, correction=correction)
    return ptcl


nbody_static_halo_scheduled = nbody_scheduled


def nbody_init(a, ptcl, cosmo, conf, correction=None):
    """The starting acceleration (nbody/solver.py:21-43)."""
    return force_state(a, ptcl, cosmo, conf, correction)


def nbody_step(a_prev, a_next, ptcl, cosmo, conf, correction=None):
    """One macro step (nbody/solver.py:46-65)."""
    return integrate(a_prev, a_next, ptcl, cosmo, conf, correction)


def nbody_collect(ptcl, cosmo, conf, collector, collector_state, reverse=False, return_final=False,
                  correction=None):
    """Forward run updating caller state after every macro step
    (nbody/solver.py:116-167): state = collector(state, a_prev, a_next, ptcl,
    cosmo, conf).  Forward only; returns the state, or (final particles,
    state) with return_final."""
    a = conf.a_nbody[::-1] if reverse else conf.a_nbody
    ptcl = nbody_init(float(a[0]), ptcl, cosmo, conf, correction)
    state = collector_state
    for a_prev, a_next in zip(a[:-1], a[1:]):
        ptcl = nbody_step(float(a_prev), float(a_next), ptcl, cosmo, conf, correction)
        state = collector(state, float(a_prev), float(a_next), ptcl, cosmo, conf)
    return (ptcl, state) if return_final else state


def _stack_tree(obs):
    """Stack a list of observation trees (tensors, numbers, dicts, tuples) along a new leading axis."""
    first = obs[0]
    if isinstance(first, dict):
        return {k: _stack_tree([o[k] for o in obs]) for k in first}
    if isinstance(first, (tuple, list)):
        return type(first)(_stack_tree([o[i] for o in obs]) for i in range(len(first)))
    if torch.is_tensor(first):
        return torch.stack(obs)
    return torch.as_tensor(np.asarray(obs))


def nbody_observe(ptcl, cosmo, conf, observer, reverse=False, include_start=False, return_final=False,
                  correction=None):
    """Forward run stacking observer(a, ptcl, cosmo, conf) after every macro
    step, and at the start with include_start (nbody/solver.py:170-227)."""
    a = conf.a_nbody[::-1] if reverse else conf.a_nbody
    ptcl = nbody_init(float(a[0]), ptcl, cosmo, conf, correction)
    obs = [observer(float(a[0]), ptcl, cosmo, conf)] if include_start else []
    for a_prev, a_next in zip(a[:-1], a[1:]):
        ptcl = nbody_step(float(a_prev), float(a_next), ptcl, cosmo, conf, correction)
        obs.append(observer(float(a_next), ptcl, cosmo, conf))
    stacked = _stack_tree(obs) if obs else None
    return (ptcl, stacked) if return_final else stacked


def nbody_adj(ptcl, ptcl_cot, cosmo, conf, reverse=False, correction=None):
    """Reverse sweep from the final state (nbody/solver.py:385-444).

    Returns (ptcl_in, ptcl_in_cot, Omega_m_cot)."""
    a = conf.a_nbody[::-1] if reverse else conf.a_nbody
    run = NBodyRun(conf, cosmo, correction)
    if conf.float_dtype == torch.float64:
        return run.adjoint(ptcl, ptcl_cot, a_nbody=a)
    _, F = force(ptcl.pmid, ptcl.disp.clone(), conf, cosmo.Omega_m, a=float(a[-1]), cosmo=cosmo,
                 correction=correction)
    return run.adjoint(ptcl, ptcl_cot, force_meshes=F, a_nbody=a)
