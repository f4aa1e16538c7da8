"""Mesh-CNN residual potential correction (corrections/mesh_cnn.py:66-265,
corrections/core.py:286-331).

A small periodic 3-D convolutional network predicts a real-space residual
potential from the Poisson source S and the PM potential phi:

    x = [S / s(S), phi / s(phi), a, Omega_m, sigma8]   (s(v) = sqrt(mean v^2 + 1e-6))
    h = gelu(conv_stem(x))
    repeat depth-1 times:  h = gelu(conv2(gelu(conv1(h))) + h)
    R = g phi + max_residual tanh(conv_out(h)) s(phi),
    g = max_residual tanh(w_gain . [a, Omega_m, sigma8] + b_gain)

and the force uses the potential spectrum plus rfft(R).  Convolutions are
haiku's Conv3D after periodic padding by one cell; parameters keep haiku's
names and shapes (w (3, 3, 3, Cin, Cout), b (Cout,)) in one flat float32
tensor.  The constant conditioning channels only add a per-channel constant
to the stem, folded into its bias.  The kernels are in csrc/meshcnn.cu; the
backward is hand-written (convolution transposes, weight gradients, the
normalisations' and the gain's derivatives), returning the cotangents of S,
phi, the parameters and the conditioning features.

Parameter values come from this module's initialiser (haiku's schemes:
fan-in truncated normal for the convolutions, zeros for the output layer,
normal of stddev output_init_scale for the gain); JAX's random streams are
not reproduced, so trained reference parameters must be loaded with
``load_params``.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ._lib import call
from .runtime import require_cuda, stream_handle

_EPS = 1e-6
_NFEAT = 3  # a, Omega_m, sigma8


def param_layout(channels=8, depth=4):
    """[(name, shape)] in the flat parameter order (haiku module names)."""
    C = channels
    lay = [("stem/w", (3, 3, 3, 2 + _NFEAT, C)), ("stem/b", (C, ))]
    for i in range(max(depth - 1, 0)):
        lay += [(f"block_{i}_conv1/w", (3, 3, 3, C, C)), (f"block_{i}_conv1/b", (C, )),
                (f"block_{i}_conv2/w", (3, 3, 3, C, C)), (f"block_{i}_conv2/b", (C, ))]
    lay += [("out/w", (3, 3, 3, C, 1)), ("out/b", (1, )), ("direct_gain/w", (_NFEAT, 1)), ("direct_gain/b", (1, ))]
    return lay


class MeshCNNCorrection:
    """Trainable real-space residual potential correction (MeshCNNPotentialCorrection)."""

    green_kernel = 0
    gradient_kernel = "spectral"
    interlacing = False
    trainable = False   # not the radial-transfer kind; its gradients accumulate in .grad
    mesh_cnn = True

    def __init__(self, channels=8, depth=4, max_residual=0.1, output_init_scale=1e-2, seed=0, device="cuda",
                 sigma8_value=0.8, allow_missing_sigma8=False):
        if channels not in (4, 8, 16):
            raise ValueError("the mesh-CNN kernels are built for 4, 8 or 16 channels")
        self.channels, self.depth = int(channels), int(depth)
        self.max_residual, self.output_init_scale = float(max_residual), float(output_init_scale)
        self.sigma8_value, self.allow_missing_sigma8 = float(sigma8_value), bool(allow_missing_sigma8)
        self.device = torch.device(device)
        self.layout = param_layout(self.channels, self.depth)
        self.offsets = {}
        off = 0
        for name, shape in self.layout:
            self.offsets[name] = (off, shape)
            off += math.prod(shape)
        self.params = torch.zeros(off, dtype=torch.float32, device=self.device)
        self.grad = torch.zeros(off, dtype=torch.float64, device=self.device)
        self.accumulate_grads = True
        self._init(seed)

    # ---- parameters ------------------------------------------------------
    def view(self, name, t=None):
        off, shape = self.offsets[name]
        t = self.params if t is None else t
        return t[off:off + math.prod(shape)].view(shape)

    def _init(self, seed):
        """haiku defaults: VarianceScaling(1, fan_in, truncated normal) for the
        convolutions, zeros for biases and the output layer, normal of stddev
        output_init_scale for the gain."""
        g = torch.Generator().manual_seed(int(seed))
        for name, shape in self.layout:
            if name.endswith("/b") or name.startswith("out/"):
                continue
            if name.startswith("direct_gain"):
                w = torch.randn(shape, generator=g) * self.output_init_scale
            else:
                fan_in = 27 * shape[3]
                std = math.sqrt(1.0 / fan_in) / 0.87962566103423978  # truncated-normal correction
                w = torch.fmod(torch.randn(shape, generator=g), 2.0) * std
            self.view(name).copy_(w.to(torch.float32))

    def load_params(self, params):
        """Set parameters from a {haiku name: array} mapping."""
        for name, shape in self.layout:
            self.view(name).copy_(torch.as_tensor(np.asarray(params[name], np.float32).reshape(shape)))

    def params_dict(self):
        return {name: self.view(name).cpu().numpy() for name, _ in self.layout}

    def transfer_tables(self, a, cosmo, conf):
        return None, None

    def features(self, a, cosmo):
        s8 = getattr(cosmo, "sigma8", None) if cosmo is not None else None
        if s8 is None or not np.isfinite(s8):
            if not self.allow_missing_sigma8 and cosmo is not None:
                raise ValueError("sigma8 is not initialised on the cosmology; run boltzmann() first or set "
                                 "allow_missing_sigma8=True")
            s8 = self.sigma8_value
        om = 0.3 if cosmo is None else float(cosmo.Omega_m)
        return [1.0 if a is None else float(a), om, float(s8)]

    # ---- forward -----------------------------------------------------------
    def _dot(self, a, b):
        out = torch.zeros(1, dtype=torch.float64, device=a.device)
        call("pmb_dot", a.data_ptr(), b.data_ptr(), a.numel(), out.data_ptr(), stream_handle(a.device))
        return out

    def _conv(self, x, ci, w, b, co, shape, act, res=None, zref=None, trans=False, want_h=True):
        nx, ny, nz = shape
        M = nx * ny * nz
        z = torch.empty((co, M), dtype=torch.float32, device=x.device)
        h = torch.empty_like(z) if (act == 1 and want_h) else None
        call("pmb_cnn_conv3d", x.data_ptr(), ci, w.data_ptr(), None if b is None else b.data_ptr(),
             None if res is None else res.data_ptr(), None if zref is None else zref.data_ptr(), act, z.data_ptr(),
             None if h is None else h.data_ptr(), co, nx, ny, nz, int(trans), stream_handle(x.device))
        return z, h

    def residual(self, S, phi, a, cosmo, keep=True):
        """R for source S and potential phi (real (nx, ny, nz) float32 meshes)."""
        require_cuda(S, phi)
        shape = tuple(S.shape)
        M = S.numel()
        C = self.channels
        S = S.contiguous()
        phi = phi.contiguous()
        f = self.features(a, cosmo)
        dev = S.device
        s2 = torch.cat([self._dot(S, S), self._dot(phi, phi)]).cpu().numpy()
        sS = math.sqrt(s2[0] / M + _EPS)
        sP = math.sqrt(s2[1] / M + _EPS)
        x0 = torch.empty((2, M), dtype=torch.float32, device=dev)
        call("pmb_cnn_stem_input", S.data_ptr(), phi.data_ptr(), M, float(1 / sS), float(1 / sP), x0.data_ptr(),
             stream_handle(dev))
        W0 = self.view("stem/w")
        w0s = W0[:, :, :, :2, :].contiguous()
        fv = torch.tensor(f, dtype=torch.float32, device=dev)
        b0 = (self.view("stem/b") + (W0[:, :, :, 2:, :] * fv[:, None]).sum(dim=(0, 1, 2, 3))).contiguous()
        z0, h = self._conv(x0, 2, w0s, b0, C, shape, 1)
        acts = [("stem", x0, z0, h)]
        for i in range(self.depth - 1):
            z1, t = self._conv(h, C, self.view(f"block_{i}_conv1/w"), self.view(f"block_{i}_conv1/b"), C, shape, 1)
            z2, h2 = self._conv(t, C, self.view(f"block_{i}_conv2/w"), self.view(f"block_{i}_conv2/b"), C, shape, 1,
                                res=h)
            acts.append((f"block_{i}", h, z1, t, z2))
            h = h2
        o, _ = self._conv(h, C, self.view("out/w"), self.view("out/b"), 1, shape, 0)
        u = float((self.view("direct_gain/w")[:, 0].double().cpu() * torch.tensor(f, dtype=torch.float64)).sum()
                  + self.view("direct_gain/b")[0].double().cpu())
        g = self.max_residual * math.tanh(u)
        c = self.max_residual * sP
        R = torch.empty_like(S)
        call("pmb_cnn_residual", phi.data_ptr(), o.data_ptr(), M, float(g), float(c), R.data_ptr(), stream_handle(dev))
        if keep:
            self._saved = dict(shape=shape, S=S, phi=phi, f=f, sS=sS, sP=sP, x0=x0, w0s=w0s, acts=acts, h=h, o=o,
                               u=u, g=g, c=c)
        return R

    # ---- backward ----------------------------------------------------------
    def residual_adjoint(self, Rc):
        """Cotangents (dS, dphi, dparams float64 flat, dfeatures [a, Omega_m,
        sigma8]) of the last residual() call given R's cotangent Rc."""
        sv = self._saved
        shape, M, C = sv["shape"], Rc.numel(), self.channels
        dev = Rc.device
        s = stream_handle(dev)
        mr = self.max_residual
        dparams = torch.zeros_like(self.grad)
        dview = lambda name: self.view(name, dparams)
        Rc = Rc.contiguous()
        dphi = torch.empty_like(Rc)
        do = torch.empty((1, M), dtype=torch.float32, device=dev)
        dots = torch.zeros(2, dtype=torch.float64, device=dev)
        call("pmb_cnn_residual_adjoint", Rc.data_ptr(), sv["phi"].data_ptr(), sv["o"].data_ptr(), M, float(sv["g"]),
             float(sv["c"]), dphi.data_ptr(), do.data_ptr(), dots.data_ptr(), s)
        dg_dc = dots.cpu().numpy()
        dsP = mr * dg_dc[1]  # c = mr sP
        du = dg_dc[0] * mr * (1.0 - math.tanh(sv["u"])**2)
        f = sv["f"]
        dfeat = np.array([du * float(self.view("direct_gain/w")[k, 0]) for k in range(_NFEAT)])
        dview("direct_gain/w")[:, 0] += torch.tensor([du * fk for fk in f], dtype=torch.float64, device=dev)
        dview("direct_gain/b")[0] += du
        # output layer
        last = sv["acts"][-1]
        zlast = last[2] if len(last) == 4 else last[4]
        dz, _ = self._conv(do, 1, self.view("out/w"), None, C, shape, 2, zref=zlast, trans=True)
        self._wgrad(sv["h"], C, do, 1, shape, dview("out/w"), dview("out/b"))
        for i in range(self.depth - 2, -1, -1):
            _, h_in, z1, t, z2 = sv["acts"][i + 1]
            dz2 = dz
            self._wgrad(t, C, dz2, C, shape, dview(f"block_{i}_conv2/w"), dview(f"block_{i}_conv2/b"))
            dz1, _ = self._conv(dz2, C, self.view(f"block_{i}_conv2/w"), None, C, shape, 2, zref=z1, trans=True)
            self._wgrad(h_in, C, dz1, C, shape, dview(f"block_{i}_conv1/w"), dview(f"block_{i}_conv1/b"))
            prev = sv["acts"][i]
            zprev = prev[2] if len(prev) == 4 else prev[4]
            dz, _ = self._conv(dz1, C, self.view(f"block_{i}_conv1/w"), None, C, shape, 2, res=dz2, zref=zprev,
                               trans=True)
        # stem: dz is its pre-activation cotangent
        dw0 = torch.zeros((27, 2, C), dtype=torch.float64, device=dev)
        db0 = torch.zeros(C, dtype=torch.float64, device=dev)
        call("pmb_cnn_conv3d_wgrad", sv["x0"].data_ptr(), 2, dz.data_ptr(), C, *shape, dw0.data_ptr(), db0.data_ptr(), s)
        W0d = dview("stem/w")
        W0d[:, :, :, :2, :] += dw0.view(3, 3, 3, 2, C)
        fv = torch.tensor(f, dtype=torch.float64, device=dev)
        W0d[:, :, :, 2:, :] += fv[:, None] * db0[None, :]
        dview("stem/b")[:] += db0
        W0c = self.view("stem/w")[:, :, :, 2:, :].double()
        dfeat += (W0c * db0[None, None, None, None, :]).sum(dim=(0, 1, 2, 4)).cpu().numpy()
        dx0, _ = self._conv(dz, C, sv["w0s"], None, 2, shape, 0, trans=True)
        # normalisations (and the potential scale inside c = mr sP)
        S, phi, sS, sP = sv["S"], sv["phi"], sv["sS"], sv["sP"]
        d = torch.cat([self._dot(dx0[0], S), self._dot(dx0[1], phi)]).cpu().numpy()
        cS = d[0] / (M * sS**3)
        cP = d[1] / (M * sP**3) - dsP / (M * sP)
        dS = torch.empty_like(S)
        call("pmb_cnn_norm_adjoint", dx0.data_ptr(), S.data_ptr(), phi.data_ptr(), M, float(1 / sS), float(cS),
             float(1 / sP), float(cP), dS.data_ptr(), dphi.data_ptr(), s)
        return dS, dphi, dparams, dfeat

    def _wgrad(self, x, ci, dout, co, shape, dW, db):
        tw = torch.zeros(dW.numel(), dtype=torch.float64, device=x.device)
        tb = torch.zeros(co, dtype=torch.float64, device=x.device)
        call("pmb_cnn_conv3d_wgrad", x.data_ptr(), ci, dout.data_ptr(), co, *shape, tw.data_ptr(), tb.data_ptr(),
             stream_handle(x.device))
        dW += tw.view(dW.shape)
        db += tb

    # ---- training ------------------------------------------------------------
    def zero_grad(self):
        self.grad.zero_()

    def adam_step(self, lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        """One Adam update of the parameters from .grad (then cleared)."""
        if not hasattr(self, "_m"):
            self._m = torch.zeros_like(self.grad)
            self._v = torch.zeros_like(self.grad)
            self._t = 0
        self._t += 1
        g = self.grad
        self._m.mul_(betas[0]).add_(g, alpha=1 - betas[0])
        self._v.mul_(betas[1]).addcmul_(g, g, value=1 - betas[1])
        mh = self._m / (1 - betas[0]**self._t)
        vh = self._v / (1 - betas[1]**self._t)
        self.params -= (lr * mh / (vh.sqrt() + eps)).to(torch.float32)
        self.zero_grad()
