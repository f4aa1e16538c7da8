"""CUDA-graph-captured runs.

A forward N-body run is a fixed sequence of C-ABI launches whose scalar
arguments (time factors, Green's-function options, the correction's
conditioning) depend only on the configuration and cosmology, so it is
captured once into a CUDA graph and replayed: replay removes the per-launch
host work that dominates small meshes.  Inputs are copied into the graph's
static buffers before each replay.  cuFFT plans and workspaces are created by
a warm-up run before capture (plan creation allocates and must not happen
inside a capture).  The graph keeps references to every workspace buffer
that existed at capture time: a later run that grows a shared workspace slot
replaces the slot's tensor, and the captured pointers must stay valid.
"""
from __future__ import annotations

import torch

from . import runtime
from .nbody import NBodyRun
from .particles import Particles


class GraphedForward:
    """Replayable forward run of NBodyRun for fixed conf / cosmology / correction."""

    def __init__(self, conf, cosmo, ptcl, correction=None, a_nbody=None, warmup=1):
        self.run = NBodyRun(conf, cosmo, correction)
        self.a = a_nbody
        self.static_in = Particles(conf, ptcl.pmid.clone(), ptcl.disp.clone(),
                                   (ptcl.vel if ptcl.vel is not None else torch.zeros_like(ptcl.disp)).clone())
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.run.forward(self.static_in, self.a)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = self.run.forward(self.static_in, self.a)
        self._workspaces = runtime.workspace_refs()

    def __call__(self, disp=None, vel=None):
        if disp is not None:
            self.static_in.disp.copy_(disp)
        if vel is not None:
            self.static_in.vel.copy_(vel)
        self.graph.replay()
        return self.out
