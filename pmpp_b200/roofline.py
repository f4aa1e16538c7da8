"""Algorithmic HBM bytes per launch of each PM stage: the roofline numerator.

N particles, M mesh cells, Mc = Mx*My*(Mz/2+1) complex cells, R = Mx*My mesh
rows, T distinct mesh cells touched by the particles' CIC corners (at most
min(M, 8N); the upper bound is used when T is not measured).  Every input is
counted once and every output once, at the sizes of the reference's data
layout (pmid int16 x 3 + disp float32 x 3 = 18 B per particle); re-reads,
halo redundancy, the pass chain's zero padding and cuFFT's extra passes are not
counted, so a stage's
achieved GB/s is directly comparable with the HBM copy bandwidth.

live = (fy, fz): the pass chain pruned to the particle-Nyquist box (pmfft.cu,
on meshes finer than the particle grid), fy the live fraction of ky and fz of
kz (Mz/2+1 values).  Its passes then need only the live part: the forward y
passes read fz of the spectrum and write fz*fy, the x passes read and write
fy*fz, the inverse y passes read fz*fy and write fz, and the z passes need
only the live fz of each spectral row (the kernels move whole rows, which
measured faster; that surplus is not counted).
"""
from __future__ import annotations


def algorithmic_bytes(op, N, M, Mc=None, R=None, T=None, live=None):
    Mc = M // 2 if Mc is None else Mc
    R = round(M ** (2 / 3)) if R is None else R
    T = min(M, 8 * N) if T is None else min(T, M)
    if live is not None:
        fy, fz = live
        pruned = {
            "fft_z_r2c": 4 * M + 8 * Mc * fz,
            "fft_z_r2c3": 3 * (4 * M + 8 * Mc * fz),
            "fft_y": 8 * Mc * fz * (1 + fy),
            "fft_y_yz": 8 * Mc * fz * (2 + fy),
            "fft_y_inv": 8 * Mc * fz * (fy + 1),
            "fft_y_inv_yz": 8 * Mc * fz * (fy + 2),
            "fft_x_green": 24 * Mc * fy * fz,
            "fft_x_green_adj": 24 * Mc * fy * fz,
            "fft_z_c2r": 8 * Mc * fz + 4 * M,
            "fft_z_c2r3": 3 * (8 * Mc * fz + 4 * M),
        }
        if op in pruned:
            return pruned[op]
    table = {
        # row sort: pmid+disp in, 16 B records + 4 B permutation out, row offsets
        "sort": 18 * N + 20 * N + 8 * R,
        "scatter": 18 * N + 4 * M,
        "scatter3": 18 * N + 12 * N + 12 * M,          # gather adjoint: 3-channel values in, 3 meshes out
        "gather": 18 * N + 12 * N + 12 * T,             # 3 force meshes in, acc out
        "gather_kick": 18 * N + 12 * N + 12 * T + 24 * N,  # ... and the folded kick: vel in and out
        "gather_kick_only": 18 * N + 12 * T + 24 * N,   # the folded kicks without storing acc
        "gather_adjoint": 18 * N + 12 * T + 12 * N + 24 * N,   # positions, meshes, acc cot, disp cot r/w
        "scatter_adjoint": 18 * N + 4 * T + 24 * N,     # positions, density cot, disp cot r/w
        "fft_r2c": 4 * M + 8 * Mc,
        "fft_r2c_x3": 3 * (4 * M + 8 * Mc),
        "fft_c2r": 8 * Mc + 4 * M,
        "fft_c2r_x3": 3 * (8 * Mc + 4 * M),
        # hand-written pass chain (pmfft.cu), complex channels counted at Mc
        "fft_z_r2c": 4 * M + 8 * Mc,
        "fft_z_r2c3": 3 * (4 * M + 8 * Mc),
        "fft_y": 16 * Mc,
        "fft_y_yz": 24 * Mc,
        "fft_y_inv": 16 * Mc,
        "fft_y_inv_yz": 24 * Mc,
        "fft_x_green": 24 * Mc,
        "fft_x_green_adj": 24 * Mc,
        "fft_x_adj": 24 * Mc,
        "fft_x_inv": 16 * Mc,
        "fft_z_c2r": 8 * Mc + 4 * M,
        "fft_z_c2r3": 3 * (8 * Mc + 4 * M),
        "green_gradient": 8 * Mc + 24 * Mc,
        "green_gradient_adjoint": 24 * Mc + 8 * Mc,
        "kdk": 6 * N + 24 * N + 24 * N + 12 * N,
    }
    if op not in table:
        raise KeyError(op)
    return table[op]
