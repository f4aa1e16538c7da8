"""Algorithmic HBM bytes per launch of each PM stage: the roofline numerator.

N particles, M mesh cells, Mc = Mx*My*(Mz/2+1) complex cells, R = Mx*My mesh
rows, T distinct mesh cells touched by the particles' CIC corners (at most
min(M, 8N); the upper bound is used when T is not measured).  Every input is
counted once and every output once, at the sizes of the reference's data
layout (pmid int16 x 3 + disp float32 x 3 = 18 B per particle); re-reads,
halo redundancy, the pass chain's zero padding and cuFFT's extra passes are not
counted, so a stage's
achieved GB/s is directly comparable with the HBM copy bandwidth.
"""
from __future__ import annotations


def algorithmic_bytes(op, N, M, Mc=None, R=None, T=None):
    Mc = M // 2 if Mc is None else Mc
    R = round(M ** (2 / 3)) if R is None else R
    T = min(M, 8 * N) if T is None else min(T, M)
    table = {
        # row sort: pmid+disp in, 16 B records + 4 B permutation out, row offsets
        "sort": 18 * N + 20 * N + 8 * R,
        "scatter": 18 * N + 4 * M,
        "scatter3": 18 * N + 12 * N + 12 * M,          # gather adjoint: 3-channel values in, 3 meshes out
        "gather": 18 * N + 12 * N + 12 * T,             # 3 force meshes in, acc out
        "gather_kick": 18 * N + 12 * N + 12 * T + 24 * N,  # ... and the folded kick: vel in and out
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
