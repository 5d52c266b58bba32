"""Algorithmic flop model of the tracker (real flops: complex multiply 6,
add 2, fused multiply-add 8, division or reciprocal 11), computed from the
sparse table, not from the instructions the kernel executes.

Per unit (one evaluation of H, H_z, H_t, one LU, one solve), with s_k the
number of nonzero homogenized exponents of term k (w included) and E_j the
largest homogenized exponent of unknown j:

    F_eval = sum_j 6 max(0, E_j - 1) + sum_k (38 s_k - 10)
    F_hom  = 6 n N + sum_i (12 d_i + 46) + 8 N
    F_LU   = sum_{r=1}^{N-1} (8 r^2 + 9 r + 11) + 3 N
    F_sol  = 8 N (N - 1) + 6 N
    F_unit = F_eval + F_hom + F_LU + F_sol

A path's flops follow from its unit counters (phc_path_out): predictor,
corrector and refine units cost F_unit, evaluation-only units F_eval + F_hom,
a cond1 call F_LU + N F_sol. In mixed precision a predictor or corrector
unit evaluates H, H_z and H_t in FP64 (F_eval + F_hom) and eliminates in
FP32 (F_LU + F_sol), unless the whole unit ran in FP64 (counter
n_fp64_retry). (The single-system kernels for n <= 7 evaluate the mixed
predictor in FP32; the model counts that evaluation as FP64.)
"""
import numpy as np


def unit_model(n, deg, hexps):
    N = n + 1
    hexps = np.asarray(hexps).reshape(-1, N)
    E = hexps.max(axis=0) if len(hexps) else np.zeros(N, dtype=int)
    s = (hexps > 0).sum(axis=1)
    deg = np.asarray(deg)
    f_eval = float(np.sum(6 * np.maximum(0, E - 1)) + np.sum(38 * s - 10))
    f_hom = float(6 * n * N + np.sum(12 * deg + 46) + 8 * N)
    f_lu = float(sum(8 * r * r + 9 * r + 11 for r in range(1, N)) + 3 * N)
    f_sol = float(8 * N * (N - 1) + 6 * N)
    return dict(F_eval=f_eval, F_hom=f_hom, F_LU=f_lu, F_sol=f_sol,
                F_unit=f_eval + f_hom + f_lu + f_sol, N=N)


def path_flops(model, paths, mixed):
    """Total (fp64_flops, fp32_flops) of a set of path records."""
    M = model
    t = paths["n_tangent"].astype(np.float64).sum()
    c = paths["n_newton"].astype(np.float64).sum()
    r = paths["n_refine"].astype(np.float64).sum()
    e = paths["n_eval"].astype(np.float64).sum()
    k = paths["n_cond"].astype(np.float64).sum()
    other64 = r * M["F_unit"] + e * (M["F_eval"] + M["F_hom"]) + k * (M["F_LU"] + M["N"] * M["F_sol"])
    if not mixed:
        return (t + c) * M["F_unit"] + other64, 0.0
    u64 = paths["n_fp64_retry"].astype(np.float64).sum()
    u32 = max(t + c - u64, 0.0)
    f64 = other64 + u64 * M["F_unit"] + u32 * (M["F_eval"] + M["F_hom"])
    f32 = u32 * (M["F_LU"] + M["F_sol"])
    return f64, f32
