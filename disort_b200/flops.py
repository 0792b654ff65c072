"""Algorithmic FP64 operation counts of one DISORT solve (the roofline numerator).

The counts are those of the reference algorithm (DisORT++ FluxSolver.cpp), not
of this engine's kernels:

* per layer (m = 0): phase matrix N^3; Cholesky, S = L^T A L, symmetric QR with
  vectors and eigenvector recovery 16.33 NN^3 + 6 NN^2; beam and thermal particular
  solutions (2/3 N^3 + 4 N^2) each when present;
* boundary-value problem: the LINPACK band factorisation count
  sum_k 2 lm_k min(ml+mu, n-k) with ml = mu = 3NN-1, n = N ncut (structural zeros
  inside the band included, as sgbfa performs them), plus the band solve
  2 sum lm_k + 2 sum (min(k, ml+mu+1) - 1);
* fluxes: (L+1)(2 N^2 + 8 N).

Transcendental calls (exp, sqrt, log, pow) are not counted.
"""
from __future__ import annotations


def layer_flops(N: int, beam: bool, thermal: bool) -> float:
    NN = N // 2
    f = N ** 3 + 16.33 * NN ** 3 + 6 * NN ** 2
    if beam:
        f += (2.0 / 3.0) * N ** 3 + 4 * N ** 2
    if thermal:
        f += (2.0 / 3.0) * N ** 3 + 4 * N ** 2
    return f


def band_lu_flops(N: int, ncut: int) -> float:
    NN = N // 2
    ml = mu = 3 * NN - 1
    n = N * ncut
    fac = 0.0
    sol = 0.0
    for k in range(1, n):
        lm = min(ml, n - k)
        fac += 2.0 * lm * min(ml + mu, n - k)
        sol += 2.0 * lm
    m1 = ml + mu + 1
    for k in range(1, n + 1):
        sol += 2.0 * (min(k, m1) - 1)
    return fac + sol


def flux_flops(N: int, L: int) -> float:
    return (L + 1) * (2.0 * N * N + 8.0 * N)


def flux_solve_flops(N: int, L: int, beam: bool, thermal: bool, ncut: int | None = None) -> dict:
    """FLOPs of one flux solve split by the engine kernel that performs each part."""
    nc = L if ncut is None else ncut
    lay = nc * layer_flops(N, beam, thermal)
    bvp = band_lu_flops(N, nc) + flux_flops(N, L)
    return {"flux_layer_kernel": lay, "flux_bvp_kernel": bvp, "total": lay + bvp}
