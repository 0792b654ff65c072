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

import functools


def layer_flops(N: int, beam: bool, thermal: bool) -> float:
    NN = N // 2
    f = N ** 3 + 16.33 * NN ** 3 + 6 * NN ** 2
    if beam:
        f += (2.0 / 3.0) * N ** 3 + 4 * N ** 2
    if thermal:
        f += (2.0 / 3.0) * N ** 3 + 4 * N ** 2
    return f


@functools.lru_cache(maxsize=None)
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


def absorption_cut(dtau, ssa, thermal: bool) -> int:
    """Layers the solvers keep (disortSet's abscut = 10 absorption depth rule)."""
    L = len(dtau)
    abstau, ncut = 0.0, L
    for lc in range(L):
        if abstau < 10.0:
            ncut = lc + 1
        abstau += (1.0 - ssa[lc]) * dtau[lc]
    lyrcut = abstau >= 10.0 and not thermal and L > 1
    return ncut if lyrcut else L


def general_solve_flops(N: int, L: int, ncut: int, modes: int, numu: int, ntau: int, beam: bool,
                        thermal: bool) -> dict:
    """FLOPs of one general (DisortSolver) solve, split by engine kernel.

    Per azimuth mode m with nact = N - m active Legendre orders, per kept layer:
    phase matrix 2 NN N nact, the eigensystem as in layer_flops, the beam source
    (2/3 N^3 + 4 N^2), the thermal source at m = 0, interpEigenvec 2 nact N^2 +
    2 numu nact N and interpSource (2 nact N + 2 numu nact per source); per mode the
    band LU, mode-0 fluxes at the ntau output depths, and the user intensities
    8 N ntau numu ncut.
    """
    NN = N // 2
    lay = bvp = inten = 0.0
    for m in range(modes):
        nact = N - m
        per = 2.0 * NN * N * nact + 16.33 * NN ** 3 + 6 * NN ** 2
        if beam:
            per += (2.0 / 3.0) * N ** 3 + 4 * N ** 2
        if thermal and m == 0:
            per += (2.0 / 3.0) * N ** 3 + 4 * N ** 2
        if numu:
            per += 2.0 * nact * N * N + 2.0 * numu * nact * N
            nsrc = (1 if beam else 0) + (2 if thermal and m == 0 else 0)
            per += nsrc * (2.0 * nact * N + 2.0 * numu * nact)
        lay += ncut * per
        bvp += band_lu_flops(N, ncut)
        if m == 0:
            bvp += ntau * (2.0 * N * N + 8.0 * N)
        if numu:
            inten += 8.0 * N * ntau * numu * ncut
    return {"gen_layer_kernel": lay, "gen_bvp_kernel": bvp, "gen_intensity_kernel": inten,
            "total": lay + bvp + inten}
