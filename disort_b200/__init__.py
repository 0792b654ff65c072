"""disort_b200 — B200-native DISORT spectral engine (FP64, sm_100a).

``import disort_b200 as disortpp`` gives the DisORT++ Python API with every
solve running on the GPU: the flux path (DisortFluxConfig, FluxResult,
DisortFluxSolver4..64, create_flux_solver, solve_flux_spectral,
solve_flux_spectral_bands) and the general path (DisortConfig, DisortFlags,
BoundaryConditions, DisortResult, DisortSolver, solve_spectral,
solve_spectral_bands), plus PhaseFunction, BoundaryConditionType, BrdfType and
the BRDF parameter structs.
The C ABI is include/dsp.h (libdsp.so under disort_b200/lib); ``capi`` is its
ctypes mirror.
"""
from . import capi  # noqa: F401

try:
    from ._disortpp import (  # noqa: F401
        AmbralsBrdfSpec,
        BoundaryConditions,
        BoundaryConditionType,
        BrdfSpecification,
        BrdfType,
        CoxMunkBrdfSpec,
        DisortConfig,
        DisortFlags,
        DisortResult,
        DisortSolver,
        HapkeBrdfSpec,
        RpvBrdfSpec,
        DisortFluxConfig,
        DisortFluxSolver4,
        DisortFluxSolver6,
        DisortFluxSolver8,
        DisortFluxSolver10,
        DisortFluxSolver12,
        DisortFluxSolver14,
        DisortFluxSolver16,
        DisortFluxSolver32,
        DisortFluxSolver64,
        FluxResult,
        PhaseFunction,
        create_flux_solver,
        solve_flux_spectral,
        solve_flux_spectral_bands,
        solve_flux_spectral_bands_arrays,
        solve_spectral,
        solve_spectral_bands,
    )
except ImportError as e:  # the native host module is the product; no Python fallback
    raise ImportError(f"disort_b200 native module not built ({e}); run __graft_entry__.build()") from e

__version__ = "0.1.0"
