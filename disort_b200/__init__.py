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

# The DisORT++ API names served by the native host module (_disortpp).  The
# module is loaded on first use of any of them, so the pure-Python helpers
# (capi, workloads, flops, replicas) can be imported without mapping the GPU
# libraries; a missing build fails loudly at that first use.
_NATIVE_NAMES = (
    "AmbralsBrdfSpec", "BoundaryConditions", "BoundaryConditionType", "BrdfSpecification", "BrdfType",
    "CoxMunkBrdfSpec", "DisortConfig", "DisortFlags", "DisortResult", "DisortSolver", "HapkeBrdfSpec",
    "RpvBrdfSpec", "DisortFluxConfig", "DisortFluxSolver4", "DisortFluxSolver6", "DisortFluxSolver8",
    "DisortFluxSolver10", "DisortFluxSolver12", "DisortFluxSolver14", "DisortFluxSolver16",
    "DisortFluxSolver32", "DisortFluxSolver64", "FluxResult", "PhaseFunction", "create_flux_solver",
    "solve_flux_spectral", "solve_flux_spectral_bands", "solve_flux_spectral_bands_arrays", "solve_spectral",
    "solve_spectral_bands",
)


def _native():
    try:
        from . import _disortpp
    except ImportError as e:  # the native host module is the product; no Python fallback
        raise ImportError(f"disort_b200 native module not built ({e}); run __graft_entry__.build()") from e
    return _disortpp


def __getattr__(name):
    if name in _NATIVE_NAMES:
        value = getattr(_native(), name)
        globals()[name] = value
        return value
    raise AttributeError(f"module 'disort_b200' has no attribute {name!r}")


def __dir__():
    return sorted(list(globals()) + list(_NATIVE_NAMES))


__all__ = list(_NATIVE_NAMES)
__version__ = "0.1.0"
