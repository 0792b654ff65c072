"""Generate tests/golden/reference_goldens.json from the reference's own tests.

Run where the DisORT++ sources are available, giving their path:

    python tests/golden/make_reference_goldens.py /path/to/DisORT

The reference's known-answer tests are C++ code (tests/test_solver.cpp).  This
script pairs each selected TEST with a transcription of its configuration (the
CASES table below, each entry citing the test's line) and extracts the expected
values and tolerances programmatically from the EXPECT_NEAR lines of that TEST's
body, so every number in the fixture comes from the reference file itself.  The
Garcia-Siewert Cloud C.1 moment table is read from src/PhaseFunction.cpp.
"""
from __future__ import annotations

import json
import math
import os
import re
import sys

PI = math.pi

# Transcribed configurations.  phase: ("iso",) | ("hg", g) | ("rayleigh",) | ("cloud",),
# one entry per layer or a single entry for all layers.  utau: None = output at the
# layer boundaries (use_user_tau = false).
CASES = [
    dict(test="ValidationDisotest1a", N=16, L=1, nmom=0, dtau=[0.03125], ssa=[0.2], phase=[("iso",)],
         fbeam=31.41592653589793, umu0=0.1, albedo=0.0),
    dict(test="ValidationDisotest1b", N=16, L=1, nmom=0, dtau=[0.03125], ssa=[1.0], phase=[("iso",)],
         fbeam=31.41592653589793, umu0=0.1, albedo=0.0),
    dict(test="ValidationDisotest1c", N=16, L=1, nmom=0, dtau=[0.03125], ssa=[0.99], phase=[("iso",)],
         fbeam=31.41592653589793, umu0=0.1, albedo=0.0),
    dict(test="ValidationDisotest1d", N=16, L=1, nmom=0, dtau=[32.0], ssa=[0.2], phase=[("iso",)],
         fbeam=31.41592653589793, umu0=0.1, albedo=0.0),
    dict(test="ValidationDisotest2a", N=16, L=1, nmom=0, dtau=[0.2], ssa=[0.5], phase=[("rayleigh",)],
         fbeam=PI, umu0=0.080442, albedo=0.0),
    dict(test="ValidationDisotest2b", N=16, L=1, nmom=0, dtau=[0.2], ssa=[1.0], phase=[("rayleigh",)],
         fbeam=PI, umu0=0.080442, albedo=0.0),
    dict(test="ValidationDisotest2c", N=16, L=1, nmom=0, dtau=[5.0], ssa=[0.5], phase=[("rayleigh",)],
         fbeam=PI, umu0=0.080442, albedo=0.0),
    dict(test="ValidationDisotest2d", N=16, L=1, nmom=0, dtau=[5.0], ssa=[1.0], phase=[("rayleigh",)],
         fbeam=PI, umu0=0.080442, albedo=0.0),
    dict(test="ValidationDisotest3a", N=16, L=1, nmom=32, dtau=[1.0], ssa=[1.0], phase=[("hg", 0.75)],
         fbeam=PI, umu0=1.0, albedo=0.0),
    dict(test="ValidationDisotest7a", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.1], phase=[("hg", 0.05)],
         thermal=True, temperature=[200.0, 300.0], wn=(300.0, 800.0), utau=[0.0, 1.0]),
    dict(test="ValidationDisotest7b", N=16, L=1, nmom=0, dtau=[100.0], ssa=[0.95], phase=[("hg", 0.75)],
         thermal=True, temperature=[200.0, 300.0], wn=(2702.99, 2703.01), utau=[0.0, 100.0],
         umu=[-1.0, 1.0], phi=[0.0]),
    dict(test="ValidationDisotest7c", N=12, L=1, nmom=0, dtau=[1.0], ssa=[0.5], phase=[("hg", 0.8)],
         thermal=True, temperature=[300.0, 200.0], wn=(0.0, 50000.0), fbeam=200.0, umu0=0.5,
         fisot=100.0, ttemp=100.0, btemp=320.0, utau=[0.0, 0.5, 1.0], umu=[-1.0, -0.1, 0.1, 1.0],
         phi=[0.0, 90.0]),
    # make9cConfig (test_solver.cpp:3309-3363)
    dict(test="ValidationDisotest9c", N=8, L=6, nmom=0, dtau=[1, 2, 3, 4, 5, 6],
         ssa=[0.65 + 0.05 * i for i in range(6)], phase=[("hg", (i + 1) / 7.0) for i in range(6)],
         thermal=True, temperature=[600.0 + 10 * i for i in range(7)], wn=(999.0, 1000.0),
         fbeam=PI, umu0=0.5, fisot=1.0, albedo=0.5, btemp=700.0, ttemp=550.0,
         utau=[0.0, 1.05, 2.1, 6.0, 21.0], umu=[-1.0, -0.2, 0.2, 1.0], phi=[60.0, 120.0, 180.0]),
    dict(test="ValidationDisotest10a", N=4, L=6, nmom=0, dtau=[1, 2, 3, 4, 5, 6],
         ssa=[0.65 + 0.05 * i for i in range(6)], phase=[("hg", (i + 1) / 7.0) for i in range(6)],
         thermal=True, temperature=[600.0 + 10 * i for i in range(7)], wn=(999.0, 1000.0),
         fbeam=PI, umu0=0.5, fisot=1.0, albedo=0.5, btemp=700.0, ttemp=550.0,
         utau=[0.0, 2.1, 21.0], umu=[-0.788675129, -0.211324871, 0.211324871, 0.788675129],
         phi=[60.0, 120.0]),
    # makeThermalConfig(tau, albedo, btemp, ttemp, temper_top, temper_bot, fbeam, umu0, ntau, utau)
    # (test_solver.cpp:3155-3213): N=16, 1 layer, ssa 0, wn [0, 50000], umu {-1,-0.1,0.1,1}
    dict(test="ThermalEmission_T1_AlbedoZero", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso0",)],
         thermal=True, temperature=[200.0, 300.0], wn=(0.0, 50000.0), albedo=0.0, btemp=300.0, ttemp=0.0,
         utau=[0.0, 1.0], umu=[-1.0, -0.1, 0.1, 1.0], phi=[0.0]),
    dict(test="ThermalEmission_T2_AlbedoHalf", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso0",)],
         thermal=True, temperature=[200.0, 300.0], wn=(0.0, 50000.0), albedo=0.5, btemp=300.0, ttemp=0.0,
         utau=[0.0, 1.0], umu=[-1.0, -0.1, 0.1, 1.0], phi=[0.0]),
    dict(test="ThermalEmission_T3_BeamPlusThermal", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso0",)],
         thermal=True, temperature=[0.0, 0.0], wn=(0.0, 50000.0), albedo=0.0, btemp=300.0, ttemp=0.0,
         fbeam=200.0, umu0=0.5, utau=[0.0, 0.5, 1.0], umu=[-1.0, -0.1, 0.1, 1.0], phi=[0.0]),
    dict(test="ThermalEmission_T4_InternalEmission", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso0",)],
         thermal=True, temperature=[250.0, 300.0], wn=(0.0, 50000.0), albedo=0.0, btemp=300.0, ttemp=250.0,
         utau=[0.0, 0.5, 1.0], umu=[-1.0, -0.1, 0.1, 1.0], phi=[0.0]),
    dict(test="HenyeyGreenstein", suite="DeltaMPlus", N=16, L=1, nmom=17, dtau=[1.0], ssa=[0.9],
         phase=[("hg", 0.85)], fbeam=1.0, umu0=0.5, albedo=0.1, dm_plus=True, utau=[0.0, 1.0],
         umu=[-1.0, -0.5, 0.5, 1.0], phi=[0.0]),
    dict(test="MultiLayer", suite="DeltaMPlus", N=16, L=6, nmom=17, dtau=[0.1, 0.2, 0.5, 1.0, 2.0, 5.0],
         ssa=[0.9] * 6, phase=[("hg", 0.9)], fbeam=1.0, umu0=0.5, albedo=0.1, dm_plus=True,
         utau=[0.0, 8.8], umu=[-1.0, -0.5, 0.5, 1.0], phi=[0.0]),
    dict(test="DisortFluxSolver", suite="DeltaMPlus", N=16, L=1, nmom=17, dtau=[1.0], ssa=[0.9],
         phase=[("hg", 0.85)], fbeam=1.0, umu0=0.5, albedo=0.1, dm_plus=True),
    dict(test="CloudGarciaSiewert", suite="DeltaMPlus", N=16, L=1, nmom=298, dtau=[5.0], ssa=[1.0],
         phase=[("cloud",)], fbeam=1.0, umu0=0.5, albedo=0.0, dm_plus=True, utau=[0.0, 5.0],
         umu=[-1.0, -0.5, 0.5, 1.0], phi=[0.0]),
    # bidirectional surfaces (general solver only).  Hapke (makeHapkeTestConfig1Layer,
    # test_solver.cpp:4038-4080; b0 1, hh 0.06, w 0.6 by default) and RPV (:4133-4190),
    # no intensity correction: fluxes and intensities pin the surface Fourier terms.
    dict(test="HapkeBRDF1", N=16, L=1, nmom=16, dtau=[1.0], ssa=[1.0], phase=[("hg", 0.75)],
         fbeam=PI, umu0=0.5, brdf=(4, [1.0, 0.06, 0.6]), utau=[0.0, 1.0],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="HapkeBRDF2", N=16, L=1, nmom=16, dtau=[0.5], ssa=[0.5], phase=[("iso",)],
         fbeam=1.0, umu0=0.8, brdf=(4, [1.0, 0.06, 0.6]), utau=[0.0, 0.5],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="RpvBRDF1", N=16, L=1, nmom=16, dtau=[0.3], ssa=[0.9], phase=[("iso",)],
         fbeam=1.0, umu0=0.6, brdf=(1, [0.1, 0.9, -0.2, 0.0, 0.0, 0.0, 1.0]), utau=[0.0, 0.3],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    # disotest 6d-6h (makeTest6dConfig, test_solver.cpp:2200-2250): Hapke surface under a
    # non-scattering layer with the intensity corrections switched on; without
    # scattering the Nakajima-Tanaka correction does not apply, the BRDF beam correction
    # of the intensities does ("intensity_corrected": the fluxes pin the surface alone)
    dict(test="ValidationDisotest6d", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso",)],
         fbeam=200.0, umu0=0.5, brdf=(4, [1.0, 0.06, 0.6]), corr=True, utau=[0.0, 0.5, 1.0],
         umu=[-1.0, -0.1, 0.1, 1.0], phi=[90.0], wn=(0.0, 50000.0)),
    dict(test="ValidationDisotest6e", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso",)],
         fbeam=200.0, umu0=0.5, brdf=(4, [1.0, 0.06, 0.6]), corr=True, utau=[0.0, 0.5, 1.0],
         umu=[-1.0, -0.1, 0.1, 1.0], phi=[90.0], thermal=True, temperature=[0.0, 0.0], wn=(0.0, 50000.0),
         btemp=300.0, ttemp=0.0),
    dict(test="ValidationDisotest6f", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso",)],
         fbeam=200.0, umu0=0.5, brdf=(4, [1.0, 0.06, 0.6]), corr=True, utau=[0.0, 0.5, 1.0],
         umu=[-1.0, -0.1, 0.1, 1.0], phi=[90.0], thermal=True, temperature=[0.0, 0.0], wn=(0.0, 50000.0),
         btemp=300.0, ttemp=250.0, fisot=100.0 / PI),
    dict(test="ValidationDisotest6g", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.0], phase=[("iso",)],
         fbeam=200.0, umu0=0.5, brdf=(4, [1.0, 0.06, 0.6]), corr=True, utau=[0.0, 0.5, 1.0],
         umu=[-1.0, -0.1, 0.1, 1.0], phi=[90.0], thermal=True, temperature=[250.0, 300.0], wn=(0.0, 50000.0),
         btemp=300.0, ttemp=250.0, fisot=100.0 / PI),
    dict(test="ValidationDisotest6h", N=16, L=1, nmom=0, dtau=[10.0], ssa=[0.0], phase=[("iso",)],
         fbeam=200.0, umu0=0.5, brdf=(4, [1.0, 0.06, 0.6]), corr=True, utau=[0.0, 1.0, 10.0],
         umu=[-1.0, -0.1, 0.1, 1.0], phi=[90.0], thermal=True, temperature=[250.0, 300.0], wn=(0.0, 50000.0),
         btemp=300.0, ttemp=250.0, fisot=100.0 / PI),
    # Nakajima-Tanaka intensity correction (makeICTestConfig1Layer, test_solver.cpp:3779-3825:
    # 16 streams, 16 moments, intensity_corr_buras and intensity_corr_nakajima on,
    # mu_user kUmu6, phi 0, black surface)
    dict(test="IntensityCorrectionIso1a", N=16, L=1, nmom=16, dtau=[0.03125], ssa=[0.2], phase=[("iso",)],
         fbeam=PI / 0.1, umu0=0.1, corr=True, utau=[0.0, 0.03125],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="IntensityCorrectionIso1b", N=16, L=1, nmom=16, dtau=[0.03125], ssa=[1.0], phase=[("iso",)],
         fbeam=PI / 0.1, umu0=0.1, corr=True, utau=[0.0, 0.03125],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="IntensityCorrectionIso1d", N=16, L=1, nmom=16, dtau=[32.0], ssa=[0.2], phase=[("iso",)],
         fbeam=PI / 0.1, umu0=0.1, corr=True, utau=[0.0, 32.0],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="IntensityCorrectionIso1e", N=16, L=1, nmom=16, dtau=[32.0], ssa=[1.0], phase=[("iso",)],
         fbeam=PI / 0.1, umu0=0.1, corr=True, utau=[0.0, 32.0],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="IntensityCorrectionHG3a", N=16, L=1, nmom=16, dtau=[1.0], ssa=[1.0], phase=[("hg", 0.75)],
         fbeam=PI, umu0=1.0, corr=True, utau=[0.0, 1.0],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="IntensityCorrectionHG3b", N=16, L=1, nmom=16, dtau=[8.0], ssa=[1.0], phase=[("hg", 0.75)],
         fbeam=PI, umu0=1.0, corr=True, utau=[0.0, 8.0],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    # Buras-Emde correction (makeNewICTestConfig1Layer, test_solver.cpp:3940-3987): the HG phase
    # function tabulated on 100 uniform cosines, intensity_corr_nakajima off
    dict(test="NewICHG3a", N=16, L=1, nmom=16, dtau=[1.0], ssa=[1.0], phase=[("hg", 0.75)],
         fbeam=PI, umu0=1.0, corr=True, tab=(0.75, 100), utau=[0.0, 1.0],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    dict(test="NewICHG3b", N=16, L=1, nmom=16, dtau=[8.0], ssa=[1.0], phase=[("hg", 0.75)],
         fbeam=PI, umu0=1.0, corr=True, tab=(0.75, 100), utau=[0.0, 8.0],
         umu=[-1.0, -0.5, -0.1, 0.1, 0.5, 1.0], phi=[0.0]),
    # ibcnd = Special (test_solver.cpp:4206-4318): albedo and transmissivity of the medium at
    # mu 0.5 with the spherical-albedo correction of a 0.5 surface albedo
    dict(test="SpecialBC13a", N=16, L=1, nmom=0, dtau=[1.0], ssa=[0.99], phase=[("hg", 0.8)],
         albedo=0.5, special=True, umu=[0.5]),
    dict(test="SpecialBC13c", N=16, L=2, nmom=0, dtau=[0.5, 0.5], ssa=[0.99, 0.5], phase=[("hg", 0.8)],
         albedo=0.5, special=True, umu=[0.5]),
    # disotest 12a (test_solver.cpp:3637-3700): 20 streams (oracle only; the engine takes 4-16, 32, 64)
    dict(test="ValidationDisotest12a", N=20, L=1, nmom=20, dtau=[20.1], ssa=[0.5], phase=[("hg", 0.9)],
         fbeam=1.0, umu0=1.0, albedo=1.0, corr=True, utau=[0.0, 10.0, 19.9, 20.1],
         umu=[-1.0, -0.1, 0.1, 1.0], phi=[0.0]),
    # pseudo-spherical beam (test_solver.cpp:4459-4533): altitudes 60/30/0 km, radius 6371 km
    dict(test="SphericalGeometry", N=16, L=2, nmom=0, dtau=[0.5, 1.0], ssa=[0.9, 0.8], phase=[("hg", 0.8)],
         fbeam=1.0, umu0=0.5, albedo=0.1, spherical=True, zalt=[60.0, 30.0, 0.0], radius=6371.0,
         umu=[-0.5, 0.1, 0.5, 1.0], phi=[0.0]),
]

FIELDS = ("flux_direct_beam", "flux_down", "flux_up", "flux_tau_divergence", "mean_intensity",
          "mean_intensity_down", "mean_intensity_up", "mean_intensity_direct_beam")


def test_bodies(text: str) -> dict:
    out = {}
    for m in re.finditer(r"TEST\((\w+),\s*(\w+)\)\s*\{", text):
        start = m.end()
        depth, i = 1, start
        while depth and i < len(text):
            if text[i] == "{":
                depth += 1
            elif text[i] == "}":
                depth -= 1
            i += 1
        line = text.count("\n", 0, m.start()) + 1
        out[(m.group(1), m.group(2))] = (text[start:i - 1], line)
    return out


def extract_expectations(body: str, body_line: int, L: int) -> tuple[list, list]:
    consts = {"nlyr": L}
    for m in re.finditer(r"(?:const\s+)?double\s+(\w+)\s*=\s*([0-9.eE+\-]+)\s*;", body):
        consts[m.group(1)] = float(m.group(2))
    # only expectations before the first re-solve of a modified config
    cut = re.search(r"\n\s*cfg\.flags\.\w+\s*=.*\n\s*auto\s+r2", body)
    body_use = body[:cut.start()] if cut else body
    fluxes, intens = [], []
    pat = re.compile(r"EXPECT_NEAR\(\s*\w+\.(%s)\[(\w+)\]\s*,\s*([-+0-9.eE]+)\s*,\s*([^;]+)\);" % "|".join(FIELDS))
    for m in pat.finditer(body_use):
        idx = m.group(2)
        idx = int(idx) if idx.isdigit() else int(consts[idx])
        tol = eval(m.group(4).replace("std::abs", "abs"), {"abs": abs}, dict(consts))
        line = body_line + body_use.count("\n", 0, m.start())
        fluxes.append(dict(field=m.group(1), index=idx, value=float(m.group(3)), tol=float(tol), line=line))
    pat2 = re.compile(r"EXPECT_NEAR\(\s*\w+\.intensities\((\d+),\s*(\d+),\s*(\d+)\)\s*,\s*([-+0-9.eE]+)\s*,\s*([^;]+)\);")
    for m in pat2.finditer(body_use):
        tol = eval(m.group(5).replace("std::abs", "abs"), {"abs": abs}, dict(consts))
        line = body_line + body_use.count("\n", 0, m.start())
        intens.append(dict(iu=int(m.group(1)), lu=int(m.group(2)), j=int(m.group(3)),
                           value=float(m.group(4)), tol=float(tol), line=line))
    return fluxes, intens


def cloud_table(src: str) -> list:
    m = re.search(r"fillCloudGarciaSiewert.*?cldmom\[\d+\]\s*=\s*\{(.*?)\};", src, re.S)
    return [float(x) for x in re.findall(r"[0-9]+\.[0-9]+", m.group(1))]


def moments(phase, nmom_nstr: int, cloud: list) -> list:
    kind = phase[0]
    pm = [0.0] * (nmom_nstr + 1)
    if kind == "hg":
        g, gk = phase[1], 1.0
        for k in range(nmom_nstr + 1):
            pm[k] = gk
            gk *= g
    elif kind in ("iso", "iso0"):
        pm[0] = 1.0
    elif kind == "rayleigh":
        pm[0] = 1.0
        if nmom_nstr >= 2:
            pm[2] = 0.1
    elif kind == "cloud":
        pm[0] = 1.0
        for k in range(1, nmom_nstr + 1):
            pm[k] = cloud[k - 1] / (2 * k + 1) if k <= 298 else 0.0
    return pm


def albtrans_expectations(body: str) -> list:
    """EXPECT_NEAR lines on albedo_medium / transmissivity_medium (ibcnd = Special)."""
    pat = re.compile(r"EXPECT_NEAR\(\s*\w+\.(albedo_medium|transmissivity_medium)\[(\d+)\]\s*,\s*([-+0-9.eE]+)\s*,"
                     r"\s*([^;]+)\);")
    return [dict(field=m.group(1), index=int(m.group(2)), value=float(m.group(3)),
                 tol=float(eval(m.group(4), {}, {}))) for m in pat.finditer(body)]


def tabulated(tab, L: int) -> dict:
    """The HG phase function on a uniform cosine grid, as makeNewICTestConfig1Layer fills it."""
    if tab is None:
        return {}
    g, n = tab
    mu = [-1.0 + 2.0 * it / (n - 1) for it in range(n)]
    val = []
    for ct in mu:
        d = 1.0 + g * g - 2.0 * g * ct
        val.append((1.0 - g * g) / (d * math.sqrt(d)))
    return dict(mu_phase_function=mu, phase_function=[val] * L)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_goldens.py /path/to/DisORT (the DisORT++ source tree)")
    ref = sys.argv[1]
    text = open(os.path.join(ref, "tests", "test_solver.cpp")).read()
    cloud = cloud_table(open(os.path.join(ref, "src", "PhaseFunction.cpp")).read())
    bodies = test_bodies(text)
    cases = []
    for c in CASES:
        suite = c.get("suite", "SolverTest")
        body, line = bodies[(suite, c["test"])]
        body = re.sub(r"//[^\n]*", "", body)  # commented-out expectations do not count
        N, L, nmom = c["N"], c["L"], c["nmom"]
        nmn = max(nmom, N)
        ph = c["phase"] if len(c["phase"]) == L else c["phase"] * L
        fl, it = extract_expectations(body, line, L)
        cases.append(dict(
            name=f"{suite}.{c['test']}", source=f"tests/test_solver.cpp:{line}",
            num_streams=N, num_layers=L, num_phase_func_moments=nmom,
            delta_tau=[float(x) for x in c["dtau"]], single_scat_albedo=[float(x) for x in c["ssa"]],
            phase_function_moments=[moments(p, nmn, cloud) for p in ph],
            use_thermal_emission=bool(c.get("thermal", False)),
            temperature=c.get("temperature", []),
            wavenumber_low=c.get("wn", (0.0, 0.0))[0], wavenumber_high=c.get("wn", (0.0, 0.0))[1],
            direct_beam_flux=c.get("fbeam", 0.0), direct_beam_mu=c.get("umu0", 0.5),
            isotropic_flux_top=c.get("fisot", 0.0), surface_albedo=c.get("albedo", 0.0),
            temperature_top=c.get("ttemp", 0.0), temperature_bottom=c.get("btemp", 0.0),
            emissivity_top=1.0, use_delta_m_plus=bool(c.get("dm_plus", False)),
            tau_user=c.get("utau"), mu_user=c.get("umu"), phi_user=c.get("phi"),
            use_spherical_beam=bool(c.get("spherical", False)), level_altitudes=c.get("zalt"),
            bottom_radius=c.get("radius", 0.0),
            brdf_type=c["brdf"][0] if "brdf" in c else 0,
            brdf_params=c["brdf"][1] if "brdf" in c else [],
            intensity_corrected=bool(c.get("corr", False)),
            special_bc=bool(c.get("special", False)), expect_albtrans=albtrans_expectations(body),
            **tabulated(c.get("tab"), L),
            expect_flux=fl, expect_intensity=it,
        ))
    out = dict(generated_by="tests/golden/make_reference_goldens.py",
               reference="DisORT++ tests/test_solver.cpp and src/PhaseFunction.cpp", cases=cases)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}: {len(cases)} cases, "
          f"{sum(len(c['expect_flux']) for c in cases)} flux and "
          f"{sum(len(c['expect_intensity']) for c in cases)} intensity expectations")


if __name__ == "__main__":
    main()
