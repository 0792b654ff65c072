"""Generate phase_tables.inc: the Garcia & Siewert (1985) Haze-L and Cloud C.1
Legendre-moment tables used by setHazeGarciaSiewert / setCloudGarciaSiewert.

These published coefficient tables must be identical to the reference's for the
phase-function helpers to agree, so they are extracted from DisORT++
src/PhaseFunction.cpp (fillHazeGarciaSiewert / fillCloudGarciaSiewert):

    python disort_b200/csrc/host/make_phase_tables.py /path/to/DisORT
"""
import os
import re
import sys


def table(src: str, func: str, name: str) -> list:
    m = re.search(func + r".*?" + name + r"\[\d+\]\s*=\s*\{(.*?)\};", src, re.S)
    return [x for x in re.findall(r"[0-9]+\.[0-9]+", m.group(1))]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_phase_tables.py /path/to/DisORT (the DisORT++ source tree)")
    ref = sys.argv[1]
    src = open(os.path.join(ref, "src", "PhaseFunction.cpp")).read()
    haze = table(src, "fillHazeGarciaSiewert", "hazelm")
    cloud = table(src, "fillCloudGarciaSiewert", "cldmom")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "phase_tables.inc")
    with open(out, "w") as f:
        f.write("// Generated by make_phase_tables.py: Garcia & Siewert (1985) Haze-L and\n")
        f.write("// Cloud C.1 phase-function Legendre coefficients (coefficient k is for moment k+1).\n")
        f.write(f"static const int kHazeCount = {len(haze)};\n")
        f.write("static const double kHazeL[] = {\n")
        for i in range(0, len(haze), 10):
            f.write("  " + ", ".join(haze[i:i + 10]) + ",\n")
        f.write("};\n")
        f.write(f"static const int kCloudCount = {len(cloud)};\n")
        f.write("static const double kCloudC1[] = {\n")
        for i in range(0, len(cloud), 12):
            f.write("  " + ", ".join(cloud[i:i + 12]) + ",\n")
        f.write("};\n")
    print(f"wrote {out}: {len(haze)} haze, {len(cloud)} cloud coefficients")


if __name__ == "__main__":
    main()
