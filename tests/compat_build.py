"""Builds tests/compat/compat_probe.cpp (test infrastructure): a
reference-style caller of the mean-field plugin table, compiled against the
oracle's shim of the reference's type declarations and
include/btam_dmd_equations.hpp, linked with bt-am_b200/lib/libbtam.so."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "compat", "compat_probe.cpp")
OUT = os.path.join(ROOT, "tests", "compat", "_build", "compat_probe")


def build_probe(defines=()):
    """The probe, compiled with the given -D macros (a separate binary per
    set: e.g. the reference's MULTIPOLE_INTEGRAL switch)."""
    lib = os.path.join(ROOT, "bt-am_b200", "lib")
    out = OUT + "".join("_" + d.split("=")[0].lower() for d in defines)
    deps = [SRC, os.path.join(ROOT, "include", "btam_dmd_equations.hpp"),
            os.path.join(ROOT, "include", "btam.h"), os.path.join(lib, "libbtam.so")]
    if os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O1", *("-D" + d for d in defines),
                    "-I", os.path.join(ROOT, "oracle", "ref_shim"),
                    "-I", os.path.join(ROOT, "include"), SRC, "-L", lib, "-lbtam",
                    "-Wl,-rpath," + lib, "-o", out], check=True)
    return out
