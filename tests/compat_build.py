"""Builds tests/compat/compat_probe.cpp (test infrastructure): a
reference-style caller of the mean-field plugin table, compiled against the
oracle's shim of the reference's type declarations and
include/btam_dmd_equations.hpp, linked with bt-am_b200/lib/libbtam.so."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "compat", "compat_probe.cpp")
OUT = os.path.join(ROOT, "tests", "compat", "_build", "compat_probe")


def build_probe():
    lib = os.path.join(ROOT, "bt-am_b200", "lib")
    deps = [SRC, os.path.join(ROOT, "include", "btam_dmd_equations.hpp"),
            os.path.join(ROOT, "include", "btam.h"), os.path.join(lib, "libbtam.so")]
    if os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "oracle", "ref_shim"),
                    "-I", os.path.join(ROOT, "include"), SRC, "-L", lib, "-lbtam",
                    "-Wl,-rpath," + lib, "-o", OUT], check=True)
    return OUT
