"""Build oracle/_ref/libmeraxes_ref.so: the reference's own reionization step, compiled unmodified
from its sources, over in-tree stand-ins for FFTW, GSL, MPI, HDF5 and mlog -- TEST INFRASTRUCTURE.

    python oracle/build_ref.py [--reference DIR] [--force]

The reference sources compiled (from DIR/src/core, default /root/reference):
find_HII_bubbles.c, ComputeTs.c, XRayHeatingFunctions.c, BrightnessTemperature.c, reionization.c,
recombinations.c, misc_tools.c, virial_properties.c, utils.c.  Nothing is copied from them: gcc
reads them where they lie.  The stand-ins (oracle/ref_shim) are:

* ``include/`` -- declarations of the third-party APIs those files include (fftw3.h,
  fftw3-mpi.h, mpi.h, hdf5.h, hdf5_hl.h, gsl/*.h, mlog.h) and the configure-time
  meraxes_conf.h with the reference's default CMake options;
* ``ref_fft.c`` (FFTW plans over a double-precision FFT), ``ref_gsl.c`` (natural cubic spline,
  QAG with the 61-point Gauss-Kronrod rule, Brent), ``ref_mpi_mlog.c`` (one MPI rank, logging),
  ``ref_driver.c`` (Meraxes' start-up for one rank and the C entry points the tests call);
* a generated ``ref_gk61.h`` (the Gauss-Kronrod table, from oracle/gk61.py) and a generated
  stub file: every other external symbol the reference objects name (HDF5 output, the galaxy
  tree readers) becomes a function that aborts with its name, since the step never calls them.

Two libraries are built: libmeraxes_ref.so (the default build) and libmeraxes_ref_mini.so
(-DUSE_MINI_HALOS, the mini-halo build).  Both go to oracle/_ref/, which git ignores.
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "ref_shim")
OUT = os.path.join(HERE, "_ref")
BUILD = os.path.join(HERE, "_build")
REF_SOURCES = ["find_HII_bubbles.c", "ComputeTs.c", "XRayHeatingFunctions.c", "BrightnessTemperature.c",
               "reionization.c", "recombinations.c", "misc_tools.c", "virial_properties.c", "utils.c"]
SHIM_SOURCES = ["ref_fft.c", "ref_gsl.c", "ref_mpi_mlog.c", "ref_driver.c"]
CFLAGS = ["-std=gnu11", "-O2", "-fPIC", "-fcommon", "-w", "-Werror=implicit-function-declaration"]
LIBS = ["/lib/x86_64-linux-gnu/libc.so.6", "/lib/x86_64-linux-gnu/libm.so.6"]


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout


def gk61_header(path):
    sys.path.insert(0, HERE)
    import gk61
    xgk, wgk, wg = gk61.rule()
    fmt = lambda a: ",\n  ".join(repr(float(v)) for v in a)
    text = ("/* The 61-point Gauss-Kronrod rule on [-1, 1], generated by oracle/build_ref.py from\n"
            "   oracle/gk61.py: nodes descending (xgk[30] = 0), Kronrod weights, Gauss weights at the\n"
            "   odd positions (zero at the Kronrod-only nodes). */\n"
            f"static const double RG_REF_XGK[31] = {{\n  {fmt(xgk)}}};\n"
            f"static const double RG_REF_WGK[31] = {{\n  {fmt(wgk)}}};\n"
            f"static const double RG_REF_WG[30] = {{\n  {fmt(wg)}}};\n")
    with open(path, "w") as f:
        f.write(text)


def runtime_symbols() -> set:
    """Symbols libc, libm and gcc's runtime library (complex arithmetic helpers) provide."""
    out = set()
    for lib in LIBS:
        if os.path.exists(lib):
            for line in run(["nm", "-D", "--defined-only", lib]).splitlines():
                parts = line.split()
                if parts:
                    out.add(parts[-1].split("@")[0])
    libgcc = run(["gcc", "-print-libgcc-file-name"]).strip()
    for line in run(["nm", "--defined-only", libgcc]).splitlines():
        parts = line.split()
        if len(parts) == 3:
            out.add(parts[2])
    return out


def build(reference: str, variant: str, force: bool) -> str:
    mini = variant == "mini"
    lib = os.path.join(OUT, "libmeraxes_ref_mini.so" if mini else "libmeraxes_ref.so")
    bdir = os.path.join(BUILD, "ref_" + variant)
    os.makedirs(bdir, exist_ok=True)
    os.makedirs(OUT, exist_ok=True)
    core = os.path.join(reference, "src", "core")
    srcs = [os.path.join(core, s) for s in REF_SOURCES] + [os.path.join(SHIM, s) for s in SHIM_SOURCES]
    newest = max(os.path.getmtime(s) for s in srcs + [__file__])
    for root, _, files in os.walk(os.path.join(SHIM, "include")):
        newest = max([newest] + [os.path.getmtime(os.path.join(root, f)) for f in files])
    if not force and os.path.exists(lib) and os.path.getmtime(lib) >= newest:
        return lib
    gk = os.path.join(BUILD, "ref_gk61.h")
    gk61_header(gk)
    inc = ["-I" + os.path.join(SHIM, "include"), "-I" + BUILD, "-I" + os.path.join(reference, "src"), "-I" + core]
    defs = ["-DUSE_MINI_HALOS"] if mini else []
    objs = []
    for s in srcs:
        o = os.path.join(bdir, os.path.basename(s) + ".o")
        run(["gcc"] + CFLAGS + defs + inc + ["-c", s, "-o", o])
        objs.append(o)
    # every external symbol nothing here defines and libc/libm do not provide: an aborting stub
    defined, undefined = set(), set()
    for o in objs:
        for line in run(["nm", o]).splitlines():
            parts = line.split()
            if len(parts) == 2 and parts[0] == "U":
                undefined.add(parts[1])
            elif len(parts) == 3 and parts[1] in "TDBCRVWtdbr" and parts[1].isupper():
                defined.add(parts[2])
    missing = sorted(undefined - defined - runtime_symbols() - {"_GLOBAL_OFFSET_TABLE_"})
    stub = os.path.join(bdir, "ref_stubs.c")
    with open(stub, "w") as f:
        f.write("/* Generated by oracle/build_ref.py: external symbols of the reference objects that the\n"
                "   reionization step never calls.  Each aborts with its name. */\n"
                "#include <stdio.h>\n#include <stdlib.h>\n"
                "static void rg_ref_unsupported(const char* what) {\n"
                "  fprintf(stderr, \"oracle/_ref: %s is not provided (outside the reionization step)\\n\", what);\n"
                "  abort();\n}\n")
        for name in missing:
            f.write(f"void {name}(void) {{ rg_ref_unsupported(\"{name}\"); }}\n")
    so = os.path.join(bdir, "ref_stubs.c.o")
    run(["gcc"] + CFLAGS + ["-c", stub, "-o", so])
    run(["gcc", "-shared", "-o", lib] + objs + [so, "-lm", "-Wl,--no-undefined"])
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    if not os.path.isdir(os.path.join(a.reference, "src", "core")):
        print("reference sources not found; nothing built")
        return
    for v in ("default", "mini"):
        print(build(a.reference, v, a.force))


if __name__ == "__main__":
    main()
