"""CPU tests of the C ABI: the library loads, exports every declared symbol, and the
ctypes mirror of each struct has the C layout.  No compute call needs a GPU here."""

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import reion_oracle as ro
import rg_b200 as rg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rg_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rg_[a-zA-Z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = rg.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", rg.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT " + n + r"\b", out), n


def test_struct_layouts_match_c():
    structs = {"rg_params": rg.rg_params, "rg_grids": rg.rg_grids, "rg_snapshot": rg.rg_snapshot,
               "rg_hii_scalars": rg.rg_hii_scalars, "rg_ts_scalars": rg.rg_ts_scalars}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rg_b200.h"', "int main(void) {"]
    for s, cls in structs.items():
        lines.append(f'printf("{s} size %zu\\n", sizeof({s}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{s} {f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-I" + os.path.dirname(HEADER), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, out):
        parts = line.split()
        cls = structs[parts[0]]
        if parts[1] == "size":
            assert C.sizeof(cls) == int(parts[2]), line
        else:
            assert getattr(cls, parts[1]).offset == int(parts[2]), line


def test_params_default_and_schedule_match_oracle():
    lib = rg.load()
    for n, box, z, rmax, filt in [(64, 64.0, 8.0, 50.0, 0), (256, 250.0, 7.0, 50.0, 1), (512, 500.0, 8.0, 1000.0, 2),
                                  (96, 96.0, 10.0, 50.0, 0), (32, 10.0, 6.5, 20.0, 0)]:
        p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=rmax, ReionFilterType=filt)
        radii = (C.c_double * 200)()
        cnt = C.c_int()
        assert lib.rg_radius_schedule(C.byref(p), z, radii, 200, C.byref(cnt)) == rg.RG_OK
        op = ro.Params(ReionGridDim=n, BoxSize=box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=rmax)
        sched = ro.radius_schedule(op, z)
        assert cnt.value == len(sched)
        assert np.allclose([radii[i] for i in range(cnt.value)], [r for r, _ in sched], rtol=0, atol=0)
    p = rg.make_params(64, 64.0)
    assert p.ReionEfficiency == pytest.approx(1.0 / 0.15714 * 4000 / (1 - 0.75 * 0.24))
    assert p.TsNumFilterSteps == 40 and p.TsHeatingFilterType == 1 and p.ReionUVBFlag == 1


def test_invalid_arguments_rejected_without_gpu():
    lib = rg.load()
    h = C.c_void_p()
    # unsupported grid size is refused before any device call
    assert lib.rg_create(0, 100, C.byref(h)) == rg.RG_EUNSUPPORTED
    assert lib.rg_create(0, 64, None) == rg.RG_EINVAL
    assert lib.rg_status_string(rg.RG_EINVAL) == b"invalid argument"
    assert lib.rg_destroy(None) == rg.RG_EINVAL
    p = rg.make_params(64, 64.0, ReionDeltaRFactor=1.0)
    cnt = C.c_int()
    assert lib.rg_radius_schedule(C.byref(p), 8.0, None, 0, C.byref(cnt)) == rg.RG_EINVAL


def test_create_without_device_reports_nodev():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = rg.load()
    h = C.c_void_p()
    assert lib.rg_create(0, 64, C.byref(h)) == rg.RG_ENODEV


def test_host_only_functions_reject_bad_arguments():
    lib = rg.load()
    n = C.c_int()
    p = rg.make_params(32, 32.0)
    assert lib.rg_power_spectrum_length(None, C.byref(n)) == rg.RG_EINVAL
    bad = rg.make_params(32, -1.0)
    assert lib.rg_power_spectrum_length(C.byref(bad), C.byref(n)) == rg.RG_EINVAL
    assert lib.rg_power_spectrum_length(C.byref(p), C.byref(n)) == rg.RG_OK and n.value > 0
    radii = (C.c_double * 8)()
    assert lib.rg_radius_schedule(C.byref(bad), 8.0, radii, 8, C.byref(n)) == rg.RG_EINVAL
    assert lib.rg_params_default(None, 32, 32.0) == rg.RG_EINVAL
