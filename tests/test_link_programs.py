"""Programs written against the reference interfaces build unchanged against
include/ and link to libdedisp.so: a C program on the C API
(src/clib/dedisp.h; its use mirrors bin/test/ctestdedisp.c:286-345) and a
C++ program on the plan classes (src/tdd/TDDPlan.hpp:17-57,
src/dedisp/DedispPlan.hpp:21-66, src/fdd/FDDGPUPlan.hpp:18-35). Both stop at
plan setup, which needs no GPU: the DM list, delays and getters."""
import os
import shutil
import subprocess

import pytest

import dedisp_tests_b200 as dd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.dirname(dd.LIB_PATH)

C_PROGRAM = r"""
#include <stdio.h>
#include "dedisp.h"

int main(void)
{
    dedisp_plan plan = 0;
    dedisp_error e = dedisp_select_implementation(DEDISP_TDD);
    if (e != DEDISP_NO_ERROR) return 10;
    e = dedisp_create_plan(&plan, 4096, 64e-6f, 1500.0f, -0.078125f);
    if (e != DEDISP_NO_ERROR || !plan) return 11;
    e = dedisp_generate_dm_list(plan, 0.f, 2000.f, 40.f, 1.25f);
    if (e != DEDISP_NO_ERROR) return 12;
    printf("%lu %lu %lu %.4f\n", (unsigned long)dedisp_get_dm_count(plan),
           (unsigned long)dedisp_get_max_delay(plan), (unsigned long)dedisp_get_channel_count(plan),
           (double)dedisp_get_df(plan));
    printf("%s\n", dedisp_get_error_string(DEDISP_TOO_FEW_NSAMPS));
    dedisp_destroy_plan(plan);
    return 0;
}
"""

CXX_PROGRAM = r"""
#include <cstdio>
#include <vector>
#include <dedisp/DedispPlan.hpp>
#include <fdd/FDDGPUPlan.hpp>
#include <tdd/TDDPlan.hpp>

int main()
{
    dedisp::TDDPlan plan(1024, 250e-6f, 1581.8f, -0.390625f);
    std::vector<float> dms(512);
    for (int i = 0; i < 512; ++i) dms[i] = 500.0f * (float)i / 511.0f;
    plan.set_dm_list(dms.data(), dms.size());
    plan.set_gulp_size(65536);
    std::printf("%lu %lu %lu\n", (unsigned long)plan.get_dm_count(),
                (unsigned long)plan.get_max_delay(), (unsigned long)plan.get_gulp_size());
    dedisp::DedispPlan legacy(4096, 64e-6f, 1500.0f, -0.078125f);
    legacy.generate_dm_list(0.f, 2000.f, 40.f, 1.25f);
    dedisp::FDDGPUPlan fdd(1024, 250e-6f, 1581.8f, -0.390625f);
    fdd.set_dm_list(dms.data(), dms.size());
    std::printf("%lu %lu %lu\n", (unsigned long)legacy.get_dm_count(), (unsigned long)legacy.get_max_delay(),
                (unsigned long)fdd.get_max_delay());
    return 0;
}
"""


def _build_and_run(tmp_path, compiler, src, name, std):
    path = tmp_path / name
    path.write_text(src)
    exe = tmp_path / (name + ".out")
    cmd = [compiler, *std, "-I" + INC, str(path), "-o", str(exe), "-L" + LIBDIR, "-ldedisp",
           "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr[-2000:])
    return r.stdout.split("\n")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_on_the_reference_c_api(tmp_path):
    out = _build_and_run(tmp_path, "gcc", C_PROGRAM, "app.c", ["-std=c99"])
    assert out[0] == "3643 35500 4096 -0.0781"
    assert out[1] == "No. samples < maximum delay"


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cxx_program_on_the_reference_plan_classes(tmp_path):
    out = _build_and_run(tmp_path, "g++", CXX_PROGRAM, "app.cpp", ["-std=c++17"])
    assert out[0] == "512 2622 65536"
    assert out[1] == "3643 35500 2622"
