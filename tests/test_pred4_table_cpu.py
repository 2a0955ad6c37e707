"""The key-frame screen's 4x4 prediction table (csrc/device/pred4_table.h)
equals the reference-restating predictor pred4_px (csrc/device/intra.cuh)
sample for sample: both are compiled for the host with g++ and compared over
every mode, sample position and availability, on random neighbours."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

HARNESS = r'''
#include <cstdio>
#include <cstdlib>
#define __device__
#define __host__
#define __forceinline__ inline
#include "pred4_table.h"
namespace fdvb {
#include "pred4_px.inc"
}
int main() {
    using namespace fdvb;
    const P4Tab tab = make_p4tab();
    srand(7);
    long bad = 0;
    for (int it = 0; it < 20000; ++it) {
        int Tn[9], Ln[5], N[14];
        for (int i = 0; i < 9; ++i) Tn[i] = rand() & 255;
        for (int i = 0; i < 5; ++i) Ln[i] = rand() & 255;
        Ln[0] = Tn[0];
        const int ht = it & 1, hl = (it >> 1) & 1;
        for (int i = 0; i < 4; ++i) N[i] = Ln[4 - i];
        N[4] = Tn[0];
        for (int i = 0; i < 8; ++i) N[5 + i] = Tn[1 + i];
        N[13] = p4_dc(Tn, Ln, ht, hl);
        for (int m = 0; m < 9; ++m)
            for (int y = 0; y < 4; ++y)
                for (int x = 0; x < 4; ++x)
                    if (pred4_px(m, Tn, Ln, ht, hl, x, y) != p4_eval(tab.op[m * 16 + y * 4 + x], N)) ++bad;
    }
    printf("%ld\n", bad);
    return bad != 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_pred4_table_equals_pred4_px(tmp_path):
    dev = os.path.join(ROOT, "fdv_b200", "csrc", "device")
    src = open(os.path.join(dev, "intra.cuh")).read()
    m = re.search(r"__device__ inline int pred4_px\(.*?\n}\n", src, re.S)
    assert m, "pred4_px not found"
    (tmp_path / "pred4_px.inc").write_text(m.group(0).replace("__device__ inline", "inline"))
    (tmp_path / "pred4_table.h").write_text(open(os.path.join(dev, "pred4_table.h")).read())
    (tmp_path / "h.cpp").write_text(HARNESS)
    exe = tmp_path / "h"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(tmp_path), "-o", str(exe), str(tmp_path / "h.cpp")],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "0", r.stdout
