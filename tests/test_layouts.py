"""Device buffer layouts: every sub-array of a window's shared memory starts
on its type's alignment (16 bytes for complex128), for every window shape
the planner can produce.  Compiled for the host with nvcc; no GPU needed."""

import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "qfb_common.cuh"
#include "qfb_window.cuh"
int main() {
    int bad = 0;
    for (int nt = 1; nt <= 2; ++nt)
      for (int b = 1; b <= 12; ++b)
        for (int L = 0; L <= 3 && L <= b; ++L)
          for (int nstr = 0; nstr <= qfbw::kWinMaxStr; nstr += (nstr < 20 ? 1 : 7))
            for (int nsteps = 0; nsteps <= nstr && nsteps <= 2 * qfbw::kWinMaxSteps;
                 nsteps += (nsteps < 8 ? 1 : 37)) {
              for (int ntab = 0; ntab <= qfbw::kWinMaxTab; ntab += 1 + ntab / 3) {
                qfbw::WinSmem m = qfbw::win_smem_layout(b, L, nstr, nsteps, nt, ntab);
                bad += (m.cs_step % 16) + (m.cs_str % 16) + (m.gtab % 16) + (m.ipw % 16) +
                       (m.steps % 8) + (m.g_step % 8) + (m.sc_str % 8) + (m.zl_str % 8) +
                       (m.q_str % 4) + (m.tab % 16);
                // the planner's largest windows fit the 227 KB a block may use
                if (nsteps <= qfbw::kWinMaxSteps && ((b <= 12 && nt == 1) || (b <= 11 && nt == 2)))
                    bad += m.total > 227u * 1024u;
              }
            }
    printf("%d\n", bad);
    return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
def test_window_shared_memory_layout_alignment():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.cu")
        exe = os.path.join(d, "layout")
        with open(src, "w") as f:
            f.write(PROGRAM)
        subprocess.run([nvcc, "-std=c++17", "-I", os.path.join(ROOT, "qforte_b200", "csrc"),
                        "-I", os.path.join(ROOT, "include"), "-o", exe, src], check=True,
                       capture_output=True)
        out = subprocess.run([exe], capture_output=True, text=True)
        assert out.returncode == 0 and out.stdout.strip() == "0", out.stdout
