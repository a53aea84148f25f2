"""The tiled 3D work queue's z chunks (chunk_count / chunk_span in
vespa.jl_b200/csrc/vb_launch.h), checked on the host: compiled by nvcc as
host code and run without a GPU.  Every (nz, kz) must give contiguous chunks
covering [0, nz) exactly once, none longer than kz; the uniform form must be
the plain ceil(nz / kz) chunks; with kz >= 16 the tapered form's tail pieces
must have at least 8 planes (all of nz when nz < 8) and its last piece fewer
than 16."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "vespa.jl_b200", "csrc")

PROGRAM = r'''
#include <cstdio>
#include "vb_launch.h"
int main()
{
    const int nzs[] = {2, 3, 7, 8, 9, 15, 16, 17, 24, 31, 33, 47, 48, 49, 64, 95, 96, 97, 100,
                       128, 129, 160, 191, 255, 256, 257, 300, 384, 512, 1000, 4096};
    const int kzs[] = {1, 2, 4, 8, 16, 24, 32, 40, 48, 64, 96, 128};
    for (int nz : nzs)
        for (int kz : kzs)
            for (int taper = 0; taper < 2; ++taper) {
                int nchu = 0;
                const int n = vb::chunk_count(nz, kz, taper != 0, &nchu);
                int prev = 0, last = 0;
                for (int c = 0; c < n; ++c) {
                    int k0, k1;
                    vb::chunk_span(nz, kz, nchu, c, k0, k1);
                    if (k0 != prev || k1 <= k0 || k1 - k0 > kz) {
                        std::printf("BAD %d %d %d chunk %d [%d, %d)\n", nz, kz, taper, c, k0, k1);
                        return 1;
                    }
                    const int minp = nz < 8 ? nz : 8;
                    if (taper && kz >= 16 && c >= nchu && k1 - k0 < minp) {
                        std::printf("BAD short tail piece %d %d chunk %d: %d\n", nz, kz, c, k1 - k0);
                        return 1;
                    }
                    prev = k1;
                    last = k1 - k0;
                }
                if (prev != nz) {
                    std::printf("BAD %d %d %d ends at %d\n", nz, kz, taper, prev);
                    return 1;
                }
                if (!taper && n != (nz + kz - 1) / kz) {
                    std::printf("BAD uniform count %d %d: %d\n", nz, kz, n);
                    return 1;
                }
                if (taper && kz >= 16 && last >= 16) {
                    std::printf("BAD taper end %d %d: %d\n", nz, kz, last);
                    return 1;
                }
            }
    std::printf("OK\n");
    return 0;
}
'''


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_chunk_partition(tmp_path):
    src = tmp_path / "chunks.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "chunks"
    subprocess.run(["nvcc", "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe)], check=True, capture_output=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stdout
