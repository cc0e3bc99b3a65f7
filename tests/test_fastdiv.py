"""The exact multiply-high division the transport uses for region indices
(FastDiv in omc_device.cuh; Granlund and Montgomery 1994) against integer
division, compiled from the header on the host: divisors 1 to 5000 and
the phantom strides the workloads use, dividends at 0, the ends of each
divisor's multiples and up to 2^31 - 1."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = r'''
#include <cstdio>
#include <cstdint>
#include "omc_device.cuh"
int main() {
    unsigned long long checked = 0, bad = 0;
    uint32_t ds[6000];
    int nd = 0;
    for (uint32_t d = 1; d <= 5000; d++) ds[nd++] = d;
    const uint32_t extra[] = {64u * 64u, 128u * 128u, 256u * 256u, 30u * 30u, 32u * 32u, 1u << 20, 65537u, 1000003u,
                              (1u << 31) - 1u, 1u << 31, (1u << 31) + 1u, 4000000000u, 4294967295u};
    for (uint32_t d : extra) ds[nd++] = d;
    for (int a = 0; a < nd; a++) {
        const uint32_t d = ds[a];
        const omc::FastDiv f = omc::FastDiv::make(d);
        uint32_t ns[16] = {0u, 1u, d - 1u, d, d + 1u, 2u * d - 1u, 2u * d, 12345678u, 2147483647u, 2147483646u,
                           (2147483647u / d) * d, (2147483647u / d) * d - 1u, 1048575u, 16777215u, 268435455u,
                           1000000007u};
        for (uint32_t n : ns) {
            if (n > 2147483647u) continue;
            checked++;
            if (f.div(n) != n / d) bad++;
        }
        for (uint32_t n = 0; n < 3000000u; n += 997u + a % 13u) {
            checked++;
            if (f.div(n) != n / d) bad++;
        }
    }
    std::printf("%llu %llu\n", checked, bad);
    return bad != 0;
}
'''


def test_fastdiv_exact(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    src = tmp_path / "fastdiv.cu"
    src.write_text(SRC)
    exe = tmp_path / "fastdiv"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-I", str(ROOT / "ompmc_b200" / "csrc"), "-o", str(exe), str(src)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    checked, bad = map(int, out.stdout.split())
    assert checked > 1_000_000
    assert bad == 0 and out.returncode == 0
