"""The C++ call-site replacement shown in INTEGRATION.md compiles and links
against include/dcore_b200.h and the shared library with the documented
command line, and runs: without a GPU every compute call returns
DC_ERR_NO_DEVICE with a message (no CPU fallback); with one it decomposes."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "dcore_b200.h"

int main() {
    std::printf("version %s\n", dc_version());
    // a 3-cycle plus one chord: kmax 1 on the cycle
    std::vector<uint32_t> src = {0, 1, 2, 0}, dst = {1, 2, 0, 2};
    dc_graph* h = nullptr;
    int rc = dc_graph_create(3, src.size(), src.data(), dst.data(), nullptr, &h);
    if (rc != DC_OK) {
        std::printf("create rc %d %s\n", rc, dc_last_error());
        return rc == DC_ERR_NO_DEVICE ? 0 : 1;
    }
    int32_t kmax = 0, lmax = 0;
    rc = dc_decompose(h, DC_METHOD_INCREMENTAL, &kmax, &lmax);
    std::printf("decompose rc %d kmax %d lmax %d\n", rc, kmax, lmax);
    std::vector<int32_t> km(3);
    if (rc == DC_OK) rc = dc_get_kmaxes(h, km.data());
    dc_graph_free(h);
    return rc == DC_OK ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_documented_cpp_driver_builds_and_runs(dc, tmp_path):
    src = tmp_path / "my_driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "my_driver"
    libdir = os.path.dirname(dc.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", str(src), "-I", os.path.join(ROOT, "include"), "-L", libdir,
                    "-ldcore_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "version" in r.stdout and "sm_100a" in r.stdout
    assert ("create rc -9" in r.stdout) or ("decompose rc 0 kmax" in r.stdout)
