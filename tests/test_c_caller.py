"""The C ABI from a C caller: a C99 program compiled against include/mcv_gpu.h
and linked with libmcv_gpu.so exercises the calls that need no GPU (grid
sizes, footprints, argument checks, the server queue).  Shows the header is
plain C and the library links as a C library would be linked by a driver."""
import os
import shutil
import subprocess

import pytest

from mcv_sw_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "mcv_gpu.h"

#define CHECK(c) do { if (!(c)) { printf("FAIL line %d\n", __LINE__); return 1; } } while (0)

int main(void) {
  int npx, n, halo;
  CHECK(mcv_grid_sizes(4, 256, &npx, &n, &halo) == MCV_OK);
  CHECK(n == 769 && halo == 3 && npx == 775);
  CHECK(mcv_footprint_bytes(4, 256, MCV_RK3_TVD, MCV_MIXED, 1) > 0);
  mcv_handle *h = NULL;
  CHECK(mcv_create(5, 32, MCV_RK4, MCV_FP64, 100.0, 6.371e6, 1, &h) == MCV_ERR_ARG);
  CHECK(strstr(mcv_last_error(), "order") != NULL);
  CHECK(mcv_step(NULL, 1) == MCV_ERR_ARG);
  mcv_server *s = NULL;
  CHECK(mcv_server_create(MCV_FP64, MCV_RK3_TVD, 6.371e6, 1LL << 30, 64LL << 20, 4, 1.0, -1, &s) == MCV_OK);
  static double z[6 * 13 * 13];
  long long id = 0;
  CHECK(mcv_grid_sizes(3, 4, &npx, &n, &halo) == MCV_OK && npx == 13);
  CHECK(mcv_server_submit(s, 3, 4, -1.0, 2, z, z, z, z, &id) == MCV_ERR_ARG);
  CHECK(mcv_server_submit(s, 3, 4, 100.0, 2, z, NULL, z, z, &id) == MCV_ERR_ARG);
  CHECK(mcv_server_submit(s, 3, 4, 100.0, 2, z, z, z, z, &id) == MCV_OK && id == 1);
  long long st[9];
  CHECK(mcv_server_stats(s, st) == MCV_OK && st[0] == 1 && st[3] == 0);
  CHECK(mcv_server_result(s, 1, NULL, NULL, NULL, NULL, NULL, NULL) == MCV_BUSY);
  CHECK(mcv_server_destroy(s) == MCV_OK);
  printf("ok\n");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_c_program_links_and_calls_the_abi(tmp_path):
    src = tmp_path / "caller.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(api.lib_path())
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", libdir, "-lmcv_gpu", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
