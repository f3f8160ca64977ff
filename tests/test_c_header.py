"""The C ABI as a C caller sees it: include/hignn_b200.h compiled as C99 by gcc, linked against
libhignn_b200.so, driven on a host-only model (device -1; no GPU needed).

The program follows the call sequence a binding of the reference's HignnModel would make
(interface/HignnInterface.cpp:17-35): create, set parameters, inspect the tree and lists, and
receive status codes for what a host-only model cannot do.
"""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(REPO, "hignn_b200")

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "hignn_b200.h"

#define CHECK(c) do { if (!(c)) { printf("FAILED line %d: %s\n", __LINE__, #c); return 1; } } while (0)

int main(void) {
  const int64_t n = 3000;
  float* xyz = (float*)malloc(sizeof(float) * 3 * n);
  unsigned s = 12345u;
  for (int64_t i = 0; i < 3 * n; i++) { s = s * 1103515245u + 12345u; xyz[i] = (float)(s >> 8) / 16777216.0f * 40.0f; }
  hignn_model* m = NULL;
  char msg[256];
  CHECK(hignn_version() >= 100);
  CHECK(hignn_create(xyz, n, 64, -1, &m) == HIGNN_OK && m != NULL);
  CHECK(hignn_set_param(m, HIGNN_P_EPSILON, 1e-3) == HIGNN_OK);
  double v = 0.0;
  CHECK(hignn_get_param(m, HIGNN_P_EPSILON, &v) == HIGNN_OK && v == 1e-3);
  CHECK(hignn_set_param(m, HIGNN_P_MAX_ITER, 0) == HIGNN_ERR_ARG);
  CHECK(hignn_last_error(msg, sizeof msg) == HIGNN_OK && strlen(msg) > 0);
  CHECK(hignn_set_param(m, 9999, 1.0) == HIGNN_ERR_ARG);
  CHECK(hignn_update_coord(m, xyz, n) == HIGNN_OK);
  CHECK(hignn_update_coord(m, xyz, n - 1) == HIGNN_ERR_ARG);
  hignn_stats st;
  memset(&st, 0, sizeof st);
  CHECK(hignn_get_stats(m, &st) == HIGNN_OK);
  CHECK(st.n == n && st.num_nodes > 3 && st.num_leaves > 1 && st.num_close > 0 && st.num_far > 0);
  int64_t* tree = (int64_t*)malloc(sizeof(int64_t) * 5 * st.num_nodes);
  int64_t* perm = (int64_t*)malloc(sizeof(int64_t) * n);
  CHECK(hignn_get_tree(m, tree, perm) == HIGNN_OK);
  CHECK(tree[0] == 3 && tree[1] == 4 && tree[2] == 0 && tree[3] == n);  /* root -> rows 3, 4 */
  char* seen = (char*)calloc(n, 1);
  for (int64_t i = 0; i < n; i++) { CHECK(perm[i] >= 0 && perm[i] < n && !seen[perm[i]]); seen[perm[i]] = 1; }
  int64_t* ci = (int64_t*)malloc(sizeof(int64_t) * st.num_close);
  int64_t* cj = (int64_t*)malloc(sizeof(int64_t) * st.num_close);
  int64_t* fi = (int64_t*)malloc(sizeof(int64_t) * st.num_far);
  int64_t* fj = (int64_t*)malloc(sizeof(int64_t) * st.num_far);
  CHECK(hignn_get_lists(m, ci, cj, fi, fj) == HIGNN_OK);
  for (int64_t q = 0; q < st.num_close; q++) CHECK(cj[q] >= ci[q]);  /* symmetric lists: J >= I */
  float* u = (float*)malloc(sizeof(float) * 3 * n);
  CHECK(hignn_dot(m, u, xyz, n) == HIGNN_ERR_NODEV);  /* no CPU fallback */
  CHECK(hignn_dot(NULL, u, xyz, n) == HIGNN_ERR_ARG);
  CHECK(hignn_create(xyz, 0, 64, -1, &m) == HIGNN_ERR_ARG);
  hignn_nbl* l = NULL;
  CHECK(hignn_nbl_create(0, &l) == HIGNN_ERR_NODEV || l != NULL);  /* no device here, or a GPU box */
  if (l) hignn_nbl_destroy(l);
  printf("C ABI OK: %lld nodes, %lld close, %lld far\n", (long long)st.num_nodes, (long long)st.num_close,
         (long long)st.num_far);
  return 0;
}
"""


def test_c_program_against_the_header(tmp_path):
    gcc = shutil.which("gcc")
    lib = os.path.join(LIBDIR, "libhignn_b200.so")
    if gcc is None or not os.path.exists(lib):
        pytest.skip("gcc or the built library is missing")
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(REPO, "include"), str(src),
                    "-L", LIBDIR, "-lhignn_b200", "-o", str(exe)], check=True, capture_output=True, text=True)
    env = dict(os.environ, LD_LIBRARY_PATH=LIBDIR + os.pathsep + os.environ.get("LD_LIBRARY_PATH", ""))
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "C ABI OK" in r.stdout
