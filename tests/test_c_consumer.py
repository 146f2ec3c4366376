"""The boundary is a C ABI: a plain C99 program (gcc -std=c99 -pedantic
-Werror) includes include/nnkifmm.h, links libnnkifmm.so and builds an octree
on the host through it, as a MEX gateway or a cgo/JNI stub would; its node
count and list lengths equal the Python mirror's, and an FMM on a machine
without a GPU fails with NNK_E_CUDA and a message."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import nnkifmm as nk
from conftest import ROOT

C_SOURCE = r"""
#include <stdio.h>
#include <stdlib.h>
#include "nnkifmm.h"

int main(int argc, char** argv) {
  int n = atoi(argv[1]), i, rc, gpu_expected = atoi(argv[2]);
  double* x = malloc(sizeof(double) * 3 * (size_t)n);
  unsigned s = 12345u;
  for (i = 0; i < 3 * n; ++i) { s = s * 1103515245u + 12345u; x[i] = (double)(s >> 8) / 16777216.0; }
  nnk_ctx* ctx = NULL;
  if (nnk_ctx_create(0, &ctx) != NNK_OK) return 2;
  nnk_tree_params p;
  p.node_capacity = 20; p.max_depth = 21; p.nearest = 0; p.builder = 1;
  nnk_tree* tree = NULL;
  rc = nnk_tree_build(ctx, x, n, x, n, NULL, 0, NULL, NULL, NULL, &p, &tree);
  if (rc != NNK_OK) { printf("tree %d %s\n", rc, nnk_last_error(ctx)); return 3; }
  nnk_tree_info info;
  nnk_tree_info_get(tree, &info);
  printf("nodes %d levels %d u %lld v %lld w %lld x %lld\n", info.node_count, info.max_level + 1,
         (long long)info.u_total, (long long)info.v_total, (long long)info.w_total, (long long)info.x_total);
  nnk_fmm_params fp = {1e-3, 1.0, 6, 1, NNK_PREC_FP64, 0, 0.0};
  nnk_fmm* fmm = NULL;
  rc = nnk_fmm_create(ctx, tree, &fp, &fmm);
  if (!gpu_expected) printf("fmm %d %s\n", rc, nnk_last_error(ctx));
  if (fmm) nnk_fmm_destroy(fmm);
  nnk_tree_destroy(tree);
  nnk_ctx_destroy(ctx);
  free(x);
  return 0;
}
"""


def _lcg_points(n):
    s = 12345
    out = np.empty(3 * n)
    for i in range(3 * n):
        s = (s * 1103515245 + 12345) % 2 ** 32
        out[i] = (s >> 8) / 16777216.0
    return out.reshape(n, 3)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not installed")
def test_plain_c_program_builds_a_tree_through_the_abi(tmp_path):
    import torch
    libdir = os.path.dirname(nk._lib.lib._name)
    src = tmp_path / "consumer.c"
    src.write_text(C_SOURCE)
    exe = tmp_path / "consumer"
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", libdir, "-lnnkifmm", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    gpu = int(torch.cuda.is_available())
    out = subprocess.run([str(exe), "1500", str(gpu)], check=True, capture_output=True, text=True).stdout.split("\n")
    x = _lcg_points(1500)
    t = nk.OcTree(x, x, nodeCapacity=20, builder="host")
    i = t.info
    assert out[0] == (f"nodes {t.nodeCount} levels {i.max_level + 1} u {i.u_total} v {i.v_total} "
                      f"w {i.w_total} x {i.x_total}")
    if not gpu:
        assert out[1].startswith(f"fmm {nk._lib.NNK_E_CUDA} ") and "no CUDA device" in out[1]
