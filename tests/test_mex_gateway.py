"""The MATLAB MEX gateway (stokes-nnkifmm_b200/mex/nnk_mex.c) compiled with gcc
against a stand-in for mex.h (tests/mex_fake/: the documented C Matrix API
names it uses, backed by a small in-memory runtime and a command-script
driver) and the real libnnkifmm.so, then run on the CPU: nearestMatrix, the
OcTree build, tree info and the four interaction lists come back in MATLAB's
layouts (sparse compressed columns, 1-based ids) and agree with the Python
mirror; an FMM without a GPU, and a tree deeper than maxDepth, come back as
MATLAB errors with the library's message and the reference's identifier.
MATLAB itself is not installed here."""
import os
import shutil
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN, ROOT

HERE = os.path.dirname(os.path.abspath(__file__))


def write_dense(d, name, a):
    a = np.atleast_2d(np.asarray(a, dtype=np.float64))
    a.T.copy().tofile(os.path.join(d, name + ".bin"))  # column-major, as MATLAB stores it
    with open(os.path.join(d, name + ".shape"), "w") as f:
        f.write(f"{a.shape[0]} {a.shape[1]}\n")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_mex_gateway_runs_on_the_c_abi(tmp_path):
    d = str(tmp_path)
    lib_dir = os.path.dirname(nk.LIB_PATH)
    exe = os.path.join(d, "mexdrv")
    cmd = ["gcc", "-std=c99", "-O1", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter",
           "-I", os.path.join(HERE, "mex_fake"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "stokes-nnkifmm_b200", "mex", "nnk_mex.c"), os.path.join(HERE, "mex_fake", "fake_mex.c"),
           "-L", lib_dir, "-lnnkifmm", f"-Wl,-rpath,{lib_dir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    g = np.load(os.path.join(GOLDEN, "sphere10_40.npz"))
    c, f = g["coarse"], g["fine"]
    NN = sp.csc_matrix(sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]), shape=(len(f), len(c))))
    write_dense(d, "coarse", c)
    write_dense(d, "fine", f)
    write_dense(d, "NN_pr", NN.data[None, :])
    write_dense(d, "NN_ir", NN.indices[None, :].astype(float))
    write_dense(d, "NN_jc", NN.indptr[None, :].astype(float))
    write_dense(d, "NN_mn", [[len(f), len(c)]])
    script = "\n".join([
        '1 "nearestMatrix" @coarse @fine',
        '1 "tree" @coarse @coarse 60 21 @fine sparse:NN',
        '1 "treeInfo" #1',
        '1 "treeList" #1 0', '1 "treeList" #1 1', '1 "treeList" #1 2', '1 "treeList" #1 3',
        '1 "fmm" #1 0.01 1',
        '0 "destroy" #1',
        '1 "tree" @coarse @coarse 60 2 @fine sparse:NN',
    ]) + "\n"
    with open(os.path.join(d, "script.txt"), "w") as fh:
        fh.write(script)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([exe, "script.txt"], cwd=d, capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    # nearestMatrix: MATLAB sparse Q x N, equal to the library's
    trip = np.fromfile(os.path.join(d, "out_0_0.bin")).reshape(-1, 3)
    M = sp.csr_matrix((trip[:, 2], (trip[:, 0].astype(int), trip[:, 1].astype(int))), shape=(len(f), len(c)))
    assert (M != nk.nearestMatrix(c, f, builder="host")).nnz == 0
    # the tree against the Python mirror of the same entry points
    t = nk.OcTree(c, c, nodeCapacity=60, nearest=1, finePoints=f, NN=sp.csr_matrix(NN), builder="host")
    info = np.fromfile(os.path.join(d, "out_2_0.bin"))
    assert info[0] == t.nodeCount and info[1] == t.nodeLevel.max()
    for k in range(4):
        raw = np.fromfile(os.path.join(d, f"out_{3 + k}_0.bin"))
        off, ids = t.interaction_list(k)
        pos, got = 0, []
        for i in range(t.nodeCount):
            cnt = int(raw[pos])
            got.append(raw[pos + 1:pos + 1 + cnt].astype(np.int32))
            pos += 1 + cnt
        assert pos == raw.size
        for i in range(t.nodeCount):
            assert np.array_equal(got[i], ids[off[i]:off[i + 1]]), (k, i)
    # no GPU here: the FMM is refused with the library's message
    assert any(ln.startswith("ERROR nnkifmm:error KIFMM: no CUDA device") for ln in lines) or "OK 7" in lines
    assert "OK 8" in lines
    assert "ERROR OcTree:maxDepth Max level reached: Increase Max Depth" in lines
