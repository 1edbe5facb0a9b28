"""CPU check of the ERI kernels' launch shapes: a host program (tests/shape_bounds.cu, built with
nvcc, launching nothing) enumerates every shape the dispatch compiles and evaluates the index
bounds the kernels static_assert (shape_violation in csrc/eri_kernel.cuh): group count, the
primitive-loop and transform regions inside each group's shared memory, one scratch buffer per
block where it lives in global memory, named-barrier ids and counts, and the block's shared-memory
total."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

NVCC = os.environ.get("NVCC", "nvcc")


@pytest.mark.skipif(shutil.which(NVCC) is None, reason="nvcc not available")
def test_every_compiled_launch_shape_keeps_its_indexes_in_bounds(tmp_path):
    exe = tmp_path / "shape_bounds"
    src = os.path.join(ROOT, "tests", "shape_bounds.cu")
    subprocess.run([NVCC, "-std=c++17", "-O0", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(exe), src],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = [r.split() for r in out if r.strip()]
    assert len({tuple(r[:4]) for r in rows}) == 120  # every (li lj | lk ll) class up to g
    bad = [r for r in rows if r[-1] != "0"]
    assert not bad, bad[:5]
    for r in rows:
        s, lanes, block, q, smem, glob = (int(r[i]) for i in (6, 7, 8, 9, 11, 12))
        assert block <= 1024 and smem <= 227 * 1024
        if glob:  # classes whose transform buffers live in global scratch: one group per block
            assert q == 1
    # the sliced and split-transfer cooperative shapes exist where the autotuner can pick them
    assert any(r[4] == "sph" and r[5] == "9" for r in rows)
    for v in ("10", "11"):
        assert any(r[4] == "sph" and r[5] == v and r[:4] == ["3", "3", "3", "0"] for r in rows)
