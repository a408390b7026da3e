"""The reference's own C++ test program (tests/test.cpp + tests/vectors.cpp),
compiled unchanged against include/vkzg.h and libvkzg.so by oracle/ref_harness.py,
run on the GPU over the consensus-spec vectors.

It covers tests/test.cpp:55-276 as the reference runs it: every proof vector one
by one, the batched path, argument validation, a zero-blob call, chunking past
max_batch_size = 4, four threads sharing one prover, and the recovery vectors
one by one and batched.  Its exit status is the verdict (tests/test.cpp:278-280).
"""
import os
import subprocess

import pytest

from spec_vectors import write_vectors_dir

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TEST_BIN = os.path.join(ROOT, "oracle", "_ref", "vkzg_ref_test")


def test_reference_test_program(tmp_path, golden_proofs, golden_recover, oracle):
    if not os.path.exists(TEST_BIN):
        pytest.skip("oracle/_ref/vkzg_ref_test not built: no reference checkout where the build ran")
    vec_dir = write_vectors_dir(str(tmp_path / "vectors"), golden_proofs, golden_recover, oracle)
    env = dict(os.environ)
    env.pop("VKZG_TABLES_PATH", None)
    run = subprocess.run([TEST_BIN, vec_dir], capture_output=True, text=True, timeout=600, env=env)
    out = run.stdout + run.stderr
    assert run.returncode == 0, out
    lines = out.splitlines()
    assert lines[-1].startswith("ok: "), out
    assert not any(line.startswith("FAIL") for line in lines), out
    # 11 proof vectors, the batched path, 4 API checks, chunking, threads,
    # 6 recovery vectors and the batched recovery (tests/test.cpp:55-276).
    assert int(lines[-1].split()[1]) == 25, out
