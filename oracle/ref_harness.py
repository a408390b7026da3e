"""Builds jtraglia/vkzg's own C++ test and bench programs, unchanged, against this
repository's include/vkzg.h and vkzg_b200/libvkzg.so (TEST INFRASTRUCTURE ONLY).

    python oracle/ref_harness.py [REFERENCE_CHECKOUT]

The checkout defaults to $VKZG_REFERENCE_DIR.  The programs are compiled from
the sources where they lie in the checkout:

    tests/test.cpp + tests/vectors.cpp  -> oracle/_ref/vkzg_ref_test
    bench/bench.cpp                     -> oracle/_ref/vkzg_ref_bench

None of them needs Vulkan: tests/test.cpp:1-11, tests/vectors.h:14-20 and
bench/bench.cpp:1-8 include only "../include/vkzg.h" and the C++ standard
library.  Because that include is relative to the source file, the sources are
reached through a staging directory of symbolic links (created in a temporary
directory and removed afterwards) whose include/vkzg.h is this repository's
header, so the programs see exactly the declarations this library exports.
The binaries find libvkzg.so through an $ORIGIN-relative run path; nothing is
copied from the checkout into the repository.
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
LIBDIR = os.path.join(ROOT, "vkzg_b200")
TEST_BIN = os.path.join(OUT, "vkzg_ref_test")
BENCH_BIN = os.path.join(OUT, "vkzg_ref_bench")

# (binary, sources relative to the checkout)
PROGRAMS = [
    (TEST_BIN, ["tests/test.cpp", "tests/vectors.cpp"]),
    (BENCH_BIN, ["bench/bench.cpp"]),
]
# Headers the sources include, relative to the checkout.
HEADERS = ["tests/vectors.h", "bench/bench_common.h"]


def reference_dir(arg=None):
    return arg or os.environ.get("VKZG_REFERENCE_DIR")


def build(ref=None, force=False):
    """Compiles both programs; returns their paths, or None when no checkout is given."""
    ref = reference_dir(ref)
    if not ref or not os.path.isdir(ref):
        return None
    lib = os.path.join(LIBDIR, "libvkzg.so")
    if not os.path.exists(lib):
        raise FileNotFoundError(f"{lib} is not built (python -m vkzg_b200.build)")
    os.makedirs(OUT, exist_ok=True)
    stage = tempfile.mkdtemp(prefix="vkzg_ref_harness_")
    try:
        for d in ("tests", "bench", "include"):
            os.makedirs(os.path.join(stage, d))
        for rel in [s for _, srcs in PROGRAMS for s in srcs] + HEADERS:
            os.symlink(os.path.join(ref, rel), os.path.join(stage, rel))
        os.symlink(os.path.join(ROOT, "include", "vkzg.h"), os.path.join(stage, "include", "vkzg.h"))
        for binary, srcs in PROGRAMS:
            deps = [os.path.join(ref, s) for s in srcs] + [lib, os.path.join(ROOT, "include", "vkzg.h")]
            if not force and os.path.exists(binary) and all(
                    os.path.getmtime(d) <= os.path.getmtime(binary) for d in deps):
                continue
            cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-Wall",
                   *[os.path.join(stage, s) for s in srcs],
                   "-o", binary, "-L", LIBDIR, "-lvkzg",
                   "-Wl,-rpath,$ORIGIN/../../vkzg_b200", "-Wl,-rpath,/usr/local/cuda/lib64"]
            subprocess.check_call(cmd)
    finally:
        shutil.rmtree(stage, ignore_errors=True)
    return TEST_BIN, BENCH_BIN


if __name__ == "__main__":
    got = build(sys.argv[1] if len(sys.argv) > 1 else None, force="--force" in sys.argv)
    if got is None:
        sys.exit("no reference checkout: pass its path or set VKZG_REFERENCE_DIR")
    print("\n".join(got))
