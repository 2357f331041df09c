"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

* ``oracle/liboracle.so``: the CPU restatement (oracle.cpp), single-threaded,
  ``-O2 -ffp-contract=off -fno-fast-math`` so every floating-point operation is
  one IEEE rounding in source order.
* ``oracle/_ref/libccircular_ref.so``: the reference's own C++ SpikeContainer
  (brian/utils/ccircular/circular.cpp) compiled from the reference tree where
  it lies, behind the small C shim ref_shim.cpp.  Built only when the
  reference tree is present (it is not on GPU hosts; the built .so travels).

Run: ``python oracle/build.py`` (also called by ``__graft_entry__.build()``);
the reference tree is taken from ``$BRIAN_REFERENCE`` when set.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libccircular_ref.so")
# the reference tree: BRIAN_REFERENCE, else where the build container mounts it
REFERENCE = os.environ.get("BRIAN_REFERENCE", "/root/reference")
CCIRC = os.path.join(REFERENCE, "brian", "utils", "ccircular")


def _stale(out, deps):
    return not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps)


def build_oracle(force=False):
    src = os.path.join(HERE, "oracle.cpp")
    if force or _stale(ORACLE_SO, [src]):
        subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-std=c++17",
                               "-shared", "-fPIC", "-o", ORACLE_SO, src])
    return ORACLE_SO


def build_reference(force=False):
    if not os.path.isdir(CCIRC):
        return None
    srcs = [os.path.join(HERE, "ref_shim.cpp"), os.path.join(CCIRC, "circular.cpp")]
    os.makedirs(REF_DIR, exist_ok=True)
    if force or _stale(REF_SO, srcs):
        subprocess.check_call(["g++", "-O2", "-shared", "-fPIC", "-w", "-I", CCIRC, "-o", REF_SO] + srcs)
    return REF_SO


def build(force=False):
    build_oracle(force)
    build_reference(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(ORACLE_SO, REF_SO if os.path.exists(REF_SO) else "(reference SpikeContainer not built)")
