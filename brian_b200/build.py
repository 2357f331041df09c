"""Build the engine's shared library in-tree with nvcc for sm_100a.

``python -m brian_b200.build`` compiles every ``csrc/*.cu`` into
``brian_b200/libbrian_b200.so`` (static cudart, NVRTC and the driver API for
generated model kernels).  The library is loaded with ctypes by
``brian_b200._lib``; nothing is JIT-compiled or cached outside the tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbrian_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         # the bit-exact FP64 path spells out every rounding with __dmul_rn /
         # __dadd_rn; no contraction anywhere else either
         "-fmad=false"]


# Headers the network engine compiles again at run time (NVRTC) around a
# generated model: embedded into bg_rtc_src.cu, which this script writes.
RTC_HEADERS = ["bg_common.cuh", "bg_expfn.h", "bg_kernels.cuh"]
RTC_OUT = os.path.join(CSRC, "bg_rtc_src.cu")


def write_rtc_sources():
    text = ""
    for h in RTC_HEADERS:
        with open(os.path.join(CSRC, h)) as f:
            for line in f:
                if line.strip().startswith('#include "'):
                    continue
                text += line
        text += "\n"
    if ")BGRTC\"" in text:
        raise RuntimeError("embedded source contains the raw-string delimiter")
    chunks, cur = [], ""
    for line in text.splitlines(True):
        if len(cur) + len(line) > 12000:
            chunks.append(cur)
            cur = ""
        cur += line
    chunks.append(cur)
    out = ("// Generated by brian_b200/build.py from %s: the network engine's kernel\n"
           "// sources, compiled again at run time around a generated model.\n"
           "#include \"bg_rtc.h\"\n\nconst char *const kNetRtcSource[] = {\n" % ", ".join(RTC_HEADERS))
    for c in chunks:
        out += 'R"BGRTC(' + c + ')BGRTC",\n'
    out += "nullptr};\n"
    old = open(RTC_OUT).read() if os.path.exists(RTC_OUT) else None
    if old != out:
        with open(RTC_OUT, "w") as f:
            f.write(out)


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "brian_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    write_rtc_sources()
    cmds, objs = [], []
    for src in sources():
        obj = os.path.join(CSRC, os.path.basename(src)[:-3] + ".o")
        cmds.append([NVCC] + ARCH + FLAGS + ["-I", os.path.join(HERE, "..", "include"), "-c", src, "-o", obj])
        objs.append(obj)
    # one nvcc per translation unit, side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
        list(ex.map(subprocess.check_call, cmds))
    link = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
        "-L" + os.path.join(CUDA_HOME, "lib64"),
        "-L" + os.path.join(CUDA_HOME, "lib64", "stubs"),
        "-lnvrtc", "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")]
    if verbose:
        print(" ".join(link))
    subprocess.check_call(link)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
