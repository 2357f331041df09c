"""The network kernels embedded for run-time compilation (a generated
model's head kernel is compiled by NVRTC around them) compile with NVRTC
for sm_100a, in FP64 and FP32.  NVRTC runs on the host, so this needs no
GPU; it catches device code that nvcc accepts but NVRTC does not."""
import os

import pytest

from brian_b200 import build as engine_build

nvrtc = pytest.importorskip("cuda.bindings.nvrtc")

_MODEL = """
namespace bg {
struct GenModel {
    static constexpr bool custom_update = true, custom_threshold = true, custom_reset = true;
    template <typename T, int NV> static __device__ __forceinline__ void update(T (&S)[NV], double t_) {
        typedef T scalar; scalar s_v = S[0]; s_v = s_v + (scalar)0.001 * ((scalar)-0.07 - s_v); S[0] = s_v; }
    template <typename T, int NV> static __device__ __forceinline__ bool threshold(const T (&S)[NV], double t_) {
        return S[0] > (T)-0.05; }
    template <typename T, int NV> static __device__ __forceinline__ void reset(T (&S)[NV], double t_) {
        S[0] = (T)-0.06; }
};
}
extern "C" __global__ void __launch_bounds__(bg::kHeadThreads, 2) bg_gen_head(const bg::HeadArgs<%s> a) {
    bg::head_body<%s, 3, bg::GenModel>(a);
}
"""


def _embedded_source():
    text = ""
    for h in engine_build.RTC_HEADERS:
        with open(os.path.join(engine_build.CSRC, h)) as f:
            for line in f:
                if not line.strip().startswith('#include "'):
                    text += line
        text += "\n"
    return text


@pytest.mark.parametrize("scalar", ["double", "float"])
def test_generated_head_compiles(scalar):
    src = "#define BG_GENERATED_MODEL 1\n" + _embedded_source() + _MODEL % (scalar, scalar)
    err, prog = nvrtc.nvrtcCreateProgram(src.encode(), b"gen_head.cu", 0, [], [])
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
    # the options the engine passes (csrc/bg_fit.cu nvrtc_compile)
    opts = [b"--gpu-architecture=sm_100a", b"-fmad=false", b"-prec-div=true", b"-prec-sqrt=true", b"-ftz=false",
            b"--std=c++17", b"-lineinfo"]
    (res,) = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
    _, n = nvrtc.nvrtcGetProgramLogSize(prog)
    log = b" " * n
    nvrtc.nvrtcGetProgramLog(prog, log)
    nvrtc.nvrtcDestroyProgram(prog)
    assert res == nvrtc.nvrtcResult.NVRTC_SUCCESS, log.decode(errors="replace")[-4000:]
