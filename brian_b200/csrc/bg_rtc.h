// bg_rtc.h -- run-time compilation shared by the fitting and network engines
// (library internal, host only).
#pragma once
#include <string>
#include <vector>

// NVRTC for sm_100a with -fmad=false, IEEE division and square root; the
// cubin of each distinct source is cached for the life of the process.
int bg_nvrtc_compile(const std::string &src, std::vector<char> *cubin, std::string *log);

// Kernel sources the network engine compiles with a generated model
// (bg_common.cuh and bg_kernels.cuh, embedded at build time), in pieces.
extern const char *const kNetRtcSource[];
