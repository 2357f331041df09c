// bg_fit.cu -- batched model fitting: the GPUModelFitting replacement
// (library/modelfitting/gpu_modelfitting.py:202-401), the gamma factor
// (tools/statistics.py:236-240) and a device-resident grouped particle swarm
// (tools/particle_swarm.py:6-111).
//
// The simulation kernel's model part (state update, threshold, reset) is
// generated from the user's equations, so its source is assembled here from
// the template in bg_fit_template.cuh and compiled by NVRTC for sm_100a at
// bg_fit_create (the reference JIT-compiles its template with PyCUDA on every
// reinit_vars call, gpu_modelfitting.py:333-336; here it happens once per
// handle).  The cubin is loaded with the runtime's library API.  Everything
// else -- state preparation, the gamma factor, the swarm update and the
// best-position reductions -- is compiled ahead of time below.
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "bg_common.cuh"
#include "bg_fit_template.cuh"
#include "../../include/brian_b200.h"

namespace {

int fail(int code, const std::string &m) { return bg_internal_fail(code, m.c_str()); }

#define FCK(call)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(BG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

constexpr int kSimThreads = 128;    // must match __launch_bounds__ in the template
constexpr int kAuxThreads = 256;

// Host image of the template's FitArgs (same field order and types).
struct FitArgsHost {
    void *S;
    const void *I;
    const long long *I_off;
    const int *nsteps;
    const int *spk;
    const long long *spk_end;
    long long *spk_idx;
    const int *delay;
    const int *refr;
    int *next_allowed;
    int *ncoinc;
    int *nspikes;
    unsigned char *flags;
    const int *order;
    int *rec;
    int *rec_n;
    int *next_task;
    long long ns;
    int Tstart, Tend, onset, rec_cap;
};

std::vector<std::string> split_names(const char *names) {
    std::vector<std::string> out;
    std::string cur;
    for (const char *p = names; p && *p; ++p) {
        if (*p == ',' || *p == ' ') {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += *p;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

bool valid_ident(const std::string &s) {
    if (s.empty() || !(isalpha((unsigned char)s[0]) || s[0] == '_')) return false;
    for (char c : s)
        if (!(isalnum((unsigned char)c) || c == '_')) return false;
    return true;
}

const char *nz(const char *p) { return p ? p : ""; }

// Full NVRTC source: scalar type, constants, the division helpers, the Model
// struct, the template.
int assemble_source(int precision, const bg_fit_model *model, double dt, int delta, int exclusive, std::string *src,
                    int *nstate) {
    if (precision != 32 && precision != 64) return fail(BG_EINVAL, "fit: precision must be 32 or 64");
    if (!(dt > 0)) return fail(BG_EINVAL, "fit: dt must be positive");
    if (delta < 0) return fail(BG_EINVAL, "fit: delta must be >= 0");
    if (!model) return fail(BG_EINVAL, "fit: null model");
    std::vector<std::string> names = split_names(model->state_names);
    if (names.empty()) return fail(BG_EINVAL, "fit: no state variables");
    for (auto &n : names)
        if (!valid_ident(n)) return fail(BG_EINVAL, "fit: bad state variable name '" + n + "'");
    const char *sc = precision == 32 ? "float" : "double";
    const bool has_fast = model->update_fast_code && *model->update_fast_code;
    char dtbuf[64];
    snprintf(dtbuf, sizeof dtbuf, "%a", dt);
    std::ostringstream o;
    o << "typedef " << sc << " scalar;\n"
      << "#define BG_DT (" << dtbuf << ")\n"
      << "#define BG_DELTA (" << delta << ")\n"
      << "#define BG_EXCLUSIVE " << (exclusive ? 1 : 0) << "\n"
      << kFitHelperSource
      << "struct Model {\n";
    for (auto &n : names) o << "    scalar s_" << n << ";\n";
    o << "    bool bg_exact;\n" << nz(model->aux_decl) << "\n";
    o << "    __device__ __forceinline__ void load(const scalar *S, long long ns, long long i) {\n";
    for (size_t k = 0; k < names.size(); ++k) o << "        s_" << names[k] << " = S[" << k << "LL * ns + i];\n";
    o << "        bg_exact = false;\n" << nz(model->setup_code) << "\n";
    o << "    }\n    __device__ __forceinline__ void store(scalar *S, long long ns, long long i) const {\n";
    for (size_t k = 0; k < names.size(); ++k) o << "        S[" << k << "LL * ns + i] = s_" << names[k] << ";\n";
    o << "    }\n    __device__ __forceinline__ void update(const scalar I_in, const scalar t) {\n"
      << nz(model->update_code) << "\n    }\n"
      << "    __device__ __forceinline__ void update_fast(const scalar I_in, const scalar t, bool &suspect) {\n"
      << (has_fast ? nz(model->update_fast_code) : "update(I_in, t);") << "\n    }\n"
      << "    __device__ __forceinline__ bool threshold(const scalar I_in, const scalar t) const {\n"
      << "        return " << (model->threshold_code && *model->threshold_code ? model->threshold_code : "false")
      << ";\n    }\n"
      << "    __device__ __forceinline__ void reset(const scalar I_in, const scalar t, const bool reset_on) {\n"
      << nz(model->reset_code) << "\n    }\n};\n"
      << kFitKernelSource;
    *src = o.str();
    *nstate = (int)names.size();
    return BG_OK;
}

// Compiled kernels of this process, keyed by their full source.
std::mutex g_cubin_mutex;
std::map<std::string, std::vector<char>> g_cubins;

int nvrtc_compile(const std::string &src, std::vector<char> *cubin, std::string *log) {
    {
        std::lock_guard<std::mutex> lock(g_cubin_mutex);
        auto it = g_cubins.find(src);
        if (it != g_cubins.end()) {
            *cubin = it->second;
            log->clear();
            return BG_OK;
        }
    }
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "bg_fit_model.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        return fail(BG_ECOMPILE, "nvrtcCreateProgram failed");
    // -fmad=false: the generated arithmetic rounds after every operation, as
    // numpy evaluates the same expressions; IEEE division and square root.
    const char *opts[] = {"--gpu-architecture=sm_100a", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
                          "-ftz=false", "--std=c++17", "-lineinfo"};
    nvrtcResult r = nvrtcCompileProgram(prog, (int)(sizeof opts / sizeof opts[0]), opts);
    size_t ls = 0;
    nvrtcGetProgramLogSize(prog, &ls);
    log->assign(ls, '\0');
    if (ls) nvrtcGetProgramLog(prog, &(*log)[0]);
    if (r != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        return fail(BG_ECOMPILE, std::string("model kernel compilation failed: ") + nvrtcGetErrorString(r) +
                                     "\n" + *log);
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    cubin->resize(n);
    nvrtcGetCUBIN(prog, cubin->data());
    nvrtcDestroyProgram(&prog);
    std::lock_guard<std::mutex> lock(g_cubin_mutex);
    g_cubins[src] = *cubin;
    return BG_OK;
}

template <typename T>
void free_ptr(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

}  // namespace

// Shared with the network engine (generated group kernels).
int bg_nvrtc_compile(const std::string &src, std::vector<char> *cubin, std::string *log) {
    return nvrtc_compile(src, cubin, log);
}

struct bg_fit {
    int device = 0;
    int precision = 64;
    size_t ssz = 8;
    int nstate = 0;
    double dt = 0;
    int delta = 0;
    cudaStream_t stream = nullptr;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern = nullptr;
    // simulations
    int64_t ns = 0, ninput = 0, nspk = 0;
    void *S = nullptr, *S0 = nullptr, *I = nullptr;
    long long *I_off = nullptr, *spk_off = nullptr, *spk_end = nullptr, *spk_idx = nullptr;
    int *nsteps = nullptr, *spk = nullptr, *delay = nullptr, *delay0 = nullptr, *refr = nullptr,
        *refr0 = nullptr, *next_allowed = nullptr, *ncoinc = nullptr, *nspikes = nullptr, *order = nullptr;
    unsigned char *flags = nullptr;
    int *rec = nullptr, *rec_n = nullptr;
    int rec_cap = 0;
    int onset = 0;
    int max_steps = 0;
    int *next_task = nullptr;
    int nsm = 148;
    int blocks_per_sm = 2;      // resident simulation blocks per SM (bg_fit_autotune)
    // gamma
    int64_t npart = 0;
    int slices = 1;
    int *tlen = nullptr;
    double *trate = nullptr, *fit = nullptr;
    double delta_s = 0;
    bool gamma_ready = false;
    // parameters and swarm
    int ndim = 0;
    int *dimvar = nullptr;
    double *X = nullptr, *V = nullptr, *Xl = nullptr, *lfit = nullptr, *Xg = nullptr, *gfit = nullptr,
           *lo = nullptr, *hi = nullptr;
    int group_size = 0, ngroups = 0;
    double omega = 0, c1 = 0, c2 = 0;
    uint64_t seed = 0;
    int64_t iter = 0;
    bool pso_ready = false;
    float last_sim_ms = 0;
    float last_eval_ms = 0;     // whole evaluation (prepare, simulate, gamma, bests)
    int64_t sim_launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

// ------------------------------------------------------------------ kernels
// State and counters of every simulation back to the start of a run, with
// the candidate parameters of X written into their state rows (ModelFitting.
// evaluate, modelfitting.py:175-199, and GPUModelFitting.reinit_vars,
// gpu_modelfitting.py:333-379).  Dimension d goes to state row dimvar[d];
// dimvar -1 is the spike delay and -2 the refractory period, both converted
// with rint(x / dt).  Simulation i holds particle i % npart (slice-major).
template <typename T>
__global__ void k_fit_prepare(int64_t ns, int nstate, T *S, const T *S0, const double *X, int ndim,
                              const int *dimvar, int64_t npart, double dt, const long long *spk_off,
                              long long *spk_idx, int *delay, const int *delay0, int *refr, const int *refr0,
                              int *next_allowed, int *ncoinc, int *nspikes, unsigned char *flags, int *rec_n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    for (int v = 0; v < nstate; ++v) S[v * ns + i] = S0[v * ns + i];
    int dl = delay0[i], rf = refr0[i];
    if (X) {
        const int64_t p = i % npart;
        for (int d = 0; d < ndim; ++d) {
            const double x = X[d * npart + p];
            const int vd = dimvar[d];
            if (vd >= 0) S[vd * ns + i] = (T)x;
            else if (vd == -1) dl = (int)rint(x / dt);
            else if (vd == -2) rf = (int)rint(x / dt);
        }
    }
    delay[i] = dl;
    refr[i] = rf;
    spk_idx[i] = spk_off[i];
    next_allowed[i] = -1;
    ncoinc[i] = 0;
    nspikes[i] = 0;
    flags[i] = 2;   // last_spike_allowed = false, next_spike_allowed = true (gpu_modelfitting.py:364-365)
    if (rec_n) rec_n[i] = 0;
}

// gamma = (Nc - 2 delta Nt r) / (0.5 (1 - 2 delta r) (Nt + Nm)), evaluated
// in the order numpy evaluates get_gamma_factor (statistics.py:236-240);
// counts are summed over slices first (modelfitting.py:221-223).
__global__ void k_gamma(int64_t npart, int slices, const int *ncoinc, const int *nspikes, const int *tlen,
                        const double *trate, double delta, double *fit) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npart) return;
    long long nc = 0, nm = 0;
    for (int s = 0; s < slices; ++s) {
        nc += ncoinc[s * npart + p];
        nm += nspikes[s * npart + p];
    }
    const double nt = (double)tlen[p], r = trate[p];
    const double avg = __dmul_rn(__dmul_rn(__dmul_rn(2.0, delta), nt), r);
    const double norm = __dmul_rn(0.5, __dadd_rn(1.0, -__dmul_rn(__dmul_rn(2.0, delta), r)));
    fit[p] = __ddiv_rn(__dadd_rn((double)nc, -avg), __dmul_rn(norm, (double)(tlen[p] + nm)));
}

// One swarm move (particle_swarm.py:68-77):
//   V = omega V + c1 R1 (X_lbest - X) + c2 R2 (X_gbest - X); X = X + V;
//   X = min(max(X, lo), hi)
// R1, R2 are Philox4x32-10 uniforms keyed (seed, 2 it [+1], d * M + p).
__global__ void k_pso_move(int64_t M, int ndim, int group_size, double *X, double *V, const double *Xl,
                           const double *Xg, const double *lo, const double *hi, double omega, double c1, double c2,
                           uint64_t seed, int64_t it) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M * ndim) return;
    const int d = (int)(k / M);
    const int64_t p = k % M;
    const int64_t g = p / group_size;
    const int64_t G = M / group_size;
    const double r1 = bg_philox_uniform(seed, 2 * it, k);
    const double r2 = bg_philox_uniform(seed, 2 * it + 1, k);
    const double x = X[k];
    const double a = __dmul_rn(omega, V[k]);
    const double b = __dmul_rn(__dmul_rn(c1, r1), __dadd_rn(Xl[k], -x));
    const double c = __dmul_rn(__dmul_rn(c2, r2), __dadd_rn(Xg[d * G + g], -x));
    const double v = __dadd_rn(__dadd_rn(a, b), c);
    double xn = __dadd_rn(x, v);
    const double l = lo[d], h = hi[d];
    xn = (xn < l) ? l : xn;   // numpy maximum/minimum: NaN stays NaN
    xn = (xn > h) ? h : xn;
    V[k] = v;
    X[k] = xn;
}

// Local and group bests after an evaluation (particle_swarm.py:88-103): a
// particle's best moves on a strictly larger fitness; a group's best moves
// to the first particle holding the group maximum when that maximum is
// strictly larger than the group's best so far.  NaN never wins.  One block
// per group.
__global__ void k_pso_best(int64_t M, int ndim, int group_size, const double *X, const double *fit, double *Xl,
                           double *lfit, double *Xg, double *gfit, double *trace, int64_t it) {
    __shared__ double sv[kAuxThreads];
    __shared__ long long si[kAuxThreads];
    const int64_t g = blockIdx.x, G = M / group_size;
    double best = -INFINITY;
    long long bi = -1;
    for (int64_t q = threadIdx.x; q < group_size; q += blockDim.x) {
        const int64_t p = g * group_size + q;
        const double f = fit[p];
        if (f > lfit[p]) {
            lfit[p] = f;
            for (int d = 0; d < ndim; ++d) Xl[d * M + p] = X[d * M + p];
        }
        if (f > best) {   // ascending q per thread: first max kept
            best = f;
            bi = p;
        }
    }
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            const double o = sv[threadIdx.x + s];
            const long long oi = si[threadIdx.x + s];
            const bool take = oi >= 0 && (si[threadIdx.x] < 0 || o > sv[threadIdx.x] ||
                                          (o == sv[threadIdx.x] && oi < si[threadIdx.x]));
            if (take) {
                sv[threadIdx.x] = o;
                si[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (si[0] >= 0 && sv[0] > gfit[g]) {
            gfit[g] = sv[0];
            for (int d = 0; d < ndim; ++d) Xg[d * G + g] = X[d * M + si[0]];
        }
        if (trace) trace[it * G + g] = gfit[g];
    }
}

// Spike-train and input features of every simulation from its recorded
// spikes (first `cap`), one warp per simulation, for the learned proposal:
//   f[0..31]  histogram of log10(ISI / s) over [-3, log10 2) in 32 equal bins
//             (outside values in the end bins), divided by the ISI count;
//   f[32]     firing_rate: (n-1) / (t_last - t_first)   (statistics.py:15-21)
//   f[33]     CV: std(ISI) / mean(ISI), population std   (statistics.py:23-30)
//   f[34..63] spike-triggered average of the input in nA over 30 ms before
//             each spike, 30 bins of 1 ms, most recent first, as
//             spike_triggered_average (statistics.py:125-153) computes it:
//             spikes with t > 30 ms contribute input[i-1-j] for j < 300,
//             i = int(t / dt), and the sum is divided by (n - 1).
// Quantities that need two spikes are 0 with fewer.  Sums run in double in
// a fixed order.
template <typename T>
__global__ void k_features(int64_t ns, const int *rec, const int *rec_n, int cap, const T *I, const long long *I_off,
                           double dt, float *out) {
    constexpr int kBins = 32, kSta = 30, kWin = 300, kPerLane = (kWin + 31) / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    __shared__ double sbin[4][kSta];
    if (i >= ns) return;
    const int n = min(rec_n[i], cap);
    const int *s = rec + i * (int64_t)cap;
    const double lo = -3.0, hi = log10(2.0), width = (hi - lo) / kBins;
    // ISI histogram: each lane counts its share into registers, bins reduced
    // across the warp
    int cnt[kBins];
#pragma unroll
    for (int b = 0; b < kBins; ++b) cnt[b] = 0;
    double sd = 0.0, sd2 = 0.0;
    for (int k = lane; k + 1 < n; k += 32) {
        const double d = (double)(s[k + 1] - s[k]) * dt;
        sd += d;
        sd2 += d * d;
        int b = (int)floor((log10(d) - lo) / width);
        b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
#pragma unroll
        for (int q = 0; q < kBins; ++q) cnt[q] += (q == b) ? 1 : 0;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sd += __shfl_xor_sync(0xffffffffu, sd, off);
        sd2 += __shfl_xor_sync(0xffffffffu, sd2, off);
    }
    float *f = out + i * 64;
    const int nisi = n > 1 ? n - 1 : 0;
#pragma unroll
    for (int q = 0; q < kBins; ++q) {
        int c = cnt[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
        if (lane == q) f[q] = nisi ? (float)((double)c / nisi) : 0.f;
    }
    if (lane == 0) {
        if (n >= 2) {
            const double t0 = (double)s[0] * dt, t1 = (double)s[n - 1] * dt;
            f[32] = (float)((double)(n - 1) / (t1 - t0));
            const double mean = sd / nisi;
            const double var = sd2 / nisi - mean * mean;
            f[33] = (float)(sqrt(var > 0 ? var : 0.0) / mean);
        } else {
            f[32] = 0.f;
            f[33] = 0.f;
        }
    }
    // spike-triggered average: lane handles window samples j = lane + 32u
    double acc[kPerLane];
#pragma unroll
    for (int u = 0; u < kPerLane; ++u) acc[u] = 0.0;
    const T *in = I + I_off[i];
    for (int k = 0; k < n; ++k) {
        const double t = (double)s[k] * dt;
        if (!(t > 0.03)) continue;   // spikes after the 30 ms window length
        const long long idx = (long long)(t / dt);
#pragma unroll
        for (int u = 0; u < kPerLane; ++u) {
            const int j = lane + 32 * u;
            if (j < kWin) acc[u] += (double)in[idx - 1 - j];
        }
    }
    if (lane < kSta) sbin[warp][lane] = 0.0;
    __syncwarp();
    // fixed-order bin sums: lanes in turn
    for (int src = 0; src < 32; ++src) {
        if (lane == src) {
#pragma unroll
            for (int u = 0; u < kPerLane; ++u) {
                const int j = lane + 32 * u;
                if (j < kWin) sbin[warp][j / 10] += acc[u];
            }
        }
        __syncwarp();
    }
    if (lane < kSta) f[34 + lane] = n >= 2 ? (float)(sbin[warp][lane] / 10.0 / (double)(n - 1) * 1e9) : 0.f;
}

int sim_launch(bg_fit *h, int Tstart, int Tend) {
    FitArgsHost a;
    a.S = h->S;
    a.I = h->I;
    a.I_off = h->I_off;
    a.nsteps = h->nsteps;
    a.spk = h->spk;
    a.spk_end = h->spk_end;
    a.spk_idx = h->spk_idx;
    a.delay = h->delay;
    a.refr = h->refr;
    a.next_allowed = h->next_allowed;
    a.ncoinc = h->ncoinc;
    a.nspikes = h->nspikes;
    a.flags = h->flags;
    a.order = h->order;
    a.rec = h->rec_cap > 0 ? h->rec : nullptr;
    a.rec_n = h->rec_cap > 0 ? h->rec_n : nullptr;
    a.next_task = h->next_task;
    a.ns = h->ns;
    a.Tstart = Tstart;
    a.Tend = Tend;
    a.onset = h->onset;
    a.rec_cap = h->rec_cap;
    void *args[] = {&a};
    // persistent warps pulling 32-simulation tasks; no more blocks than tasks
    const long long ntasks = (h->ns + 31) / 32;
    const long long want = (long long)h->nsm * h->blocks_per_sm;
    const unsigned grid = (unsigned)std::max(1LL, std::min(want, (ntasks + kSimThreads / 32 - 1) / (kSimThreads / 32)));
    FCK(cudaMemsetAsync(h->next_task, 0, sizeof(int), h->stream));
    FCK(cudaLaunchKernel((const void *)h->kern, dim3(grid), dim3(kSimThreads), args, 0, h->stream));
    ++h->sim_launches;
    return BG_OK;
}

int prepare_launch(bg_fit *h, const double *dX) {
    const unsigned grid = (unsigned)((h->ns + kAuxThreads - 1) / kAuxThreads);
    if (h->precision == 32)
        k_fit_prepare<float><<<grid, kAuxThreads, 0, h->stream>>>(
            h->ns, h->nstate, (float *)h->S, (const float *)h->S0, dX, h->ndim, h->dimvar, h->npart ? h->npart : h->ns,
            h->dt, h->spk_off, h->spk_idx, h->delay, h->delay0, h->refr, h->refr0, h->next_allowed, h->ncoinc,
            h->nspikes, h->flags, h->rec_cap > 0 ? h->rec_n : nullptr);
    else
        k_fit_prepare<double><<<grid, kAuxThreads, 0, h->stream>>>(
            h->ns, h->nstate, (double *)h->S, (const double *)h->S0, dX, h->ndim, h->dimvar,
            h->npart ? h->npart : h->ns, h->dt, h->spk_off, h->spk_idx, h->delay, h->delay0, h->refr, h->refr0,
            h->next_allowed, h->ncoinc, h->nspikes, h->flags, h->rec_cap > 0 ? h->rec_n : nullptr);
    FCK(cudaGetLastError());
    return BG_OK;
}

int gamma_launch(bg_fit *h) {
    const unsigned grid = (unsigned)((h->npart + kAuxThreads - 1) / kAuxThreads);
    k_gamma<<<grid, kAuxThreads, 0, h->stream>>>(h->npart, h->slices, h->ncoinc, h->nspikes, h->tlen, h->trate,
                                                 h->delta_s, h->fit);
    FCK(cudaGetLastError());
    return BG_OK;
}

int check_sims(bg_fit *h) {
    if (!h) return fail(BG_EINVAL, "fit: null handle");
    if (h->ns <= 0 || !h->S) return fail(BG_ESTATE, "fit: bg_fit_set_sims not called");
    if (!h->I) return fail(BG_ESTATE, "fit: bg_fit_set_input not called");
    if (!h->spk) return fail(BG_ESTATE, "fit: bg_fit_set_targets not called");
    return BG_OK;
}

template <typename T>
int upload(T **dst, const T *src, size_t n, cudaStream_t st) {
    free_ptr(*dst);
    if (n == 0) return BG_OK;
    if (cudaMalloc((void **)dst, n * sizeof(T)) != cudaSuccess) return fail(BG_ENOMEM, "fit: cudaMalloc failed");
    if (src) FCK(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return BG_OK;
}

// Host doubles -> device scalars (the reference converts with
// array(..., dtype=mydtype), gpu_modelfitting.py:352-353).
int upload_scalar(bg_fit *h, void **dst, const double *src, size_t n) {
    if (h->precision == 64) return upload((double **)dst, src, n, h->stream);
    std::vector<float> f(n);
    for (size_t k = 0; k < n; ++k) f[k] = (float)src[k];
    int rc = upload((float **)dst, f.data(), n, h->stream);
    if (rc) return rc;
    FCK(cudaStreamSynchronize(h->stream));
    return BG_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

BG_API int bg_fit_compile_check(int precision, const bg_fit_model *model, double dt, int delta_steps,
                                int exclusive, char *log, int64_t log_len) {
    std::string src, lg;
    int nstate = 0;
    int rc = assemble_source(precision, model, dt, delta_steps, exclusive, &src, &nstate);
    if (rc) return rc;
    std::vector<char> cubin;
    rc = nvrtc_compile(src, &cubin, &lg);
    if (log && log_len > 0) {
        snprintf(log, (size_t)log_len, "%s", lg.c_str());
    }
    return rc;
}

BG_API int bg_fit_create(bg_fit **out, int device, int precision, const bg_fit_model *model, double dt,
                         int delta_steps, int exclusive) {
    if (!out) return fail(BG_EINVAL, "fit: null output pointer");
    *out = nullptr;
    std::string src, lg;
    int nstate = 0;
    int rc = assemble_source(precision, model, dt, delta_steps, exclusive, &src, &nstate);
    if (rc) return rc;
    std::vector<char> cubin;
    rc = nvrtc_compile(src, &cubin, &lg);
    if (rc) return rc;
    FCK(cudaSetDevice(device));
    bg_fit *h = new bg_fit();
    h->device = device;
    h->precision = precision;
    h->ssz = precision == 32 ? 4 : 8;
    h->nstate = nstate;
    h->dt = dt;
    h->delta = delta_steps;
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaLibraryLoadData(&h->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&h->kern, h->lib, "bg_fit_sim");
    if (e == cudaSuccess) e = cudaMalloc((void **)&h->next_task, sizeof(int));
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
    if (e != cudaSuccess) {
        std::string m = std::string("fit: loading the model kernel failed: ") + cudaGetErrorString(e);
        bg_fit_destroy(h);
        return fail(BG_ECUDA, m);
    }
    *out = h;
    return BG_OK;
}

BG_API int bg_fit_destroy(bg_fit *h) {
    if (!h) return BG_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_ptr(h->S); free_ptr(h->S0); free_ptr(h->I); free_ptr(h->I_off); free_ptr(h->spk_off);
    free_ptr(h->spk_end); free_ptr(h->spk_idx); free_ptr(h->nsteps); free_ptr(h->spk); free_ptr(h->delay);
    free_ptr(h->delay0); free_ptr(h->refr); free_ptr(h->refr0); free_ptr(h->next_allowed); free_ptr(h->ncoinc);
    free_ptr(h->nspikes); free_ptr(h->order); free_ptr(h->flags); free_ptr(h->rec); free_ptr(h->rec_n);
    free_ptr(h->tlen); free_ptr(h->trate); free_ptr(h->fit); free_ptr(h->dimvar); free_ptr(h->X); free_ptr(h->V);
    free_ptr(h->Xl); free_ptr(h->lfit); free_ptr(h->Xg); free_ptr(h->gfit); free_ptr(h->lo); free_ptr(h->hi);
    free_ptr(h->next_task);
    if (h->lib) cudaLibraryUnload(h->lib);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return BG_OK;
}

BG_API int bg_fit_set_input(bg_fit *h, const double *I, int64_t n) {
    if (!h || !I || n <= 0) return fail(BG_EINVAL, "fit: bad input array");
    FCK(cudaSetDevice(h->device));
    int rc = upload_scalar(h, &h->I, I, (size_t)n);
    if (rc) return rc;
    h->ninput = n;
    return BG_OK;
}

BG_API int bg_fit_set_targets(bg_fit *h, const int32_t *spiketimes, int64_t n) {
    if (!h || !spiketimes || n < 2) return fail(BG_EINVAL, "fit: bad target spike array");
    FCK(cudaSetDevice(h->device));
    int rc = upload(&h->spk, (const int *)spiketimes, (size_t)n, h->stream);
    if (rc) return rc;
    FCK(cudaStreamSynchronize(h->stream));
    h->nspk = n;
    return BG_OK;
}

BG_API int bg_fit_set_sims(bg_fit *h, int64_t nsims, const double *S0, const int64_t *I_offset,
                           const int32_t *nsteps, const int64_t *spk_offset, const int64_t *spk_end,
                           const int32_t *delay, const int32_t *refractory, int32_t onset) {
    if (!h || nsims <= 0 || !S0 || !I_offset || !nsteps || !spk_offset || !spk_end)
        return fail(BG_EINVAL, "fit: bad simulation arrays");
    if (nsims > (int64_t)INT32_MAX) return fail(BG_EINVAL, "fit: too many simulations");
    if (!h->I || !h->spk) return fail(BG_ESTATE, "fit: set the input and the targets before the simulations");
    int max_steps = 0;
    for (int64_t i = 0; i < nsims; ++i) {
        if (nsteps[i] < 0 || I_offset[i] < 0 || I_offset[i] + nsteps[i] > h->ninput)
            return fail(BG_EINVAL, "fit: simulation " + std::to_string(i) + " reads past the input");
        if (spk_offset[i] < 0 || spk_end[i] > h->nspk || spk_end[i] - spk_offset[i] < 2)
            return fail(BG_EINVAL, "fit: simulation " + std::to_string(i) + " has a bad target train range");
        max_steps = std::max(max_steps, (int)nsteps[i]);
    }
    FCK(cudaSetDevice(h->device));
    // Longest simulations first; equal lengths keep their input together so
    // that a warp reads one input row.
    std::vector<int> order(nsims);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        if (nsteps[a] != nsteps[b]) return nsteps[a] > nsteps[b];
        return I_offset[a] < I_offset[b];
    });
    const size_t n = (size_t)nsims;
    std::vector<int> zero(n, 0);
    int rc = 0;
    h->ns = nsims;
    h->max_steps = max_steps;
    h->onset = onset;
    if ((rc = upload_scalar(h, &h->S0, S0, n * h->nstate))) return rc;
    if (h->precision == 64) {
        if ((rc = upload((double **)&h->S, (const double *)nullptr, n * h->nstate, h->stream))) return rc;
    } else {
        if ((rc = upload((float **)&h->S, (const float *)nullptr, n * h->nstate, h->stream))) return rc;
    }
    if ((rc = upload(&h->I_off, (const long long *)I_offset, n, h->stream))) return rc;
    if ((rc = upload(&h->nsteps, (const int *)nsteps, n, h->stream))) return rc;
    if ((rc = upload(&h->spk_off, (const long long *)spk_offset, n, h->stream))) return rc;
    if ((rc = upload(&h->spk_end, (const long long *)spk_end, n, h->stream))) return rc;
    if ((rc = upload(&h->spk_idx, (const long long *)nullptr, n, h->stream))) return rc;
    if ((rc = upload(&h->delay0, delay ? (const int *)delay : zero.data(), n, h->stream))) return rc;
    if ((rc = upload(&h->refr0, refractory ? (const int *)refractory : zero.data(), n, h->stream))) return rc;
    if ((rc = upload(&h->delay, (const int *)nullptr, n, h->stream))) return rc;
    if ((rc = upload(&h->refr, (const int *)nullptr, n, h->stream))) return rc;
    if ((rc = upload(&h->next_allowed, (const int *)nullptr, n, h->stream))) return rc;
    if ((rc = upload(&h->ncoinc, (const int *)nullptr, n, h->stream))) return rc;
    if ((rc = upload(&h->nspikes, (const int *)nullptr, n, h->stream))) return rc;
    if ((rc = upload(&h->flags, (const unsigned char *)nullptr, n, h->stream))) return rc;
    if ((rc = upload(&h->order, order.data(), n, h->stream))) return rc;
    if ((rc = upload(&h->rec_n, (const int *)nullptr, n, h->stream))) return rc;
    if (h->rec_cap > 0 && (rc = upload(&h->rec, (const int *)nullptr, n * (size_t)h->rec_cap, h->stream)))
        return rc;
    FCK(cudaStreamSynchronize(h->stream));
    h->gamma_ready = h->pso_ready = false;
    return bg_fit_reinit(h);
}

BG_API int bg_fit_set_record(bg_fit *h, int32_t cap) {
    if (!h || cap < 0) return fail(BG_EINVAL, "fit: bad record capacity");
    FCK(cudaSetDevice(h->device));
    h->rec_cap = cap;
    free_ptr(h->rec);
    if (cap > 0 && h->ns > 0) {
        int rc = upload(&h->rec, (const int *)nullptr, (size_t)h->ns * cap, h->stream);
        if (rc) return rc;
    }
    return BG_OK;
}

BG_API int bg_fit_reinit(bg_fit *h) {
    int rc = check_sims(h);
    if (rc) return rc;
    FCK(cudaSetDevice(h->device));
    return prepare_launch(h, nullptr);
}

BG_API int bg_fit_run(bg_fit *h, int32_t Tstart, int32_t Tend) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (Tstart < 0 || Tend < Tstart) return fail(BG_EINVAL, "fit: bad time window");
    FCK(cudaSetDevice(h->device));
    FCK(cudaEventRecord(h->ev0, h->stream));
    if ((rc = sim_launch(h, Tstart, Tend))) return rc;
    FCK(cudaEventRecord(h->ev1, h->stream));
    FCK(cudaStreamSynchronize(h->stream));
    FCK(cudaEventElapsedTime(&h->last_sim_ms, h->ev0, h->ev1));
    return BG_OK;
}

BG_API int bg_fit_read(bg_fit *h, int32_t *coinc, int32_t *nspikes, double *state) {
    int rc = check_sims(h);
    if (rc) return rc;
    FCK(cudaSetDevice(h->device));
    FCK(cudaStreamSynchronize(h->stream));
    const size_t n = (size_t)h->ns;
    if (coinc) FCK(cudaMemcpy(coinc, h->ncoinc, n * sizeof(int), cudaMemcpyDeviceToHost));
    if (nspikes) FCK(cudaMemcpy(nspikes, h->nspikes, n * sizeof(int), cudaMemcpyDeviceToHost));
    if (state) {
        const size_t m = n * h->nstate;
        if (h->precision == 64) {
            FCK(cudaMemcpy(state, h->S, m * sizeof(double), cudaMemcpyDeviceToHost));
        } else {
            std::vector<float> f(m);
            FCK(cudaMemcpy(f.data(), h->S, m * sizeof(float), cudaMemcpyDeviceToHost));
            for (size_t k = 0; k < m; ++k) state[k] = f[k];
        }
    }
    return BG_OK;
}

BG_API int bg_fit_read_spikes(bg_fit *h, int32_t *counts, int32_t *steps) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (h->rec_cap <= 0) return fail(BG_ESTATE, "fit: spike recording is off (bg_fit_set_record)");
    FCK(cudaSetDevice(h->device));
    FCK(cudaStreamSynchronize(h->stream));
    if (counts) FCK(cudaMemcpy(counts, h->rec_n, (size_t)h->ns * sizeof(int), cudaMemcpyDeviceToHost));
    if (steps)
        FCK(cudaMemcpy(steps, h->rec, (size_t)h->ns * h->rec_cap * sizeof(int), cudaMemcpyDeviceToHost));
    return BG_OK;
}

BG_API int bg_fit_features(bg_fit *h, float *out) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (h->rec_cap <= 0) return fail(BG_ESTATE, "fit: spike recording is off (bg_fit_set_record)");
    if (!out) return fail(BG_EINVAL, "fit: null output");
    FCK(cudaSetDevice(h->device));
    float *d = nullptr;
    if (cudaMalloc((void **)&d, (size_t)h->ns * 64 * sizeof(float)) != cudaSuccess)
        return fail(BG_ENOMEM, "fit: cudaMalloc failed");
    const unsigned grid = (unsigned)((h->ns + 3) / 4);
    if (h->precision == 32)
        k_features<float><<<grid, 128, 0, h->stream>>>(h->ns, h->rec, h->rec_n, h->rec_cap, (const float *)h->I,
                                                       h->I_off, h->dt, d);
    else
        k_features<double><<<grid, 128, 0, h->stream>>>(h->ns, h->rec, h->rec_n, h->rec_cap, (const double *)h->I,
                                                        h->I_off, h->dt, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, (size_t)h->ns * 64 * sizeof(float), cudaMemcpyDeviceToHost,
                                              h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("fit: features failed: ") + cudaGetErrorString(e));
    return BG_OK;
}

BG_API int bg_spike_features(int device, int64_t ntrains, const int32_t *steps, const int64_t *offsets,
                             const double *I, const int64_t *I_offset, int64_t ninput, double dt, float *out) {
    if (ntrains <= 0 || !steps || !offsets || !I || !I_offset || ninput <= 0 || !out || !(dt > 0))
        return fail(BG_EINVAL, "features: bad arguments");
    int cap = 1;
    for (int64_t i = 0; i < ntrains; ++i) {
        if (offsets[i + 1] < offsets[i]) return fail(BG_EINVAL, "features: offsets must not decrease");
        cap = std::max(cap, (int)(offsets[i + 1] - offsets[i]));
        for (int64_t k = offsets[i]; k < offsets[i + 1]; ++k) {
            // the window reads 300 samples before every spike after 30 ms
            const double t = (double)steps[k] * dt;
            const long long idx = (long long)(t / dt);
            if (steps[k] < 0 || I_offset[i] < 0 || I_offset[i] + idx > ninput ||
                (t > 0.03 && I_offset[i] + idx - 300 < 0))
                return fail(BG_EINVAL, "features: spike " + std::to_string(k) + " lies outside its input");
        }
    }
    std::vector<int> rec((size_t)ntrains * cap, 0), cnt((size_t)ntrains);
    for (int64_t i = 0; i < ntrains; ++i) {
        cnt[i] = (int)(offsets[i + 1] - offsets[i]);
        for (int k = 0; k < cnt[i]; ++k) rec[(size_t)i * cap + k] = steps[offsets[i] + k];
    }
    FCK(cudaSetDevice(device));
    int *drec = nullptr, *dcnt = nullptr;
    double *dI = nullptr;
    long long *doff = nullptr;
    float *dout = nullptr;
    cudaError_t e = cudaMalloc((void **)&drec, rec.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&dcnt, cnt.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&dI, (size_t)ninput * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void **)&doff, (size_t)ntrains * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc((void **)&dout, (size_t)ntrains * 64 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(drec, rec.data(), rec.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dcnt, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dI, I, (size_t)ninput * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(doff, I_offset, (size_t)ntrains * sizeof(long long), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_features<double><<<(unsigned)((ntrains + 3) / 4), 128>>>(ntrains, drec, dcnt, cap, dI, doff, dt, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, (size_t)ntrains * 64 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(drec);
    cudaFree(dcnt);
    cudaFree(dI);
    cudaFree(doff);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("features: ") + cudaGetErrorString(e));
    return BG_OK;
}

BG_API int bg_fit_train_features(bg_fit *h, int64_t ntrains, const int32_t *steps, const int64_t *offsets,
                                 const int64_t *I_offset, float *out, float *gpu_ms) {
    if (!h || !h->I) return fail(BG_ESTATE, "fit: bg_fit_set_input not called");
    if (ntrains <= 0 || !steps || !offsets || !I_offset || !out) return fail(BG_EINVAL, "fit: bad feature arguments");
    int cap = 1;
    for (int64_t i = 0; i < ntrains; ++i) {
        if (offsets[i + 1] < offsets[i]) return fail(BG_EINVAL, "fit: offsets must not decrease");
        cap = std::max(cap, (int)(offsets[i + 1] - offsets[i]));
        for (int64_t k = offsets[i]; k < offsets[i + 1]; ++k) {
            const double t = (double)steps[k] * h->dt;
            const long long idx = (long long)(t / h->dt);
            if (steps[k] < 0 || I_offset[i] < 0 || I_offset[i] + idx > h->ninput ||
                (t > 0.03 && I_offset[i] + idx - 300 < 0))
                return fail(BG_EINVAL, "fit: spike " + std::to_string(k) + " lies outside its input");
        }
    }
    std::vector<int> rec((size_t)ntrains * cap, 0), cnt((size_t)ntrains);
    for (int64_t i = 0; i < ntrains; ++i) {
        cnt[i] = (int)(offsets[i + 1] - offsets[i]);
        for (int k = 0; k < cnt[i]; ++k) rec[(size_t)i * cap + k] = steps[offsets[i] + k];
    }
    FCK(cudaSetDevice(h->device));
    int *drec = nullptr, *dcnt = nullptr;
    long long *doff = nullptr;
    float *dout = nullptr;
    cudaError_t e = cudaMalloc((void **)&drec, rec.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&dcnt, cnt.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void **)&doff, (size_t)ntrains * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc((void **)&dout, (size_t)ntrains * 64 * sizeof(float));
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    if (e == cudaSuccess) cudaEventRecord(a, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(drec, rec.data(), rec.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dcnt, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(doff, I_offset, (size_t)ntrains * sizeof(long long), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        const unsigned grid = (unsigned)((ntrains + 3) / 4);
        if (h->precision == 32)
            k_features<float><<<grid, 128, 0, h->stream>>>(ntrains, drec, dcnt, cap, (const float *)h->I, doff, h->dt,
                                                           dout);
        else
            k_features<double><<<grid, 128, 0, h->stream>>>(ntrains, drec, dcnt, cap, (const double *)h->I, doff,
                                                            h->dt, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dout, (size_t)ntrains * 64 * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) cudaEventRecord(b, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    float ms = 0;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, a, b);
    if (gpu_ms) *gpu_ms = ms;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(drec);
    cudaFree(dcnt);
    cudaFree(doff);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("fit: features failed: ") + cudaGetErrorString(e));
    return BG_OK;
}

BG_API int bg_fit_set_gamma(bg_fit *h, int64_t nparticles, int32_t slices, const int32_t *target_length,
                            const double *target_rate, double delta) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (nparticles <= 0 || slices <= 0 || nparticles * slices != h->ns || !target_length || !target_rate)
        return fail(BG_EINVAL, "fit: particles x slices must equal the number of simulations");
    FCK(cudaSetDevice(h->device));
    h->npart = nparticles;
    h->slices = slices;
    h->delta_s = delta;
    if ((rc = upload(&h->tlen, (const int *)target_length, (size_t)nparticles, h->stream))) return rc;
    if ((rc = upload(&h->trate, target_rate, (size_t)nparticles, h->stream))) return rc;
    if ((rc = upload(&h->fit, (const double *)nullptr, (size_t)nparticles, h->stream))) return rc;
    FCK(cudaStreamSynchronize(h->stream));
    h->gamma_ready = true;
    return BG_OK;
}

BG_API int bg_fit_set_params(bg_fit *h, int32_t ndim, const int32_t *dim_var) {
    if (!h || ndim < 0 || (ndim > 0 && !dim_var)) return fail(BG_EINVAL, "fit: bad parameter map");
    for (int d = 0; d < ndim; ++d)
        if (dim_var[d] < -2 || dim_var[d] >= h->nstate) return fail(BG_EINVAL, "fit: parameter maps to no state row");
    FCK(cudaSetDevice(h->device));
    h->ndim = ndim;
    int rc = upload(&h->dimvar, (const int *)dim_var, (size_t)ndim, h->stream);
    if (rc) return rc;
    FCK(cudaStreamSynchronize(h->stream));
    h->pso_ready = false;
    return BG_OK;
}

BG_API int bg_fit_evaluate(bg_fit *h, const double *X, double *gamma_out) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (!h->gamma_ready) return fail(BG_ESTATE, "fit: bg_fit_set_gamma not called");
    if (!X && h->ndim > 0) return fail(BG_EINVAL, "fit: null parameter matrix");
    FCK(cudaSetDevice(h->device));
    double *dX = nullptr;
    const size_t nx = (size_t)h->ndim * h->npart;
    if (nx) {
        if (cudaMalloc((void **)&dX, nx * sizeof(double)) != cudaSuccess) return fail(BG_ENOMEM, "fit: cudaMalloc failed");
        cudaError_t e = cudaMemcpyAsync(dX, X, nx * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        if (e != cudaSuccess) {
            cudaFree(dX);
            return fail(BG_ECUDA, std::string("fit: copy of X failed: ") + cudaGetErrorString(e));
        }
    }
    cudaEvent_t e_start = nullptr;
    cudaEventCreate(&e_start);
    cudaEventRecord(e_start, h->stream);
    rc = prepare_launch(h, dX);
    if (!rc) {
        cudaEventRecord(h->ev0, h->stream);
        rc = sim_launch(h, 0, h->max_steps);
        cudaEventRecord(h->ev1, h->stream);
    }
    if (!rc) rc = gamma_launch(h);
    cudaEvent_t e_end = nullptr;
    cudaEventCreate(&e_end);
    cudaEventRecord(e_end, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (dX) cudaFree(dX);
    if (!rc && e == cudaSuccess) cudaEventElapsedTime(&h->last_eval_ms, e_start, e_end);
    cudaEventDestroy(e_start);
    cudaEventDestroy(e_end);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("fit: evaluation failed: ") + cudaGetErrorString(e));
    FCK(cudaEventElapsedTime(&h->last_sim_ms, h->ev0, h->ev1));
    if (gamma_out) FCK(cudaMemcpy(gamma_out, h->fit, (size_t)h->npart * sizeof(double), cudaMemcpyDeviceToHost));
    return BG_OK;
}

BG_API int bg_fit_set_blocks_per_sm(bg_fit *h, int32_t blocks_per_sm) {
    if (!h || blocks_per_sm < 1 || blocks_per_sm > 16) return fail(BG_EINVAL, "fit: blocks per SM must be in 1..16");
    h->blocks_per_sm = blocks_per_sm;
    return BG_OK;
}

BG_API int bg_fit_autotune(bg_fit *h, const double *X, int32_t *blocks_per_sm, float *ms_out) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (X && !h->npart) return fail(BG_ESTATE, "fit: bg_fit_set_gamma not called");
    FCK(cudaSetDevice(h->device));
    double *dX = nullptr;
    const size_t nx = X ? (size_t)h->ndim * h->npart : 0;
    if (nx) {
        if (cudaMalloc((void **)&dX, nx * sizeof(double)) != cudaSuccess) return fail(BG_ENOMEM, "fit: cudaMalloc failed");
        cudaMemcpy(dX, X, nx * sizeof(double), cudaMemcpyHostToDevice);
    }
    // every candidate launch shape runs the same simulations; results do not
    // depend on it, only the time does
    static const int cand[] = {1, 2, 3, 4, 6, 8};
    float best = INFINITY;
    int bestb = h->blocks_per_sm;
    for (int k = 0; k < (int)(sizeof cand / sizeof cand[0]) && !rc; ++k) {
        h->blocks_per_sm = cand[k];
        rc = prepare_launch(h, dX);
        if (!rc) rc = sim_launch(h, 0, h->max_steps);      // warm
        if (!rc) rc = prepare_launch(h, dX);
        if (!rc) {
            cudaEventRecord(h->ev0, h->stream);
            rc = sim_launch(h, 0, h->max_steps);
            cudaEventRecord(h->ev1, h->stream);
        }
        if (!rc && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = fail(BG_ECUDA, "fit: autotune run failed");
        float ms = 0;
        if (!rc) cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        if (ms_out) ms_out[k] = ms;
        if (!rc && ms < best) {
            best = ms;
            bestb = cand[k];
        }
    }
    h->blocks_per_sm = bestb;
    if (!rc) rc = prepare_launch(h, dX);
    cudaStreamSynchronize(h->stream);
    if (dX) cudaFree(dX);
    if (blocks_per_sm) *blocks_per_sm = bestb;
    return rc;
}

BG_API int bg_fit_pso_init(bg_fit *h, int32_t group_size, const double *X0, const double *xmin, const double *xmax,
                           double omega, double c1, double c2, uint64_t seed) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (!h->gamma_ready) return fail(BG_ESTATE, "fit: bg_fit_set_gamma not called");
    if (h->ndim <= 0) return fail(BG_ESTATE, "fit: bg_fit_set_params not called");
    if (group_size <= 0 || h->npart % group_size != 0 || !X0 || !xmin || !xmax)
        return fail(BG_EINVAL, "fit: the group size must divide the number of particles");
    FCK(cudaSetDevice(h->device));
    const size_t M = (size_t)h->npart, D = (size_t)h->ndim, G = M / group_size;
    h->group_size = group_size;
    h->ngroups = (int)G;
    h->omega = omega;
    h->c1 = c1;
    h->c2 = c2;
    h->seed = seed;
    h->iter = 0;
    // X0 clipped into the bounds (particle_swarm.py:51-52); X_lbest = X0,
    // X_gbest = the first particle of each group (particle_swarm.py:56-57).
    std::vector<double> X(X0, X0 + D * M), Xg(D * G), mfit(M, -INFINITY), gf(G, -INFINITY), zero(D * M, 0.0);
    for (size_t d = 0; d < D; ++d)
        for (size_t p = 0; p < M; ++p) {
            double &x = X[d * M + p];
            x = (x < xmin[d]) ? xmin[d] : x;
            x = (x > xmax[d]) ? xmax[d] : x;
        }
    for (size_t d = 0; d < D; ++d)
        for (size_t g = 0; g < G; ++g) Xg[d * G + g] = X[d * M + g * group_size];
    if ((rc = upload(&h->X, X.data(), D * M, h->stream))) return rc;
    if ((rc = upload(&h->V, zero.data(), D * M, h->stream))) return rc;
    if ((rc = upload(&h->Xl, X.data(), D * M, h->stream))) return rc;
    if ((rc = upload(&h->lfit, mfit.data(), M, h->stream))) return rc;
    if ((rc = upload(&h->Xg, Xg.data(), D * G, h->stream))) return rc;
    if ((rc = upload(&h->gfit, gf.data(), G, h->stream))) return rc;
    if ((rc = upload(&h->lo, xmin, D, h->stream))) return rc;
    if ((rc = upload(&h->hi, xmax, D, h->stream))) return rc;
    FCK(cudaStreamSynchronize(h->stream));
    h->pso_ready = true;
    return BG_OK;
}

BG_API int bg_fit_pso_run(bg_fit *h, int32_t iterations, double *trace, float *iter_ms) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (!h->pso_ready) return fail(BG_ESTATE, "fit: bg_fit_pso_init not called");
    if (iterations < 0) return fail(BG_EINVAL, "fit: negative iteration count");
    FCK(cudaSetDevice(h->device));
    const int64_t M = h->npart, G = h->ngroups;
    double *dtrace = nullptr;
    if (trace && iterations > 0 &&
        cudaMalloc((void **)&dtrace, (size_t)iterations * G * sizeof(double)) != cudaSuccess)
        return fail(BG_ENOMEM, "fit: cudaMalloc failed");
    std::vector<cudaEvent_t> ev;
    if (iter_ms) {
        ev.resize((size_t)iterations + 1);
        for (auto &e : ev) cudaEventCreate(&e);
        cudaEventRecord(ev[0], h->stream);
    }
    const unsigned gmove = (unsigned)((M * h->ndim + kAuxThreads - 1) / kAuxThreads);
    for (int k = 0; k < iterations && !rc; ++k) {
        k_pso_move<<<gmove, kAuxThreads, 0, h->stream>>>(M, h->ndim, h->group_size, h->X, h->V, h->Xl, h->Xg, h->lo,
                                                         h->hi, h->omega, h->c1, h->c2, h->seed, h->iter);
        rc = prepare_launch(h, h->X);
        if (!rc) rc = sim_launch(h, 0, h->max_steps);
        if (!rc) rc = gamma_launch(h);
        if (!rc) {
            k_pso_best<<<(unsigned)G, kAuxThreads, 0, h->stream>>>(M, h->ndim, h->group_size, h->X, h->fit, h->Xl,
                                                                   h->lfit, h->Xg, h->gfit, dtrace, k);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = fail(BG_ECUDA, std::string("fit: swarm kernels: ") + cudaGetErrorString(e));
        }
        if (iter_ms) cudaEventRecord(ev[(size_t)k + 1], h->stream);
        ++h->iter;
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (!rc && e != cudaSuccess) rc = fail(BG_ECUDA, std::string("fit: swarm run failed: ") + cudaGetErrorString(e));
    if (!rc && trace && dtrace)
        if (cudaMemcpy(trace, dtrace, (size_t)iterations * G * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(BG_ECUDA, "fit: trace read failed");
    if (iter_ms) {
        for (int k = 0; k < iterations; ++k)
            if (!rc) cudaEventElapsedTime(&iter_ms[k], ev[k], ev[(size_t)k + 1]);
        for (auto &x : ev) cudaEventDestroy(x);
    }
    if (dtrace) cudaFree(dtrace);
    return rc;
}

BG_API int bg_fit_pso_evaluate_initial(bg_fit *h) {
    int rc = check_sims(h);
    if (rc) return rc;
    if (!h->pso_ready) return fail(BG_ESTATE, "fit: bg_fit_pso_init not called");
    FCK(cudaSetDevice(h->device));
    FCK(cudaEventRecord(h->ev0, h->stream));
    if ((rc = prepare_launch(h, h->X))) return rc;
    if ((rc = sim_launch(h, 0, h->max_steps))) return rc;
    if ((rc = gamma_launch(h))) return rc;
    k_pso_best<<<(unsigned)h->ngroups, kAuxThreads, 0, h->stream>>>(h->npart, h->ndim, h->group_size, h->X, h->fit,
                                                                    h->Xl, h->lfit, h->Xg, h->gfit, nullptr, 0);
    FCK(cudaGetLastError());
    FCK(cudaEventRecord(h->ev1, h->stream));
    FCK(cudaStreamSynchronize(h->stream));
    FCK(cudaEventElapsedTime(&h->last_eval_ms, h->ev0, h->ev1));
    return BG_OK;
}

BG_API int bg_fit_pso_best(bg_fit *h, double *X_gbest, double *fit_gbest) {
    if (!h || !h->pso_ready) return fail(BG_ESTATE, "fit: no swarm");
    FCK(cudaSetDevice(h->device));
    FCK(cudaStreamSynchronize(h->stream));
    const size_t G = (size_t)h->ngroups;
    if (X_gbest) FCK(cudaMemcpy(X_gbest, h->Xg, (size_t)h->ndim * G * sizeof(double), cudaMemcpyDeviceToHost));
    if (fit_gbest) FCK(cudaMemcpy(fit_gbest, h->gfit, G * sizeof(double), cudaMemcpyDeviceToHost));
    return BG_OK;
}

BG_API int bg_fit_pso_state(bg_fit *h, double *X, double *V, double *X_lbest, double *fit_lbest) {
    if (!h || !h->pso_ready) return fail(BG_ESTATE, "fit: no swarm");
    FCK(cudaSetDevice(h->device));
    FCK(cudaStreamSynchronize(h->stream));
    const size_t n = (size_t)h->ndim * h->npart;
    if (X) FCK(cudaMemcpy(X, h->X, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (V) FCK(cudaMemcpy(V, h->V, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (X_lbest) FCK(cudaMemcpy(X_lbest, h->Xl, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (fit_lbest) FCK(cudaMemcpy(fit_lbest, h->lfit, (size_t)h->npart * sizeof(double), cudaMemcpyDeviceToHost));
    return BG_OK;
}

// out[0] = GPU ms of the last simulation launch, out[1] = simulation
// launches so far, out[2] = neuron-steps of one full run, out[3] = longest
// simulation (steps), out[4] = GPU ms of the last whole evaluation.
BG_API int bg_fit_stats(bg_fit *h, double *out, int n) {
    if (!h || !out) return fail(BG_EINVAL, "fit: bad stats call");
    long long steps = 0;
    if (h->ns > 0) {
        std::vector<int> ns((size_t)h->ns);
        cudaSetDevice(h->device);
        FCK(cudaMemcpy(ns.data(), h->nsteps, ns.size() * sizeof(int), cudaMemcpyDeviceToHost));
        for (int v : ns) steps += v;
    }
    const double v[5] = {h->last_sim_ms, (double)h->sim_launches, (double)steps, (double)h->max_steps,
                         h->last_eval_ms};
    for (int k = 0; k < n && k < 5; ++k) out[k] = v[k];
    return BG_OK;
}

}  // extern "C"
