// bg_net.cu -- host runtime of the clock-driven network engine (C ABI).
//
// A bg_net holds the device image of a Brian Network: per-group state
// matrices, bit-per-neuron spike history rings, CSR connection matrices,
// DelayConnection rings, STDP traces and monitor buffers.  bg_net_prepare
// freezes the schedule into a per-step list of kernel launches; bg_net_run
// replays it from a CUDA graph of kGraphSteps steps, draining monitor
// buffers to host memory between chunks.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "bg_kernels.cuh"
#include "bg_persist.cuh"
#include "bg_synpersist.cuh"
#include "bg_batch.cuh"
#include "bg_rtc.h"
#include "../../include/brian_b200.h"

namespace {

thread_local std::string g_err;
int fail(int code, const std::string &m) { g_err = m; return code; }

#define BG_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(BG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

constexpr int kGraphSteps = 32;
constexpr int64_t kChunkSteps = 1024;

struct HGroup {
    int64_t n = 0, npad = 0; int nvar = 0;
    std::vector<double> S0;
    bool linear = false, useC = false; std::vector<double> A, C;
    int thr_kind = 0, thr_var = 0, thr_var2 = 0; double thr_val = 0;
    int rate_var = 0; uint64_t seed = 0;
    std::vector<int64_t> gen_steps; std::vector<int32_t> gen_idx;
    int reset_kind = 0, reset_var = 0, reset_var2 = 0; double reset_val = 0;
    bool refr = false; double refr_time = 0; int period = 0; int clamp_var = 0; double clamp_val = 0;
    int depth = 1;
    void *dS = nullptr; uint32_t *dHist = nullptr; double *dNext = nullptr; int32_t *dLast = nullptr;
    int borrowed = -1;                  // index into bg_net::imports when the state lives in a caller's buffer
    int64_t *dGenSteps = nullptr; int32_t *dGenIdx = nullptr;
    std::vector<int> delivs, recs;
    int emp_steps = 0;                  // EmpiricalThreshold window (steps), 0: off
    struct Setter {                     // TimedArraySetter (see bg::SetDev)
        int var, mode; int64_t origin, count, nrows, ncols; double t_init, adt; int64_t first;
        std::vector<double> vals; std::vector<int64_t> bp;
        void *dVals = nullptr; int64_t *dBp = nullptr;
    };
    std::vector<Setter> setters;
    // generated model (update / threshold / reset as C over s_<name>),
    // compiled with the head kernel by NVRTC at prepare
    std::vector<std::string> gen_names;
    std::string gen_update, gen_threshold, gen_reset;
    cudaLibrary_t gen_lib = nullptr; cudaKernel_t gen_kernel = nullptr;
    bool generated() const { return !gen_update.empty() || !gen_threshold.empty() || !gen_reset.empty(); }
};
// A std::vector that leaves new elements uninitialised: the large host
// copies of the connectivity are filled by parallel copies, which also
// spreads the first touch of their pages over threads.
template <typename T> struct NoInitAlloc : std::allocator<T> {
    template <typename U> struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <typename U> NoInitAlloc(const NoInitAlloc<U> &) {}
    template <typename U> void construct(U *p) noexcept { ::new ((void *)p) U; }
    template <typename U, typename... A> void construct(U *p, A &&...a) { ::new ((void *)p) U(std::forward<A>(a)...); }
};
template <typename T> using hvec = std::vector<T, NoInitAlloc<T>>;

// f(lo, hi, t) over [0, n) split into contiguous parts, one per host thread
// (at most 32, at least `grain` items each); t is the part's index.
template <typename F> void parallel_for(int64_t n, F f, int64_t grain = (int64_t)1 << 22) {
    int nt = (int)std::min<int64_t>(std::min<unsigned>(32u, std::max(1u, std::thread::hardware_concurrency())),
                                    (n + grain - 1) / grain);
    if (nt <= 1) { f((int64_t)0, n, 0); return; }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; ++t) th.emplace_back([&f, n, nt, t] { f(n * t / nt, n * (t + 1) / nt, t); });
    for (auto &x : th) x.join();
}
static int parallel_parts(int64_t n, int64_t grain = (int64_t)1 << 22) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(std::min<unsigned>(32u, std::max(1u, std::thread::hardware_concurrency())),
                                                       (n + grain - 1) / grain));
}

// device helpers of the network set-up (grid-stride loops)
__global__ void k_fill_u32(uint32_t *p, int64_t n, uint32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_fill_u64(unsigned long long *p, int64_t n, unsigned long long v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
// in-degree of every target (columns validated to lie in [0, tn))
__global__ void k_indegree(const int32_t *cols, int64_t n, int32_t *deg) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(deg + cols[i], 1);
}
// persistent push words: target | delay << 24
// (d null: every delay is zero)
__global__ void k_pack_synapses(const int32_t *cols, const uint8_t *d, int64_t n, uint32_t *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)cols[i] | ((uint32_t)(d ? d[i] : 0) << 24);
}

struct HConn {
    int32_t src = 0, tgt = 0; int64_t so = 0, sn = 0, to = 0, tn = 0; int var = 0;
    bool dense = false; int64_t nnz = 0;
    std::vector<int64_t> rowptr; hvec<int32_t> cols; hvec<char> w; int w_bits = 64;
    bool wshared = false;      // w holds the one weight every synapse shares (the device array is filled)
    int32_t delay = 0; bool hetero = false; hvec<uint8_t> d; int md = 0; int mod_var = -1;
    bool homogeneous = false; int parts = 1; int stdp = -1; bool fused_push = false;
    uint16_t *dCRing = nullptr; int64_t tnp = 0; void *dTable = nullptr; int tablen = 0;   // count ring (shared weight)
    int64_t *dRow = nullptr; int32_t *dCols = nullptr; void *dW = nullptr; uint8_t *dD = nullptr; void *dRing = nullptr;
    uint32_t *dPacked = nullptr;       // persistent path: target | delay << 24 (count rings, targets < 2^24)
    // persistent path, zero-delay Connection: its own count ring of dir_md
    // rows and the table {0, w} (not part of the saved state: every launch
    // ends with the ring delivered)
    uint16_t *dDirRing = nullptr; void *dDirTable = nullptr; int dir_md = 0;
    int64_t *dColptr = nullptr, *dColk = nullptr; int32_t *dColsrc = nullptr;
    int64_t wcount() const { return dense ? sn * tn : nnz; }
};
struct HStdp {
    int cid; double a_pre, c_pre, a_post, c_post, Ap, Am, wmin, wmax; int inter; int pre_delay, post_delay;
    double *dApre = nullptr, *dApost = nullptr; bool fused = false;
    int pre_mode = 0, post_mode = 0; double wx = 0.0;   // update forms of the w lines (stdp_w)
    // DelayConnection: trace histories of hlen steps and per-synapse lags
    bool delayed = false; int hlen = 0; std::vector<uint8_t> lag_pre, lag_post;
    double *dHpre = nullptr, *dHpost = nullptr; uint8_t *dLagPre = nullptr, *dLagPostC = nullptr;
};
// Synapses: incoming synapses of each target in queue order (delay
// descending, source, synapse index), as words source | (delay+1) << 24
// with the statements' terms permuted alike.
struct HSyn {
    int32_t src = 0, tgt = 0; int64_t so = 0, sn = 0, to = 0, tn = 0, nsyn = 0; int nops = 0, dmax = 0;
    std::vector<int32_t> op_var, op_sub;
    std::vector<int64_t> colptr, perm; std::vector<uint32_t> word; std::vector<double> terms;   // terms: [nops][nsyn], synapse order
    int64_t *dColptr = nullptr; uint32_t *dWord = nullptr; double *dTerm = nullptr;
    // event path (rows by source): per source, its synapses by (delay, synapse
    // index) with their target and column position; event bins and flags
    bool events = false;
    std::vector<int64_t> srcptr; std::vector<uint8_t> sd; std::vector<int32_t> stgt, sq;
    int64_t *dSrcPtr = nullptr; uint8_t *dSd = nullptr; int32_t *dStgt = nullptr, *dSq = nullptr;
    int *dBinCnt = nullptr; unsigned long long *dBinKey = nullptr; int32_t *dBinQ = nullptr; int *dUsePull = nullptr;
    int32_t *dDoff = nullptr;           // per source, start of each delay in its row (when it fits 256 MB)
    int nbins = 0;
    int32_t *dSlist = nullptr; int *dScnt = nullptr; int sdepth = 0;   // spike lists of the last sdepth steps
    double *dTermSrc = nullptr;         // persistent kernel: the statement's term per synapse, by-source order
    // synapses with code (bg_synapses_set_code): synaptic variables [nsv][nsyn]
    // (synapse order on the host, column order on the device), the generated
    // pre/post code, the target variables it uses (slots; `writes` those it
    // assigns) and the source variables it reads
    bool coded = false; int nsv = 0; std::vector<double> sv; double *dSv = nullptr;
    std::string pre_code, post_code; std::vector<int32_t> slot_var, pre_var, writes;
    cudaLibrary_t code_lib = nullptr; cudaKernel_t code_kernel = nullptr;
};
struct HSpikeMon {
    int gid; int64_t origin, n; int delay;
    long long *dCnt = nullptr, *dBase = nullptr; int32_t *dIdx = nullptr, *dSteps = nullptr; int64_t cap = 0;
    std::vector<int64_t> steps; std::vector<int32_t> idx;
};
struct HStateMon {
    int gid; int var; std::vector<int32_t> idx; int timestep; long long start = 0;
    std::vector<int32_t> sorted, pos, blk_lo;
    int32_t *dIdx = nullptr, *dPos = nullptr, *dBlk = nullptr; void *dBuf = nullptr; long long *dRowBase = nullptr;
    int32_t *dBlkP = nullptr;          // blk_lo for the persistent kernel's blocks
    int64_t cap_rows = 0; long long rows_done = 0;
    std::vector<double> vals; std::vector<int64_t> steps;
};
enum { IT_CONN = 0, IT_SPIKEMON = 1, IT_STDP_PRE = 2, IT_STDP_POST = 3 };
struct Item { int kind; int id; };

using Launch = std::function<cudaError_t(cudaStream_t, int tail, int last)>;

}  // namespace

struct bg_net {
    int device = 0, precision = 64, deterministic = 1; double dt = 1e-4;
    int allow_persist = 1;
    int persist_th = 0;                 // forced threads per block of the persistent kernel (0: automatic)
    int persist_used = 0;               // threads per block of the built persistent kernel (0: none)
    void *stage[2] = {nullptr, nullptr};                 // pinned staging of large uploads (prepare only)
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    bool stage_used[2] = {false, false};
    uint32_t *dMonWords = nullptr;      // persistent path with spike monitors: spike words per step of a chunk
    long long *dMonOff = nullptr;       //   and per-step record offsets
    cudaStream_t stream = nullptr;
    std::vector<HGroup> groups; std::vector<HConn> conns; std::vector<HStdp> stdps; std::vector<HSyn> syns;
    std::vector<HSpikeMon> smons; std::vector<HStateMon> stmons; std::vector<Item> items;
    std::vector<int> mon_kind, mon_idx;
    DevCtl *dCtl = nullptr;
    bool prepared = false; long long nstep = 0;
    std::vector<Launch> step_launches;     // per-step kernels in schedule order
    std::vector<std::string> item_names;   // one per step launch
    unsigned long long *dCounters = nullptr; // [groups] spikes, then [conns] events
    std::vector<Launch> finalize_launches; // tail-only head kernels
    cudaGraphExec_t gexec = nullptr;
    // step launches [side0, side1) (the SpikeMonitors, right after the group
    // kernels) only read the spike history the group kernels wrote: in the
    // step graph they run on a side stream beside the launches after them
    // and join before the step's last launch (the one that advances the step)
    size_t side0 = 0, side1 = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // persistent single-launch path (see bg_persist.cuh); empty when the
    // network does not have its shape
    std::function<cudaError_t(cudaStream_t, int nsteps)> persist;
    unsigned int *dArrived = nullptr;
    int *dUsePull3 = nullptr;           // Synapses persistent kernel: overflow flags by step mod 3
    int *dPBinCnt = nullptr; unsigned long long *dPBinKey = nullptr; double *dPBinT = nullptr;   //   and its bins
    int64_t launches = 0; double last_ms = 0;
    unsigned int spin_limit = BG_SPIN_LIMIT;   // polls of a bounded inter-block wait
    int hold_block = -1;                // test hook: a persistent block that never arrives
    int check_finite = 0;               // check the states for NaN/inf after every run
    bool failed = false;                // a device error stopped the network
    int syn_events_forced = 0;          // Synapses: event path whatever the size (tests)
    bool syn_lists_stale = true;        // Synapses spike lists to rebuild from the history before the next step
    std::vector<void *> allocs;
    struct Import { void *ptr; int64_t bytes; int dtype; };
    std::vector<Import> imports;        // borrowed device buffers (the caller owns and frees them)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t chunk_steps = kChunkSteps;

    template <typename P> cudaError_t alloc(P **p, size_t bytes) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
        if (e == cudaSuccess) { allocs.push_back(q); *p = (P *)q; }
        return e;
    }
};

namespace {

size_t tsize(const bg_net *n) { return n->precision == 64 ? 8 : 4; }

bool gid_ok(const bg_net *n, int32_t g) { return n && g >= 0 && g < (int32_t)n->groups.size(); }

// ------------------------------------------------------------------ launches
template <typename T, int NV>
cudaError_t launch_head_nv(const bg::HeadArgs<T> &a, int64_t blocks, cudaStream_t s) {
    bg::k_head<T, NV><<<(unsigned)blocks, bg::kHeadThreads, 0, s>>>(a);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_head(const bg::HeadArgs<T> &a, int nvar, int64_t blocks, cudaStream_t s) {
    switch (nvar) {
    case 0: case 1: return launch_head_nv<T, 1>(a, blocks, s);
    case 2: return launch_head_nv<T, 2>(a, blocks, s);
    case 3: return launch_head_nv<T, 3>(a, blocks, s);
    case 4: return launch_head_nv<T, 4>(a, blocks, s);
    case 5: return launch_head_nv<T, 5>(a, blocks, s);
    case 6: return launch_head_nv<T, 6>(a, blocks, s);
    case 7: return launch_head_nv<T, 7>(a, blocks, s);
    default: return launch_head_nv<T, 8>(a, blocks, s);
    }
}

// The head kernel of a group with a generated model: the engine's kernel
// sources with a model policy over the group's registers (head_body).
template <typename T>
int compile_generated_head(HGroup &g) {
    if (g.gen_kernel) return BG_OK;
    const char *sc = sizeof(T) == 8 ? "double" : "float";
    std::string src = "#define BG_GENERATED_MODEL 1\n";
    for (const char *const *p = kNetRtcSource; *p; ++p) src += *p;
    auto load = [&](bool cnst) {
        std::string o;
        for (size_t k = 0; k < g.gen_names.size(); ++k)
            o += std::string("        ") + (cnst ? "const " : "") + "scalar s_" + g.gen_names[k] + " = S[" +
                 std::to_string(k) + "];\n";
        return o;
    };
    auto store = [&]() {
        std::string o;
        for (size_t k = 0; k < g.gen_names.size(); ++k)
            o += "        S[" + std::to_string(k) + "] = s_" + g.gen_names[k] + ";\n";
        return o;
    };
    src += "namespace bg {\nstruct GenModel {\n";
    src += std::string("    static constexpr bool custom_update = ") + (g.gen_update.empty() ? "false" : "true") +
           ", custom_threshold = " + (g.gen_threshold.empty() ? "false" : "true") +
           ", custom_reset = " + (g.gen_reset.empty() ? "false" : "true") + ";\n";
    src += "    template <typename T, int NV> static __device__ __forceinline__ void update(T (&S)[NV], double t_) {\n"
           "        typedef T scalar; const scalar t = (scalar)t_; const scalar I_in = (scalar)0; (void)t; (void)I_in;\n" +
           load(false) + g.gen_update + "\n" + store() + "    }\n";
    src += "    template <typename T, int NV> static __device__ __forceinline__ bool threshold(const T (&S)[NV], double t_) {\n"
           "        typedef T scalar; const scalar t = (scalar)t_; const scalar I_in = (scalar)0; (void)t; (void)I_in;\n" +
           load(true) + "        return (bool)(" + (g.gen_threshold.empty() ? std::string("false") : g.gen_threshold) +
           ");\n    }\n";
    src += "    template <typename T, int NV> static __device__ __forceinline__ void reset(T (&S)[NV], double t_) {\n"
           "        typedef T scalar; const scalar t = (scalar)t_; const scalar I_in = (scalar)0; const bool reset_on = true;\n"
           "        (void)t; (void)I_in; (void)reset_on;\n" +
           load(false) + g.gen_reset + "\n" + store() + "    }\n";
    src += "};\n}  // namespace bg\n";
    src += std::string("extern \"C\" __global__ void __launch_bounds__(bg::kHeadThreads, 2) bg_gen_head(const bg::HeadArgs<") +
           sc + "> a) {\n    bg::head_body<" + sc + ", " + std::to_string(std::max(1, g.nvar)) + ", bg::GenModel>(a);\n}\n";
    std::vector<char> cubin;
    std::string log;
    int rc = bg_nvrtc_compile(src, &cubin, &log);
    if (rc) return rc;
    cudaError_t e = cudaLibraryLoadData(&g.gen_lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&g.gen_kernel, g.gen_lib, "bg_gen_head");
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("generated group kernel: ") + cudaGetErrorString(e));
    return BG_OK;
}

template <typename T>
cudaError_t launch_generated_head(cudaKernel_t k, const bg::HeadArgs<T> &a, int64_t blocks, cudaStream_t s) {
    void *args[] = {(void *)&a};
    return cudaLaunchKernel((const void *)k, dim3((unsigned)blocks), dim3(bg::kHeadThreads), args, 0, s);
}

template <typename T>
int build_group(bg_net *net, int gid) {
    HGroup &g = net->groups[gid];
    bg::HeadArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.S = (T *)g.dS; a.n = g.n; a.npad = g.npad; a.nvar = g.nvar;
    a.linear = g.linear; a.useC = g.useC;
    for (int j = 0; j < g.nvar && g.linear; ++j) {
        for (int k = 0; k < g.nvar; ++k) a.A[j * g.nvar + k] = (T)g.A[j * g.nvar + k];
        a.C[j] = g.useC ? (T)g.C[j] : T(0);
    }
    bg::set_linear_masks(a, g.nvar);
    a.thr_kind = g.thr_kind; a.thr_var = g.thr_var; a.thr_var2 = g.thr_var2; a.thr_val = (T)g.thr_val;
    a.dt = net->dt; a.seed = g.seed; a.rate_var = g.rate_var;
    a.gen_steps = g.dGenSteps; a.gen_idx = g.dGenIdx; a.gen_n = (int64_t)g.gen_steps.size();
    a.reset_kind = g.reset_kind; a.reset_var = g.reset_var; a.reset_var2 = g.reset_var2; a.reset_val = (T)g.reset_val;
    a.refr = g.refr; a.refr_time = g.refr_time; a.period = g.period; a.clamp_var = g.clamp_var; a.clamp_val = (T)g.clamp_val;
    a.next_allowed = g.dNext; a.last_spike = g.dLast; a.emp_steps = g.emp_steps;
    a.hist = g.dHist; a.depth = g.depth; a.nwords = g.npad / 32;
    if ((int)g.delivs.size() > bg::kMaxDeliv) return fail(BG_ENOSYS, "too many DelayConnections into one group");
    a.ndeliv = (int)g.delivs.size();
    for (int k = 0; k < a.ndeliv; ++k) {
        const HConn &c = net->conns[g.delivs[k]];
        a.deliv[k].ring = (T *)c.dRing; a.deliv[k].tn = c.tn; a.deliv[k].to = c.to; a.deliv[k].md = c.md; a.deliv[k].var = c.var;
        a.deliv[k].cring = c.dCRing; a.deliv[k].tnp = c.tnp; a.deliv[k].table = (const T *)c.dTable; a.deliv[k].tablen = c.tablen;
    }
    a.npush = 0;
    for (size_t ci = 0; ci < net->conns.size(); ++ci) {
        const HConn &c = net->conns[ci];
        if (!c.fused_push || c.src != gid) continue;
        if (a.npush == bg::kMaxPush) return fail(BG_ENOSYS, "too many delayed connections from one group");
        bg::Push<T> &q = a.push[a.npush++];
        q.ring = (T *)c.dRing; q.md = c.md; q.so = c.so; q.sn = c.sn; q.tn = c.tn;
        q.rowptr = c.dRow; q.cols = c.dCols; q.w = c.dW; q.w_bits = c.w_bits; q.d = c.dD;
        q.events = net->dCounters + net->groups.size() + ci;
        q.cring = c.dCRing; q.tnp = c.tnp;
    }
    a.nset = (int)g.setters.size();
    for (int k = 0; k < a.nset; ++k) {
        const HGroup::Setter &h = g.setters[k];
        bg::SetDev<T> &d = a.set[k];
        d.var = h.var; d.mode = h.mode; d.origin = h.origin; d.count = h.count; d.nrows = h.nrows; d.ncols = h.ncols;
        d.t_init = h.t_init; d.adt = h.adt; d.first = h.first; d.vals = (const T *)h.dVals; d.bp = h.dBp;
    }
    if ((int)g.recs.size() > bg::kMaxRec) return fail(BG_ENOSYS, "too many StateMonitors on one group");
    a.nrec = (int)g.recs.size();
    for (int k = 0; k < a.nrec; ++k) {
        const HStateMon &m = net->stmons[g.recs[k]];
        bg::RecDev &r = a.rec[k];
        r.var = m.var; r.nidx = (int)m.idx.size(); r.idx = m.dIdx; r.pos = m.dPos; r.blk_lo = m.dBlk;
        r.buf = m.dBuf; r.row_base = m.dRowBase; r.timestep = m.timestep; r.start = m.start;
    }
    const int64_t blocks = g.npad / bg::kBlockNeurons;
    const int nvar = g.nvar;
    a.spikes = net->dCounters + gid;
    if (g.generated()) {
        int st = compile_generated_head<T>(g);
        if (st) return st;
        const bool has_tail = a.ndeliv || g.reset_kind || !g.gen_reset.empty() || g.period > 0 || a.nrec;
        const cudaKernel_t k = g.gen_kernel;
        net->item_names.push_back("genhead[g" + std::to_string(gid) + "]");
        net->step_launches.push_back([a, k, blocks](cudaStream_t s, int tail, int last) {
            bg::HeadArgs<T> b = a; b.tail = tail; b.update = 1; b.last = last;
            return launch_generated_head<T>(k, b, blocks, s);
        });
        if (has_tail)
            net->finalize_launches.push_back([a, k, blocks](cudaStream_t s, int, int) {
                bg::HeadArgs<T> b = a; b.tail = 1; b.update = 0; b.last = 0;
                return launch_generated_head<T>(k, b, blocks, s);
            });
        return BG_OK;
    }
    if (nvar > bg::kMaxVars) return fail(BG_ENOSYS, "more than 8 state variables in a linear group");
    const bool has_tail = a.ndeliv || g.reset_kind || g.period > 0 || a.nrec;
    net->item_names.push_back("head[g" + std::to_string(gid) + "]");
    net->step_launches.push_back([a, nvar, blocks](cudaStream_t s, int tail, int last) {
        bg::HeadArgs<T> b = a; b.tail = tail; b.update = 1; b.last = last;
        return launch_head<T>(b, nvar, blocks, s);
    });
    if (has_tail)
        net->finalize_launches.push_back([a, nvar, blocks](cudaStream_t s, int, int) {
            bg::HeadArgs<T> b = a; b.tail = 1; b.update = 0; b.last = 0;
            return launch_head<T>(b, nvar, blocks, s);
        });
    return BG_OK;
}

template <typename T, typename WT>
cudaError_t launch_prop(const bg::PropArgs<T> &a, int mode, int64_t grid, cudaStream_t s) {
    switch (mode) {
    case 5: bg::k_prop_dense<T, WT, 64><<<(unsigned)grid, 64, 0, s>>>(a); break;
    case 0: bg::k_prop_atomic<T, WT, false><<<(unsigned)grid, 256, 0, s>>>(a); break;
    case 1: bg::k_prop_atomic<T, WT, true><<<(unsigned)grid, 256, 0, s>>>(a); break;
    case 2: bg::k_prop_ordered<T, WT, false><<<(unsigned)grid, bg::kOrdThreads, 0, s>>>(a); break;
    case 3: bg::k_prop_ordered<T, WT, true><<<(unsigned)grid, bg::kOrdThreads, 0, s>>>(a); break;
    default: bg::k_prop_dense<T, WT><<<(unsigned)grid, bg::kDenseThreads, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

int sm_count() {
    static int n = 0;
    if (!n) { int dev = 0; cudaGetDevice(&dev); cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev); if (n <= 0) n = 148; }
    return n;
}

template <typename T>
int build_conn(bg_net *net, int cid) {
    HConn &c = net->conns[cid];
    const HGroup &gs = net->groups[c.src];
    HGroup &gt = net->groups[c.tgt];
    bg::PropArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.hist = gs.dHist; a.depth = gs.depth; a.nwords = gs.npad / 32;
    a.delay = c.hetero ? 0 : c.delay; a.so = c.so; a.sn = c.sn; a.to = c.to; a.tn = c.tn;
    a.sv = (T *)gt.dS + (int64_t)c.var * gt.npad + c.to;
    a.ring = (T *)c.dRing; a.md = c.md;
    a.rowptr = c.dRow; a.cols = c.dCols; a.w = c.dW; a.d = c.dD; a.dense = c.dense;
    a.mod = c.mod_var >= 0 ? (const T *)gs.dS + (int64_t)c.mod_var * gs.npad + c.so : nullptr;
    const double avg = c.sn ? (double)c.nnz / (double)c.sn : 0.0;
    c.parts = std::max(1, std::min(32, (int)((avg + 63.0) / 64.0)));
    a.parts = c.parts;
    if (c.stdp >= 0 && net->stdps[c.stdp].fused) {
        HStdp &s = net->stdps[c.stdp];
        a.stdp = 1; a.A_pre = s.dApre; a.A_post = s.dApost; a.Ap = s.Ap;
        a.pre_set = (s.inter == BG_STDP_NEAREST || s.inter == BG_STDP_NEAREST_PRE);
        a.wmin = s.wmin; a.wmax = s.wmax; a.wmode = s.pre_mode; a.wx = s.wx;
    }
    if (c.fused_push) return BG_OK;   // pushed by the source group's head kernel
    int mode; int64_t grid;
    // equal weights sum to the same value in any order; STDP makes them differ
    const bool use_atomic = !c.dense && c.mod_var < 0 && ((c.homogeneous && c.stdp < 0) || !net->deterministic) && !a.stdp;
    if (c.dense) {
        // one thread per target column; blocks of 64 when blocks of 256
        // would leave most SMs idle
        mode = (c.tn + bg::kDenseThreads - 1) / bg::kDenseThreads < sm_count() ? 5 : 4;
        const int th = mode == 5 ? 64 : bg::kDenseThreads;
        grid = (c.tn + th - 1) / th;
    }
    else if (use_atomic) {
        mode = c.hetero ? 1 : 0;
        const int64_t nch = ((c.so + c.sn + 31) / 32 - c.so / 32 + 31) / 32;
        const int64_t warps = std::max<int64_t>(1, nch * c.parts);
        grid = std::min<int64_t>((warps + 7) / 8, (int64_t)sm_count() * 8);
    } else {
        mode = c.hetero ? 3 : 2;
        grid = std::max<int64_t>(1, (c.tn + bg::kOrdTB - 1) / bg::kOrdTB);
    }
    const int wb = c.w_bits;
    a.events = net->dCounters + net->groups.size() + cid;
    static const char *kModeName[] = {"prop_atomic", "prop_ring_atomic", "prop_ordered", "prop_ring_ordered", "prop_dense",
                                      "prop_dense"};
    net->item_names.push_back(std::string(kModeName[mode]) + "[c" + std::to_string(cid) + "]");
    net->step_launches.push_back([a, mode, grid, wb](cudaStream_t s, int, int last) {
        bg::PropArgs<T> b = a; b.last = last;
        return wb == 64 ? launch_prop<T, double>(b, mode, grid, s) : launch_prop<T, float>(b, mode, grid, s);
    });
    return BG_OK;
}

int build_stdp_pre_delayed(bg_net *net, int sid) {
    HStdp &s = net->stdps[sid];
    HConn &c = net->conns[s.cid];
    const HGroup &gs = net->groups[c.src];
    bg::DelayedPreArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.hist = gs.dHist; a.depth = gs.depth; a.nwords = gs.npad / 32; a.delay = s.pre_delay;
    a.so = c.so; a.sn = c.sn; a.tn = c.tn; a.rowptr = c.dRow; a.cols = c.dCols; a.w = c.dW;
    a.A_pre = s.dApre; a.Ap = s.Ap; a.pre_set = (s.inter == BG_STDP_NEAREST || s.inter == BG_STDP_NEAREST_PRE);
    a.H_post = s.dHpost; a.hlen = s.hlen; a.lag = s.dLagPre; a.wmin = s.wmin; a.wmax = s.wmax;
    a.wmode = s.pre_mode; a.wx = s.wx;
    const int64_t nwords = (c.so + c.sn + 31) / 32 - c.so / 32;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((nwords + 255) / 256, (int64_t)sm_count() * 4));
    const int wb = c.w_bits;
    net->item_names.push_back("stdp_pre_delayed[s" + std::to_string(sid) + "]");
    net->step_launches.push_back([a, grid, wb](cudaStream_t st, int, int last) {
        bg::DelayedPreArgs b = a; b.last = last;
        if (wb == 64) bg::k_dstdp_pre<double><<<(unsigned)grid, 256, 0, st>>>(b);
        else bg::k_dstdp_pre<float><<<(unsigned)grid, 256, 0, st>>>(b);
        return cudaGetLastError();
    });
    return BG_OK;
}

int build_stdp_pre(bg_net *net, int sid) {
    HStdp &s = net->stdps[sid];
    if (s.fused) return BG_OK;
    if (s.delayed) return build_stdp_pre_delayed(net, sid);
    HConn &c = net->conns[s.cid];
    const HGroup &gs = net->groups[c.src];
    bg::PropArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.hist = gs.dHist; a.depth = gs.depth; a.nwords = gs.npad / 32; a.delay = s.pre_delay;
    a.so = c.so; a.sn = c.sn; a.to = c.to; a.tn = c.tn; a.rowptr = c.dRow; a.cols = c.dCols; a.w = c.dW; a.dense = c.dense;
    a.stdp = 1; a.A_pre = s.dApre; a.A_post = s.dApost; a.Ap = s.Ap;
    a.pre_set = (s.inter == BG_STDP_NEAREST || s.inter == BG_STDP_NEAREST_PRE); a.wmin = s.wmin; a.wmax = s.wmax;
    a.wmode = s.pre_mode; a.wx = s.wx;
    const int64_t nwords = (c.so + c.sn + 31) / 32 - c.so / 32;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((nwords + 255) / 256, (int64_t)sm_count() * 4));
    const int wb = c.w_bits;
    net->item_names.push_back("stdp_pre[s" + std::to_string(sid) + "]");
    net->step_launches.push_back([a, grid, wb](cudaStream_t st, int, int last) {
        bg::PropArgs<double> b = a; b.last = last;
        if (wb == 64) bg::k_stdp_pre<double><<<(unsigned)grid, 256, 0, st>>>(b);
        else bg::k_stdp_pre<float><<<(unsigned)grid, 256, 0, st>>>(b);
        return cudaGetLastError();
    });
    return BG_OK;
}

int build_stdp_post(bg_net *net, int sid) {
    HStdp &s = net->stdps[sid];
    HConn &c = net->conns[s.cid];
    const HGroup &gt = net->groups[c.tgt];
    bg::PostArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.hist = gt.dHist; a.depth = gt.depth; a.nwords = gt.npad / 32; a.delay = s.post_delay;
    a.to = c.to; a.tn = c.tn; a.sn = c.sn; a.w = c.dW; a.dense = c.dense;
    a.colptr = c.dColptr; a.colk = c.dColk; a.colsrc = c.dColsrc;
    a.A_post = s.dApost; a.A_pre = s.dApre; a.Am = s.Am;
    a.post_set = (s.inter != BG_STDP_ALL);   // 'nearest_pre' writes A_post=+Am (stdp.py:500-502)
    a.wmin = s.wmin; a.wmax = s.wmax; a.wmode = s.post_mode; a.wx = s.wx;
    if (s.delayed) { a.H_pre = s.dHpre; a.hlen = s.hlen; a.lagc = s.dLagPostC; }
    const int wb = c.w_bits;
    if (c.dense) {
        // one pass over the rows applies every column update of the step
        const int64_t bands = (c.sn + bg::kPostRows - 1) / bg::kPostRows;
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(bands, (int64_t)sm_count() * 8));
        net->item_names.push_back("stdp_post_rows[s" + std::to_string(sid) + "]");
        net->step_launches.push_back([a, grid, wb](cudaStream_t st, int, int last) {
            bg::PostArgs b = a; b.last = last;
            if (wb == 64) bg::k_stdp_post_rows<double><<<(unsigned)grid, bg::kPostThreads, 0, st>>>(b);
            else bg::k_stdp_post_rows<float><<<(unsigned)grid, bg::kPostThreads, 0, st>>>(b);
            return cudaGetLastError();
        });
        return BG_OK;
    }
    const int64_t grid = 8;
    net->item_names.push_back("stdp_post[s" + std::to_string(sid) + "]");
    net->step_launches.push_back([a, grid, wb](cudaStream_t st, int, int last) {
        bg::PostArgs b = a; b.last = last;
        if (wb == 64) bg::k_stdp_post<double><<<(unsigned)grid, 256, 0, st>>>(b);
        else bg::k_stdp_post<float><<<(unsigned)grid, 256, 0, st>>>(b);
        return cudaGetLastError();
    });
    return BG_OK;
}

// The generated kernel of a Synapses object with code: the policy struct
// (pre and post bodies over X(slot), SV(var), PRE(k), T) around
// bg::syn_code_body, compiled by NVRTC with the engine's kernel sources.
int compile_syn_code(HSyn &y) {
    if (y.code_kernel) return BG_OK;
    std::string src = "#define BG_GENERATED_MODEL 1\n";
    for (const char *const *p = kNetRtcSource; *p; ++p) src += *p;
    src += "namespace bg {\nstruct SynCode {\n"
           "#define X(s) x_[s]\n#define SV(k) sv_[k][q_]\n#define PRE(k) pre_[k]\n#define T t_\n"
           "    static __device__ __forceinline__ void pre(double *x_, double *const *sv_, int64_t q_, double t_, const double *pre_) {\n"
           "        (void)x_; (void)sv_; (void)q_; (void)t_; (void)pre_;\n" + y.pre_code + "\n    }\n"
           "    static __device__ __forceinline__ void post(double *x_, double *const *sv_, int64_t q_, double t_) {\n"
           "        (void)x_; (void)sv_; (void)q_; (void)t_;\n" + y.post_code + "\n    }\n"
           "#undef X\n#undef SV\n#undef PRE\n#undef T\n};\n}  // namespace bg\n"
           "extern \"C\" __global__ void __launch_bounds__(bg::kSynThreads) bg_syn_code(const bg::SynCodeArgs a) {\n"
           "    bg::syn_code_body<bg::SynCode>(a);\n}\n";
    std::vector<char> cubin;
    std::string log;
    int rc = bg_nvrtc_compile(src, &cubin, &log);
    if (rc) return rc;
    cudaError_t e = cudaLibraryLoadData(&y.code_lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&y.code_kernel, y.code_lib, "bg_syn_code");
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("synaptic code kernel: ") + cudaGetErrorString(e));
    return BG_OK;
}

// The event path's arguments of Synapses object yi.
bg::SynEvArgs syn_ev_args(bg_net *net, int yi) {
    HSyn &y = net->syns[yi];
    const HGroup &gs = net->groups[y.src];
    HGroup &gt = net->groups[y.tgt];
    bg::SynEvArgs e;
    std::memset(&e, 0, sizeof(e));
    e.ctl = net->dCtl; e.hist = gs.dHist; e.depth = gs.depth; e.nwords = gs.npad / 32;
    e.so = y.so; e.sn = y.sn; e.tn = y.tn; e.dmax = y.dmax;
    e.srcptr = y.dSrcPtr; e.sd = y.dSd; e.stgt = y.dStgt; e.sq = y.dSq; e.doff = y.dDoff;
    e.colptr = y.dColptr; e.word = y.dWord;
    e.bin_cnt = y.dBinCnt; e.bin_key = y.dBinKey; e.bin_q = y.dBinQ; e.nbins = y.nbins; e.use_pull = y.dUsePull;
    e.slist = y.dSlist; e.scnt = y.dScnt; e.sdepth = y.sdepth;
    e.term = y.dTerm; e.nsyn = y.nsyn; e.nops = y.nops;
    for (int k = 0; k < y.nops; ++k) {
        int sl = -1;
        for (int q = 0; q < e.nslots; ++q) if (e.slot_var[q] == y.op_var[k]) sl = q;
        if (sl < 0) { sl = e.nslots++; e.slot_var[sl] = y.op_var[k]; }
        e.slot_of[k] = sl; e.sub[k] = y.op_sub[k];
    }
    e.S = (double *)gt.dS; e.npad = gt.npad; e.to = y.to;
    return e;
}

// Event path of the Synapses objects `ids` (consecutive in the schedule,
// targets' variables disjoint): one gather launch over all their (delay,
// history word) items, then one launch over all their bins (which fall back
// to the pull's test for an object whose events overflowed in a step).
int build_syn_events(bg_net *net, const std::vector<int> &ids) {
    bg::SynEvGroup g;
    std::memset(&g, 0, sizeof(g));
    g.nobj = (int)ids.size(); g.ctl = net->dCtl;
    std::string tag;
    for (int k = 0; k < g.nobj; ++k) {
        const HSyn &y = net->syns[ids[k]];
        g.o[k] = syn_ev_args(net, ids[k]);
        const int64_t nw = (y.so + y.sn + 31) / 32 - y.so / 32;
        g.item0[k + 1] = g.item0[k] + nw;
        g.pair0[k + 1] = g.pair0[k] + y.dmax;
        g.bin0[k + 1] = g.bin0[k] + y.nbins;
        tag += (k ? ",y" : "y") + std::to_string(ids[k]);
    }
    // every (object, delay) list split over nparts blocks (about four list
    // blocks per SM in all), then the blocks of this step's history words
    const int npair = g.pair0[g.nobj];
    g.nparts = npair ? std::max(1, sm_count() * 4 / npair) : 1;
    const int64_t ggrid = (int64_t)npair * g.nparts +
                          std::max<int64_t>(1, std::min<int64_t>((g.item0[g.nobj] + 255) / 256, (int64_t)sm_count() * 4));
    if (ggrid >= ((int64_t)1 << 31)) return fail(BG_ENOSYS, "Synapses event path: too many gather blocks");
    const size_t bsmem = (size_t)bg::kSynBinCap * (8 + 4);
    cudaFuncSetAttribute(bg::k_syn_bins, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsmem);
    net->item_names.push_back("syn_gather[" + tag + "]");
    net->step_launches.push_back([g, ggrid](cudaStream_t st, int, int last) {
        bg::SynEvGroup b = g; b.last = last;
        bg::k_syn_gather<<<(unsigned)ggrid, 256, 0, st>>>(b);
        return cudaGetLastError();
    });
    net->item_names.push_back("syn_bins[" + tag + "]");
    net->step_launches.push_back([g, bsmem](cudaStream_t st, int, int last) {
        bg::SynEvGroup b = g; b.last = last;
        bg::k_syn_bins<<<(unsigned)b.bin0[b.nobj], bg::kSynBinThreads, bsmem, st>>>(b);
        return cudaGetLastError();
    });
    return BG_OK;
}

// Whether Synapses objects a and b may apply their events in either order:
// no target variable on overlapping target ranges is written by both.
bool syn_disjoint(const HSyn &a, const HSyn &b) {
    if (a.tgt != b.tgt || a.to >= b.to + b.tn || b.to >= a.to + a.tn) return true;
    for (int u : a.op_var)
        for (int v : b.op_var)
            if (u == v) return false;
    return true;
}

int build_syn_code(bg_net *net, int yi) {
    HSyn &y = net->syns[yi];
    const HGroup &gs = net->groups[y.src];
    HGroup &gt = net->groups[y.tgt];
    int st = compile_syn_code(y);
    if (st) return st;
    bg::SynCodeArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.hist = gs.dHist; a.depth = gs.depth; a.nwords = gs.npad / 32;
    a.thist = gt.dHist; a.tdepth = gt.depth; a.tnwords = gt.npad / 32;
    a.so = y.so; a.to = y.to; a.tn = y.tn; a.colptr = y.dColptr; a.word = y.dWord;
    for (int v = 0; v < y.nsv; ++v) a.sv[v] = y.dSv + (size_t)v * y.nsyn;
    a.nslots = (int)y.slot_var.size();
    for (int k = 0; k < a.nslots; ++k) a.slot_var[k] = y.slot_var[k];
    a.S = (double *)gt.dS; a.npad = gt.npad;
    a.Ssrc = (const double *)gs.dS; a.snpad = gs.npad; a.npre = (int)y.pre_var.size();
    for (int k = 0; k < a.npre; ++k) a.pre_var[k] = y.pre_var[k];
    a.dt = net->dt;
    a.has_post = y.post_code.empty() ? 0 : 1;
    const int64_t ntiles = (y.tn + bg::kSynTile - 1) / bg::kSynTile;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)sm_count() * 8));
    const cudaKernel_t k = y.code_kernel;
    net->item_names.push_back("syn_code[y" + std::to_string(yi) + "]");
    net->step_launches.push_back([a, k, grid](cudaStream_t s, int, int last) {
        bg::SynCodeArgs b = a; b.last = last;
        void *args[] = {(void *)&b};
        return cudaLaunchKernel((const void *)k, dim3(grid), dim3(bg::kSynThreads), args, 0, s);
    });
    return BG_OK;
}

int build_syn(bg_net *net, int yi) {
    HSyn &y = net->syns[yi];
    if (y.coded) return build_syn_code(net, yi);
    const HGroup &gs = net->groups[y.src];
    HGroup &gt = net->groups[y.tgt];
    bg::SynArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.hist = gs.dHist; a.depth = gs.depth; a.nwords = gs.npad / 32;
    a.so = y.so; a.to = y.to; a.tn = y.tn; a.colptr = y.dColptr; a.word = y.dWord; a.term = y.dTerm; a.nsyn = y.nsyn;
    a.nops = y.nops;
    for (int k = 0; k < y.nops; ++k) {
        int sl = -1;
        for (int q = 0; q < a.nslots; ++q) if (a.slot_var[q] == y.op_var[k]) sl = q;
        if (sl < 0) { sl = a.nslots++; a.slot_var[sl] = y.op_var[k]; }
        a.slot_of[k] = sl; a.sub[k] = y.op_sub[k];
    }
    a.S = (double *)gt.dS; a.npad = gt.npad;
    const int64_t ntiles = (y.tn + bg::kSynTile - 1) / bg::kSynTile;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)sm_count() * 8));
    if (y.events) return build_syn_events(net, {yi});
    net->item_names.push_back("syn_deliver[y" + std::to_string(yi) + "]");
    net->step_launches.push_back([a, grid](cudaStream_t st, int, int last) {
        bg::SynArgs b = a; b.last = last;
        bg::k_syn_deliver<<<(unsigned)grid, bg::kSynThreads, 0, st>>>(b);
        return cudaGetLastError();
    });
    return BG_OK;
}

int build_spikemon(bg_net *net, int k) {
    HSpikeMon &m = net->smons[k];
    const HGroup &g = net->groups[m.gid];
    bg::MonArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.hist = g.dHist; a.depth = g.depth; a.nwords = g.npad / 32; a.delay = m.delay;
    a.origin = m.origin; a.n = m.n; a.cnt = m.dCnt; a.cap = m.cap; a.idx = m.dIdx; a.steps = m.dSteps; a.step_base = m.dBase;
    net->item_names.push_back("spikemon[m" + std::to_string(k) + "]");
    net->step_launches.push_back([a](cudaStream_t st, int, int last) {
        bg::MonArgs b = a; b.last = last;
        bg::k_spikemon<<<1, bg::kMonThreads, 0, st>>>(b);
        return cudaGetLastError();
    });
    return BG_OK;
}

int build_decay(bg_net *net, int sid) {
    HStdp &s = net->stdps[sid];
    const HConn &c = net->conns[s.cid];
    bg::DecayArgs a;
    std::memset(&a, 0, sizeof(a));
    if (s.delayed) { a.H_pre = s.dHpre; a.H_post = s.dHpost; a.hlen = s.hlen; }
    a.A_pre = s.dApre; a.npre = c.sn; a.a_pre = s.a_pre; a.c_pre = s.c_pre;
    a.A_post = s.dApost; a.npost = c.tn; a.a_post = s.a_post; a.c_post = s.c_post; a.ctl = net->dCtl; a.last = 0;
    const int64_t grid = std::max<int64_t>(1, (c.sn + c.tn + 255) / 256);
    net->item_names.push_back("stdp_decay[s" + std::to_string(sid) + "]");
    net->step_launches.push_back([a, grid](cudaStream_t st, int, int last) {
        bg::DecayArgs b = a; b.last = last;
        bg::k_stdp_decay<<<(unsigned)grid, 256, 0, st>>>(b);
        return cudaGetLastError();
    });
    return BG_OK;
}

// Host-to-device copy.  Large arrays (the connectivity) go through two
// pinned staging buffers: all host threads copy one chunk in while the DMA
// of the previous chunk runs (a pageable copy is staged by the driver one
// thread at a time).  The buffers live until the end of bg_net_prepare.
constexpr size_t kStageBytes = (size_t)64 << 20;

int upload(bg_net *net, void *dst, const void *src, size_t bytes) {
    if (bytes < 2 * kStageBytes || net->prepared) {
        BG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, net->stream));
        return BG_OK;
    }
    if (!net->stage[0]) {
        for (int b = 0; b < 2; ++b) {
            if (cudaHostAlloc(&net->stage[b], kStageBytes, cudaHostAllocDefault) != cudaSuccess ||
                cudaEventCreateWithFlags(&net->stage_ev[b], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                BG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, net->stream));
                return BG_OK;
            }
        }
        net->stage_used[0] = net->stage_used[1] = false;
    }
    size_t k = 0;
    for (size_t off = 0; off < bytes; off += kStageBytes, ++k) {
        const int b = (int)(k & 1);
        const size_t len = std::min(kStageBytes, bytes - off);
        if (net->stage_used[b]) BG_CUDA(cudaEventSynchronize(net->stage_ev[b]));
        char *stg = (char *)net->stage[b];
        const char *s = (const char *)src + off;
        parallel_for((int64_t)len, [&](int64_t lo, int64_t hi, int) { std::memcpy(stg + lo, s + lo, hi - lo); },
                     (int64_t)4 << 20);
        BG_CUDA(cudaMemcpyAsync((char *)dst + off, stg, len, cudaMemcpyHostToDevice, net->stream));
        BG_CUDA(cudaEventRecord(net->stage_ev[b], net->stream));
        net->stage_used[b] = true;
    }
    return BG_OK;
}

void release_staging(bg_net *net) {
    for (int b = 0; b < 2; ++b) {
        if (net->stage_ev[b]) { cudaEventSynchronize(net->stage_ev[b]); cudaEventDestroy(net->stage_ev[b]); }
        if (net->stage[b]) cudaFreeHost(net->stage[b]);
        net->stage[b] = nullptr; net->stage_ev[b] = nullptr; net->stage_used[b] = false;
    }
}

int upload_state(bg_net *net, HGroup &g, int var, const double *in) {
    if (net->precision == 64) return upload(net, (double *)g.dS + (size_t)var * g.npad, in, g.n * 8);
    std::vector<float> tmp(g.n);
    for (int64_t i = 0; i < g.n; ++i) tmp[i] = (float)in[i];
    int st = upload(net, (float *)g.dS + (size_t)var * g.npad, tmp.data(), g.n * 4);
    if (st) return st;
    BG_CUDA(cudaStreamSynchronize(net->stream));
    return BG_OK;
}

int reset_dynamic(bg_net *net) {
    net->syn_lists_stale = true;
    for (auto &g : net->groups) {
        BG_CUDA(cudaMemsetAsync(g.dHist, 0, (size_t)g.depth * (g.npad / 32) * 4, net->stream));
        if (g.dNext) {
            std::vector<double> m1(g.npad, -1.0);
            BG_CUDA(cudaMemcpyAsync(g.dNext, m1.data(), g.npad * 8, cudaMemcpyHostToDevice, net->stream));
            BG_CUDA(cudaStreamSynchronize(net->stream));
        }
        if (g.dLast) {
            std::vector<int32_t> m(g.npad, -(1 << 30));
            BG_CUDA(cudaMemcpyAsync(g.dLast, m.data(), g.npad * 4, cudaMemcpyHostToDevice, net->stream));
            BG_CUDA(cudaStreamSynchronize(net->stream));
        }
    }
    for (auto &c : net->conns) {
        if (c.dRing) BG_CUDA(cudaMemsetAsync(c.dRing, 0, (size_t)c.md * c.tn * tsize(net), net->stream));
        if (c.dCRing) BG_CUDA(cudaMemsetAsync(c.dCRing, 0, (size_t)c.md * c.tnp * 2, net->stream));
    }
    for (auto &s : net->stdps) {
        const HConn &c = net->conns[s.cid];
        BG_CUDA(cudaMemsetAsync(s.dApre, 0, c.sn * 8, net->stream));
        BG_CUDA(cudaMemsetAsync(s.dApost, 0, c.tn * 8, net->stream));
        if (s.delayed) {
            BG_CUDA(cudaMemsetAsync(s.dHpre, 0, (size_t)s.hlen * c.sn * 8, net->stream));
            BG_CUDA(cudaMemsetAsync(s.dHpost, 0, (size_t)s.hlen * c.tn * 8, net->stream));
        }
    }
    return BG_OK;
}

int check_device_error(bg_net *net) {
    DevCtl h;
    BG_CUDA(cudaMemcpyAsync(&h, net->dCtl, sizeof(h), cudaMemcpyDeviceToHost, net->stream));
    BG_CUDA(cudaStreamSynchronize(net->stream));
    if (h.err) net->failed = true;       // the network's device state is no longer consistent
    if (h.err == BG_DERR_MONITOR_OVERFLOW) return fail(BG_ESTATE, "spike monitor buffer overflow");
    if (h.err == BG_DERR_TIMEOUT) return fail(BG_ETIMEOUT, "inter-block wait timed out at step " + std::to_string(h.err_info));
    if (h.err == BG_DERR_NONFINITE)
        return fail(BG_ENUMERIC, "non-finite state: group " + std::to_string(h.err_info >> 48) + ", variable " +
                    std::to_string((h.err_info >> 40) & 0xff) + ", neuron " + std::to_string(h.err_info & 0xffffffffffll));
    if (h.err == BG_DERR_RANGE) return fail(BG_EINVAL, "device range check failed (entry " + std::to_string(h.err_info) + ")");
    if (h.err) return fail(BG_ESTATE, "device error " + std::to_string(h.err));
    return BG_OK;
}

// NaN/inf in the first n entries of each of the nvar rows (stride npad) of a
// group's state: raises BG_DERR_NONFINITE with (group, variable, neuron).
template <typename T>
__global__ void k_check_finite(const T *S, int64_t n, int64_t npad, int nvar, int gid, DevCtl *ctl) {
    const int64_t total = n * nvar;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t var = q / n, i = q - var * n;
        const T x = S[var * npad + i];
        if (!isfinite(x)) bg_raise(ctl, BG_DERR_NONFINITE, ((long long)gid << 48) | ((long long)var << 40) | i);
    }
}

int check_finite_states(bg_net *n) {
    for (size_t gi = 0; gi < n->groups.size(); ++gi) {
        const HGroup &g = n->groups[gi];
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((g.n * g.nvar + 255) / 256, 1184));
        if (n->precision == 64) k_check_finite<double><<<grid, 256, 0, n->stream>>>((const double *)g.dS, g.n, g.npad, g.nvar, (int)gi, n->dCtl);
        else k_check_finite<float><<<grid, 256, 0, n->stream>>>((const float *)g.dS, g.n, g.npad, g.nvar, (int)gi, n->dCtl);
        BG_CUDA(cudaGetLastError());
    }
    return check_device_error(n);
}

// Copy monitor records of the finished chunk to host memory.
// `tail_done_upto`: last step whose 'end' slot has run.
// Move one spike monitor's device records (steps relative to
// chunk_base_cs) to host memory and empty its buffer.
int drain_spikemon(bg_net *net, HSpikeMon &m, long long chunk_base_cs) {
    long long cnt = 0;
    BG_CUDA(cudaMemcpy(&cnt, m.dCnt, 8, cudaMemcpyDeviceToHost));
    if (cnt > m.cap) return fail(BG_ESTATE, "spike monitor buffer overflow");
    if (cnt > 0) {
        std::vector<int32_t> idx(cnt), st(cnt);
        BG_CUDA(cudaMemcpy(idx.data(), m.dIdx, cnt * 4, cudaMemcpyDeviceToHost));
        BG_CUDA(cudaMemcpy(st.data(), m.dSteps, cnt * 4, cudaMemcpyDeviceToHost));
        for (long long k = 0; k < cnt; ++k) { m.idx.push_back(idx[k]); m.steps.push_back(chunk_base_cs + st[k]); }
        long long z = 0;
        BG_CUDA(cudaMemcpy(m.dCnt, &z, 8, cudaMemcpyHostToDevice));
    }
    return BG_OK;
}

int drain(bg_net *net, long long chunk_base_cs, long long tail_done_upto, long long off) {
    BG_CUDA(cudaStreamSynchronize(net->stream));
    for (auto &m : net->smons) {
        int st = drain_spikemon(net, m, chunk_base_cs);
        if (st) return st;
    }
    for (auto &m : net->stmons) {
        // records exist for ps in [start, tail_done_upto] with (ps-start) % timestep == 0
        long long total = tail_done_upto < m.start ? 0 : (tail_done_upto - m.start) / m.timestep + 1;
        long long fresh = total - m.rows_done;
        if (fresh <= 0) continue;
        if (fresh > m.cap_rows) return fail(BG_ESTATE, "state monitor buffer overflow");
        const size_t w = m.idx.size();
        const size_t ts = tsize(net);
        std::vector<char> buf(fresh * w * ts);
        if (buf.size()) BG_CUDA(cudaMemcpy(buf.data(), m.dBuf, buf.size(), cudaMemcpyDeviceToHost));
        for (long long r = 0; r < fresh; ++r) {
            for (size_t j = 0; j < w; ++j)
                m.vals.push_back(ts == 8 ? ((double *)buf.data())[r * w + j] : (double)((float *)buf.data())[r * w + j]);
            const long long ps = m.start + (m.rows_done + r) * m.timestep;
            m.steps.push_back(ps + off);   // clock step of the record
        }
        m.rows_done = total;
        BG_CUDA(cudaMemcpy(m.dRowBase, &m.rows_done, 8, cudaMemcpyHostToDevice));
    }
    return BG_OK;
}

}  // namespace

namespace {

// Shapes of the persistent kernel: threads per block x neurons per thread,
// 512 x 2 or 256 x 4, both 1024-neuron blocks.
constexpr int persist_npt(int th) { return th == 256 ? 4 : 2; }

template <typename T, int NV, int TH>
cudaError_t launch_persist_nv(bg::PersistArgs<T> a, bool diag, int64_t blocks, cudaStream_t s) {
    void *args[] = {(void *)&a};
    const void *k = diag ? (const void *)bg::k_persist<T, NV, TH, persist_npt(TH), true>
                         : (const void *)bg::k_persist<T, NV, TH, persist_npt(TH), false>;
    return cudaLaunchCooperativeKernel(k, dim3((unsigned)blocks), dim3(TH), args, 0, s);
}

template <typename T, int TH>
cudaError_t launch_persist_th(bg::PersistArgs<T> a, int nvar, bool diag, int64_t blocks, cudaStream_t s) {
    switch (nvar) {
    case 1: return launch_persist_nv<T, 1, TH>(a, diag, blocks, s);
    case 2: return launch_persist_nv<T, 2, TH>(a, diag, blocks, s);
    case 3: return launch_persist_nv<T, 3, TH>(a, diag, blocks, s);
    default: return launch_persist_nv<T, 4, TH>(a, diag, blocks, s);
    }
}

// Co-resident blocks of the persistent kernel of one shape on the device
// (the DIAG instance has the same limits or fewer registers).
template <typename T, int TH>
int64_t persist_slots(int nvar) {
    constexpr int NPT = persist_npt(TH);
    int per_sm = 0;
    cudaError_t e;
    switch (nvar) {
    case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bg::k_persist<T, 1, TH, NPT, false>, TH, 0); break;
    case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bg::k_persist<T, 2, TH, NPT, false>, TH, 0); break;
    case 3: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bg::k_persist<T, 3, TH, NPT, false>, TH, 0); break;
    default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bg::k_persist<T, 4, TH, NPT, false>, TH, 0); break;
    }
    if (e != cudaSuccess) { cudaGetLastError(); return 0; }
    return (int64_t)per_sm * sm_count();
}

// Threads per block of the persistent kernel: 512 x 2 (32 warps per SM at
// two blocks per SM) hides more of each step's dependent latencies than
// 256 x 4; both fit the same networks.  0 when no shape fits co-resident.
template <typename T>
int persist_threads(int64_t n, int nvar, int forced) {
    auto blocks = [n](int th) { return (n + (int64_t)th * persist_npt(th) - 1) / ((int64_t)th * persist_npt(th)); };
    auto fits = [&](int th) {
        return th == 256 ? blocks(256) <= persist_slots<T, 256>(nvar) : blocks(512) <= persist_slots<T, 512>(nvar);
    };
    if (forced) return fits(forced) ? forced : 0;
    if (fits(512)) return 512;
    if (fits(256)) return 256;
    return 0;
}

// The persistent path applies to one linear group (at most 4 variables, no
// refractoriness, no Poisson/generator input) whose every connection is a
// shared-weight DelayConnection or zero-delay Connection from the group onto
// itself, with undelayed spike monitors, StateMonitors and no plasticity --
// the CUBA benchmark topology.
// Steps per persistent launch when spike monitors record: the spike words of
// a launch are converted to records after it (32 KB per step at 262144
// neurons), in step ranges that fit each monitor's record buffer.
constexpr int64_t kPersistMonSteps = bg::kMonWordsThreads;

// Largest in-degree of a connection, counted on the device from its uploaded columns.
int max_indegree(bg_net *n, const HConn &c, int64_t *kmax) {
    *kmax = 0;
    if (c.nnz <= 0) return BG_OK;
    int32_t *dDeg = nullptr;
    BG_CUDA(cudaMalloc(&dDeg, c.tn * 4));
    std::vector<int32_t> indeg(c.tn);
    cudaError_t e = cudaMemsetAsync(dDeg, 0, c.tn * 4, n->stream);
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((c.nnz + 255) / 256, (int64_t)sm_count() * 8));
    if (e == cudaSuccess) { k_indegree<<<grid, 256, 0, n->stream>>>(c.dCols, c.nnz, dDeg); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaMemcpyAsync(indeg.data(), dDeg, c.tn * 4, cudaMemcpyDeviceToHost, n->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(n->stream);
    cudaFree(dDeg);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("in-degree: ") + cudaGetErrorString(e));
    for (int32_t k : indeg) *kmax = std::max<int64_t>(*kmax, k);
    return BG_OK;
}

// A zero-delay Connection of the group onto itself with one shared weight
// and nothing else on it: the persistent kernel counts its events per target
// in a ring and adds the weight once per event at delivery.
bool persist_direct(const HConn &c) {
    return !c.hetero && !c.dense && c.delay == 0 && c.mod_var < 0 && c.stdp < 0 && c.homogeneous && c.src == 0 &&
           c.tgt == 0 && c.tn <= (1 << 24);
}

template <typename T>
int build_persist(bg_net *net) {
    net->persist = nullptr;
    if (net->groups.size() != 1 || !net->stdps.empty() || !net->syns.empty()) return BG_OK;
    for (const HSpikeMon &m : net->smons)
        if (m.gid != 0 || m.delay != 0) return BG_OK;
    if ((int)net->stmons.size() > bg::kMaxRec) return BG_OK;

    const HGroup &g = net->groups[0];
    if (!g.linear || g.nvar < 1 || g.nvar > 4 || g.refr || g.period > 0) return BG_OK;
    if (g.generated() || g.emp_steps > 0 || !g.setters.empty()) return BG_OK;
    if (g.thr_kind != BG_THR_CONST && g.thr_kind != BG_THR_VAR && g.thr_kind != BG_THR_NONE) return BG_OK;
    if (net->conns.empty() || (int)net->conns.size() > bg::kPersistMaxPush) return BG_OK;
    int min_d = 255, ndirect = 0;
    for (const HConn &c : net->conns) {
        if (persist_direct(c)) { ++ndirect; min_d = 0; continue; }
        if (!c.fused_push || c.src != 0 || c.tgt != 0) return BG_OK;
        for (uint8_t d : c.d) min_d = std::min<int>(min_d, d);
    }
    if (ndirect + (int)g.delivs.size() > bg::kPersistMaxDeliv) return BG_OK;
    {
        int dev = 0, coop = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return BG_OK;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (!coop) return BG_OK;
    }
    const int th = persist_threads<T>(g.n, g.nvar, net->persist_th);
    cudaGetLastError();
    if (!th) return BG_OK;
    const int64_t bn = (int64_t)th * persist_npt(th), blocks = (g.n + bn - 1) / bn;
    net->persist_used = 0;
    // a block's synapse rows must span fewer than 2^32 entries (32-bit
    // offsets in shared memory)
    for (const HConn &c : net->conns)
        for (int64_t b = 0; b < blocks; ++b) {
            const int64_t lo = std::min(std::max(b * bn - c.so, (int64_t)0), c.sn);
            const int64_t hi = std::min(std::max((b + 1) * bn - c.so, (int64_t)0), c.sn);
            if (c.rowptr[hi] - c.rowptr[lo] >= ((int64_t)1 << 32)) return BG_OK;
        }
    if (net->alloc(&net->dArrived, 64) != cudaSuccess) return fail(BG_ENOMEM, "arrival counter");
    bg::PersistArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.S = (T *)g.dS; a.n = g.n; a.npad = g.npad; a.useC = g.useC;
    for (int j = 0; j < g.nvar; ++j) {
        for (int k = 0; k < g.nvar; ++k) a.A[j * g.nvar + k] = (T)g.A[j * g.nvar + k];
        a.C[j] = g.useC ? (T)g.C[j] : T(0);
    }
    bg::set_linear_masks(a, g.nvar);
    a.thr_kind = g.thr_kind; a.thr_var = g.thr_var; a.thr_var2 = g.thr_var2; a.thr_val = (T)g.thr_val;
    a.reset_kind = g.reset_kind; a.reset_var = g.reset_var; a.reset_var2 = g.reset_var2; a.reset_val = (T)g.reset_val;
    a.hist = g.dHist; a.depth = g.depth; a.nwords = g.npad / 32;
    // zero-delay Connections: a count ring of 3 rows (a push of step t lands
    // in row t mod 3, delivered at the top of step t+1; blocks are at most
    // one step apart) and the table {0, w}
    for (HConn &c : net->conns) {
        if (!persist_direct(c) || c.dDirRing) continue;
        int64_t kmax = 0;
        int st = max_indegree(net, c, &kmax);
        if (st) return st;
        if (kmax >= 65535) return BG_OK;                     // 16-bit counts
        c.dir_md = 3;
        c.tnp = (c.tn + 1) & ~1ll;
        if (net->alloc(&c.dDirRing, (size_t)c.dir_md * c.tnp * 2) != cudaSuccess ||
            net->alloc(&c.dDirTable, 2 * sizeof(T)) != cudaSuccess)
            return fail(BG_ENOMEM, "count ring");
        BG_CUDA(cudaMemsetAsync(c.dDirRing, 0, (size_t)c.dir_md * c.tnp * 2, net->stream));
        const double w0 = c.w_bits == 64 ? *(const double *)c.w.data() : (double)*(const float *)c.w.data();
        const T tab[2] = {T(0), (T)w0};
        st = upload(net, c.dDirTable, tab, sizeof(tab));
        if (st) return st;
        BG_CUDA(cudaStreamSynchronize(net->stream));
    }
    // deliveries in the order of the stepped path: the zero-delay
    // Connections (propagated in the step's connection slot), then the
    // DelayConnections' due rows
    a.ndeliv = 0;
    for (const HConn &c : net->conns) {
        if (!persist_direct(c)) continue;
        a.direct_mask |= 1u << a.ndeliv;
        bg::Deliv<T> &dv = a.deliv[a.ndeliv++];
        dv.ring = nullptr; dv.tn = c.tn; dv.to = c.to; dv.md = c.dir_md; dv.var = c.var;
        dv.cring = c.dDirRing; dv.tnp = c.tnp; dv.table = (const T *)c.dDirTable; dv.tablen = 2;
    }
    for (int k = 0; k < (int)g.delivs.size(); ++k) {
        const HConn &c = net->conns[g.delivs[k]];
        bg::Deliv<T> &dv = a.deliv[a.ndeliv++];
        dv.ring = (T *)c.dRing; dv.tn = c.tn; dv.to = c.to; dv.md = c.md; dv.var = c.var;
        dv.cring = c.dCRing; dv.tnp = c.tnp; dv.table = (const T *)c.dTable; dv.tablen = c.tablen;
    }
    a.npush = (int)net->conns.size();
    for (int p = 0; p < a.npush; ++p) {
        HConn &c = net->conns[p];
        bg::Push<T> &q = a.push[p];
        const bool direct = persist_direct(c);
        q.ring = (T *)c.dRing; q.md = direct ? c.dir_md : c.md; q.so = c.so; q.sn = c.sn; q.tn = c.tn;
        q.rowptr = c.dRow; q.cols = c.dCols; q.w = c.dW; q.w_bits = c.w_bits; q.d = c.dD;
        q.events = net->dCounters + net->groups.size() + p;
        q.cring = direct ? c.dDirRing : c.dCRing; q.tnp = c.tnp;
        // one word per synapse for the scatter: a single load (and a single
        // stream of cache lines and pages) per synapse instead of two
        if (q.cring && c.tn <= (1 << 24) && c.nnz > 0 && c.dCols && (c.dD || direct)) {
            if (!c.dPacked) {
                if (net->alloc(&c.dPacked, c.nnz * 4) != cudaSuccess) return fail(BG_ENOMEM, "packed synapses");
                const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((c.nnz + 255) / 256, (int64_t)sm_count() * 8));
                k_pack_synapses<<<grid, 256, 0, net->stream>>>(c.dCols, c.dD, c.nnz, c.dPacked);
                BG_CUDA(cudaGetLastError());
            }
            q.packed = c.dPacked;
        }
    }
    a.spikes = net->dCounters;
    a.arrived = net->dArrived;
    a.lag = min_d >= 1 ? 2 : 1;
    a.spin_limit = net->spin_limit;
    a.hold_block = net->hold_block;
    // StateMonitors: the recorded neurons of each persistent block (the
    // monitor's sorted indices split at multiples of bn)
    a.nrec = (int)net->stmons.size();
    for (int k = 0; k < a.nrec; ++k) {
        HStateMon &m = net->stmons[k];
        if (!m.dBlkP) {
            std::vector<int32_t> lo(blocks + 1, 0);
            const int64_t w = (int64_t)m.sorted.size();
            for (int64_t b = 0, e = 0; b <= blocks; ++b) {
                while (e < w && m.sorted[e] < b * bn) ++e;
                lo[b] = (int32_t)e;
            }
            if (net->alloc(&m.dBlkP, (blocks + 1) * 4) != cudaSuccess) return fail(BG_ENOMEM, "state monitor");
            BG_CUDA(cudaMemcpy(m.dBlkP, lo.data(), (blocks + 1) * 4, cudaMemcpyHostToDevice));
        }
        bg::RecDev &r = a.rec[k];
        r.var = m.var; r.nidx = (int)m.idx.size(); r.idx = m.dIdx; r.pos = m.dPos; r.blk_lo = m.dBlkP;
        r.buf = m.dBuf; r.row_base = m.dRowBase; r.timestep = m.timestep; r.start = m.start;
    }
    if (!net->smons.empty()) {
        // spike monitors: the kernel writes each step's spike words; the
        // monitor kernels turn a launch's words into records (one launch per
        // chunk of at most chunk_steps steps)
        a.mon_stride = g.npad / 32;
        if (!net->dMonWords &&
            (net->alloc(&net->dMonWords, (size_t)kPersistMonSteps * a.mon_stride * 4) != cudaSuccess ||
             net->alloc(&net->dMonOff, (size_t)kPersistMonSteps * 8) != cudaSuccess))
            return fail(BG_ENOMEM, "spike words");
        a.mon_words = net->dMonWords;
    }
    const int nvar = g.nvar;
    unsigned int *arr = net->dArrived;
    // first row full, other rows diagonal, C at most in its first entry
    // (read from the masks of the coefficients as the kernel's type holds them)
    bool diag = (a.cnz & ~1u) == 0;
    for (int j = 0; j < g.nvar; ++j)
        for (int k = 0; k < g.nvar; ++k)
            if ((((a.anz >> (j * g.nvar + k)) & 1ull) != 0) != (j == 0 || j == k)) diag = false;
    net->persist_used = th;
    net->persist = [a, blocks, nvar, arr, th, diag](cudaStream_t s, int nsteps) {
        cudaError_t e = cudaMemsetAsync(arr, 0, 64, s);
        if (e != cudaSuccess) return e;
        bg::PersistArgs<T> b = a; b.nsteps = nsteps;
        return th == 256 ? launch_persist_th<T, 256>(b, nvar, diag, blocks, s)
                         : launch_persist_th<T, 512>(b, nvar, diag, blocks, s);
    };
    return BG_OK;
}

// The persistent kernel's copy of a Synapses object's terms in by-source
// order (its one statement), from the column-order terms on the device.
int refresh_term_src(bg_net *net, const HSyn &y) {
    if (!y.dTermSrc || y.nsyn == 0) return BG_OK;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((y.nsyn + 255) / 256, (int64_t)sm_count() * 8));
    bg::k_syn_term_src<<<grid, 256, 0, net->stream>>>(y.dSq, y.dTerm, y.nsyn, y.dTermSrc);
    BG_CUDA(cudaGetLastError());
    BG_CUDA(cudaStreamSynchronize(net->stream));
    return BG_OK;
}

// The persistent kernel of CUBA through Synapses (bg_synpersist.cuh): one
// linear FP64 group whose event-path Synapses (static variables, additive
// statements) all connect it to itself, bins aligned with the kernel's
// 1024-neuron blocks, every block co-resident.  Otherwise the stepped path.
// Whether the network has the shape of the persistent kernel for Synapses
// (device limits aside): one linear FP64 group, Synapses only, each with one
// statement, onto the group itself, one target range starting at a bin
// boundary; monitors of that group.
bool syn_persist_shape(const bg_net *net) {
    if (!net->allow_persist) return false;
    if (net->groups.size() != 1 || !net->conns.empty() || !net->stdps.empty() || net->syns.empty()) return false;
    if (net->precision != 64 || (int)net->syns.size() > bg::kSynEvMerge) return false;
    for (const HSyn &y : net->syns) {
        if (y.coded || y.src != 0 || y.tgt != 0 || y.to % bg::kSynBin != 0) return false;
        // one statement; one target range for all (the bins are shared, the
        // key holds target * 4 + object below 2^24); sources below 2^24
        if (y.nops != 1 || y.to != net->syns[0].to || y.tn != net->syns[0].tn) return false;
        if (y.tn > ((int64_t)1 << 22) || y.sn >= ((int64_t)1 << 24)) return false;
    }
    for (const HSpikeMon &m : net->smons)
        if (m.gid != 0 || m.delay != 0) return false;
    if ((int)net->stmons.size() > bg::kMaxRec) return false;
    const HGroup &g = net->groups[0];
    if (!g.linear || g.nvar < 1 || g.nvar > 4 || g.refr || g.period > 0) return false;
    if (g.generated() || g.emp_steps > 0 || !g.setters.empty()) return false;
    return g.thr_kind == BG_THR_CONST || g.thr_kind == BG_THR_VAR || g.thr_kind == BG_THR_NONE;
}

int build_syn_persist(bg_net *net) {
    net->persist = nullptr;
    if (!syn_persist_shape(net)) return BG_OK;
    for (const HSyn &y : net->syns)
        if (!y.events || !y.dScnt) return BG_OK;
    const HGroup &g = net->groups[0];
    {
        int dev = 0, coop = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return BG_OK;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (!coop) return BG_OK;
    }
    const int64_t blocks = (g.n + bg::kSPBn - 1) / bg::kSPBn;
    const size_t smem = (size_t)bg::kSynBinCap * (8 + 8);
    const void *kern[4][2] = {{(const void *)bg::k_syn_persist<1, false>, (const void *)bg::k_syn_persist<1, true>},
                              {(const void *)bg::k_syn_persist<2, false>, (const void *)bg::k_syn_persist<2, true>},
                              {(const void *)bg::k_syn_persist<3, false>, (const void *)bg::k_syn_persist<3, true>},
                              {(const void *)bg::k_syn_persist<4, false>, (const void *)bg::k_syn_persist<4, true>}};
    int64_t slots = -1;
    for (int d = 0; d < 2; ++d) {
        const void *k = kern[g.nvar - 1][d];
        int per_sm = 0;
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, bg::kSPTh, smem) != cudaSuccess) {
            cudaGetLastError();
            return BG_OK;
        }
        const int64_t sl = (int64_t)per_sm * sm_count();
        slots = slots < 0 ? sl : std::min(slots, sl);
    }
    if (blocks > slots) return BG_OK;
    if (!net->dArrived && net->alloc(&net->dArrived, 64) != cudaSuccess) return fail(BG_ENOMEM, "arrival counter");
    if (!net->dUsePull3) {
        if (net->alloc(&net->dUsePull3, 16) != cudaSuccess) return fail(BG_ENOMEM, "overflow flags");
        BG_CUDA(cudaMemsetAsync(net->dUsePull3, 0, 16, net->stream));
    }
    bg::SynPersistArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = net->dCtl; a.S = (double *)g.dS; a.n = g.n; a.npad = g.npad;
    for (int j = 0; j < g.nvar; ++j) {
        for (int k = 0; k < g.nvar; ++k) {
            a.A[j * g.nvar + k] = g.A[j * g.nvar + k];
            if (a.A[j * g.nvar + k] != 0) a.anz |= 1ull << (j * g.nvar + k);
        }
        a.C[j] = g.useC ? g.C[j] : 0.0;
        if (a.C[j] != 0) a.cnz |= 1u << j;
    }
    a.thr_kind = g.thr_kind; a.thr_var = g.thr_var; a.thr_var2 = g.thr_var2; a.thr_val = g.thr_val;
    a.reset_kind = g.reset_kind; a.reset_var = g.reset_var; a.reset_var2 = g.reset_var2; a.reset_val = g.reset_val;
    a.hist = g.dHist; a.depth = g.depth; a.nwords = g.npad / 32;
    a.nobj = (int)net->syns.size();
    const HSyn &y0 = net->syns[0];
    a.nbins = y0.nbins; a.blk0 = (int)(y0.to / bg::kSynBin); a.tn = y0.tn;
    if (!net->dPBinCnt) {
        if (net->alloc(&net->dPBinCnt, (size_t)2 * a.nbins * 4) != cudaSuccess ||
            net->alloc(&net->dPBinKey, (size_t)2 * a.nbins * bg::kSynBinCap * 8) != cudaSuccess ||
            net->alloc(&net->dPBinT, (size_t)2 * a.nbins * bg::kSynBinCap * 8) != cudaSuccess)
            return fail(BG_ENOMEM, "synapse event bins");
        BG_CUDA(cudaMemsetAsync(net->dPBinCnt, 0, (size_t)2 * a.nbins * 4, net->stream));
    }
    a.bin_cnt = net->dPBinCnt; a.bin_key = net->dPBinKey; a.bin_t = net->dPBinT;
    for (int k = 0; k < a.nobj; ++k) {
        HSyn &y = net->syns[k];
        if (!y.dTermSrc) {
            if (net->alloc(&y.dTermSrc, (size_t)std::max<int64_t>(1, y.nsyn) * 8) != cudaSuccess)
                return fail(BG_ENOMEM, "synapse terms by source");
            int st = refresh_term_src(net, y);
            if (st) return st;
        }
        bg::SynPersistObj &o = a.o[k];
        o.e = syn_ev_args(net, k);
        o.term_src = y.dTermSrc;
        o.var = y.op_var[0]; o.sub = y.op_sub[0];
        a.pair0[k + 1] = a.pair0[k] + y.dmax;
    }
    const int npair = a.pair0[a.nobj];
    a.nparts = npair ? std::max<int>(1, (int)(blocks / npair)) : 1;
    a.use_pull = net->dUsePull3;
    a.spikes = net->dCounters;
    a.arrived = net->dArrived;
    a.spin_limit = net->spin_limit;
    a.hold_block = net->hold_block;
    a.nrec = (int)net->stmons.size();
    for (int k = 0; k < a.nrec; ++k) {
        HStateMon &m = net->stmons[k];
        if (!m.dBlkP) {
            std::vector<int32_t> lo(blocks + 1, 0);
            const int64_t w = (int64_t)m.sorted.size();
            for (int64_t b = 0, e = 0; b <= blocks; ++b) {
                while (e < w && m.sorted[e] < b * bg::kSPBn) ++e;
                lo[b] = (int32_t)e;
            }
            if (net->alloc(&m.dBlkP, (blocks + 1) * 4) != cudaSuccess) return fail(BG_ENOMEM, "state monitor");
            BG_CUDA(cudaMemcpy(m.dBlkP, lo.data(), (blocks + 1) * 4, cudaMemcpyHostToDevice));
        }
        bg::RecDev &r = a.rec[k];
        r.var = m.var; r.nidx = (int)m.idx.size(); r.idx = m.dIdx; r.pos = m.dPos; r.blk_lo = m.dBlkP;
        r.buf = m.dBuf; r.row_base = m.dRowBase; r.timestep = m.timestep; r.start = m.start;
    }
    if (!net->smons.empty()) {
        a.mon_stride = g.npad / 32;
        if (!net->dMonWords &&
            (net->alloc(&net->dMonWords, (size_t)kPersistMonSteps * a.mon_stride * 4) != cudaSuccess ||
             net->alloc(&net->dMonOff, (size_t)kPersistMonSteps * 8) != cudaSuccess))
            return fail(BG_ENOMEM, "spike words");
        a.mon_words = net->dMonWords;
    }
    bool diag = (a.cnz & ~1u) == 0;
    for (int j = 0; j < g.nvar; ++j)
        for (int k = 0; k < g.nvar; ++k)
            if ((((a.anz >> (j * g.nvar + k)) & 1ull) != 0) != (j == 0 || j == k)) diag = false;
    const void *k = kern[g.nvar - 1][diag ? 1 : 0];
    unsigned int *arr = net->dArrived;
    int *flags = net->dUsePull3;
    net->persist_used = bg::kSPTh;
    net->persist = [a, blocks, k, smem, arr, flags](cudaStream_t s, int nsteps) {
        cudaError_t e = cudaMemsetAsync(arr, 0, 64, s);
        if (e != cudaSuccess) return e;
        e = cudaMemsetAsync(flags, 0, 16, s);
        if (e != cudaSuccess) return e;
        bg::SynPersistArgs b = a; b.nsteps = nsteps;
        void *args[] = {(void *)&b};
        return cudaLaunchCooperativeKernel(k, dim3((unsigned)blocks), dim3(bg::kSPTh), args, smem, s);
    };
    return BG_OK;
}

// Runs nsteps with the persistent kernel (one launch) and advances the step
// counter on the host and device.
int run_persist(bg_net *n, int64_t nsteps) {
    cudaError_t e = n->persist(n->stream, (int)nsteps);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("persistent launch: ") + cudaGetErrorString(e));
    n->launches += 1;
    n->nstep += nsteps;
    long long ns = n->nstep;
    BG_CUDA(cudaMemcpyAsync(&n->dCtl->nstep, &ns, 8, cudaMemcpyHostToDevice, n->stream));
    BG_CUDA(cudaStreamSynchronize(n->stream));
    return BG_OK;
}

}  // namespace

int bg_internal_fail(int code, const char *msg) { return fail(code, msg); }

// ============================================================== C ABI
extern "C" {

int bg_version(void) { return 1; }

int bg_last_error(char *buf, int64_t len) {
    if (!buf || len <= 0) return BG_EINVAL;
    std::strncpy(buf, g_err.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
    return BG_OK;
}

int bg_net_create(int device, int precision, int deterministic, double dt, bg_net **out) {
    if (!out || !(dt > 0)) return fail(BG_EINVAL, "bg_net_create: bad dt or out");
    if (precision != 64 && precision != 32) return fail(BG_EINVAL, "precision must be 64 or 32");
    int ndev = 0;
    BG_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(BG_EINVAL, "no such CUDA device");
    BG_CUDA(cudaSetDevice(device));
    bg_net *n = new bg_net();
    n->device = device; n->precision = precision; n->deterministic = deterministic; n->dt = dt;
    cudaError_t e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete n; return fail(BG_ECUDA, cudaGetErrorString(e)); }
    if (n->alloc(&n->dCtl, sizeof(DevCtl)) != cudaSuccess) { delete n; return fail(BG_ENOMEM, "ctl"); }
    cudaMemset(n->dCtl, 0, sizeof(DevCtl));
    cudaEventCreate(&n->ev0); cudaEventCreate(&n->ev1);
    *out = n;
    return BG_OK;
}

int bg_net_destroy(bg_net *n) {
    if (!n) return BG_OK;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    release_staging(n);
    if (n->gexec) cudaGraphExecDestroy(n->gexec);
    for (auto &g : n->groups)
        if (g.gen_lib) cudaLibraryUnload(g.gen_lib);
    for (void *p : n->allocs) cudaFree(p);
    if (n->ev0) cudaEventDestroy(n->ev0);
    if (n->ev1) cudaEventDestroy(n->ev1);
    if (n->ev_fork) cudaEventDestroy(n->ev_fork);
    if (n->ev_join) cudaEventDestroy(n->ev_join);
    if (n->side) cudaStreamDestroy(n->side);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
    return BG_OK;
}

int bg_group_add(bg_net *n, int64_t N, int nvar, const double *S0, int32_t *gid) {
    if (!n || N < 0 || nvar < 0 || (N > 0 && nvar > 0 && !S0) || !gid) return fail(BG_EINVAL, "bg_group_add");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    if (nvar > bg::kMaxVars) return fail(BG_ENOSYS, "at most 8 state variables per group");
    HGroup g; g.n = N; g.nvar = nvar;
    g.npad = std::max<int64_t>(bg::kBlockNeurons, (N + bg::kBlockNeurons - 1) / bg::kBlockNeurons * bg::kBlockNeurons);
    g.S0.assign(S0, S0 + (size_t)N * nvar);
    n->groups.push_back(std::move(g));
    *gid = (int32_t)n->groups.size() - 1;
    return BG_OK;
}

int bg_group_set_linear(bg_net *n, int32_t gid, const double *A, const double *C) {
    if (!gid_ok(n, gid) || !A) return fail(BG_EINVAL, "bg_group_set_linear");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HGroup &g = n->groups[gid];
    g.linear = true; g.A.assign(A, A + g.nvar * g.nvar);
    g.useC = C != nullptr; if (C) g.C.assign(C, C + g.nvar);
    return BG_OK;
}

int bg_group_set_timed_array(bg_net *n, int32_t gid, int var, int64_t origin, int64_t count, const double *values,
                             int64_t nrows, int64_t ncols, int mode, double t_init, double adt, int64_t first_step,
                             const int64_t *bp) {
    if (!gid_ok(n, gid) || !values) return fail(BG_EINVAL, "bg_group_set_timed_array");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HGroup &g = n->groups[gid];
    if (var < 0 || var >= g.nvar) return fail(BG_EINVAL, "timed array: variable out of range");
    if (origin < 0 || count < 1 || origin + count > g.n) return fail(BG_EINVAL, "timed array: neuron range");
    if (nrows < 1 || (ncols != 1 && ncols != count)) return fail(BG_EINVAL, "timed array: shape is (T,) or (T, count)");
    if (mode != 0 && mode != 1) return fail(BG_EINVAL, "timed array: mode 0 (clock) or 1 (times)");
    if (mode == 0 && !(adt > 0) ) return fail(BG_EINVAL, "timed array: dt must be positive");
    if (mode == 1 && nrows > 1 && !bp) return fail(BG_EINVAL, "timed array: breakpoints missing");
    if ((int)g.setters.size() >= bg::kMaxSet) return fail(BG_ENOSYS, "more than 4 TimedArraySetters on one group");
    HGroup::Setter h;
    h.var = var; h.mode = mode; h.origin = origin; h.count = count; h.nrows = nrows; h.ncols = ncols;
    h.t_init = t_init; h.adt = adt; h.first = first_step;
    h.vals.assign(values, values + nrows * ncols);
    if (mode == 1 && nrows > 1) {
        h.bp.assign(bp, bp + (nrows - 1));
        for (size_t k = 1; k < h.bp.size(); ++k)
            if (h.bp[k] < h.bp[k - 1]) return fail(BG_EINVAL, "timed array: breakpoints must ascend");
    }
    g.setters.push_back(std::move(h));
    return BG_OK;
}

int bg_group_set_threshold(bg_net *n, int32_t gid, int kind, int var, double value, int var2) {
    if (!gid_ok(n, gid) || kind < 0 || kind > 2) return fail(BG_EINVAL, "bg_group_set_threshold");
    HGroup &g = n->groups[gid];
    if (kind && (var < 0 || var >= g.nvar)) return fail(BG_EINVAL, "threshold variable out of range");
    if (kind == 2 && (var2 < 0 || var2 >= g.nvar)) return fail(BG_EINVAL, "threshold variable out of range");
    g.thr_kind = kind; g.thr_var = var; g.thr_val = value; g.thr_var2 = var2;
    return BG_OK;
}

int bg_group_set_poisson(bg_net *n, int32_t gid, int rate_var, uint64_t seed) {
    if (!gid_ok(n, gid)) return fail(BG_EINVAL, "bg_group_set_poisson");
    HGroup &g = n->groups[gid];
    if (rate_var < 0 || rate_var >= g.nvar) return fail(BG_EINVAL, "rate variable out of range");
    g.thr_kind = BG_THR_POISSON; g.rate_var = rate_var; g.seed = seed;
    return BG_OK;
}

int bg_group_set_generator(bg_net *n, int32_t gid, int64_t ns, const int64_t *steps, const int32_t *idx) {
    if (!gid_ok(n, gid) || ns < 0 || (ns > 0 && (!steps || !idx))) return fail(BG_EINVAL, "bg_group_set_generator");
    HGroup &g = n->groups[gid];
    for (int64_t k = 0; k < ns; ++k) {
        if (idx[k] < 0 || idx[k] >= g.n) return fail(BG_EINVAL, "generator index out of range");
        if (k && (steps[k] < steps[k - 1] || (steps[k] == steps[k - 1] && idx[k] < idx[k - 1])))
            return fail(BG_EINVAL, "generator spikes not sorted by (step, index)");
    }
    g.thr_kind = BG_THR_GENERATOR; g.gen_steps.assign(steps, steps + ns); g.gen_idx.assign(idx, idx + ns);
    return BG_OK;
}

int bg_group_set_reset(bg_net *n, int32_t gid, int kind, int var, double value, int var2) {
    if (!gid_ok(n, gid) || kind < 0 || kind > 2) return fail(BG_EINVAL, "bg_group_set_reset");
    HGroup &g = n->groups[gid];
    if (kind && (var < 0 || var >= g.nvar)) return fail(BG_EINVAL, "reset variable out of range");
    if (kind == 2 && (var2 < 0 || var2 >= g.nvar)) return fail(BG_EINVAL, "reset variable out of range");
    g.reset_kind = kind; g.reset_var = var; g.reset_val = value; g.reset_var2 = var2;
    return BG_OK;
}

int bg_group_set_refractory(bg_net *n, int32_t gid, double rt, int32_t period, int var, double value) {
    if (!gid_ok(n, gid) || period < 0) return fail(BG_EINVAL, "bg_group_set_refractory");
    HGroup &g = n->groups[gid];
    if (period > 0 && (var < 0 || var >= g.nvar)) return fail(BG_EINVAL, "clamp variable out of range");
    // rt <= 0: no spike filter (refractory < 0.9*dt), clamp only
    g.refr = rt > 0; g.refr_time = rt; g.period = period; g.clamp_var = var; g.clamp_val = value;
    return BG_OK;
}

int bg_group_set_empirical(bg_net *n, int32_t gid, int32_t steps) {
    if (!gid_ok(n, gid) || steps < 0) return fail(BG_EINVAL, "bg_group_set_empirical");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    n->groups[gid].emp_steps = steps;
    return BG_OK;
}

int bg_group_set_model(bg_net *n, int32_t gid, const bg_fit_model *m) {
    if (!gid_ok(n, gid) || !m || !m->state_names) return fail(BG_EINVAL, "bg_group_set_model");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HGroup &g = n->groups[gid];
    std::vector<std::string> names;
    std::string cur;
    for (const char *p = m->state_names;; ++p) {
        if (*p == ',' || *p == 0) {
            if (cur.empty()) return fail(BG_EINVAL, "empty state variable name");
            names.push_back(cur);
            cur.clear();
            if (*p == 0) break;
        } else if (std::isalnum((unsigned char)*p) || *p == '_') {
            cur += *p;
        } else if (*p != ' ') {
            return fail(BG_EINVAL, "bad state variable name");
        }
    }
    if ((int)names.size() != g.nvar) return fail(BG_EINVAL, "model names do not match the group's variables");
    if (g.nvar > 16) return fail(BG_ENOSYS, "more than 16 state variables in a generated model");
    g.gen_names = names;
    g.gen_update = m->update_code ? m->update_code : "";
    g.gen_threshold = m->threshold_code ? m->threshold_code : "";
    g.gen_reset = m->reset_code ? m->reset_code : "";
    if (!g.gen_update.empty()) g.linear = false;
    return BG_OK;
}

static int conn_common(bg_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to, int64_t tn,
                       int var, int32_t delay, int mod_var, HConn &c) {
    if (!gid_ok(n, src) || !gid_ok(n, tgt)) return fail(BG_EINVAL, "connection group id");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    const HGroup &gs = n->groups[src], &gt = n->groups[tgt];
    if (so < 0 || sn < 0 || so + sn > gs.n || to < 0 || tn < 0 || to + tn > gt.n) return fail(BG_EINVAL, "connection ranges");
    if (var < 0 || var >= gt.nvar) return fail(BG_EINVAL, "connection target variable");
    if (delay < 0 || delay > 1 << 20) return fail(BG_EINVAL, "connection delay");
    if (mod_var >= gs.nvar) return fail(BG_EINVAL, "modulation variable");
    c.src = src; c.tgt = tgt; c.so = so; c.sn = sn; c.to = to; c.tn = tn; c.var = var; c.delay = delay; c.mod_var = mod_var;
    return BG_OK;
}

// shared_w: w points to the one weight of every synapse
static int conn_add_impl(bg_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to, int64_t tn, int var,
                         int64_t nnz, const int64_t *rowptr, const int32_t *cols, const void *w, bool shared_w,
                         int w_bits, int32_t delay, const uint8_t *delays, int32_t ring_depth, int mod_var,
                         int32_t *cid) {
    HConn c;
    int st = conn_common(n, src, so, sn, tgt, to, tn, var, delay, mod_var, c);
    if (st) return st;
    if (w_bits != 32 && w_bits != 64) return fail(BG_EINVAL, "w_bits must be 32 or 64");
    if (!rowptr || nnz < 0 || (nnz > 0 && (!cols || !w)) || !cid) return fail(BG_EINVAL, "CSR arrays");
    if (rowptr[0] != 0 || rowptr[sn] != nnz) return fail(BG_EINVAL, "rowptr must start at 0 and end at nnz");
    for (int64_t i = 0; i < sn; ++i)
        if (rowptr[i + 1] < rowptr[i]) return fail(BG_EINVAL, "rowptr not monotone");
    {
        // rows in parallel (about 4M synapses per part); the first bad row
        // (lowest index) decides the message
        const int64_t row_grain = std::max<int64_t>(1, ((int64_t)1 << 22) / std::max<int64_t>(1, nnz / std::max<int64_t>(1, sn)));
        const int parts = parallel_parts(sn, row_grain);
        std::vector<int64_t> bad_row(parts, sn);
        std::vector<int> bad_kind(parts, 0);
        parallel_for(sn, [&](int64_t lo, int64_t hi, int t) {
            for (int64_t i = lo; i < hi; ++i)
                for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
                    const int kind = (cols[k] < 0 || cols[k] >= tn) ? 1 : (k > rowptr[i] && cols[k] <= cols[k - 1]) ? 2 : 0;
                    if (kind) { bad_row[t] = i; bad_kind[t] = kind; return; }
                }
        }, row_grain);
        int64_t r = sn; int kind = 0;
        for (int t = 0; t < parts; ++t) if (bad_row[t] < r) { r = bad_row[t]; kind = bad_kind[t]; }
        if (kind == 1) return fail(BG_EINVAL, "column index out of range");
        if (kind == 2) return fail(BG_EINVAL, "columns not strictly ascending in a row");
    }
    c.nnz = nnz; c.rowptr.assign(rowptr, rowptr + sn + 1);
    c.cols.resize(nnz);
    parallel_for(nnz, [&](int64_t lo, int64_t hi, int) { std::memcpy(c.cols.data() + lo, cols + lo, (hi - lo) * 4); });
    c.w_bits = w_bits;
    // one shared weight (bit pattern) is kept once and filled on the device
    if (shared_w) {
        c.homogeneous = true;
    } else {
        const int parts = parallel_parts(nnz);
        std::vector<char> same(parts, 1);
        parallel_for(nnz, [&](int64_t lo, int64_t hi, int t) {
            if (w_bits == 32) {
                const uint32_t *p = (const uint32_t *)w; const uint32_t v = p[0]; bool ok = true;
                for (int64_t k = lo; k < hi; ++k) ok &= p[k] == v;
                same[t] = ok;
            } else {
                const uint64_t *p = (const uint64_t *)w; const uint64_t v = p[0]; bool ok = true;
                for (int64_t k = lo; k < hi; ++k) ok &= p[k] == v;
                same[t] = ok;
            }
        });
        c.homogeneous = true;
        for (char x : same) c.homogeneous = c.homogeneous && x;
    }
    const int64_t wb = w_bits / 8;
    if (c.homogeneous && nnz > 0) {
        c.wshared = true;
        c.w.assign((const char *)w, (const char *)w + wb);
    } else {
        c.w.resize(nnz * wb);
        parallel_for(nnz, [&](int64_t lo, int64_t hi, int) { std::memcpy(c.w.data() + lo * wb, (const char *)w + lo * wb, (hi - lo) * wb); });
    }
    if (delays) {
        if (ring_depth < 1 || ring_depth > 255) return fail(BG_EINVAL, "ring depth must be in [1, 255]");
        const int parts = parallel_parts(nnz);
        std::vector<int> dmax(parts, 0);
        parallel_for(nnz, [&](int64_t lo, int64_t hi, int t) {
            uint8_t m = 0;
            for (int64_t k = lo; k < hi; ++k) m = std::max(m, delays[k]);
            dmax[t] = m;
        });
        for (int m : dmax) if (m >= ring_depth) return fail(BG_EINVAL, "delay >= ring depth");
        // two spare rows beyond the reference's int(max_delay/dt)+1: the rows
        // written at step t never include the rows delivered at steps t-1 and
        // t-2, which lets the spike push ride on the source group's update
        // kernel and lets blocks of the persistent kernel drift by one step
        c.hetero = true; c.md = ring_depth + 2;
        c.d.resize(nnz);
        parallel_for(nnz, [&](int64_t lo, int64_t hi, int) { std::memcpy(c.d.data() + lo, delays + lo, hi - lo); });
    }
    n->conns.push_back(std::move(c));
    *cid = (int32_t)n->conns.size() - 1;
    n->items.push_back({IT_CONN, *cid});
    return BG_OK;
}

int bg_conn_add(bg_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to, int64_t tn, int var,
                int64_t nnz, const int64_t *rowptr, const int32_t *cols, const void *w, int w_bits, int32_t delay,
                const uint8_t *delays, int32_t ring_depth, int mod_var, int32_t *cid) {
    return conn_add_impl(n, src, so, sn, tgt, to, tn, var, nnz, rowptr, cols, w, false, w_bits, delay, delays,
                         ring_depth, mod_var, cid);
}

int bg_conn_add_shared(bg_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to, int64_t tn, int var,
                       int64_t nnz, const int64_t *rowptr, const int32_t *cols, double weight, int w_bits,
                       int32_t delay, const uint8_t *delays, int32_t ring_depth, int mod_var, int32_t *cid) {
    const float wf = (float)weight;
    const void *w = w_bits == 32 ? (const void *)&wf : (const void *)&weight;
    return conn_add_impl(n, src, so, sn, tgt, to, tn, var, nnz, rowptr, cols, w, true, w_bits, delay, delays,
                         ring_depth, mod_var, cid);
}

int bg_conn_add_dense(bg_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to, int64_t tn, int var,
                      const void *W, int w_bits, int32_t delay, int mod_var, int32_t *cid) {
    HConn c;
    int st = conn_common(n, src, so, sn, tgt, to, tn, var, delay, mod_var, c);
    if (st) return st;
    if ((w_bits != 32 && w_bits != 64) || (!W && sn * tn > 0) || !cid) return fail(BG_EINVAL, "dense weights");
    c.dense = true; c.w_bits = w_bits; c.nnz = sn * tn;
    c.w.assign((const char *)W, (const char *)W + sn * tn * (w_bits / 8));
    n->conns.push_back(std::move(c));
    *cid = (int32_t)n->conns.size() - 1;
    n->items.push_back({IT_CONN, *cid});
    return BG_OK;
}

// A shared weight kept once on the host becomes a full host array (for
// reading weights back or changing them).
static void expand_shared_weight(HConn &c) {
    if (!c.wshared) return;
    const int64_t wb = c.w_bits / 8, cnt = c.wcount();
    hvec<char> full(cnt * wb);
    parallel_for(cnt, [&](int64_t lo, int64_t hi, int) {
        for (int64_t k = lo; k < hi; ++k) std::memcpy(full.data() + k * wb, c.w.data(), wb);
    });
    c.w.swap(full);
    c.wshared = false;
}

int bg_conn_get_weights(bg_net *n, int32_t cid, double *out) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !out) return fail(BG_EINVAL, "bg_conn_get_weights");
    HConn &c = n->conns[cid];
    const int64_t cnt = c.wcount();
    expand_shared_weight(c);
    if (n->prepared) {
        BG_CUDA(cudaStreamSynchronize(n->stream));
        BG_CUDA(cudaMemcpy(c.w.data(), c.dW, c.w.size(), cudaMemcpyDeviceToHost));
    }
    for (int64_t k = 0; k < cnt; ++k)
        out[k] = c.w_bits == 64 ? ((const double *)c.w.data())[k] : (double)((const float *)c.w.data())[k];
    return BG_OK;
}

int bg_conn_set_weights(bg_net *n, int32_t cid, const double *in) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !in) return fail(BG_EINVAL, "bg_conn_set_weights");
    HConn &c = n->conns[cid];
    const int64_t cnt = c.wcount();
    if (n->prepared && c.dCRing && cnt > 0) {
        // the count ring delivers k-fold sums of one weight: a new shared
        // value rebuilds the sum table, unequal weights cannot be taken
        const double w0 = c.w_bits == 64 ? in[0] : (double)(float)in[0];
        for (int64_t k = 1; k < cnt; ++k)
            if ((c.w_bits == 64 ? in[k] : (double)(float)in[k]) != w0 || std::signbit(in[k]) != std::signbit(in[0]))
                return fail(BG_ENOSYS, "weights of a shared-weight delayed connection must stay equal after prepare");
        if (n->precision == 64) {
            std::vector<double> tab(c.tablen, 0.0);
            for (int k = 1; k < c.tablen; ++k) tab[k] = tab[k - 1] + w0;
            int st = upload(n, c.dTable, tab.data(), tab.size() * 8); if (st) return st;
        } else {
            std::vector<float> tab(c.tablen, 0.0f);
            for (int k = 1; k < c.tablen; ++k) tab[k] = tab[k - 1] + (float)w0;
            int st = upload(n, c.dTable, tab.data(), tab.size() * 4); if (st) return st;
        }
    }
    expand_shared_weight(c);
    for (int64_t k = 0; k < cnt; ++k) {
        if (c.w_bits == 64) ((double *)c.w.data())[k] = in[k];
        else ((float *)c.w.data())[k] = (float)in[k];
    }
    if (n->prepared) {
        BG_CUDA(cudaStreamSynchronize(n->stream));
        BG_CUDA(cudaMemcpy(c.dW, c.w.data(), c.w.size(), cudaMemcpyHostToDevice));
    }
    return BG_OK;
}

int bg_stdp_add(bg_net *n, int32_t cid, const double *decay, double Ap, double Am, double wmin, double wmax, int inter,
                int32_t pre_delay, int32_t post_delay, int32_t *sid) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !decay || !sid) return fail(BG_EINVAL, "bg_stdp_add");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HConn &c = n->conns[cid];
    if (c.hetero) return fail(BG_ENOSYS, "STDP on a DelayConnection is not supported");
    if (c.stdp >= 0) return fail(BG_ENOSYS, "one STDP rule per connection");
    if (pre_delay < 0 || post_delay < 0 || inter < 0 || inter > 3) return fail(BG_EINVAL, "STDP parameters");
    HStdp s; s.cid = cid; s.a_pre = decay[0]; s.c_pre = decay[1]; s.a_post = decay[2]; s.c_post = decay[3];
    s.Ap = Ap; s.Am = Am; s.wmin = wmin; s.wmax = wmax; s.inter = inter; s.pre_delay = pre_delay; s.post_delay = post_delay;
    n->stdps.push_back(s);
    *sid = (int32_t)n->stdps.size() - 1;
    c.stdp = *sid;
    n->items.push_back({IT_STDP_PRE, *sid});
    n->items.push_back({IT_STDP_POST, *sid});
    return BG_OK;
}

int bg_synapses_add(bg_net *n, int32_t src_gid, int64_t src_origin, int64_t src_n, int32_t tgt_gid, int64_t tgt_origin,
                    int64_t tgt_n, int64_t nsyn, const int32_t *pre, const int32_t *post, const int32_t *delay, int nops,
                    const int32_t *op_var, const int32_t *op_sub, const double *terms, int32_t *sid) {
    if (!gid_ok(n, src_gid) || !gid_ok(n, tgt_gid) || nsyn < 0 || nops < 0 || nops > bg::kSynMaxOps || !sid ||
        (nsyn > 0 && (!pre || !post || !delay)) || (nops > 0 && (!op_var || !op_sub || (nsyn > 0 && !terms))))
        return fail(BG_EINVAL, "bg_synapses_add");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    if (n->precision != 64) return fail(BG_ENOSYS, "Synapses run on the FP64 network path");
    const HGroup &gs = n->groups[src_gid], &gt = n->groups[tgt_gid];
    if (src_origin < 0 || src_n < 0 || src_origin + src_n > gs.n || tgt_origin < 0 || tgt_n < 0 || tgt_origin + tgt_n > gt.n)
        return fail(BG_EINVAL, "synapse ranges");
    if (src_n > (1 << 24)) return fail(BG_ENOSYS, "Synapses from more than 2^24 sources");
    for (int k = 0; k < nops; ++k) if (op_var[k] < 0 || op_var[k] >= gt.nvar) return fail(BG_EINVAL, "synaptic statement");
    HSyn y; y.src = src_gid; y.tgt = tgt_gid; y.so = src_origin; y.sn = src_n; y.to = tgt_origin; y.tn = tgt_n;
    y.nsyn = nsyn; y.nops = nops; y.op_var.assign(op_var, op_var + nops); y.op_sub.assign(op_sub, op_sub + nops);
    for (int64_t k = 0; k < nsyn; ++k) {
        if (pre[k] < 0 || pre[k] >= src_n || post[k] < 0 || post[k] >= tgt_n) return fail(BG_EINVAL, "synapse index");
        if (delay[k] < 0 || delay[k] > 253) return fail(BG_ENOSYS, "synaptic delay beyond 253 bins");
        y.dmax = std::max(y.dmax, (int)delay[k]);
    }
    // queue order per target: later insertion (shorter delay) last, then
    // ascending source, then ascending synapse index
    // three stable counting passes (least significant key first): source,
    // delay descending, target
    std::vector<int64_t> cur(nsyn), nxt(nsyn);
    for (int64_t k = 0; k < nsyn; ++k) cur[k] = k;
    auto pass = [&](int64_t range, auto key) {
        std::vector<int64_t> cnt(range + 1, 0);
        for (int64_t k = 0; k < nsyn; ++k) cnt[key(cur[k]) + 1]++;
        for (int64_t r = 0; r < range; ++r) cnt[r + 1] += cnt[r];
        for (int64_t k = 0; k < nsyn; ++k) nxt[cnt[key(cur[k])]++] = cur[k];
        cur.swap(nxt);
    };
    pass(src_n, [&](int64_t k) { return (int64_t)pre[k]; });
    pass(254, [&](int64_t k) { return (int64_t)(253 - delay[k]); });
    pass(tgt_n, [&](int64_t k) { return (int64_t)post[k]; });
    y.perm = cur;
    y.colptr.assign(tgt_n + 1, 0);
    for (int64_t k = 0; k < nsyn; ++k) y.colptr[post[k] + 1]++;
    for (int64_t j = 0; j < tgt_n; ++j) y.colptr[j + 1] += y.colptr[j];
    y.word.resize(nsyn);
    for (int64_t p = 0; p < nsyn; ++p) {
        const int64_t k = y.perm[p];
        y.word[p] = (uint32_t)pre[k] | ((uint32_t)(delay[k] + 1) << 24);
    }
    if (nops > 0 && nsyn > 0) y.terms.assign(terms, terms + (size_t)nops * nsyn);
    // rows by source for the event path: synapses of a source by (delay,
    // synapse index) -- two stable counting passes -- with their targets and
    // column positions (the index of their terms)
    y.events = tgt_n < (int64_t(1) << 24) && nsyn > 0 && nsyn < (int64_t(1) << 31);
    if (y.events) {
        std::vector<int64_t> colpos(nsyn);
        for (int64_t p = 0; p < nsyn; ++p) colpos[y.perm[p]] = p;
        for (int64_t k = 0; k < nsyn; ++k) cur[k] = k;
        pass(254, [&](int64_t k) { return (int64_t)delay[k]; });
        pass(src_n, [&](int64_t k) { return (int64_t)pre[k]; });
        y.srcptr.assign(src_n + 1, 0);
        for (int64_t k = 0; k < nsyn; ++k) y.srcptr[pre[k] + 1]++;
        for (int64_t i = 0; i < src_n; ++i) y.srcptr[i + 1] += y.srcptr[i];
        y.sd.resize(nsyn); y.stgt.resize(nsyn); y.sq.resize(nsyn);
        for (int64_t p = 0; p < nsyn; ++p) {
            const int64_t k = cur[p];
            y.sd[p] = (uint8_t)delay[k]; y.stgt[p] = post[k]; y.sq[p] = (int32_t)colpos[k];
        }
    }
    n->syns.push_back(std::move(y));
    *sid = (int32_t)n->syns.size() - 1;
    return BG_OK;
}

int bg_synapses_set_code(bg_net *n, int32_t yid, int32_t nsv, const double *sv, const char *pre_code,
                         const char *post_code, int32_t nslots, const int32_t *slot_var, int32_t nwrites,
                         const int32_t *writes, int32_t npre, const int32_t *pre_var) {
    if (!n || yid < 0 || yid >= (int32_t)n->syns.size() || nsv < 0 || nsv > bg::kSynMaxVars || nslots < 0 ||
        nslots > bg::kSynMaxOps || npre < 0 || npre > bg::kSynMaxOps || nwrites < 0 || nwrites > nslots ||
        (nslots && !slot_var) || (npre && !pre_var) || (nwrites && !writes))
        return fail(BG_EINVAL, "bg_synapses_set_code");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HSyn &y = n->syns[yid];
    if (y.nops) return fail(BG_EINVAL, "Synapses with code take no separate statements");
    const HGroup &gs = n->groups[y.src], &gt = n->groups[y.tgt];
    for (int k = 0; k < nslots; ++k) if (slot_var[k] < 0 || slot_var[k] >= gt.nvar) return fail(BG_EINVAL, "target variable");
    for (int k = 0; k < nwrites; ++k) if (writes[k] < 0 || writes[k] >= gt.nvar) return fail(BG_EINVAL, "target variable");
    for (int k = 0; k < npre; ++k) if (pre_var[k] < 0 || pre_var[k] >= gs.nvar) return fail(BG_EINVAL, "source variable");
    y.coded = true; y.nsv = nsv;
    if (sv) y.sv.assign(sv, sv + (size_t)nsv * y.nsyn);
    else y.sv.assign((size_t)nsv * y.nsyn, 0.0);
    y.pre_code = pre_code ? pre_code : ""; y.post_code = post_code ? post_code : "";
    y.slot_var.assign(slot_var, slot_var + nslots); y.writes.assign(writes, writes + nwrites);
    y.pre_var.assign(pre_var, pre_var + npre);
    return BG_OK;
}

int bg_synapses_get_var(bg_net *n, int32_t yid, int32_t k, double *out) {
    if (!n || yid < 0 || yid >= (int32_t)n->syns.size() || !out) return fail(BG_EINVAL, "bg_synapses_get_var");
    HSyn &y = n->syns[yid];
    if (!y.coded || k < 0 || k >= y.nsv) return fail(BG_EINVAL, "synaptic variable");
    if (!n->prepared || y.nsyn == 0) { std::copy(y.sv.begin() + (size_t)k * y.nsyn, y.sv.begin() + (size_t)(k + 1) * y.nsyn, out); return BG_OK; }
    std::vector<double> col(y.nsyn);
    BG_CUDA(cudaStreamSynchronize(n->stream));
    BG_CUDA(cudaMemcpy(col.data(), y.dSv + (size_t)k * y.nsyn, y.nsyn * 8, cudaMemcpyDeviceToHost));
    for (int64_t p = 0; p < y.nsyn; ++p) out[y.perm[p]] = col[p];
    return BG_OK;
}

int bg_synapses_set_var(bg_net *n, int32_t yid, int32_t k, const double *in) {
    if (!n || yid < 0 || yid >= (int32_t)n->syns.size() || !in) return fail(BG_EINVAL, "bg_synapses_set_var");
    HSyn &y = n->syns[yid];
    if (!y.coded || k < 0 || k >= y.nsv) return fail(BG_EINVAL, "synaptic variable");
    std::copy(in, in + y.nsyn, y.sv.begin() + (size_t)k * y.nsyn);
    if (!n->prepared || y.nsyn == 0) return BG_OK;
    std::vector<double> col(y.nsyn);
    for (int64_t p = 0; p < y.nsyn; ++p) col[p] = in[y.perm[p]];
    BG_CUDA(cudaStreamSynchronize(n->stream));
    BG_CUDA(cudaMemcpy(y.dSv + (size_t)k * y.nsyn, col.data(), y.nsyn * 8, cudaMemcpyHostToDevice));
    return BG_OK;
}

// Upload the statements' terms in column order (from `terms` in synapse
// order, or from the stored copy when null).
static int bg_synapses_set_terms_impl(bg_net *n, int yi, const double *terms) {
    HSyn &y = n->syns[yi];
    if (terms && !y.terms.empty()) std::copy(terms, terms + (size_t)y.nops * y.nsyn, y.terms.begin());
    if (!y.dTerm || y.nops == 0 || y.nsyn == 0) return BG_OK;
    std::vector<double> col((size_t)y.nops * y.nsyn);
    for (int k = 0; k < y.nops; ++k)
        for (int64_t p = 0; p < y.nsyn; ++p) col[(size_t)k * y.nsyn + p] = y.terms[(size_t)k * y.nsyn + y.perm[p]];
    BG_CUDA(cudaStreamSynchronize(n->stream));
    BG_CUDA(cudaMemcpy(y.dTerm, col.data(), col.size() * 8, cudaMemcpyHostToDevice));
    return refresh_term_src(n, y);
}

int bg_synapses_set_terms(bg_net *n, int32_t sid, const double *terms) {
    if (!n || sid < 0 || sid >= (int32_t)n->syns.size() || !terms) return fail(BG_EINVAL, "bg_synapses_set_terms");
    return bg_synapses_set_terms_impl(n, sid, terms);
}

int bg_stdp_add_delayed(bg_net *n, int32_t cid, const double *decay, double Ap, double Am, double wmin, double wmax,
                        int inter, int32_t pre_delay, int32_t hist_len, const uint8_t *lag_pre, const uint8_t *lag_post,
                        int32_t *sid) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !decay || !sid) return fail(BG_EINVAL, "bg_stdp_add_delayed");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HConn &c = n->conns[cid];
    if (!c.hetero || c.dense) return fail(BG_EINVAL, "delayed STDP needs a sparse DelayConnection");
    if (c.stdp >= 0) return fail(BG_ENOSYS, "one STDP rule per connection");
    if (pre_delay < 0 || inter < 0 || inter > 3 || hist_len < 1 || hist_len > 256) return fail(BG_EINVAL, "STDP parameters");
    if (c.nnz > 0 && (!lag_pre || !lag_post)) return fail(BG_EINVAL, "STDP lags");
    for (int64_t k = 0; k < c.nnz; ++k)
        if (lag_pre[k] >= hist_len || lag_post[k] >= hist_len) return fail(BG_EINVAL, "STDP lag beyond the trace history");
    HStdp s; s.cid = cid; s.a_pre = decay[0]; s.c_pre = decay[1]; s.a_post = decay[2]; s.c_post = decay[3];
    s.Ap = Ap; s.Am = Am; s.wmin = wmin; s.wmax = wmax; s.inter = inter; s.pre_delay = pre_delay; s.post_delay = 0;
    s.delayed = true; s.hlen = hist_len;
    s.lag_pre.assign(lag_pre, lag_pre + c.nnz); s.lag_post.assign(lag_post, lag_post + c.nnz);
    n->stdps.push_back(std::move(s));
    *sid = (int32_t)n->stdps.size() - 1;
    c.stdp = *sid;
    n->items.push_back({IT_STDP_PRE, *sid});
    n->items.push_back({IT_STDP_POST, *sid});
    return BG_OK;
}

int bg_stdp_set_update(bg_net *n, int32_t sid, int pre_mode, int post_mode, double wmax_exact) {
    if (!n || sid < 0 || sid >= (int32_t)n->stdps.size() || pre_mode < 0 || pre_mode > 2 || post_mode < 0 ||
        post_mode > 2)
        return fail(BG_EINVAL, "bg_stdp_set_update");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HStdp &s = n->stdps[sid];
    if ((pre_mode || post_mode) && n->conns[s.cid].w_bits != 64)
        return fail(BG_ENOSYS, "multiplicative STDP updates need FP64 weights");
    s.pre_mode = pre_mode; s.post_mode = post_mode; s.wx = wmax_exact;
    return BG_OK;
}

int bg_stdp_get_traces(bg_net *n, int32_t sid, double *a_pre, double *a_post) {
    if (!n || sid < 0 || sid >= (int32_t)n->stdps.size()) return fail(BG_EINVAL, "bg_stdp_get_traces");
    if (!n->prepared) return fail(BG_ESTATE, "network not prepared");
    const HStdp &s = n->stdps[sid]; const HConn &c = n->conns[s.cid];
    BG_CUDA(cudaStreamSynchronize(n->stream));
    if (a_pre) BG_CUDA(cudaMemcpy(a_pre, s.dApre, c.sn * 8, cudaMemcpyDeviceToHost));
    if (a_post) BG_CUDA(cudaMemcpy(a_post, s.dApost, c.tn * 8, cudaMemcpyDeviceToHost));
    return BG_OK;
}

int bg_spikemon_add(bg_net *n, int32_t gid, int64_t origin, int64_t cnt, int32_t delay, int32_t *mid) {
    if (!gid_ok(n, gid) || origin < 0 || cnt < 0 || origin + cnt > n->groups[gid].n || delay < 0 || !mid)
        return fail(BG_EINVAL, "bg_spikemon_add");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HSpikeMon m; m.gid = gid; m.origin = origin; m.n = cnt; m.delay = delay;
    n->smons.push_back(m);
    n->items.push_back({IT_SPIKEMON, (int)n->smons.size() - 1});
    n->mon_kind.push_back(0); n->mon_idx.push_back((int)n->smons.size() - 1);
    *mid = (int32_t)n->mon_kind.size() - 1;
    return BG_OK;
}

int bg_statemon_add(bg_net *n, int32_t gid, int var, int64_t nidx, const int32_t *idx, int32_t timestep, int32_t *mid) {
    if (!gid_ok(n, gid) || var < 0 || var >= n->groups[gid].nvar || timestep < 1 || nidx < 0 || !mid)
        return fail(BG_EINVAL, "bg_statemon_add");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    HStateMon m; m.gid = gid; m.var = var; m.timestep = timestep;
    const HGroup &g = n->groups[gid];
    if (idx) m.idx.assign(idx, idx + nidx);
    else { m.idx.resize(g.n); for (int64_t i = 0; i < g.n; ++i) m.idx[i] = (int32_t)i; }
    for (int32_t i : m.idx) if (i < 0 || i >= g.n) return fail(BG_EINVAL, "state monitor index out of range");
    n->stmons.push_back(std::move(m));
    n->mon_kind.push_back(1); n->mon_idx.push_back((int)n->stmons.size() - 1);
    *mid = (int32_t)n->mon_kind.size() - 1;
    return BG_OK;
}

static bool mon_ok(const bg_net *n, int32_t mid, int kind) {
    return n && mid >= 0 && mid < (int32_t)n->mon_kind.size() && n->mon_kind[mid] == kind;
}

int bg_spikemon_count(bg_net *n, int32_t mid, int64_t *cnt) {
    if (!mon_ok(n, mid, 0) || !cnt) return fail(BG_EINVAL, "spike monitor id");
    *cnt = (int64_t)n->smons[n->mon_idx[mid]].idx.size();
    return BG_OK;
}

int bg_spikemon_read(bg_net *n, int32_t mid, int64_t *steps, int32_t *idx, int64_t cap, int64_t *cnt) {
    if (!mon_ok(n, mid, 0) || !cnt || cap < 0) return fail(BG_EINVAL, "spike monitor id");
    const HSpikeMon &m = n->smons[n->mon_idx[mid]];
    const int64_t k = std::min<int64_t>(cap, (int64_t)m.idx.size());
    if (k > 0) {
        if (steps) std::memcpy(steps, m.steps.data(), k * 8);
        if (idx) std::memcpy(idx, m.idx.data(), k * 4);
    }
    *cnt = k;
    return BG_OK;
}

int bg_statemon_count(bg_net *n, int32_t mid, int64_t *rows) {
    if (!mon_ok(n, mid, 1) || !rows) return fail(BG_EINVAL, "state monitor id");
    *rows = (int64_t)n->stmons[n->mon_idx[mid]].steps.size();
    return BG_OK;
}

int bg_statemon_read(bg_net *n, int32_t mid, double *vals, int64_t *steps, int64_t cap, int64_t *rows) {
    if (!mon_ok(n, mid, 1) || !rows || cap < 0) return fail(BG_EINVAL, "state monitor id");
    const HStateMon &m = n->stmons[n->mon_idx[mid]];
    const int64_t r = std::min<int64_t>(cap, (int64_t)m.steps.size());
    const int64_t w = (int64_t)m.idx.size();
    if (r > 0) {
        if (vals) std::memcpy(vals, m.vals.data(), r * w * 8);
        if (steps) std::memcpy(steps, m.steps.data(), r * 8);
    }
    *rows = r;
    return BG_OK;
}

int bg_monitor_clear(bg_net *n, int32_t mid) {
    if (!n || mid < 0 || mid >= (int32_t)n->mon_kind.size()) return fail(BG_EINVAL, "monitor id");
    if (n->mon_kind[mid] == 0) {
        HSpikeMon &m = n->smons[n->mon_idx[mid]]; m.steps.clear(); m.idx.clear();
    } else {
        HStateMon &m = n->stmons[n->mon_idx[mid]];
        if (n->prepared) return fail(BG_ENOSYS, "clearing a state monitor after prepare is not supported; create a new network");
        m.steps.clear(); m.vals.clear();
    }
    return BG_OK;
}

static int prepare_impl(bg_net *n);

int bg_net_prepare(bg_net *n) {
    const int st = prepare_impl(n);
    if (n) release_staging(n);
    return st;
}

static int prepare_impl(bg_net *n) {
    if (!n) return fail(BG_EINVAL, "net");
    if (n->prepared) return BG_OK;
    BG_CUDA(cudaSetDevice(n->device));
    const size_t ts = tsize(n);
    // spike-history depth per group (neurongroup.py:459-473)
    for (auto &g : n->groups) g.depth = std::max(1, g.period);
    for (auto &c : n->conns) { HGroup &g = n->groups[c.src]; g.depth = std::max(g.depth, (c.hetero ? 0 : c.delay) + 1); }
    for (auto &s : n->stdps) {
        const HConn &c = n->conns[s.cid];
        n->groups[c.src].depth = std::max(n->groups[c.src].depth, s.pre_delay + 1);
        n->groups[c.tgt].depth = std::max(n->groups[c.tgt].depth, s.post_delay + 1);
    }
    for (auto &m : n->smons) { HGroup &g = n->groups[m.gid]; g.depth = std::max(g.depth, m.delay + 1); }
    for (auto &y : n->syns) { HGroup &g = n->groups[y.src]; g.depth = std::max(g.depth, y.dmax + 2); }
    // the reference adds a DelayConnection's due row (after_connections)
    // before the Synapses slot; here the row is added in the next step's
    // head kernel, after the Synapses kernel: refuse targets fed by both
    for (const auto &y : n->syns)
        for (const auto &c : n->conns)
            if (c.hetero && c.tgt == y.tgt && c.to < y.to + y.tn && y.to < c.to + c.tn) {
                for (int v : y.op_var)
                    if (v == c.var)
                        return fail(BG_ENOSYS, "a variable fed by both a DelayConnection and Synapses");
                for (int v : y.writes)
                    if (v == c.var)
                        return fail(BG_ENOSYS, "a variable fed by both a DelayConnection and Synapses");
            }
    // chunk length bounded by monitor buffer sizes
    int64_t chunk = kChunkSteps;
    for (auto &m : n->smons) chunk = std::min<int64_t>(chunk, std::max<int64_t>(kGraphSteps, (int64_t)(1 << 25) / std::max<int64_t>(1, m.n)));
    for (auto &m : n->stmons) chunk = std::min<int64_t>(chunk, std::max<int64_t>(kGraphSteps, (int64_t)(1 << 26) / std::max<int64_t>(1, (int64_t)m.idx.size())));
    chunk = std::max<int64_t>(kGraphSteps, chunk / kGraphSteps * kGraphSteps);
    n->chunk_steps = chunk;
    // ---- device allocations
    for (auto &g : n->groups) {
        const size_t sbytes = (size_t)std::max(1, g.nvar) * g.npad * ts;
        if (g.borrowed >= 0) {
            const bg_net::Import &im = n->imports[g.borrowed];
            if ((size_t)im.bytes < sbytes)
                return fail(BG_EINVAL, "borrowed buffer smaller than the group state (" + std::to_string(sbytes) + " bytes)");
            if (im.dtype != (n->precision == 64 ? BG_DTYPE_F64 : BG_DTYPE_F32))
                return fail(BG_EINVAL, "borrowed buffer type differs from the network precision");
            g.dS = im.ptr;
        } else if (n->alloc(&g.dS, sbytes) != cudaSuccess) return fail(BG_ENOMEM, "group state");
        BG_CUDA(cudaMemsetAsync(g.dS, 0, sbytes, n->stream));
        for (int v = 0; v < g.nvar; ++v) { int st = upload_state(n, g, v, g.S0.data() + (size_t)v * g.n); if (st) return st; }
        if (n->alloc(&g.dHist, (size_t)g.depth * (g.npad / 32) * 4) != cudaSuccess) return fail(BG_ENOMEM, "spike history");
        if (g.refr && n->alloc(&g.dNext, g.npad * 8) != cudaSuccess) return fail(BG_ENOMEM, "refractory");
        if ((g.period > 0 || g.emp_steps > 0) && n->alloc(&g.dLast, g.npad * 4) != cudaSuccess)
            return fail(BG_ENOMEM, "refractory");
        for (auto &h : g.setters) {
            const size_t nv = h.vals.size();
            if (n->alloc(&h.dVals, nv * ts) != cudaSuccess || n->alloc(&h.dBp, std::max<size_t>(1, h.bp.size()) * 8) != cudaSuccess)
                return fail(BG_ENOMEM, "timed array");
            int st;
            if (ts == 8) st = upload(n, h.dVals, h.vals.data(), nv * 8);
            else {
                std::vector<float> f(h.vals.begin(), h.vals.end());
                st = upload(n, h.dVals, f.data(), nv * 4);
                if (!st) BG_CUDA(cudaStreamSynchronize(n->stream));
            }
            if (st) return st;
            if (!h.bp.empty()) { st = upload(n, h.dBp, h.bp.data(), h.bp.size() * 8); if (st) return st; }
        }
        if (!g.gen_steps.empty()) {
            if (n->alloc(&g.dGenSteps, g.gen_steps.size() * 8) != cudaSuccess || n->alloc(&g.dGenIdx, g.gen_idx.size() * 4) != cudaSuccess)
                return fail(BG_ENOMEM, "generator");
            int st = upload(n, g.dGenSteps, g.gen_steps.data(), g.gen_steps.size() * 8); if (st) return st;
            st = upload(n, g.dGenIdx, g.gen_idx.data(), g.gen_idx.size() * 4); if (st) return st;
        }
    }
    for (size_t ci = 0; ci < n->conns.size(); ++ci) {
        HConn &c = n->conns[ci];
        const int64_t wbytes = c.wcount() * (c.w_bits / 8);
        if (n->alloc(&c.dW, wbytes) != cudaSuccess) return fail(BG_ENOMEM, "weights");
        int st = BG_OK;
        if (c.wshared) {
            const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((c.wcount() + 255) / 256, (int64_t)sm_count() * 8));
            if (c.w_bits == 32) k_fill_u32<<<grid, 256, 0, n->stream>>>((uint32_t *)c.dW, c.wcount(), *(const uint32_t *)c.w.data());
            else k_fill_u64<<<grid, 256, 0, n->stream>>>((unsigned long long *)c.dW, c.wcount(), *(const unsigned long long *)c.w.data());
            BG_CUDA(cudaGetLastError());
        } else {
            st = upload(n, c.dW, c.w.data(), wbytes); if (st) return st;
        }
        if (!c.dense) {
            if (n->alloc(&c.dRow, (c.sn + 1) * 8) != cudaSuccess || n->alloc(&c.dCols, c.nnz * 4) != cudaSuccess)
                return fail(BG_ENOMEM, "CSR");
            st = upload(n, c.dRow, c.rowptr.data(), (c.sn + 1) * 8); if (st) return st;
            st = upload(n, c.dCols, c.cols.data(), c.nnz * 4); if (st) return st;
        }
        c.fused_push = c.hetero && !c.dense && c.mod_var < 0 && c.stdp < 0 && (c.homogeneous || !n->deterministic);
        if (c.hetero) {
            if (n->alloc(&c.dD, c.nnz) != cudaSuccess) return fail(BG_ENOMEM, "delays");
            st = upload(n, c.dD, c.d.data(), c.nnz); if (st) return st;
            // A shared weight on the atomic path: the ring counts events per
            // (row, target) and delivery looks up the k-fold sum of the weight.
            // A row entry collects at most one event per synapse, so counts
            // stay below the largest in-degree.
            int64_t kmax = 0;
            if (c.fused_push && c.homogeneous && c.nnz > 0) { st = max_indegree(n, c, &kmax); if (st) return st; }
            if (kmax > 0 && kmax < 65535) {
                c.tablen = (int)kmax + 1;
                c.tnp = (c.tn + 1) & ~1ll;
                if (n->alloc(&c.dCRing, (size_t)c.md * c.tnp * 2) != cudaSuccess) return fail(BG_ENOMEM, "count ring");
                if (n->alloc(&c.dTable, (size_t)(kmax + 1) * ts) != cudaSuccess) return fail(BG_ENOMEM, "count table");
                const double w0 = c.w_bits == 64 ? *(const double *)c.w.data() : (double)*(const float *)c.w.data();
                if (n->precision == 64) {
                    std::vector<double> tab(kmax + 1, 0.0);
                    for (int64_t k = 1; k <= kmax; ++k) tab[k] = tab[k - 1] + w0;
                    st = upload(n, c.dTable, tab.data(), tab.size() * 8); if (st) return st;
                } else {
                    std::vector<float> tab(kmax + 1, 0.0f);
                    const float wf = (float)w0;
                    for (int64_t k = 1; k <= kmax; ++k) tab[k] = tab[k - 1] + wf;
                    st = upload(n, c.dTable, tab.data(), tab.size() * 4); if (st) return st;
                }
                BG_CUDA(cudaStreamSynchronize(n->stream));
            } else if (n->alloc(&c.dRing, (size_t)c.md * c.tn * ts) != cudaSuccess) {
                return fail(BG_ENOMEM, "delay ring");
            }
            n->groups[c.tgt].delivs.push_back((int)ci);
        }
        if (c.stdp >= 0 && !c.dense) {
            // column access (connectionmatrix.py:317-333): ascending source per target column
            std::vector<int64_t> colptr(c.tn + 1, 0), colk(c.nnz); std::vector<int32_t> colsrc(c.nnz);
            for (int32_t j : c.cols) colptr[j + 1]++;
            for (int64_t j = 0; j < c.tn; ++j) colptr[j + 1] += colptr[j];
            std::vector<int64_t> fill(colptr.begin(), colptr.end() - 1);
            for (int64_t i = 0; i < c.sn; ++i)
                for (int64_t k = c.rowptr[i]; k < c.rowptr[i + 1]; ++k) { int64_t p = fill[c.cols[k]]++; colk[p] = k; colsrc[p] = (int32_t)i; }
            if (n->alloc(&c.dColptr, (c.tn + 1) * 8) != cudaSuccess || n->alloc(&c.dColk, c.nnz * 8) != cudaSuccess ||
                n->alloc(&c.dColsrc, c.nnz * 4) != cudaSuccess) return fail(BG_ENOMEM, "column index");
            st = upload(n, c.dColptr, colptr.data(), (c.tn + 1) * 8); if (st) return st;
            st = upload(n, c.dColk, colk.data(), c.nnz * 8); if (st) return st;
            st = upload(n, c.dColsrc, colsrc.data(), c.nnz * 4); if (st) return st;
            HStdp &s = n->stdps[c.stdp];
            if (s.delayed && c.nnz > 0) {
                std::vector<uint8_t> lagc(c.nnz);
                for (int64_t p = 0; p < c.nnz; ++p) lagc[p] = s.lag_post[colk[p]];
                if (n->alloc(&s.dLagPre, c.nnz) != cudaSuccess || n->alloc(&s.dLagPostC, c.nnz) != cudaSuccess)
                    return fail(BG_ENOMEM, "STDP lags");
                st = upload(n, s.dLagPre, s.lag_pre.data(), c.nnz); if (st) return st;
                st = upload(n, s.dLagPostC, lagc.data(), c.nnz); if (st) return st;
            }
            BG_CUDA(cudaStreamSynchronize(n->stream));
        }
    }
    for (auto &s : n->stdps) {
        const HConn &c = n->conns[s.cid];
        if (n->alloc(&s.dApre, std::max<int64_t>(1, c.sn) * 8) != cudaSuccess || n->alloc(&s.dApost, std::max<int64_t>(1, c.tn) * 8) != cudaSuccess)
            return fail(BG_ENOMEM, "STDP traces");
        if (s.delayed && (n->alloc(&s.dHpre, (size_t)s.hlen * std::max<int64_t>(1, c.sn) * 8) != cudaSuccess ||
                          n->alloc(&s.dHpost, (size_t)s.hlen * std::max<int64_t>(1, c.tn) * 8) != cudaSuccess))
            return fail(BG_ENOMEM, "STDP trace histories");
        // the presynaptic update rides on the propagation kernel when it reads
        // the same spikes and the items are adjacent (connection, then updater)
        s.fused = !s.delayed && (s.pre_delay == c.delay);
        if (s.fused) {
            for (size_t k = 0; k + 1 < n->items.size(); ++k)
                if (n->items[k + 1].kind == IT_STDP_PRE && n->items[k + 1].id == (int)(&s - &n->stdps[0])) {
                    s.fused = n->items[k].kind == IT_CONN && n->items[k].id == s.cid;
                    break;
                }
        }
    }
    for (auto &m : n->smons) {
        m.cap = std::max<int64_t>(1024, m.n * (n->chunk_steps + 1));
        if (n->alloc(&m.dCnt, 8) != cudaSuccess || n->alloc(&m.dBase, 8) != cudaSuccess ||
            n->alloc(&m.dIdx, m.cap * 4) != cudaSuccess || n->alloc(&m.dSteps, m.cap * 4) != cudaSuccess)
            return fail(BG_ENOMEM, "spike monitor");
        BG_CUDA(cudaMemsetAsync(m.dCnt, 0, 8, n->stream));
        BG_CUDA(cudaMemsetAsync(m.dBase, 0, 8, n->stream));
    }
    for (size_t k = 0; k < n->stmons.size(); ++k) {
        HStateMon &m = n->stmons[k];
        HGroup &g = n->groups[m.gid];
        const int64_t w = (int64_t)m.idx.size();
        std::vector<int32_t> order(w);
        for (int64_t e = 0; e < w; ++e) order[e] = (int32_t)e;
        std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return m.idx[a] < m.idx[b]; });
        m.sorted.resize(w); m.pos.resize(w);
        for (int64_t e = 0; e < w; ++e) { m.sorted[e] = m.idx[order[e]]; m.pos[e] = order[e]; }
        const int64_t nb = g.npad / bg::kBlockNeurons;
        m.blk_lo.assign(nb + 1, 0);
        for (int64_t b = 0, e = 0; b <= nb; ++b) {
            while (e < w && m.sorted[e] < b * bg::kBlockNeurons) ++e;
            m.blk_lo[b] = (int32_t)e;
        }
        m.cap_rows = n->chunk_steps / m.timestep + 2;
        m.start = n->nstep;
        if (n->alloc(&m.dIdx, std::max<int64_t>(1, w) * 4) != cudaSuccess || n->alloc(&m.dPos, std::max<int64_t>(1, w) * 4) != cudaSuccess ||
            n->alloc(&m.dBlk, (nb + 1) * 4) != cudaSuccess || n->alloc(&m.dBuf, std::max<int64_t>(1, w) * m.cap_rows * ts) != cudaSuccess ||
            n->alloc(&m.dRowBase, 8) != cudaSuccess)
            return fail(BG_ENOMEM, "state monitor");
        int st;
        if (w) { st = upload(n, m.dIdx, m.sorted.data(), w * 4); if (st) return st; st = upload(n, m.dPos, m.pos.data(), w * 4); if (st) return st; }
        st = upload(n, m.dBlk, m.blk_lo.data(), (nb + 1) * 4); if (st) return st;
        BG_CUDA(cudaMemsetAsync(m.dRowBase, 0, 8, n->stream));
        g.recs.push_back((int)k);
    }
    for (auto &y : n->syns) {
        if (n->alloc(&y.dColptr, (y.tn + 1) * 8) != cudaSuccess || n->alloc(&y.dWord, std::max<int64_t>(1, y.nsyn) * 4) != cudaSuccess ||
            n->alloc(&y.dTerm, std::max<int64_t>(1, (int64_t)y.nops * y.nsyn) * 8) != cudaSuccess)
            return fail(BG_ENOMEM, "synapses");
        int st = upload(n, y.dColptr, y.colptr.data(), (y.tn + 1) * 8); if (st) return st;
        if (y.nsyn) { st = upload(n, y.dWord, y.word.data(), y.nsyn * 4); if (st) return st; }
        if (y.coded) {
            y.events = false;                   // the code runs on the pull's per-target walk
            if (n->alloc(&y.dSv, std::max<int64_t>(1, (int64_t)y.nsv * y.nsyn) * 8) != cudaSuccess)
                return fail(BG_ENOMEM, "synaptic variables");
            std::vector<double> col((size_t)y.nsv * y.nsyn);
            for (int v = 0; v < y.nsv; ++v)
                for (int64_t p = 0; p < y.nsyn; ++p) col[(size_t)v * y.nsyn + p] = y.sv[(size_t)v * y.nsyn + y.perm[p]];
            if (!col.empty()) { st = upload(n, y.dSv, col.data(), col.size() * 8); if (st) return st; }
            BG_CUDA(cudaStreamSynchronize(n->stream));
        }
        // the event path pays off once the pull's synapse words no longer
        // stay in L2 (it reads every word every step); below that the pull
        // is cheaper than the event path's extra launches -- unless the
        // network runs in the persistent kernel for Synapses (no launches)
        if (n->syn_events_forced == 2) y.events = false;
        if (y.events && !syn_persist_shape(n)) {
            int dev = 0, l2 = 0;
            cudaGetDevice(&dev);
            if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess) l2 = 0;
            int64_t words = 0;
            for (const auto &o : n->syns) words += o.nsyn;
            if (!n->syn_events_forced && words * 4 <= (int64_t)l2 / 2) y.events = false;
        }
        // the spike lists hold every source for dmax + 2 steps
        if (y.events && (int64_t)(y.dmax + 2) * y.sn * 4 > ((int64_t)1 << 30)) y.events = false;
        if (y.events) {
            y.nbins = (int)((y.tn + bg::kSynBin - 1) / bg::kSynBin);
            if (n->alloc(&y.dSrcPtr, (y.sn + 1) * 8) != cudaSuccess || n->alloc(&y.dSd, y.nsyn) != cudaSuccess ||
                n->alloc(&y.dStgt, y.nsyn * 4) != cudaSuccess || n->alloc(&y.dSq, y.nsyn * 4) != cudaSuccess ||
                n->alloc(&y.dBinCnt, (size_t)y.nbins * 4) != cudaSuccess ||
                n->alloc(&y.dBinKey, (size_t)y.nbins * bg::kSynBinCap * 8) != cudaSuccess ||
                n->alloc(&y.dBinQ, (size_t)y.nbins * bg::kSynBinCap * 4) != cudaSuccess || n->alloc(&y.dUsePull, 8) != cudaSuccess)
                return fail(BG_ENOMEM, "synapse events");
            y.sdepth = y.dmax + 2;
            if (n->alloc(&y.dSlist, (size_t)y.sdepth * std::max<int64_t>(1, y.sn) * 4) != cudaSuccess ||
                n->alloc(&y.dScnt, (size_t)y.sdepth * 4) != cudaSuccess)
                return fail(BG_ENOMEM, "synapse spike lists");
            BG_CUDA(cudaMemsetAsync(y.dScnt, 0, (size_t)y.sdepth * 4, n->stream));
            if ((st = upload(n, y.dSrcPtr, y.srcptr.data(), (y.sn + 1) * 8)) || (st = upload(n, y.dSd, y.sd.data(), y.nsyn)) ||
                (st = upload(n, y.dStgt, y.stgt.data(), y.nsyn * 4)) || (st = upload(n, y.dSq, y.sq.data(), y.nsyn * 4)))
                return st;
            BG_CUDA(cudaMemsetAsync(y.dBinCnt, 0, (size_t)y.nbins * 4, n->stream));
            BG_CUDA(cudaMemsetAsync(y.dUsePull, 0, 8, n->stream));
            const int64_t dw = y.dmax + 2;
            if (y.sn * dw * 4 <= ((int64_t)256 << 20)) {
                std::vector<int32_t> doff((size_t)(y.sn * dw));
                for (int64_t i = 0; i < y.sn; ++i) {
                    const int64_t r0 = y.srcptr[i], r1 = y.srcptr[i + 1];
                    int64_t p = r0;
                    for (int d = 0; d < dw; ++d) {
                        while (p < r1 && y.sd[p] < d) ++p;
                        doff[i * dw + d] = (int32_t)(p - r0);
                    }
                }
                if (n->alloc(&y.dDoff, doff.size() * 4) != cudaSuccess) return fail(BG_ENOMEM, "synapse delay offsets");
                if ((st = upload(n, y.dDoff, doff.data(), doff.size() * 4))) return st;
            }
        }
    }
    for (size_t yi = 0; yi < n->syns.size(); ++yi) {
        int st = bg_synapses_set_terms_impl(n, (int)yi, nullptr); if (st) return st;
    }
    const size_t ncount = n->groups.size() + n->conns.size();
    if (n->alloc(&n->dCounters, std::max<size_t>(1, ncount) * 8) != cudaSuccess) return fail(BG_ENOMEM, "counters");
    BG_CUDA(cudaMemsetAsync(n->dCounters, 0, std::max<size_t>(1, ncount) * 8, n->stream));
    BG_CUDA(cudaStreamSynchronize(n->stream));
    int st = reset_dynamic(n);
    if (st) return st;
    // ---- per-step launch list: groups, trace decay, connections slot
    for (size_t gi = 0; gi < n->groups.size(); ++gi) {
        st = n->precision == 64 ? build_group<double>(n, (int)gi) : build_group<float>(n, (int)gi);
        if (st) return st;
    }
    const size_t nhead = n->step_launches.size();
    std::vector<size_t> mon_launch;
    for (size_t si = 0; si < n->stdps.size(); ++si) { st = build_decay(n, (int)si); if (st) return st; }
    for (const Item &it : n->items) {
        switch (it.kind) {
        case IT_CONN: st = n->precision == 64 ? build_conn<double>(n, it.id) : build_conn<float>(n, it.id); break;
        case IT_SPIKEMON: mon_launch.push_back(n->step_launches.size()); st = build_spikemon(n, it.id); break;
        // STDP keeps FP64 traces and weight arithmetic on both paths (the
        // FP32 path moves the neuron state and the propagation to FP32)
        case IT_STDP_PRE: st = build_stdp_pre(n, it.id); break;
        case IT_STDP_POST: st = build_stdp_post(n, it.id); break;
        }
        if (st) return st;
    }
    // the 'synapses' slot: after the connections, before the resets
    // (DelayConnection rows and resets of this step run in the next step's
    // head kernel, so a target variable fed by both is refused at prepare)
    // consecutive event-path objects with disjoint targets share their launches
    for (size_t yi = 0; yi < n->syns.size();) {
        if (!n->syns[yi].events || n->syns[yi].coded) { st = build_syn(n, (int)yi); if (st) return st; ++yi; continue; }
        std::vector<int> grp{(int)yi};
        size_t yj = yi + 1;
        while (yj < n->syns.size() && (int)grp.size() < bg::kSynEvMerge && n->syns[yj].events && !n->syns[yj].coded) {
            bool ok = true;
            for (int k : grp) ok = ok && syn_disjoint(n->syns[k], n->syns[yj]);
            if (!ok) break;
            grp.push_back((int)yj++);
        }
        st = build_syn_events(n, grp);
        if (st) return st;
        yi = yj;
    }
    if (n->step_launches.empty()) return fail(BG_EINVAL, "empty network");
    {
        // SpikeMonitors move to right after the group kernels (they read
        // nothing but the spike history, which only the group kernels write)
        std::vector<Launch> L;
        std::vector<std::string> names;
        std::vector<char> is_mon(n->step_launches.size(), 0);
        for (size_t i : mon_launch) is_mon[i] = 1;
        for (size_t i = 0; i < nhead; ++i) { L.push_back(n->step_launches[i]); names.push_back(n->item_names[i]); }
        for (size_t i : mon_launch) { L.push_back(n->step_launches[i]); names.push_back(n->item_names[i]); }
        for (size_t i = nhead; i < n->step_launches.size(); ++i)
            if (!is_mon[i]) { L.push_back(n->step_launches[i]); names.push_back(n->item_names[i]); }
        n->step_launches.swap(L);
        n->item_names.swap(names);
        n->side0 = nhead;
        n->side1 = nhead + mon_launch.size();
    }
    if (n->allow_persist) st = n->precision == 64 ? build_persist<double>(n) : build_persist<float>(n);
    if (!st && n->allow_persist && !n->persist) st = build_syn_persist(n);
    if (st) return st;
    BG_CUDA(cudaStreamSynchronize(n->stream));
    n->prepared = true;
    return BG_OK;
}

// The event path's spike lists of the last dmax steps, rebuilt from the
// spike history when it did not come from the gather launches.
static int refresh_syn_lists(bg_net *n) {
    if (!n->syn_lists_stale) return BG_OK;
    for (size_t yi = 0; yi < n->syns.size(); ++yi) {
        const HSyn &y = n->syns[yi];
        if (!y.events || y.coded || !y.dScnt) continue;
        BG_CUDA(cudaMemsetAsync(y.dScnt, 0, (size_t)y.sdepth * 4, n->stream));
        if (y.dmax == 0) continue;
        const bg::SynEvArgs a = syn_ev_args(n, (int)yi);
        const int64_t nw = (y.so + y.sn + 31) / 32 - y.so / 32;
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((nw * y.dmax + 255) / 256, (int64_t)sm_count() * 8));
        bg::k_syn_lists<<<(unsigned)grid, 256, 0, n->stream>>>(a);
        BG_CUDA(cudaGetLastError());
        n->launches += 1;
    }
    n->syn_lists_stale = false;
    return BG_OK;
}

static int launch_step(bg_net *n, int tail) {
    const size_t k = n->step_launches.size();
    for (size_t i = 0; i < k; ++i) {
        cudaError_t e = n->step_launches[i](n->stream, tail, i + 1 == k);
        if (e != cudaSuccess) return fail(BG_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    n->launches += (int64_t)k;
    return BG_OK;
}

// one step into the graph being captured, the side launches on the side
// stream (forked after the group kernels, joined before the last launch)
static int capture_step_forked(bg_net *n) {
    const size_t k = n->step_launches.size();
    for (size_t i = 0; i < k; ++i) {
        cudaStream_t st = n->stream;
        if (i == n->side0) {
            BG_CUDA(cudaEventRecord(n->ev_fork, n->stream));
            BG_CUDA(cudaStreamWaitEvent(n->side, n->ev_fork, 0));
        }
        if (i >= n->side0 && i < n->side1) st = n->side;
        if (i == n->side1) BG_CUDA(cudaEventRecord(n->ev_join, n->side));
        if (i + 1 == k) BG_CUDA(cudaStreamWaitEvent(n->stream, n->ev_join, 0));
        cudaError_t e = n->step_launches[i](st, 1, i + 1 == k);
        if (e != cudaSuccess) return fail(BG_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    n->launches += (int64_t)k;
    return BG_OK;
}

static int ensure_graph(bg_net *n) {
    if (n->gexec) return BG_OK;
    // the side launches fork only when a launch follows them
    const bool fork = n->side1 > n->side0 && n->side1 < n->step_launches.size();
    if (fork && !n->side) {
        BG_CUDA(cudaStreamCreateWithFlags(&n->side, cudaStreamNonBlocking));
        BG_CUDA(cudaEventCreateWithFlags(&n->ev_fork, cudaEventDisableTiming));
        BG_CUDA(cudaEventCreateWithFlags(&n->ev_join, cudaEventDisableTiming));
    }
    cudaGraph_t graph;
    BG_CUDA(cudaStreamBeginCapture(n->stream, cudaStreamCaptureModeThreadLocal));
    int st = BG_OK;
    for (int s = 0; s < kGraphSteps && st == BG_OK; ++s) st = fork ? capture_step_forked(n) : launch_step(n, 1);
    cudaError_t e = cudaStreamEndCapture(n->stream, &graph);
    n->launches -= (int64_t)kGraphSteps * (int64_t)n->step_launches.size();
    if (st) return st;
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&n->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return BG_OK;
}

static int net_run_steps(bg_net *n, int64_t nsteps, int64_t cs0);

int bg_net_run(bg_net *n, int64_t nsteps, int64_t cs0) {
    if (!n || nsteps < 0) return fail(BG_EINVAL, "bg_net_run");
    if (n->failed) return fail(BG_ESTATE, "the network stopped after a device error; rebuild it");
    int st = net_run_steps(n, nsteps, cs0);
    if (st == BG_OK && n->check_finite && n->prepared) st = check_finite_states(n);
    return st;
}

static int net_run_steps(bg_net *n, int64_t nsteps, int64_t cs0) {
    if (!n->prepared) { int st = bg_net_prepare(n); if (st) return st; }
    if (nsteps == 0) return BG_OK;
    if (n->nstep + nsteps >= (1ll << 31) - 1) return fail(BG_EINVAL, "a network runs at most 2^31-1 steps");
    BG_CUDA(cudaSetDevice(n->device));
    if (n->persist) {
        int st0 = refresh_syn_lists(n);
        if (st0) return st0;
        long long off0 = cs0 - n->nstep;
        BG_CUDA(cudaMemcpyAsync(&n->dCtl->clock_off, &off0, 8, cudaMemcpyHostToDevice, n->stream));
        BG_CUDA(cudaEventRecord(n->ev0, n->stream));
        const bool mons = !n->smons.empty();
        int64_t chunk = mons ? kPersistMonSteps : (int64_t)1 << 20;
        if (!n->stmons.empty()) chunk = std::min<int64_t>(chunk, n->chunk_steps);   // rows of the monitor buffers
        std::vector<long long> cnt;
        for (int64_t done = 0; done < nsteps;) {
            const int64_t c = std::min(chunk, nsteps - done);
            int st = run_persist(n, c);
            if (st) return st;
            if (mons) {
                const HGroup &g = n->groups[0];
                for (auto &m : n->smons) {
                    bg::MonWordsArgs w;
                    w.ctl = n->dCtl; w.words = n->dMonWords; w.stride = g.npad / 32; w.nsteps = (int)c; w.s0 = 0;
                    w.origin = m.origin; w.n = m.n; w.cnt = m.dCnt; w.cap = m.cap; w.idx = m.dIdx; w.steps = m.dSteps;
                    w.off = n->dMonOff;
                    bg::k_monw_count<<<(unsigned)c, bg::kMonWordsThreads, 0, n->stream>>>(w);
                    BG_CUDA(cudaGetLastError());
                    n->launches += 1;
                    cnt.resize(c);
                    BG_CUDA(cudaMemcpyAsync(cnt.data(), n->dMonOff, c * 8, cudaMemcpyDeviceToHost, n->stream));
                    BG_CUDA(cudaStreamSynchronize(n->stream));
                    // step ranges whose records fit the (empty) buffer; a step
                    // alone always fits (at most m.n records, cap >= m.n)
                    for (int64_t s0 = 0; s0 < c;) {
                        int64_t s1 = s0, tot = 0;
                        while (s1 < c && tot + cnt[s1] <= m.cap) tot += cnt[s1++];
                        bg::MonWordsArgs r = w;
                        r.words = n->dMonWords + s0 * w.stride; r.off = n->dMonOff + s0;
                        r.nsteps = (int)(s1 - s0); r.s0 = (int)s0;
                        bg::k_monw_scan<<<1, bg::kMonWordsThreads, 0, n->stream>>>(r);
                        bg::k_monw_write<<<(unsigned)(s1 - s0), bg::kMonWordsThreads, 0, n->stream>>>(r);
                        BG_CUDA(cudaGetLastError());
                        n->launches += 2;
                        BG_CUDA(cudaStreamSynchronize(n->stream));
                        st = check_device_error(n);
                        if (st) return st;
                        st = drain_spikemon(n, m, cs0 + done);
                        if (st) return st;
                        s0 = s1;
                    }
                }
            }
            // the launch ran the 'end' slot of its last step
            if (!n->stmons.empty()) { st = drain(n, cs0 + done, n->nstep - 1, off0); if (st) return st; }
            done += c;
        }
        BG_CUDA(cudaEventRecord(n->ev1, n->stream));
        BG_CUDA(cudaEventSynchronize(n->ev1));
        float ms = 0;
        BG_CUDA(cudaEventElapsedTime(&ms, n->ev0, n->ev1));
        n->last_ms = ms;
        return check_device_error(n);
    }
    int st = ensure_graph(n);
    if (st) return st;
    if ((st = refresh_syn_lists(n))) return st;
    long long off = cs0 - n->nstep;
    BG_CUDA(cudaMemcpyAsync(&n->dCtl->clock_off, &off, 8, cudaMemcpyHostToDevice, n->stream));
    BG_CUDA(cudaStreamSynchronize(n->stream));
    BG_CUDA(cudaEventRecord(n->ev0, n->stream));
    float total_ms = 0;
    int64_t done = 0;
    while (done < nsteps) {
        const int64_t c = std::min<int64_t>(n->chunk_steps, nsteps - done);
        const long long chunk_cs = cs0 + done;
        for (auto &m : n->smons) BG_CUDA(cudaMemcpyAsync(m.dBase, &chunk_cs, 8, cudaMemcpyHostToDevice, n->stream));
        BG_CUDA(cudaStreamSynchronize(n->stream));
        int64_t k = 0;
        if (done == 0) { st = launch_step(n, 0); if (st) return st; k = 1; }
        while (c - k >= kGraphSteps) {
            BG_CUDA(cudaGraphLaunch(n->gexec, n->stream));
            n->launches += (int64_t)kGraphSteps * (int64_t)n->step_launches.size();
            k += kGraphSteps;
        }
        for (; k < c; ++k) { st = launch_step(n, 1); if (st) return st; }
        done += c;
        n->nstep += c;
        const bool last_chunk = done == nsteps;
        if (last_chunk) {
            for (auto &f : n->finalize_launches) {
                cudaError_t e = f(n->stream, 1, 0);
                if (e != cudaSuccess) return fail(BG_ECUDA, cudaGetErrorString(e));
                n->launches++;
            }
        }
        BG_CUDA(cudaEventRecord(n->ev1, n->stream));
        BG_CUDA(cudaEventSynchronize(n->ev1));
        float ms = 0;
        BG_CUDA(cudaEventElapsedTime(&ms, n->ev0, n->ev1));
        total_ms += ms;
        st = check_device_error(n);
        if (st) return st;
        // 'end' slot has run for steps < nstep-1, and for nstep-1 after finalize
        st = drain(n, chunk_cs, last_chunk ? n->nstep - 1 : n->nstep - 2, off);
        if (st) return st;
        BG_CUDA(cudaEventRecord(n->ev0, n->stream));
    }
    n->last_ms = total_ms;
    return BG_OK;
}

int bg_group_get_state(bg_net *n, int32_t gid, int var, double *out) {
    if (!gid_ok(n, gid) || var < 0 || var >= n->groups[gid].nvar || !out) return fail(BG_EINVAL, "bg_group_get_state");
    HGroup &g = n->groups[gid];
    if (!n->prepared) { std::memcpy(out, g.S0.data() + (size_t)var * g.n, g.n * 8); return BG_OK; }
    BG_CUDA(cudaStreamSynchronize(n->stream));
    if (n->precision == 64) BG_CUDA(cudaMemcpy(out, (double *)g.dS + (size_t)var * g.npad, g.n * 8, cudaMemcpyDeviceToHost));
    else {
        std::vector<float> tmp(g.n);
        BG_CUDA(cudaMemcpy(tmp.data(), (float *)g.dS + (size_t)var * g.npad, g.n * 4, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < g.n; ++i) out[i] = tmp[i];
    }
    return BG_OK;
}

int bg_group_set_state(bg_net *n, int32_t gid, int var, const double *in) {
    if (!gid_ok(n, gid) || var < 0 || var >= n->groups[gid].nvar || !in) return fail(BG_EINVAL, "bg_group_set_state");
    HGroup &g = n->groups[gid];
    if (!n->prepared) { std::memcpy(g.S0.data() + (size_t)var * g.n, in, g.n * 8); return BG_OK; }
    BG_CUDA(cudaStreamSynchronize(n->stream));
    int st = upload_state(n, g, var, in);
    if (st) return st;
    BG_CUDA(cudaStreamSynchronize(n->stream));
    return BG_OK;
}

int bg_net_set_persistent(bg_net *n, int enable) {
    if (!n) return fail(BG_EINVAL, "net");
    if (n->prepared) return fail(BG_ESTATE, "set before prepare");
    if (enable != 0 && enable != 1 && enable != 256 && enable != 512)
        return fail(BG_EINVAL, "persistent: 0, 1, 256 or 512");
    n->allow_persist = enable ? 1 : 0;
    n->persist_th = enable > 1 ? enable : 0;
    return BG_OK;
}

}  // extern "C"

// ---- checkpoint / resume ----------------------------------------------------
// The dynamic state of a prepared network as one byte string: the step
// counter, every group's state rows, spike history, refractory and
// empirical-threshold bookkeeping, the delay rings (value and count rings),
// plastic weights and STDP traces (with their trace records), the spike and
// event counters and the monitors' records.  Ring cursors and the Poisson
// draws are functions of the step counter.  Static data (connectivity, fixed
// weights, model code) is not included: the state is loaded into a network
// built the same way, and every section's size is checked.
namespace {
constexpr uint64_t kStateMagic = 0x3153544e47425242ull;   // "BRBGNTS1"

struct StateWriter {
    bg_net *n; std::vector<char> out; int err = 0;
    void raw(const void *p, size_t b) { const char *c = (const char *)p; out.insert(out.end(), c, c + b); }
    template <typename V> void val(const V &v) { raw(&v, sizeof(v)); }
    void dev(const void *d, size_t b) {
        val((uint64_t)b);
        if (!b || err) return;
        const size_t o = out.size();
        out.resize(o + b);
        if (cudaMemcpy(out.data() + o, d, b, cudaMemcpyDeviceToHost) != cudaSuccess) err = 1;
    }
    template <typename V> void vec(const std::vector<V> &v) { val((uint64_t)v.size()); raw(v.data(), v.size() * sizeof(V)); }
};
struct StateReader {
    const char *p; size_t left; std::string err;
    bool raw(void *d, size_t b) { if (b > left) { err = "truncated state"; return false; } std::memcpy(d, p, b); p += b; left -= b; return true; }
    template <typename V> bool val(V &v) { return raw(&v, sizeof(v)); }
    bool expect(uint64_t want, const char *what) {
        uint64_t got = 0;
        if (!val(got)) return false;
        if (got != want) { err = std::string("state does not match this network (") + what + ")"; return false; }
        return true;
    }
    bool dev(void *d, size_t b, const char *what) {
        if (!expect(b, what)) return false;
        if (!b) return true;
        if (b > left) { err = "truncated state"; return false; }
        if (cudaMemcpy(d, p, b, cudaMemcpyHostToDevice) != cudaSuccess) { err = "copy to the device failed"; return false; }
        p += b; left -= b;
        return true;
    }
    template <typename V> bool vec(std::vector<V> &v) {
        uint64_t k = 0;
        if (!val(k) || k * sizeof(V) > left) { err = "truncated state"; return false; }
        v.resize(k);
        return raw(v.data(), k * sizeof(V));
    }
};

// visits every dynamic buffer in one fixed order for the writer and the reader
template <typename F> void visit_state(bg_net *n, F &&f) {
    const size_t ts = tsize(n);
    f.devbuf(n->dCounters, (n->groups.size() + n->conns.size()) * 8, "counters");
    for (auto &g : n->groups) {
        f.devbuf(g.dS, (size_t)g.nvar * g.npad * ts, "group state");
        f.devbuf(g.dHist, (size_t)g.depth * (g.npad / 32) * 4, "spike history");
        f.devbuf(g.dNext, g.dNext ? (size_t)g.npad * 8 : 0, "refractory");
        f.devbuf(g.dLast, g.dLast ? (size_t)g.npad * 4 : 0, "empirical threshold");
    }
    for (auto &c : n->conns) {
        f.devbuf(c.dRing, c.dRing ? (size_t)c.md * c.tn * ts : 0, "delay ring");
        f.devbuf(c.dCRing, c.dCRing ? (size_t)c.md * c.tnp * 2 : 0, "count ring");
        f.devbuf(c.stdp >= 0 ? c.dW : nullptr, c.stdp >= 0 ? (size_t)c.wcount() * (c.w_bits / 8) : 0, "plastic weights");
    }
    for (auto &st : n->stdps) {
        const HConn &c = n->conns[st.cid];
        f.devbuf(st.dApre, (size_t)c.sn * 8, "presynaptic trace");
        f.devbuf(st.dApost, (size_t)c.tn * 8, "postsynaptic trace");
        f.devbuf(st.delayed ? st.dHpre : nullptr, st.delayed ? (size_t)st.hlen * c.sn * 8 : 0, "trace records");
        f.devbuf(st.delayed ? st.dHpost : nullptr, st.delayed ? (size_t)st.hlen * c.tn * 8 : 0, "trace records");
    }
    for (auto &y : n->syns) f.devbuf(y.coded ? y.dSv : nullptr, y.coded ? (size_t)y.nsv * y.nsyn * 8 : 0, "synaptic variables");
    for (auto &m : n->smons) { f.hostvec(m.steps); f.hostvec(m.idx); }
    for (auto &m : n->stmons) { f.hostvec(m.vals); f.hostvec(m.steps); f.hostval(m.rows_done); }
}

struct SizeVisitor {
    int64_t *t;
    void devbuf(const void *, size_t b, const char *) { *t += 8 + (int64_t)b; }
    template <typename V> void hostvec(const std::vector<V> &v) { *t += 8 + (int64_t)(v.size() * sizeof(V)); }
    template <typename V> void hostval(const V &) { *t += sizeof(V); }
};
struct SaveVisitor {
    StateWriter *w;
    void devbuf(const void *d, size_t b, const char *) { w->dev(d, b); }
    template <typename V> void hostvec(const std::vector<V> &v) { w->vec(v); }
    template <typename V> void hostval(const V &v) { w->val(v); }
};
struct LoadVisitor {
    StateReader *r; bool *ok;
    void devbuf(void *d, size_t b, const char *what) { if (*ok) *ok = r->dev(d, b, what); }
    template <typename V> void hostvec(std::vector<V> &v) { if (*ok) *ok = r->vec(v); }
    template <typename V> void hostval(V &v) { if (*ok) *ok = r->val(v); }
};
uint64_t state_shape(const bg_net *n) {
    return (uint64_t)(n->groups.size() | (n->conns.size() << 16) | (n->stdps.size() << 32) |
                      ((n->smons.size() + n->stmons.size()) << 48));
}
}  // namespace

extern "C" {

int bg_net_state_bytes(bg_net *n, int64_t *bytes) {
    if (!n || !bytes) return fail(BG_EINVAL, "bg_net_state_bytes");
    if (!n->prepared) { int st = bg_net_prepare(n); if (st) return st; }
    int64_t total = 8 * 4;
    SizeVisitor f{&total};
    visit_state(n, f);
    *bytes = total;
    return BG_OK;
}

int bg_net_save_state(bg_net *n, void *buf, int64_t cap, int64_t *written) {
    if (!n || (!buf && cap > 0) || cap < 0) return fail(BG_EINVAL, "bg_net_save_state");
    if (n->failed) return fail(BG_ESTATE, "the network stopped after a device error");
    if (!n->prepared) { int st = bg_net_prepare(n); if (st) return st; }
    BG_CUDA(cudaSetDevice(n->device));
    BG_CUDA(cudaStreamSynchronize(n->stream));
    StateWriter w{n};
    w.val(kStateMagic); w.val((uint64_t)n->precision); w.val((int64_t)n->nstep); w.val(state_shape(n));
    SaveVisitor f{&w};
    visit_state(n, f);
    if (w.err) return fail(BG_ECUDA, "reading the device state failed");
    if ((int64_t)w.out.size() > cap) return fail(BG_EINVAL, "buffer too small for the state (" + std::to_string(w.out.size()) + " bytes)");
    std::memcpy(buf, w.out.data(), w.out.size());
    if (written) *written = (int64_t)w.out.size();
    return BG_OK;
}

int bg_net_load_state(bg_net *n, const void *buf, int64_t bytes) {
    if (!n || !buf || bytes < 0) return fail(BG_EINVAL, "bg_net_load_state");
    if (!n->prepared) { int st = bg_net_prepare(n); if (st) return st; }
    BG_CUDA(cudaSetDevice(n->device));
    BG_CUDA(cudaStreamSynchronize(n->stream));
    StateReader r{(const char *)buf, (size_t)bytes};
    uint64_t magic = 0, prec = 0, shape = 0; int64_t nstep = 0;
    if (!r.val(magic) || magic != kStateMagic) return fail(BG_EINVAL, "not a saved network state");
    if (!r.val(prec) || prec != (uint64_t)n->precision) return fail(BG_EINVAL, "state saved at another precision");
    if (!r.val(nstep) || nstep < 0) return fail(BG_EINVAL, "bad step counter");
    if (!r.val(shape) || shape != state_shape(n)) return fail(BG_EINVAL, "state does not match this network (objects)");
    bool ok = true;
    LoadVisitor f{&r, &ok};
    visit_state(n, f);
    if (!ok) { n->failed = true; return fail(BG_EINVAL, r.err + "; the network must be rebuilt"); }
    if (r.left) { n->failed = true; return fail(BG_EINVAL, "state has trailing bytes; the network must be rebuilt"); }
    n->nstep = nstep;
    n->syn_lists_stale = true;
    long long ns = nstep;
    BG_CUDA(cudaMemcpy(&n->dCtl->nstep, &ns, 8, cudaMemcpyHostToDevice));
    for (auto &m : n->stmons) BG_CUDA(cudaMemcpy(m.dRowBase, &m.rows_done, 8, cudaMemcpyHostToDevice));
    n->failed = false;
    return BG_OK;
}

int bg_net_save(bg_net *n, const char *path) {
    if (!n || !path) return fail(BG_EINVAL, "bg_net_save");
    int64_t bytes = 0;
    int st = bg_net_state_bytes(n, &bytes); if (st) return st;
    std::vector<char> buf((size_t)bytes);
    int64_t written = 0;
    st = bg_net_save_state(n, buf.data(), bytes, &written); if (st) return st;
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(BG_EINVAL, std::string("cannot open ") + path);
    const bool good = std::fwrite(buf.data(), 1, (size_t)written, f) == (size_t)written;
    if (std::fclose(f) != 0 || !good) return fail(BG_EINVAL, std::string("writing ") + path + " failed");
    return BG_OK;
}

int bg_net_load(bg_net *n, const char *path) {
    if (!n || !path) return fail(BG_EINVAL, "bg_net_load");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(BG_EINVAL, std::string("cannot open ") + path);
    std::vector<char> buf;
    char tmp[1 << 16];
    size_t k;
    while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
    std::fclose(f);
    return bg_net_load_state(n, buf.data(), (int64_t)buf.size());
}

int bg_import_device_ptr(bg_net *n, void *ptr, int64_t bytes, int dtype, int32_t *buf_id) {
    if (!n || !ptr || bytes <= 0 || !buf_id) return fail(BG_EINVAL, "bg_import_device_ptr");
    if (dtype != BG_DTYPE_F64 && dtype != BG_DTYPE_F32) return fail(BG_EINVAL, "dtype must be BG_DTYPE_F64 or BG_DTYPE_F32");
    if (((uintptr_t)ptr & 255) != 0) return fail(BG_EINVAL, "borrowed buffer must be 256-byte aligned");
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        return fail(BG_EINVAL, "borrowed pointer is not device memory");
    }
    if (at.device != n->device) return fail(BG_EINVAL, "borrowed buffer lives on another device");
    n->imports.push_back({ptr, bytes, dtype});
    *buf_id = (int32_t)n->imports.size() - 1;
    return BG_OK;
}

int bg_group_use_buffer(bg_net *n, int32_t gid, int32_t buf_id) {
    if (!gid_ok(n, gid) || buf_id < 0 || buf_id >= (int32_t)n->imports.size()) return fail(BG_EINVAL, "bg_group_use_buffer");
    if (n->prepared) return fail(BG_ESTATE, "network already prepared");
    for (const HGroup &g : n->groups)
        if (g.borrowed == buf_id) return fail(BG_EINVAL, "buffer already holds another group's state");
    n->groups[gid].borrowed = buf_id;
    return BG_OK;
}

int bg_group_padded_size(bg_net *n, int32_t gid, int64_t *npad) {
    if (!gid_ok(n, gid) || !npad) return fail(BG_EINVAL, "bg_group_padded_size");
    *npad = n->groups[gid].npad;
    return BG_OK;
}

int bg_net_set_synapse_events(bg_net *n, int mode) {
    if (!n || mode < 0 || mode > 2) return fail(BG_EINVAL, "synapse events: 0 (by size), 1 (always) or 2 (never)");
    if (n->prepared) return fail(BG_ESTATE, "set before prepare");
    n->syn_events_forced = mode;
    return BG_OK;
}

int bg_net_set_spin_limit(bg_net *n, int64_t polls) {
    if (!n || polls < 1 || polls > 0xffffffffll) return fail(BG_EINVAL, "spin limit: 1 .. 2^32-1 polls");
    if (n->prepared) return fail(BG_ESTATE, "set before prepare");
    n->spin_limit = (unsigned int)polls;
    return BG_OK;
}

int bg_net_debug_hold_arrival(bg_net *n, int32_t block) {
    if (!n || block < -1) return fail(BG_EINVAL, "block index");
    if (n->prepared) return fail(BG_ESTATE, "set before prepare");
    n->hold_block = block;
    return BG_OK;
}

int bg_net_set_check_finite(bg_net *n, int enable) {
    if (!n || (enable != 0 && enable != 1)) return fail(BG_EINVAL, "check_finite: 0 or 1");
    n->check_finite = enable;
    return BG_OK;
}

int bg_net_persistent_threads(bg_net *n, int32_t *threads) {
    if (!n || !threads) return fail(BG_EINVAL, "net");
    if (!n->prepared) { int st = bg_net_prepare(n); if (st) return st; }
    *threads = n->persist ? n->persist_used : 0;
    return BG_OK;
}

int bg_net_reinit(bg_net *n) {
    if (!n) return fail(BG_EINVAL, "net");
    if (!n->prepared) return BG_OK;
    BG_CUDA(cudaStreamSynchronize(n->stream));
    int st = reset_dynamic(n);
    if (st) return st;
    BG_CUDA(cudaStreamSynchronize(n->stream));
    return BG_OK;
}

int bg_net_counters(bg_net *n, int64_t *group_spikes, int64_t *conn_events) {
    if (!n) return fail(BG_EINVAL, "net");
    if (!n->prepared) return fail(BG_ESTATE, "network not prepared");
    BG_CUDA(cudaStreamSynchronize(n->stream));
    std::vector<unsigned long long> h(n->groups.size() + n->conns.size());
    if (!h.empty()) BG_CUDA(cudaMemcpy(h.data(), n->dCounters, h.size() * 8, cudaMemcpyDeviceToHost));
    for (size_t g = 0; g < n->groups.size(); ++g) if (group_spikes) group_spikes[g] = (int64_t)h[g];
    for (size_t c = 0; c < n->conns.size(); ++c) if (conn_events) conn_events[c] = (int64_t)h[n->groups.size() + c];
    return BG_OK;
}

int bg_net_profile(bg_net *n, int64_t nsteps, int64_t cs0, double *ms, int64_t cap, int64_t *nitems) {
    if (!n || nsteps <= 0 || !nitems) return fail(BG_EINVAL, "bg_net_profile");
    if (!n->prepared) { int st = bg_net_prepare(n); if (st) return st; }
    if (!n->smons.empty() || !n->stmons.empty())
        return fail(BG_ENOSYS, "profiling runs networks without monitors");
    BG_CUDA(cudaSetDevice(n->device));
    if (n->persist) {
        int st0 = refresh_syn_lists(n);
        if (st0) return st0;
        *nitems = 1;
        cudaEvent_t e0, e1;
        BG_CUDA(cudaEventCreate(&e0)); BG_CUDA(cudaEventCreate(&e1));
        BG_CUDA(cudaEventRecord(e0, n->stream));
        int st = run_persist(n, nsteps);
        if (st) return st;
        BG_CUDA(cudaEventRecord(e1, n->stream));
        BG_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0); cudaEventDestroy(e1);
        if (ms && cap > 0) ms[0] = t / (double)nsteps;   // per simulation step
        return check_device_error(n);
    }
    const size_t k = n->step_launches.size();
    *nitems = (int64_t)k;
    int st0 = refresh_syn_lists(n);
    if (st0) return st0;
    long long off = cs0 - n->nstep;
    BG_CUDA(cudaMemcpyAsync(&n->dCtl->clock_off, &off, 8, cudaMemcpyHostToDevice, n->stream));
    std::vector<cudaEvent_t> ev(k + 1);
    for (auto &e : ev) BG_CUDA(cudaEventCreate(&e));
    std::vector<double> acc(k, 0.0);
    int st = BG_OK;
    for (int64_t s = 0; s < nsteps && st == BG_OK; ++s) {
        BG_CUDA(cudaEventRecord(ev[0], n->stream));
        for (size_t i = 0; i < k; ++i) {
            cudaError_t e = n->step_launches[i](n->stream, s > 0 ? 1 : 0, i + 1 == k);
            if (e != cudaSuccess) { st = fail(BG_ECUDA, cudaGetErrorString(e)); break; }
            BG_CUDA(cudaEventRecord(ev[i + 1], n->stream));
        }
        BG_CUDA(cudaEventSynchronize(ev[k]));
        for (size_t i = 0; i < k; ++i) { float t = 0; cudaEventElapsedTime(&t, ev[i], ev[i + 1]); acc[i] += t; }
        n->launches += (int64_t)k;
    }
    n->nstep += nsteps;
    for (auto &f : n->finalize_launches) { cudaError_t e = f(n->stream, 1, 0); if (e != cudaSuccess && st == BG_OK) st = fail(BG_ECUDA, cudaGetErrorString(e)); }
    BG_CUDA(cudaStreamSynchronize(n->stream));
    for (auto &e : ev) cudaEventDestroy(e);
    if (st) return st;
    for (size_t i = 0; i < k && (int64_t)i < cap; ++i) if (ms) ms[i] = acc[i] / (double)nsteps;
    return check_device_error(n);
}

int bg_net_item_name(bg_net *n, int64_t idx, char *buf, int64_t len) {
    if (n && n->persist && buf && len > 0 && idx == 0) {
        std::strncpy(buf, "persist[g0] (per step)", (size_t)len - 1);
        buf[len - 1] = 0;
        return BG_OK;
    }
    if (!n || !buf || len <= 0 || idx < 0 || idx >= (int64_t)n->item_names.size()) return fail(BG_EINVAL, "bg_net_item_name");
    std::strncpy(buf, n->item_names[idx].c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
    return BG_OK;
}

int bg_net_stats(bg_net *n, int64_t *steps, int64_t *launches, double *ms) {
    if (!n) return fail(BG_EINVAL, "net");
    if (steps) *steps = n->nstep;
    if (launches) *launches = n->launches;
    if (ms) *ms = n->last_ms;
    return BG_OK;
}

}  // extern "C"

// ============================================================== batches
// Independent networks in one launch of bg::k_batch, one block each.  The
// batch works on the networks' own device state (group state, count rings,
// counters, control block) and appends the monitor records of every launch
// to the networks' host-side records, so each network reads and continues
// as if it had run alone.
struct bg_batch {
    std::vector<bg_net *> nets;
    int device = 0, precision = 64, nvar = 0, max_n = 0;
    int shape = -1, lanes = 32;
    size_t smem = 0;                       // dynamic shared memory per block (largest layout)
    std::vector<int32_t> smem_ring[bg::kBatchMaxConn];   // per network: ring offsets (-1: global)
    std::vector<int32_t> smem_rows[bg::kBatchMaxConn];
    std::vector<int32_t> smem_pos;
    std::vector<uint32_t *> packed[bg::kBatchMaxConn];   // target | delay << 24, per network and connection
    // launch outputs and monitor regions (one region per network and monitor)
    int32_t *dOut = nullptr, *dOrder = nullptr; void *dNets = nullptr;
    std::vector<int64_t> sreg, rreg;       // region starts: spike records / state values, [net * max + k]
    std::vector<int32_t> scap, rcap;       // region capacities (records / rows)
    int32_t *dSIdx = nullptr, *dSStep = nullptr; void *dRows = nullptr;
    int32_t *dCIdx = nullptr, *dCStep = nullptr; void *dCRows = nullptr;   // compacted copies
    int64_t *dGather = nullptr; int64_t gather_cap = 0;                     // region starts, lengths, targets
    int64_t nsrec = 0, nrval = 0;
    std::vector<std::pair<uint16_t *, uint16_t *>> snap;   // global rings and their copies (autotuning)
    std::vector<size_t> snap_bytes;
    std::vector<void *> allocs;
    cudaStream_t stream = nullptr; cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0; int64_t launches = 0;
    template <typename P> cudaError_t alloc(P **p, size_t bytes) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
        if (e == cudaSuccess) { allocs.push_back(q); *p = (P *)q; }
        return e;
    }
    ~bg_batch() {
        for (void *q : allocs) cudaFree(q);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// copies the regions [src + soff[r], + len[r]) to dst + doff[r] (32-bit words)
__global__ void k_batch_gather(const uint32_t *src, const int64_t *g, int nreg, uint32_t *dst) {
    for (int r = blockIdx.x; r < nreg; r += gridDim.x) {
        const int64_t so = g[r], len = g[nreg + r], dof = g[2 * nreg + r];
        for (int64_t k = threadIdx.x; k < len; k += blockDim.x) dst[dof + k] = src[so + k];
    }
}

bool batch_direct(const HConn &c) {
    return !c.hetero && !c.dense && c.delay == 0 && c.mod_var < 0 && c.stdp < 0 && c.homogeneous && c.src == 0 && c.tgt == 0;
}

// Why a network cannot run in a batch ("" when it can).
std::string batch_refusal(const bg_net *n) {
    if (n->failed) return "the network stopped after a device error";
    if (n->groups.size() != 1) return "a batched network has exactly one NeuronGroup";
    const HGroup &g = n->groups[0];
    if (!g.linear || g.nvar < 1 || g.nvar > 4) return "the group is not linear with 1-4 variables";
    if (g.refr || g.period > 0 || g.emp_steps > 0 || g.generated()) return "refractoriness and generated models are not batched";
    if (!g.setters.empty()) return "TimedArraySetters are not batched";
    if (g.thr_kind != BG_THR_CONST && g.thr_kind != BG_THR_VAR && g.thr_kind != BG_THR_NONE) return "threshold kind";
    if (g.reset_kind != BG_RESET_NONE && g.reset_kind != BG_RESET_CONST && g.reset_kind != BG_RESET_VAR) return "reset kind";
    if (g.n > bg::kBatchMaxNeurons) return "more than 4096 neurons";
    if (!n->stdps.empty() || !n->syns.empty()) return "STDP and Synapses are not batched";
    if ((int)n->conns.size() > bg::kBatchMaxConn) return "more than 2 connections";
    for (const HConn &c : n->conns) {
        if (batch_direct(c)) continue;
        if (!(c.hetero && c.fused_push && c.dCRing && c.homogeneous && c.src == 0 && c.tgt == 0))
            return "a connection that is neither a zero-delay shared-weight Connection nor a shared-weight DelayConnection onto the group";
    }
    if ((int)n->smons.size() > bg::kBatchMaxSmon) return "more than 2 spike monitors";
    for (const HSpikeMon &m : n->smons) if (m.gid != 0 || m.delay != 0) return "a delayed spike monitor";
    if ((int)n->stmons.size() > bg::kBatchMaxRec) return "more than 4 StateMonitors";
    for (const HStateMon &m : n->stmons) {
        if (m.gid != 0) return "a StateMonitor on another group";
        for (size_t e = 1; e < m.sorted.size(); ++e)
            if (m.sorted[e] == m.sorted[e - 1]) return "a StateMonitor that records a neuron twice";
    }
    return "";
}

template <typename T>
void batch_image(bg_batch *b, const std::vector<int64_t> &nsteps, int dry, std::vector<bg::BatchNet<T>> &img) {
    img.assign(b->nets.size(), bg::BatchNet<T>());
    for (size_t i = 0; i < b->nets.size(); ++i) {
        bg_net *n = b->nets[i];
        const HGroup &g = n->groups[0];
        bg::BatchNet<T> &N = img[i];
        std::memset(&N, 0, sizeof(N));
        const int nv = g.nvar;
        for (int j = 0; j < nv; ++j) {
            for (int k = 0; k < nv; ++k) {
                N.A[j * nv + k] = (T)g.A[j * nv + k];
                if (N.A[j * nv + k] != T(0)) N.anz |= 1ull << (j * nv + k);
            }
            N.C[j] = g.useC ? (T)g.C[j] : T(0);
            if (N.C[j] != T(0)) N.cnz |= 1u << j;
        }
        N.diag = (N.cnz & ~1u) == 0;
        for (int j = 0; j < nv; ++j)
            for (int k = 0; k < nv; ++k)
                if ((((N.anz >> (j * nv + k)) & 1ull) != 0) != (j == 0 || j == k)) N.diag = 0;
        N.thr_kind = g.thr_kind; N.thr_var = g.thr_var; N.thr_var2 = g.thr_var2; N.thr_val = (T)g.thr_val;
        N.reset_kind = g.reset_kind; N.reset_var = g.reset_var; N.reset_var2 = g.reset_var2; N.reset_val = (T)g.reset_val;
        N.S = (T *)g.dS; N.npad = g.npad; N.n = (int32_t)g.n;
        N.nconn = (int32_t)n->conns.size();
        for (int c = 0; c < N.nconn; ++c) {
            const HConn &hc = n->conns[c];
            bg::BatchConn<T> &q = N.conn[c];
            q.so = (int32_t)hc.so; q.sn = (int32_t)hc.sn; q.to = (int32_t)hc.to; q.tn = (int32_t)hc.tn; q.var = hc.var;
            q.direct = batch_direct(hc) ? 1 : 0;
            q.md = q.direct ? 2 : hc.md;           // a Connection's row of step t (parity), pushed and delivered
            q.tnp = (int32_t)((hc.tn + 1) & ~1ll);
            q.smem_ring = b->smem_ring[c][i]; q.smem_rows = b->smem_rows[c][i];
            const double w0 = hc.w_bits == 64 ? *(const double *)hc.w.data() : (double)*(const float *)hc.w.data();
            q.w = (T)w0;
            q.rowptr = hc.dRow; q.packed = b->packed[c][i];
            q.ring = q.direct ? nullptr : hc.dCRing;
        }
        // deliveries: the Connections (the step's connection slot), then the
        // DelayConnections' due rows, each in connection order
        N.ndeliv = 0;
        for (int pass = 0; pass < 2; ++pass)
            for (int c = 0; c < N.nconn; ++c)
                if ((N.conn[c].direct == 1) == (pass == 0)) N.deliv[N.ndeliv++] = c;
        const int ms = bg::kBatchMaxSmon, mr = bg::kBatchMaxRec;
        N.nsmon = (int32_t)n->smons.size();
        for (int m = 0; m < N.nsmon; ++m) {
            const HSpikeMon &h = n->smons[m];
            bg::BatchSmon &M = N.smon[m];
            M.origin = (int32_t)h.origin; M.n = (int32_t)h.n; M.cap = b->scap[i * ms + m];
            M.idx = b->dSIdx + b->sreg[i * ms + m]; M.step = b->dSStep + b->sreg[i * ms + m];
        }
        N.nrec = (int32_t)n->stmons.size();
        for (int r = 0; r < N.nrec; ++r) {
            const HStateMon &h = n->stmons[r];
            bg::BatchRec &R = N.rec[r];
            R.var = h.var; R.nidx = (int32_t)h.idx.size(); R.timestep = h.timestep; R.cap_rows = b->rcap[i * mr + r];
            R.start = h.start; R.row0 = h.rows_done; R.idx = h.dIdx; R.pos = h.dPos;
            R.buf = (T *)b->dRows + b->rreg[i * mr + r];
        }
        N.smem_pos = b->smem_pos[i];
        N.ctl = n->dCtl; N.counters = n->dCounters;
        N.t0 = n->nstep; N.nsteps = (int32_t)nsteps[i];
        N.out = b->dOut + i * bg::kBatchOut;
        (void)dry;
    }
}

// One launch over every network with steps left; returns the steps each ran.
template <typename T>
int batch_launch(bg_batch *b, const std::vector<int64_t> &want, int dry, std::vector<int32_t> *ran, float *ms) {
    std::vector<bg::BatchNet<T>> img;
    batch_image<T>(b, want, dry, img);
    // longest remaining runs first (their blocks start in the first wave)
    std::vector<int32_t> order(b->nets.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int32_t)i;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return want[x] > want[y]; });
    BG_CUDA(cudaMemcpyAsync(b->dNets, img.data(), img.size() * sizeof(img[0]), cudaMemcpyHostToDevice, b->stream));
    BG_CUDA(cudaMemcpyAsync(b->dOrder, order.data(), order.size() * 4, cudaMemcpyHostToDevice, b->stream));
    BG_CUDA(cudaEventRecord(b->ev0, b->stream));
    cudaError_t e = bg_batch_launch(b->precision, b->nvar, b->shape, b->dNets, b->dOrder, (int)b->nets.size(), b->lanes,
                                    dry, b->smem, b->stream);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    BG_CUDA(cudaEventRecord(b->ev1, b->stream));
    BG_CUDA(cudaEventSynchronize(b->ev1));
    BG_CUDA(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    b->launches++;
    if (ran) {
        ran->assign(b->nets.size() * bg::kBatchOut, 0);
        BG_CUDA(cudaMemcpy(ran->data(), b->dOut, ran->size() * 4, cudaMemcpyDeviceToHost));
    }
    return BG_OK;
}

// Monitor records of the last launch into the networks' host records.
template <typename T>
int batch_collect(bg_batch *b, const std::vector<int32_t> &out, const std::vector<int64_t> &t0,
                  const std::vector<long long> &off) {
    const int ms = bg::kBatchMaxSmon, mr = bg::kBatchMaxRec, K = bg::kBatchOut;
    const size_t nn = b->nets.size();
    // spike records: regions (start, length, target), gathered into one block
    std::vector<int64_t> so, len, dof;
    int64_t tot = 0;
    for (size_t i = 0; i < nn; ++i)
        for (int m = 0; m < (int)b->nets[i]->smons.size(); ++m) {
            const int64_t c = out[i * K + 1 + m];
            if (c > 0) { so.push_back(b->sreg[i * ms + m]); len.push_back(c); dof.push_back(tot); tot += c; }
        }
    auto gather = [&](const uint32_t *src, uint32_t *dst, const std::vector<int64_t> &a, const std::vector<int64_t> &l,
                      const std::vector<int64_t> &d, int words) -> int {
        const int nreg = (int)a.size();
        if (!nreg) return BG_OK;
        std::vector<int64_t> g(3 * nreg);
        for (int r = 0; r < nreg; ++r) { g[r] = a[r] * words; g[nreg + r] = l[r] * words; g[2 * nreg + r] = d[r] * words; }
        if (3 * nreg > b->gather_cap) return fail(BG_ESTATE, "batch gather table");
        BG_CUDA(cudaMemcpyAsync(b->dGather, g.data(), g.size() * 8, cudaMemcpyHostToDevice, b->stream));
        k_batch_gather<<<(unsigned)std::min(nreg, 4096), 256, 0, b->stream>>>(src, b->dGather, nreg, dst);
        BG_CUDA(cudaGetLastError());
        BG_CUDA(cudaStreamSynchronize(b->stream));
        return BG_OK;
    };
    if (tot > 0) {
        int st = gather((const uint32_t *)b->dSIdx, (uint32_t *)b->dCIdx, so, len, dof, 1); if (st) return st;
        st = gather((const uint32_t *)b->dSStep, (uint32_t *)b->dCStep, so, len, dof, 1); if (st) return st;
        std::vector<int32_t> idx(tot), stp(tot);
        BG_CUDA(cudaMemcpy(idx.data(), b->dCIdx, tot * 4, cudaMemcpyDeviceToHost));
        BG_CUDA(cudaMemcpy(stp.data(), b->dCStep, tot * 4, cudaMemcpyDeviceToHost));
        int64_t p = 0;
        for (size_t i = 0; i < nn; ++i)
            for (int m = 0; m < (int)b->nets[i]->smons.size(); ++m) {
                HSpikeMon &h = b->nets[i]->smons[m];
                const int64_t c = out[i * K + 1 + m];
                const long long cs = t0[i] + off[i];
                for (int64_t k = 0; k < c; ++k, ++p) { h.idx.push_back(idx[p]); h.steps.push_back(cs + stp[p]); }
            }
    }
    // state rows
    so.clear(); len.clear(); dof.clear(); tot = 0;
    for (size_t i = 0; i < nn; ++i)
        for (int r = 0; r < (int)b->nets[i]->stmons.size(); ++r) {
            const int64_t rows = out[i * K + 1 + ms + r], w = (int64_t)b->nets[i]->stmons[r].idx.size();
            if (rows > 0 && w > 0) { so.push_back(b->rreg[i * mr + r]); len.push_back(rows * w); dof.push_back(tot); tot += rows * w; }
        }
    std::vector<T> vals(tot);
    if (tot > 0) {
        const int words = (int)(sizeof(T) / 4);
        int st = gather((const uint32_t *)b->dRows, (uint32_t *)b->dCRows, so, len, dof, words); if (st) return st;
        BG_CUDA(cudaMemcpy(vals.data(), b->dCRows, tot * sizeof(T), cudaMemcpyDeviceToHost));
    }
    int64_t p = 0;
    for (size_t i = 0; i < nn; ++i)
        for (int r = 0; r < (int)b->nets[i]->stmons.size(); ++r) {
            HStateMon &h = b->nets[i]->stmons[r];
            const int64_t rows = out[i * K + 1 + ms + r], w = (int64_t)h.idx.size();
            for (int64_t q = 0; q < rows; ++q) {
                for (int64_t j = 0; j < w; ++j) h.vals.push_back((double)vals[p++]);
                const long long ps = h.start + (h.rows_done + q) * h.timestep;
                h.steps.push_back(ps + off[i]);
            }
            h.rows_done += rows;
        }
    return BG_OK;
}

template <typename T>
int batch_run_impl(bg_batch *b, const int64_t *nsteps, const int64_t *cs0) {
    const size_t nn = b->nets.size();
    std::vector<int64_t> left(nsteps, nsteps + nn), t0(nn);
    std::vector<long long> off(nn);
    for (size_t i = 0; i < nn; ++i) {
        if (left[i] < 0) return fail(BG_EINVAL, "negative step count");
        if (b->nets[i]->nstep + left[i] >= (1ll << 31) - 1) return fail(BG_EINVAL, "a network runs at most 2^31-1 steps");
        off[i] = cs0[i] - b->nets[i]->nstep;
    }
    double total_ms = 0;
    std::vector<int32_t> out;
    for (;;) {
        bool any = false;
        for (size_t i = 0; i < nn; ++i) any |= left[i] > 0;
        if (!any) break;
        std::vector<int64_t> want(nn);
        for (size_t i = 0; i < nn; ++i) { want[i] = std::min<int64_t>(left[i], (int64_t)1 << 30); t0[i] = b->nets[i]->nstep; }
        float ms = 0;
        int st = batch_launch<T>(b, want, 0, &out, &ms);
        if (st) return st;
        total_ms += ms;
        bool progress = false;
        for (size_t i = 0; i < nn; ++i) {
            const int32_t ran = out[i * bg::kBatchOut];
            if (ran < 0 || ran > want[i]) return fail(BG_ESTATE, "batch launch reported a bad step count");
            progress |= ran > 0 || want[i] == 0;
        }
        st = batch_collect<T>(b, out, t0, off);
        if (st) return st;
        for (size_t i = 0; i < nn; ++i) {
            const int32_t ran = out[i * bg::kBatchOut];
            b->nets[i]->nstep += ran;
            b->nets[i]->launches += want[i] > 0 ? 1 : 0;
            left[i] -= ran;
        }
        if (!progress) return fail(BG_ESTATE, "batch launch made no progress");
    }
    // the networks' own monitor bookkeeping follows (a later run alone
    // writes its rows after the ones taken here)
    for (bg_net *n : b->nets) {
        for (HStateMon &m : n->stmons) BG_CUDA(cudaMemcpy(m.dRowBase, &m.rows_done, 8, cudaMemcpyHostToDevice));
        n->last_ms = total_ms;
    }
    b->last_ms = total_ms;
    return BG_OK;
}

// Shapes whose blocks hold the largest network and whose instance takes the layout.
std::vector<int> batch_shapes(bg_batch *b) {
    std::vector<int> v;
    for (int sh = 0; sh < bg::kBatchNumShapes; ++sh)
        if (bg::kBatchShapes[sh].threads * bg::kBatchShapes[sh].npt >= b->max_n &&
            bg_batch_prepare_shape(b->precision, b->nvar, sh, b->smem) > 0)
            v.push_back(sh);
    return v;
}

int batch_snapshot(bg_batch *b, bool restore) {
    for (size_t k = 0; k < b->snap.size(); ++k) {
        uint16_t *ring = b->snap[k].first, *copy = b->snap[k].second;
        BG_CUDA(cudaMemcpyAsync(restore ? ring : copy, restore ? copy : ring, b->snap_bytes[k], cudaMemcpyDeviceToDevice, b->stream));
    }
    BG_CUDA(cudaStreamSynchronize(b->stream));
    return BG_OK;
}

}  // namespace

extern "C" {

int bg_batch_create(bg_net *const *nets, int32_t count, bg_batch **out) {
    if (!nets || count <= 0 || !out) return fail(BG_EINVAL, "bg_batch_create");
    *out = nullptr;
    for (int32_t i = 0; i < count; ++i) {
        if (!nets[i]) return fail(BG_EINVAL, "null network");
        for (int32_t k = 0; k < i; ++k) if (nets[k] == nets[i]) return fail(BG_EINVAL, "a network appears twice in the batch");
        if (nets[i]->device != nets[0]->device || nets[i]->precision != nets[0]->precision)
            return fail(BG_EINVAL, "the networks of a batch share the device and the precision");
        if (!nets[i]->prepared) { int st = bg_net_prepare(nets[i]); if (st) return st; }
        const std::string why = batch_refusal(nets[i]);
        if (!why.empty()) return fail(BG_ENOSYS, "network " + std::to_string(i) + ": " + why);
        if (nets[i]->groups[0].nvar != nets[0]->groups[0].nvar) return fail(BG_EINVAL, "the networks of a batch share the number of state variables");
    }
    BG_CUDA(cudaSetDevice(nets[0]->device));
    std::unique_ptr<bg_batch> b(new bg_batch());
    b->nets.assign(nets, nets + count);
    b->device = nets[0]->device; b->precision = nets[0]->precision; b->nvar = nets[0]->groups[0].nvar;
    BG_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BG_CUDA(cudaEventCreate(&b->ev0));
    BG_CUDA(cudaEventCreate(&b->ev1));
    const size_t ts = b->precision == 64 ? 8 : 4;
    // shared-memory layout of each network (32-bit words): staged row starts,
    // StateMonitor columns, then the rings -- a Connection's single row
    // always, a DelayConnection's rows while the block stays under the budget
    const int64_t kBudget = 100 * 1024 / 4;
    int64_t ntot_s = 0, ntot_w = 0;
    for (bg_net *n : b->nets) { ntot_s += (int64_t)n->smons.size(); for (auto &m : n->stmons) ntot_w += (int64_t)m.idx.size(); }
    for (int c = 0; c < bg::kBatchMaxConn; ++c) { b->smem_ring[c].assign(count, -1); b->smem_rows[c].assign(count, 0); b->packed[c].assign(count, nullptr); }
    b->smem_pos.assign(count, 0);
    b->sreg.assign((size_t)count * bg::kBatchMaxSmon, 0); b->scap.assign((size_t)count * bg::kBatchMaxSmon, 0);
    b->rreg.assign((size_t)count * bg::kBatchMaxRec, 0); b->rcap.assign((size_t)count * bg::kBatchMaxRec, 0);
    int64_t maxw = 0, nreg = 0;
    const int64_t scap_all = std::max<int64_t>(1024, std::min<int64_t>(1 << 16, ((int64_t)1 << 25) / std::max<int64_t>(1, ntot_s)));
    const int64_t rcap_all = std::max<int64_t>(1, std::min<int64_t>(4096, ((int64_t)1 << 25) / std::max<int64_t>(1, ntot_w)));
    for (int32_t i = 0; i < count; ++i) {
        bg_net *n = b->nets[i];
        const HGroup &g = n->groups[0];
        b->max_n = std::max<int>(b->max_n, (int)g.n);
        int64_t w = 0;
        for (size_t c = 0; c < n->conns.size(); ++c) {
            HConn &hc = n->conns[c];
            if (hc.rowptr[hc.sn] - hc.rowptr[0] >= ((int64_t)1 << 32)) return fail(BG_ENOSYS, "more than 2^32 synapses in one connection");
            if (hc.tn > (1 << 24)) return fail(BG_ENOSYS, "target range above 2^24");
            b->smem_rows[c][i] = (int32_t)w; w += hc.sn + 1;
            // packed synapse words (delay 0 for a Connection)
            uint32_t *pk = nullptr;
            if (b->alloc(&pk, std::max<int64_t>(1, hc.nnz) * 4) != cudaSuccess) return fail(BG_ENOMEM, "batch synapses");
            if (hc.nnz > 0) {
                const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((hc.nnz + 255) / 256, (int64_t)sm_count() * 8));
                k_pack_synapses<<<grid, 256, 0, b->stream>>>(hc.dCols, batch_direct(hc) ? nullptr : hc.dD, hc.nnz, pk);
                BG_CUDA(cudaGetLastError());
            }
            b->packed[c][i] = pk;
            if (batch_direct(hc)) {
                int64_t kmax = 0;
                int st = max_indegree(n, hc, &kmax);
                if (st) return st;
                if (kmax >= 65535) return fail(BG_ENOSYS, "in-degree above 65534 (16-bit counts)");
            }
        }
        b->smem_pos[i] = (int32_t)w; w += (int64_t)n->stmons.size() * ((g.n + 1) / 2);
        for (size_t c = 0; c < n->conns.size(); ++c) {        // Connections: two rows (step parity)
            const HConn &hc = n->conns[c];
            if (!batch_direct(hc)) continue;
            b->smem_ring[c][i] = (int32_t)w; w += (hc.tn + 1) & ~1ll;
        }
        for (size_t c = 0; c < n->conns.size(); ++c) {        // DelayConnections: md rows, if they fit
            const HConn &hc = n->conns[c];
            if (batch_direct(hc)) continue;
            const int64_t rw = (int64_t)hc.md * hc.tnp / 2;
            if (w + rw <= kBudget) { b->smem_ring[c][i] = (int32_t)w; w += rw; }
            else {
                uint16_t *copy = nullptr;
                const size_t bytes = (size_t)hc.md * hc.tnp * 2;
                if (b->alloc(&copy, bytes) != cudaSuccess) return fail(BG_ENOMEM, "batch ring copy");
                b->snap.push_back({hc.dCRing, copy}); b->snap_bytes.push_back(bytes);
            }
        }
        maxw = std::max(maxw, w);
        for (size_t m = 0; m < n->smons.size(); ++m) {
            b->sreg[i * bg::kBatchMaxSmon + m] = b->nsrec;
            const int64_t cap = std::max<int64_t>(n->smons[m].n, scap_all);
            b->scap[i * bg::kBatchMaxSmon + m] = (int32_t)cap;
            b->nsrec += cap; ++nreg;
        }
        for (size_t r = 0; r < n->stmons.size(); ++r) {
            b->rreg[i * bg::kBatchMaxRec + r] = b->nrval;
            b->rcap[i * bg::kBatchMaxRec + r] = (int32_t)rcap_all;
            b->nrval += rcap_all * (int64_t)n->stmons[r].idx.size(); ++nreg;
        }
    }
    b->smem = (size_t)maxw * 4;
    if (b->nsrec > ((int64_t)1 << 31) || b->nrval > ((int64_t)1 << 31)) return fail(BG_ENOSYS, "batch monitor buffers above 2^31 entries");
    b->gather_cap = 3 * std::max<int64_t>(1, nreg);
    if (b->alloc(&b->dNets, (size_t)count * std::max(sizeof(bg::BatchNet<double>), sizeof(bg::BatchNet<float>))) != cudaSuccess ||
        b->alloc(&b->dOrder, (size_t)count * 4) != cudaSuccess ||
        b->alloc(&b->dOut, (size_t)count * bg::kBatchOut * 4) != cudaSuccess ||
        b->alloc(&b->dSIdx, std::max<int64_t>(1, b->nsrec) * 4) != cudaSuccess ||
        b->alloc(&b->dSStep, std::max<int64_t>(1, b->nsrec) * 4) != cudaSuccess ||
        b->alloc(&b->dCIdx, std::max<int64_t>(1, b->nsrec) * 4) != cudaSuccess ||
        b->alloc(&b->dCStep, std::max<int64_t>(1, b->nsrec) * 4) != cudaSuccess ||
        b->alloc(&b->dRows, std::max<int64_t>(1, b->nrval) * ts) != cudaSuccess ||
        b->alloc(&b->dCRows, std::max<int64_t>(1, b->nrval) * ts) != cudaSuccess ||
        b->alloc(&b->dGather, b->gather_cap * 8) != cudaSuccess)
        return fail(BG_ENOMEM, "batch buffers");
    BG_CUDA(cudaStreamSynchronize(b->stream));
    // default shape: the most threads among the shapes that hold the largest network
    std::vector<int> ok = batch_shapes(b.get());
    if (ok.empty()) return fail(BG_ENOSYS, "no block shape takes the batch's shared-memory layout");
    b->shape = ok.back();
    for (int sh : ok) if (bg::kBatchShapes[sh].threads > bg::kBatchShapes[b->shape].threads) b->shape = sh;
    b->lanes = 32;
    // every network's earlier work is finished before the batch's stream uses its state
    for (bg_net *n : b->nets) BG_CUDA(cudaStreamSynchronize(n->stream));
    *out = b.release();
    return BG_OK;
}

int bg_batch_free(bg_batch *b) {
    if (!b) return fail(BG_EINVAL, "batch");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    delete b;
    return BG_OK;
}

int bg_batch_run(bg_batch *b, const int64_t *nsteps, const int64_t *cs0) {
    if (!b || !nsteps || !cs0) return fail(BG_EINVAL, "bg_batch_run");
    BG_CUDA(cudaSetDevice(b->device));
    for (bg_net *n : b->nets) {
        if (n->failed) return fail(BG_ESTATE, "a network of the batch stopped after a device error");
        BG_CUDA(cudaStreamSynchronize(n->stream));
    }
    return b->precision == 64 ? batch_run_impl<double>(b, nsteps, cs0) : batch_run_impl<float>(b, nsteps, cs0);
}

int bg_batch_set_shape(bg_batch *b, int32_t shape, int32_t lanes) {
    if (!b) return fail(BG_EINVAL, "batch");
    if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) return fail(BG_EINVAL, "lanes per spike row: 4, 8, 16 or 32");
    std::vector<int> ok = batch_shapes(b);
    if (std::find(ok.begin(), ok.end(), shape) == ok.end()) return fail(BG_EINVAL, "block shape does not hold the batch");
    b->shape = shape; b->lanes = lanes;
    return BG_OK;
}

int bg_batch_get_shape(bg_batch *b, int32_t *shape, int32_t *threads, int32_t *npt, int32_t *lanes) {
    if (!b || b->shape < 0) return fail(BG_EINVAL, "batch");
    if (shape) *shape = b->shape;
    if (threads) *threads = bg::kBatchShapes[b->shape].threads;
    if (npt) *npt = bg::kBatchShapes[b->shape].npt;
    if (lanes) *lanes = b->lanes;
    return BG_OK;
}

int bg_batch_autotune(bg_batch *b, int32_t steps, double *best_ms) {
    if (!b || steps <= 0) return fail(BG_EINVAL, "bg_batch_autotune");
    BG_CUDA(cudaSetDevice(b->device));
    for (bg_net *n : b->nets) BG_CUDA(cudaStreamSynchronize(n->stream));
    std::vector<int64_t> want(b->nets.size(), steps);
    const int keep_shape = b->shape, keep_lanes = b->lanes;
    double best = -1;
    int bs = keep_shape, bl = keep_lanes;
    int st = batch_snapshot(b, false);
    if (st) return st;
    for (int sh : batch_shapes(b)) {
        for (int lanes : {4, 8, 16, 32}) {
            b->shape = sh; b->lanes = lanes;
            float ms = 0;
            for (int rep = 0; rep < 2 && st == BG_OK; ++rep) {      // warm-up, then timed
                st = b->precision == 64 ? batch_launch<double>(b, want, 1, nullptr, &ms) : batch_launch<float>(b, want, 1, nullptr, &ms);
                if (st == BG_OK) st = batch_snapshot(b, true);      // dry runs still push into rings kept in global memory
            }
            if (st) { b->shape = keep_shape; b->lanes = keep_lanes; return st; }
            if (best < 0 || ms < best) { best = ms; bs = sh; bl = lanes; }
        }
    }
    b->shape = bs; b->lanes = bl;
    if (best_ms) *best_ms = best;
    return BG_OK;
}

int bg_batch_stats(bg_batch *b, int64_t *launches, double *ms) {
    if (!b) return fail(BG_EINVAL, "batch");
    if (launches) *launches = b->launches;
    if (ms) *ms = b->last_ms;
    return BG_OK;
}

}  // extern "C"
