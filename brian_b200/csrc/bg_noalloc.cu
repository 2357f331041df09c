// bg_noalloc.cu -- an entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running inside another
// framework's memory pool (its caching allocator owns the device memory and
// a cudaMalloc behind its back can fail or fragment it), or a process whose
// device memory is fully reserved up front.  bg_delay_group_run_noalloc runs
// the same fused update / delayed push kernel as the network engine (k_head)
// for one linear group with
// shared-weight DelayConnections onto itself, with every scratch buffer --
// control block, spike history, count rings, k-fold-sum tables -- carved out
// of one file-scope device array of fixed size.  The caller owns and passes
// the inputs (connection rows, delays) and the in/out state.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "bg_kernels.cuh"
#include "../../include/brian_b200.h"

namespace {

// Scratch of the allocation-free entry point.  Lives for the process on every
// device that loads this library; shared by all calls (see the header).
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;   // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
constexpr int kNoAllocMaxConn = 4;
constexpr int kTableLen = 65536;           // counts stay below 65535

std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kNoAllocMaxDevices] = {nullptr};

int fail(int code, const std::string &m) { return bg_internal_fail(code, m.c_str()); }

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Row pointers of one connection: rowptr[0] >= 0, non-decreasing, every row
// shorter than 2^31 entries.  Runs (and its flag is read on the host) before
// any kernel walks the rows, so a malformed rowptr never drives a read of
// cols or delays outside the rows it claims.
__global__ void k_rowcheck(const int64_t *rowptr, int64_t sn, DevCtl *ctl) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < sn; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = rowptr[i], b = rowptr[i + 1];
        if ((i == 0 && a < 0) || b < a || b - a >= (int64_t(1) << 31)) bg_raise(ctl, BG_DERR_RANGE, i);
    }
    if (sn == 0 && blockIdx.x == 0 && threadIdx.x == 0 && rowptr[0] < 0) bg_raise(ctl, BG_DERR_RANGE, 0);
}

// In-degree histogram of one connection, with range checks of the caller's
// rows (targets in [0, n), delays below the ring depth).
__global__ void k_indegree(const int64_t *rowptr, int64_t sn, const int32_t *cols, const uint8_t *d, int64_t n,
                           int depth, unsigned int *hist, DevCtl *ctl) {
    const int64_t k0 = rowptr[0], k1 = rowptr[sn];
    for (int64_t k = k0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < k1; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = cols[k];
        if (c < 0 || c >= n || d[k] >= depth) { bg_raise(ctl, BG_DERR_RANGE, k); continue; }
        atomicAdd(hist + c, 1u);
    }
}

// Largest count, then table[k] = table[k-1] + w, the value a reference ring
// entry reaches after k additions of the shared weight.
__global__ void k_count_table(const unsigned int *hist, int64_t n, double w, double *table, DevCtl *ctl) {
    __shared__ unsigned int mx;
    if (threadIdx.x == 0) mx = 0;
    __syncthreads();
    unsigned int m = 0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) m = max(m, hist[j]);
    atomicMax(&mx, m);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (mx >= (unsigned int)(kTableLen - 1)) { bg_raise(ctl, BG_DERR_RANGE, mx); return; }
        double acc = 0.0;
        table[0] = 0.0;
        for (unsigned int k = 1; k <= mx; ++k) { acc = __dadd_rn(acc, w); table[k] = acc; }
    }
}

template <int NV>
cudaError_t launch(const bg::HeadArgs<double> &a, unsigned int blocks, cudaStream_t s) {
    bg::k_head<double, NV><<<blocks, bg::kHeadThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_nv(const bg::HeadArgs<double> &a, int nvar, unsigned int blocks, cudaStream_t s) {
    switch (nvar) {
    case 1: return launch<1>(a, blocks, s);
    case 2: return launch<2>(a, blocks, s);
    case 3: return launch<3>(a, blocks, s);
    default: return launch<4>(a, blocks, s);
    }
}

// Device address of the scratch array for the current device: looked up
// once per device (cudaGetSymbolAddress), then reused for the life of the
// process.  A cudaDeviceReset unloads the module and may move the array, so
// the entry point must not be called on a device after the caller reset it.
int scratch_for_current_device(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(BG_EINVAL, "device index beyond the supported range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(BG_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_ptr[dev];
    return BG_OK;
}

}  // namespace

extern "C" {

BG_API int bg_noalloc_scratch_bytes(int64_t *bytes) {
    if (!bytes) return BG_EINVAL;
    *bytes = (int64_t)kNoAllocScratchBytes;
    return BG_OK;
}

BG_API int bg_delay_group_run_noalloc(int64_t n, int nvar, double *S, const double *A, const double *C, int thr_var,
                                      double thr_val, int reset_var, double reset_val, int nconn,
                                      const int64_t *src_origin, const int64_t *src_n, const int *tgt_var,
                                      const int64_t *const *rowptr, const int32_t *const *cols,
                                      const uint8_t *const *delays, const double *weight, const int32_t *ring_depth,
                                      int64_t nsteps, void *stream, int64_t *spikes_out) {
    // ---- arguments (host side; device rows are range-checked on the device)
    if (n <= 0 || n > (int64_t(1) << 30) || nvar < 1 || nvar > 4 || !S || !A) return fail(BG_EINVAL, "group arguments");
    if (thr_var < 0 || thr_var >= nvar || reset_var < 0 || reset_var >= nvar) return fail(BG_EINVAL, "threshold/reset variable");
    if (nconn < 0 || nconn > kNoAllocMaxConn) return fail(BG_EINVAL, "at most 4 connections");
    if (nconn && (!src_origin || !src_n || !tgt_var || !rowptr || !cols || !delays || !weight || !ring_depth))
        return fail(BG_EINVAL, "connection arrays");
    if (nsteps < 0 || nsteps >= (int64_t(1) << 31) - 1) return fail(BG_EINVAL, "nsteps");
    for (int c = 0; c < nconn; ++c) {
        if (src_origin[c] < 0 || src_n[c] < 0 || src_origin[c] + src_n[c] > n) return fail(BG_EINVAL, "source range");
        if (tgt_var[c] < 0 || tgt_var[c] >= nvar) return fail(BG_EINVAL, "target variable");
        if (ring_depth[c] < 1 || ring_depth[c] > 255) return fail(BG_EINVAL, "ring depth must be in [1, 255]");
        if (!rowptr[c] || !cols[c] || !delays[c]) return fail(BG_EINVAL, "connection pointers");
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *scr = nullptr;
    int st = scratch_for_current_device(&scr);
    if (st) return st;
    // ---- scratch layout
    const int64_t nblocks = (n + bg::kBlockNeurons - 1) / bg::kBlockNeurons;
    const int64_t nwords = nblocks * (bg::kBlockNeurons / 32);
    const int64_t tnp = (n + 1) & ~int64_t(1);
    size_t off = 0;
    const size_t o_ctl = off; off = align256(off + sizeof(DevCtl));
    const size_t o_cnt = off; off = align256(off + sizeof(unsigned long long) * (1 + kNoAllocMaxConn));
    const size_t o_hist = off; off = align256(off + sizeof(uint32_t) * nwords);
    const size_t o_deg = off; off = align256(off + sizeof(unsigned int) * n);
    size_t o_tab[kNoAllocMaxConn], o_ring[kNoAllocMaxConn];
    for (int c = 0; c < nconn; ++c) { o_tab[c] = off; off = align256(off + sizeof(double) * kTableLen); }
    for (int c = 0; c < nconn; ++c) { o_ring[c] = off; off = align256(off + sizeof(uint16_t) * (ring_depth[c] + 2) * tnp); }
    if (off > kNoAllocScratchBytes)
        return fail(BG_EINVAL, "network needs " + std::to_string(off) + " bytes of scratch; the allocation-free entry "
                    "point has " + std::to_string(kNoAllocScratchBytes));
    DevCtl *ctl = (DevCtl *)(scr + o_ctl);
    unsigned long long *cnt = (unsigned long long *)(scr + o_cnt);
    // every call starts from cleared control block, counters, history and rings
    cudaError_t e = cudaMemsetAsync(scr, 0, off, s);
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("clear scratch: ") + cudaGetErrorString(e));
    DevCtl h;
    // ---- the caller's row pointers, checked before anything walks the rows
    for (int c = 0; c < nconn; ++c) {
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((src_n[c] + 255) / 256, 1184));
        k_rowcheck<<<grid, 256, 0, s>>>(rowptr[c], src_n[c], ctl);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(BG_ECUDA, cudaGetErrorString(e));
    }
    if ((e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(BG_ECUDA, cudaGetErrorString(e));
    if (h.err) return fail(BG_EINVAL, "connection rows: rowptr negative, decreasing or a row of 2^31 entries or "
                           "more (row " + std::to_string(h.err_info) + ")");
    // ---- count tables (one in-degree histogram per connection)
    for (int c = 0; c < nconn; ++c) {
        unsigned int *deg = (unsigned int *)(scr + o_deg);
        if ((e = cudaMemsetAsync(deg, 0, sizeof(unsigned int) * n, s)) != cudaSuccess)
            return fail(BG_ECUDA, cudaGetErrorString(e));
        k_indegree<<<296, 256, 0, s>>>(rowptr[c], src_n[c], cols[c], delays[c], n, ring_depth[c], deg, ctl);
        k_count_table<<<1, 1024, 0, s>>>(deg, n, weight[c], (double *)(scr + o_tab[c]), ctl);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(BG_ECUDA, cudaGetErrorString(e));
    }
    if ((e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(BG_ECUDA, cudaGetErrorString(e));
    if (h.err) return fail(BG_EINVAL, "connection rows: target, delay or in-degree out of range (entry " +
                           std::to_string(h.err_info) + ")");
    // ---- the step loop: the network engine's fused head kernel
    bg::HeadArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = ctl; a.S = S; a.n = n; a.npad = n; a.nvar = nvar;   // caller's rows have stride n
    a.linear = 1; a.useC = C != nullptr;
    for (int j = 0; j < nvar; ++j) {
        for (int k = 0; k < nvar; ++k) a.A[j * nvar + k] = A[j * nvar + k];
        a.C[j] = C ? C[j] : 0.0;
    }
    bg::set_linear_masks(a, nvar);
    a.thr_kind = BG_THR_CONST; a.thr_var = thr_var; a.thr_val = thr_val;
    a.reset_kind = BG_RESET_CONST; a.reset_var = reset_var; a.reset_val = reset_val;
    a.hist = (uint32_t *)(scr + o_hist); a.depth = 1; a.nwords = nwords;
    a.ndeliv = nconn; a.npush = nconn;
    for (int c = 0; c < nconn; ++c) {
        bg::Deliv<double> &dv = a.deliv[c];
        dv.ring = nullptr; dv.tn = n; dv.to = 0; dv.md = ring_depth[c] + 2; dv.var = tgt_var[c];
        dv.cring = (uint16_t *)(scr + o_ring[c]); dv.tnp = tnp; dv.table = (const double *)(scr + o_tab[c]);
        bg::Push<double> &q = a.push[c];
        q.ring = nullptr; q.md = ring_depth[c] + 2; q.so = src_origin[c]; q.sn = src_n[c]; q.tn = n;
        q.rowptr = rowptr[c]; q.cols = cols[c]; q.w = nullptr; q.w_bits = 64; q.d = delays[c];
        q.events = cnt + 1 + c; q.cring = dv.cring; q.tnp = tnp;
    }
    a.spikes = cnt;
    for (int64_t k = 0; k < nsteps; ++k) {
        a.tail = k > 0; a.update = 1; a.last = 1;
        if ((e = launch_nv(a, nvar, (unsigned)nblocks, s)) != cudaSuccess) return fail(BG_ECUDA, cudaGetErrorString(e));
    }
    if (nsteps > 0) {   // deliveries and resets of the last step
        a.tail = 1; a.update = 0; a.last = 0;
        if ((e = launch_nv(a, nvar, (unsigned)nblocks, s)) != cudaSuccess) return fail(BG_ECUDA, cudaGetErrorString(e));
    }
    unsigned long long spikes = 0;
    if ((e = cudaMemcpyAsync(&spikes, cnt, sizeof(spikes), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(BG_ECUDA, cudaGetErrorString(e));
    if (h.err) return fail(BG_ESTATE, "device error " + std::to_string(h.err));
    if (spikes_out) *spikes_out = (int64_t)spikes;
    return BG_OK;
}

}  // extern "C"
