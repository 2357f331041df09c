// bg_batch.cuh -- many independent small networks in one launch, one thread
// block per network (the batched form of Network.run).
//
// A network here is what the persistent kernel runs (one linear group, its
// shared-weight Connections / DelayConnections onto itself, undelayed spike
// monitors and StateMonitors) with at most kBatchMaxNeurons neurons, so one
// block holds all of it: the state in registers, the staged row starts and
// the count rings in shared memory.  A step needs no grid-wide wait -- only
// the block's own barriers -- and the networks of a launch run at their own
// pace, each for its own number of steps (uneven durations: a block whose
// network is done exits and the hardware schedules the next one).
//
// Step t of a network, in the reference's order (network.py:403-430):
//   update (x = A s + C, ascending terms, zero coefficients skipped) ->
//   threshold -> spike list (ascending) and spike-monitor records ->
//   push of the spikes into the count rings -> delivery of the rows due at
//   t: the Connections first (w added once per event), then the
//   DelayConnections (the k-fold sum 0 + w + ... + w added once) -> reset
//   -> StateMonitor records.
// The ring layout and row mapping (a push of step s with delay d lands in
// row (s + d) mod md) are the engine's, so a DelayConnection's rows are
// loaded from and saved to the engine's own count ring around a launch, or
// used in place when they do not fit in shared memory.
#pragma once
#include "bg_kernels.cuh"
#include "../../include/brian_b200.h"

namespace bg {

constexpr int kBatchMaxConn = 2;
constexpr int kBatchMaxSmon = 2;
constexpr int kBatchMaxRec = 4;
constexpr int kBatchMaxNeurons = 4096;
constexpr int kBatchOut = 1 + kBatchMaxSmon + kBatchMaxRec;   // per-network launch outputs

template <typename T> struct BatchConn {
    int32_t so, sn, to, tn;     // source and target ranges in the group
    int32_t var;                // target variable
    int32_t direct;             // 1: Connection (w added per event); 0: DelayConnection
    int32_t md, tnp;            // ring rows, row stride (entries, even)
    int32_t smem_ring;          // ring offset in dynamic shared memory (32-bit words), -1: global
    int32_t smem_rows;          // offset of the staged row starts (sn + 1 words)
    T w;                        // the shared weight
    const int64_t *rowptr;      // CSR row starts (sn + 1)
    const uint32_t *packed;     // target | delay << 24 per synapse
    uint16_t *ring;             // the engine's count ring (md x tnp); null for a Connection
};
struct BatchSmon {              // spike monitor of the range [origin, origin + n)
    int32_t origin, n, cap;
    int32_t *idx, *step;        // records of the launch: index - origin, launch-relative step
};
struct BatchRec {               // StateMonitor of variable var on nidx neurons every timestep steps
    int32_t var, nidx, timestep, cap_rows;
    long long start;            // first recorded engine step
    long long row0;             // records already taken before this launch
    const int32_t *idx, *pos;   // recorded neurons ascending, and their columns in a row
    void *buf;                  // rows of the launch (cap_rows x nidx of T)
};
template <typename T> struct BatchNet {
    T A[16], C[4]; uint64_t anz; uint32_t cnz;   // A row-major with stride NV
    int32_t thr_kind, thr_var, thr_var2; T thr_val;
    int32_t reset_kind, reset_var, reset_var2; T reset_val;
    T *S; int64_t npad; int32_t n;
    int32_t nconn, ndeliv; int32_t deliv[kBatchMaxConn];   // delivery order (connection indices)
    BatchConn<T> conn[kBatchMaxConn];
    int32_t nsmon; BatchSmon smon[kBatchMaxSmon];
    int32_t nrec; BatchRec rec[kBatchMaxRec];
    int32_t smem_sl, smem_stash;                 // offsets (32-bit words) of the spike list and the record stash (n entries each)
    DevCtl *ctl; unsigned long long *counters;   // spikes of the group, then events per connection
    long long t0; int32_t nsteps;                // engine step at the launch, steps asked for
    int32_t *out;                                // [kBatchOut]: steps run, records per spike monitor, rows per StateMonitor
};

template <typename T, int NV, int TH, int NPT>
__global__ void __launch_bounds__(TH) k_batch(const BatchNet<T> *nets, const int32_t *order, int lanes, int dry) {
    constexpr int BN = TH * NPT;
    static_assert(BN <= kBatchMaxNeurons && BN % 32 == 0, "block shape");
    extern __shared__ __align__(16) uint32_t bsm[];
    __shared__ T sA[16], sC[4];
    __shared__ uint32_t words[BN / 32];
    __shared__ int nspk, bnd[2 * (kBatchMaxConn + kBatchMaxSmon)];
    const BatchNet<T> &N = nets[order[blockIdx.x]];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = N.n, nsteps = N.nsteps;
    if (nsteps <= 0) {                                       // uniform
        if (tid == 0 && !dry) for (int k = 0; k < kBatchOut; ++k) N.out[k] = 0;
        return;
    }
    if (tid < NV * NV) sA[tid] = N.A[tid];
    if (tid < NV) sC[tid] = N.C[tid];
    // ring rows of the current step: per connection (pushes) and per
    // delivery slot (the same rows, in delivery order)
    int64_t r00[kBatchMaxConn];
    int cur[kBatchMaxConn], dcur[kBatchMaxConn];
#pragma unroll
    for (int c = 0; c < kBatchMaxConn; ++c) {
        r00[c] = 0; cur[c] = 0; dcur[c] = 0;
        if (c < N.ndeliv) dcur[c] = (int)(N.t0 % N.conn[N.deliv[c]].md);
        if (c >= N.nconn) continue;
        const BatchConn<T> &q = N.conn[c];
        r00[c] = q.rowptr[0];
        cur[c] = (int)(N.t0 % q.md);
        uint32_t *rows = bsm + q.smem_rows;
        for (int j = tid; j <= q.sn; j += TH) rows[j] = (uint32_t)(q.rowptr[j] - r00[c]);
        if (q.smem_ring >= 0) {
            uint32_t *r = bsm + q.smem_ring;
            const int nw = q.md * q.tnp / 2;
            const uint32_t *g = reinterpret_cast<const uint32_t *>(q.ring);
            for (int k = tid; k < nw; k += TH) r[k] = q.direct ? 0u : g[k];
        }
    }
    T s[NPT][NV];
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
        const int li = u * TH + tid;
#pragma unroll
        for (int k = 0; k < NV; ++k) s[u][k] = li < n ? N.S[k * N.npad + li] : T(0);
    }
    int32_t *sl = reinterpret_cast<int32_t *>(bsm + N.smem_sl);
    T *stash = reinterpret_cast<T *>(bsm + N.smem_stash);
    int scnt[kBatchMaxSmon] = {0, 0};
    int rrows[kBatchMaxRec] = {0, 0, 0, 0};
    unsigned long long my_spikes = 0, my_events[kBatchMaxConn] = {0, 0};
    const int group = tid / lanes, gl = tid - group * lanes, ngroups = TH / lanes;
    __syncthreads();

    int st = 0;
    for (; st < nsteps; ++st) {
        const long long t = N.t0 + st;
        // a monitor buffer that might not hold this step's records ends the
        // launch before the step (every thread decides alike)
        if (!dry) {
            bool full = false;
#pragma unroll
            for (int m = 0; m < kBatchMaxSmon; ++m) full |= m < N.nsmon && scnt[m] + N.smon[m].n > N.smon[m].cap;
#pragma unroll
            for (int r = 0; r < kBatchMaxRec; ++r) {
                if (r >= N.nrec) break;
                const long long rel = t - N.rec[r].start;
                full |= rel >= 0 && rel % N.rec[r].timestep == 0 && rrows[r] >= N.rec[r].cap_rows;
            }
            if (full) break;
        }
        // ---- update: each row of A s (+ C) summed over k ascending with the
        // zero coefficients skipped (the order of linear_row)
#pragma unroll
        for (int u = 0; u < NPT; ++u) {
            T x[NV];
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                x[j] = T(0);
#pragma unroll
                for (int k = 0; k < NV; ++k)
                    if (N.anz & (1ull << (j * NV + k))) x[j] = rn<T>::add(x[j], rn<T>::mul(sA[j * NV + k], s[u][k]));
                if (N.cnz & (1u << j)) x[j] = rn<T>::add(x[j], sC[j]);
            }
#pragma unroll
            for (int j = 0; j < NV; ++j) s[u][j] = x[j];
        }
        // ---- threshold
        uint32_t spk = 0;
#pragma unroll
        for (int u = 0; u < NPT; ++u) {
            const int li = u * TH + tid;
            bool f = false;
            if (N.thr_kind == BG_THR_CONST) f = uget<T, NV>(s[u], N.thr_var) > N.thr_val;
            else if (N.thr_kind == BG_THR_VAR) f = uget<T, NV>(s[u], N.thr_var) > uget<T, NV>(s[u], N.thr_var2);
            f = f && li < n;
            spk |= (f ? 1u : 0u) << u;
            const uint32_t ball = __ballot_sync(0xffffffffu, f);
            if (lane == 0) { words[u * (TH / 32) + warp] = ball; my_spikes += __popc(ball); }
        }
        __syncthreads();
        // ---- spike list, ascending (warp 0), and its ranges per connection
        // source and per spike monitor
        if (warp == 0) {
            int acc = 0;
#pragma unroll
            for (int c0 = 0; c0 < BN / 32; c0 += 32) {
                uint32_t w = c0 + lane < BN / 32 ? words[c0 + lane] : 0u;
                const int c = __popc(w);
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += v; }
                int off = acc + incl - c;
                while (w) { const int b = __ffs(w) - 1; w &= w - 1; sl[off++] = (c0 + lane) * 32 + b; }
                acc += __shfl_sync(0xffffffffu, incl, 31);
            }
            __syncwarp();
            // first list position >= v, by lanes 0.. (one range end each)
            auto lower = [&](int v) { int lo = 0, hi = acc; while (lo < hi) { const int m = (lo + hi) >> 1; if (sl[m] < v) lo = m + 1; else hi = m; } return lo; };
            const int nb = 2 * (N.nconn + N.nsmon);
            if (lane < nb) {
                const int k = lane >> 1;
                int v;
                if (k < N.nconn) v = (lane & 1) ? N.conn[k].so + N.conn[k].sn : N.conn[k].so;
                else { const BatchSmon &m = N.smon[k - N.nconn]; v = (lane & 1) ? m.origin + m.n : m.origin; }
                bnd[lane] = lower(v);
            }
            if (lane == 0) nspk = acc;
        }
        __syncthreads();
        if (nspk) {                                          // uniform
            if (!dry) {
#pragma unroll
                for (int m = 0; m < kBatchMaxSmon; ++m) {
                    if (m >= N.nsmon) break;
                    const BatchSmon &M = N.smon[m];
                    const int lo = bnd[2 * (N.nconn + m)], hi = bnd[2 * (N.nconn + m) + 1];
                    for (int e = lo + tid; e < hi; e += TH) {
                        M.idx[scnt[m] + e - lo] = sl[e] - M.origin;
                        M.step[scnt[m] + e - lo] = st;
                    }
                    scnt[m] += hi - lo;
                }
            }
            // ---- push: one group of `lanes` threads per spike row
#pragma unroll
            for (int c = 0; c < kBatchMaxConn; ++c) {
                if (c >= N.nconn) break;
                const BatchConn<T> &q = N.conn[c];
                const uint32_t *rows = bsm + q.smem_rows;
                const uint32_t *pk0 = q.packed + r00[c];
                uint32_t *sring = q.smem_ring >= 0 ? bsm + q.smem_ring : nullptr;
                const int lo = bnd[2 * c], hi = bnd[2 * c + 1];
                for (int e = lo + group; e < hi; e += ngroups) {
                    const int j = sl[e] - q.so;
                    const uint32_t k0 = rows[j], k1 = rows[j + 1];
                    if (gl == 0) my_events[c] += k1 - k0;
                    for (uint32_t k = k0 + gl; k < k1; k += 4u * lanes) {
                        uint32_t w4[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) w4[i] = k + i * lanes < k1 ? __ldg(pk0 + k + i * lanes) : 0xffffffffu;
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            if (w4[i] == 0xffffffffu) continue;
                            const int tgt = (int)(w4[i] & 0xffffffu);
                            const int r = cur[c] + (int)(w4[i] >> 24);
                            const int row = r >= q.md ? r - q.md : r;
                            if (sring) atomicAdd(sring + ((row * q.tnp + tgt) >> 1), 1u << ((tgt & 1) << 4));
                            else cring_add(q.ring + (int64_t)row * q.tnp, tgt);
                        }
                    }
                }
            }
            __syncthreads();
        }
        // ---- delivery of the rows due at step t, in the reference's order
#pragma unroll
        for (int di = 0; di < kBatchMaxConn; ++di) {
            if (di >= N.ndeliv) break;
            const BatchConn<T> &q = N.conn[N.deliv[di]];
            const int row = dcur[di];
            uint16_t *sr = q.smem_ring >= 0 ? reinterpret_cast<uint16_t *>(bsm + q.smem_ring) + row * q.tnp : nullptr;
            uint16_t *gr = q.ring ? q.ring + (int64_t)row * q.tnp : nullptr;
            const T w = q.w;
            on_var<NV>(q.var, [&](auto K) {
                constexpr int k = decltype(K)::value;
#pragma unroll
                for (int u = 0; u < NPT; ++u) {
                    const int li = u * TH + tid;
                    if (li < q.to || li >= q.to + q.tn) continue;
                    const int e = li - q.to;
                    const int cnt = sr ? sr[e] : __ldcg(gr + e);
                    if (!cnt) continue;
                    if (sr) sr[e] = 0; else gr[e] = 0;
                    if (q.direct) {
                        for (int i = 0; i < cnt; ++i) s[u][k] = rn<T>::add(s[u][k], w);
                    } else {
                        T v = T(0);
                        for (int i = 0; i < cnt; ++i) v = rn<T>::add(v, w);
                        s[u][k] = rn<T>::add(s[u][k], v);
                    }
                }
            });
        }
#pragma unroll
        for (int c = 0; c < kBatchMaxConn; ++c) {
            if (c < N.nconn) cur[c] = cur[c] + 1 == N.conn[c].md ? 0 : cur[c] + 1;
            if (c < N.ndeliv) dcur[c] = dcur[c] + 1 == N.conn[N.deliv[c]].md ? 0 : dcur[c] + 1;
        }
        // ---- reset
        if (N.reset_kind == BG_RESET_CONST) {
#pragma unroll
            for (int u = 0; u < NPT; ++u)
                if ((spk >> u) & 1u) uset<T, NV>(s[u], N.reset_var, N.reset_val);
        } else if (N.reset_kind == BG_RESET_VAR) {
#pragma unroll
            for (int u = 0; u < NPT; ++u)
                if ((spk >> u) & 1u) uset<T, NV>(s[u], N.reset_var, uget<T, NV>(s[u], N.reset_var2));
        }
        // ---- StateMonitors ('end' slot)
        if (!dry) {
#pragma unroll
            for (int r = 0; r < kBatchMaxRec; ++r) {
                if (r >= N.nrec) break;
                const BatchRec &R = N.rec[r];
                const long long rel = t - R.start;
                if (rel < 0 || rel % R.timestep) continue;       // uniform
#pragma unroll
                for (int u = 0; u < NPT; ++u)
                    if (u * TH + tid < n) stash[u * TH + tid] = uget<T, NV>(s[u], R.var);
                __syncthreads();
                T *dst = (T *)R.buf + (int64_t)rrows[r] * R.nidx;
                for (int e = tid; e < R.nidx; e += TH) dst[R.pos[e]] = stash[R.idx[e]];
                ++rrows[r];
                __syncthreads();
            }
        }
    }
    if (dry) return;
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
        const int li = u * TH + tid;
        if (li < n) {
#pragma unroll
            for (int k = 0; k < NV; ++k) N.S[k * N.npad + li] = s[u][k];
        }
    }
    // a DelayConnection's ring held in shared memory goes back to the engine's ring
    for (int c = 0; c < N.nconn; ++c) {
        const BatchConn<T> &q = N.conn[c];
        if (q.smem_ring < 0 || q.direct) continue;
        const uint32_t *r = bsm + q.smem_ring;
        uint32_t *g = reinterpret_cast<uint32_t *>(q.ring);
        for (int k = tid; k < q.md * q.tnp / 2; k += TH) g[k] = r[k];
    }
    block_count(N.counters, my_spikes);
#pragma unroll
    for (int c = 0; c < kBatchMaxConn; ++c)
        if (c < N.nconn) block_count(N.counters + 1 + c, my_events[c]);
    if (tid == 0) {
        N.out[0] = st;
#pragma unroll
        for (int m = 0; m < kBatchMaxSmon; ++m) N.out[1 + m] = scnt[m];
#pragma unroll
        for (int r = 0; r < kBatchMaxRec; ++r) N.out[1 + kBatchMaxSmon + r] = rrows[r];
        N.ctl->nstep = N.t0 + st;
    }
}

// Block shapes (threads x neurons per thread) the batch kernel is built for.
struct BatchShape { int threads, npt; };
constexpr BatchShape kBatchShapes[] = {{128, 4}, {256, 4}, {512, 4}, {512, 8}, {1024, 4}};
constexpr int kBatchNumShapes = (int)(sizeof(kBatchShapes) / sizeof(kBatchShapes[0]));

}  // namespace bg

// Launches k_batch<T, nvar, shape> over `blocks` networks (bg_batch.cu).
cudaError_t bg_batch_launch(int precision, int nvar, int shape, const void *nets, const int32_t *order, int blocks,
                            int lanes, int dry, size_t smem, cudaStream_t s);
// Largest dynamic shared memory of the instance (after raising its limit to `smem`); 0 when unavailable.
int bg_batch_prepare_shape(int precision, int nvar, int shape, size_t smem);
