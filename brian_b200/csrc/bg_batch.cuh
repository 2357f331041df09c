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
    int32_t diag;                                // A's nonzeros are its first row and its diagonal, C's at most C[0]
    int32_t thr_kind, thr_var, thr_var2; T thr_val;
    int32_t reset_kind, reset_var, reset_var2; T reset_val;
    T *S; int64_t npad; int32_t n;
    int32_t nconn, ndeliv; int32_t deliv[kBatchMaxConn];   // delivery order (connection indices)
    BatchConn<T> conn[kBatchMaxConn];
    int32_t nsmon; BatchSmon smon[kBatchMaxSmon];
    int32_t nrec; BatchRec rec[kBatchMaxRec];
    int32_t smem_pos;                            // offset (32-bit words) of the StateMonitor columns
                                                 // (nrec x n int16, rows of n rounded up to even)
    DevCtl *ctl; unsigned long long *counters;   // spikes of the group, then events per connection
    long long t0; int32_t nsteps;                // engine step at the launch, steps asked for
    int32_t *out;                                // [kBatchOut]: steps run, records per spike monitor, rows per StateMonitor
};

template <typename T, int NV, int TH, int NPT>
__global__ void __launch_bounds__(TH) k_batch(const BatchNet<T> *nets, const int32_t *order, int lanes, int dry) {
    constexpr int BN = TH * NPT, NW = TH / 32;
    static_assert(BN <= 2 * kBatchMaxNeurons && BN % 32 == 0, "block shape");
    extern __shared__ __align__(16) uint32_t bsm[];
    __shared__ BatchNet<T> N;                   // the network's description, read many times a step
    constexpr int NWORDS = BN / 32, NQ = (NWORDS + 31) / 32;   // spike words; warps that read them
    __shared__ uint32_t words[3][NWORDS];       // spike words of step s in slot s % 3 (spike monitors)
    __shared__ int stepcnt[3][kBatchMaxSmon];   // monitored spikes of step s in slot s % 3
    __shared__ unsigned long long bcount[1 + kBatchMaxConn];   // spikes, events per connection
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(nets + order[blockIdx.x]);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&N);
        for (int k = tid; k < (int)(sizeof(BatchNet<T>) / 4); k += TH) dst[k] = src[k];
        if (tid < 3 * kBatchMaxSmon) stepcnt[tid / kBatchMaxSmon][tid % kBatchMaxSmon] = 0;
        for (int k = tid; k < 3 * NWORDS; k += TH) words[k / NWORDS][k % NWORDS] = 0u;
        if (tid <= kBatchMaxConn) bcount[tid] = 0ull;
    }
    __syncthreads();
    const int n = N.n, nsteps = N.nsteps;
    if (nsteps <= 0) {                                       // uniform
        if (tid == 0 && !dry) for (int k = 0; k < kBatchOut; ++k) N.out[k] = 0;
        return;
    }
    // ring rows of the current step: per connection (pushes) and per
    // delivery slot (the same rows, in delivery order)
    int cur[kBatchMaxConn], dcur[kBatchMaxConn];
#pragma unroll
    for (int c = 0; c < kBatchMaxConn; ++c) {
        cur[c] = 0; dcur[c] = 0;
        if (c < N.ndeliv) dcur[c] = (int)(N.t0 % N.conn[N.deliv[c]].md);
        if (c >= N.nconn) continue;
        const BatchConn<T> &q = N.conn[c];
        cur[c] = (int)(N.t0 % q.md);
        uint32_t *rows = bsm + q.smem_rows;
        const int64_t r0 = q.rowptr[0];
        for (int j = tid; j <= q.sn; j += TH) rows[j] = (uint32_t)(q.rowptr[j] - r0);
        if (q.smem_ring >= 0) {
            uint32_t *r = bsm + q.smem_ring;
            const int nw = q.md * q.tnp / 2;
            const uint32_t *g = reinterpret_cast<const uint32_t *>(q.ring);
            for (int k = tid; k < nw; k += TH) r[k] = q.direct ? 0u : g[k];
        }
    }
    // StateMonitors: column of each recorded neuron (-1: not recorded)
    int16_t *posmap = reinterpret_cast<int16_t *>(bsm + N.smem_pos);
    const int pstride = (n + 1) & ~1;
    for (int k = tid; k < N.nrec * pstride; k += TH) posmap[k] = -1;
    __syncthreads();
    for (int r = 0; r < N.nrec; ++r)
        for (int e = tid; e < N.rec[r].nidx; e += TH) posmap[r * pstride + N.rec[r].idx[e]] = (int16_t)N.rec[r].pos[e];
    T s[NPT][NV];
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
        const int li = u * TH + tid;
#pragma unroll
        for (int k = 0; k < NV; ++k) s[u][k] = li < n ? N.S[k * N.npad + li] : T(0);
    }
    // block-uniform values kept in registers
    const uint64_t anz = N.anz; const uint32_t cnz = N.cnz;
    const int thr_kind = N.thr_kind, thr_var = N.thr_var, thr_var2 = N.thr_var2;
    const T thr_val = N.thr_val;
    const int reset_kind = N.reset_kind, reset_var = N.reset_var, reset_var2 = N.reset_var2;
    const T reset_val = N.reset_val;
    const int nconn = N.nconn, ndeliv = N.ndeliv, nsmon = N.nsmon, nrec = N.nrec;
    const bool diag = N.diag != 0;
    uint32_t vmask = 0;                                      // bit u: neuron u * TH + tid exists
#pragma unroll
    for (int u = 0; u < NPT; ++u) vmask |= (u * TH + tid < n ? 1u : 0u) << u;
    int scnt[kBatchMaxSmon] = {0, 0};
    int rrows[kBatchMaxRec] = {0, 0, 0, 0};
    // steps until each StateMonitor's next record (no division in the loop)
    int rnext[kBatchMaxRec] = {0, 0, 0, 0};
#pragma unroll
    for (int r = 0; r < kBatchMaxRec; ++r) {
        if (r >= nrec) break;
        const long long rel = N.t0 - N.rec[r].start;
        rnext[r] = rel < 0 ? (int)-rel : (int)((N.rec[r].timestep - rel % N.rec[r].timestep) % N.rec[r].timestep);
    }
    // which of the thread's neurons each delivery targets (bit u)
    uint32_t dmask[kBatchMaxConn] = {0u, 0u};
#pragma unroll
    for (int di = 0; di < kBatchMaxConn; ++di) {
        if (di >= ndeliv) break;
        const BatchConn<T> &q = N.conn[N.deliv[di]];
#pragma unroll
        for (int u = 0; u < NPT; ++u) {
            const int li = u * TH + tid;
            if (li < n && li >= q.to && li < q.to + q.tn) dmask[di] |= 1u << u;
        }
    }
    const int G = 32 / lanes, grp = lane / lanes, gl = lane - grp * lanes;   // groups of `lanes` lanes in a warp
    __syncthreads();

    int st = 0;
    for (; st < nsteps; ++st) {
        const int slot = st % 3;
        // a monitor buffer that might not hold this step's records ends the
        // launch before the step (the counts are uniform: every thread
        // decides alike)
        if (!dry) {
            bool full = false;
#pragma unroll
            for (int m = 0; m < kBatchMaxSmon; ++m) full |= m < nsmon && scnt[m] + N.smon[m].n > N.smon[m].cap;
#pragma unroll
            for (int r = 0; r < kBatchMaxRec; ++r) {
                if (r >= nrec) break;
                full |= rnext[r] == 0 && rrows[r] >= N.rec[r].cap_rows;
            }
            if (full) break;
        }
        // ---- update: each row of A s (+ C) summed over k ascending with the
        // zero coefficients skipped (the order of linear_row)
        if (diag) {
            // the same sums with the zero terms left out at compile time:
            // first row full, the other rows diagonal, C in its first entry
            // at most (the masks guarantee it; a select-free update)
            // (coefficients re-read from shared memory each step rather than
            // kept in registers: the block shapes that hold 4096 neurons
            // have 64 registers a thread)
            const volatile T *sA = N.A;
            const T c0 = N.C[0];
#pragma unroll
            for (int u = 0; u < NPT; ++u) {
                T acc = T(0);
#pragma unroll
                for (int k = 0; k < NV; ++k) acc = rn<T>::add(acc, rn<T>::mul(sA[k], s[u][k]));
                if (cnz & 1u) acc = rn<T>::add(acc, c0);
#pragma unroll
                for (int j = 1; j < NV; ++j) s[u][j] = rn<T>::add(T(0), rn<T>::mul(sA[j * NV + j], s[u][j]));
                s[u][0] = acc;
            }
        } else {
            const volatile T *sA = N.A, *sC = N.C;
#pragma unroll
            for (int u = 0; u < NPT; ++u) {
                T x[NV];
#pragma unroll
                for (int j = 0; j < NV; ++j) {
                    x[j] = T(0);
#pragma unroll
                    for (int k = 0; k < NV; ++k)
                        if (anz & (1ull << (j * NV + k))) x[j] = rn<T>::add(x[j], rn<T>::mul(sA[j * NV + k], s[u][k]));
                    if (cnz & (1u << j)) x[j] = rn<T>::add(x[j], sC[j]);
                }
#pragma unroll
                for (int j = 0; j < NV; ++j) s[u][j] = x[j];
            }
        }
        // ---- threshold; spike words and monitored counts; push of the
        // warp's own spikes (counts commute: no order is needed here)
        uint32_t spk = 0;
        if (thr_kind == BG_THR_CONST) {
            on_var<NV>(thr_var, [&](auto K) {
                constexpr int k = decltype(K)::value;
#pragma unroll
                for (int u = 0; u < NPT; ++u) spk |= (s[u][k] > thr_val ? 1u : 0u) << u;
            });
        } else if (thr_kind == BG_THR_VAR) {
#pragma unroll
            for (int u = 0; u < NPT; ++u) spk |= (uget<T, NV>(s[u], thr_var) > uget<T, NV>(s[u], thr_var2) ? 1u : 0u) << u;
        }
        spk &= vmask;                                        // neurons of the network
#pragma unroll
        for (int u = 0; u < NPT; ++u) {
            const bool f = (spk >> u) & 1u;
            const uint32_t ball = __ballot_sync(0xffffffffu, f);
            if (!ball) continue;                             // warp-uniform
            const int wbase = u * TH + warp * 32;            // neuron of bit 0
            if (lane == 0) {
                atomicAdd(&bcount[0], (unsigned long long)__popc(ball));
                if (nsmon) words[slot][u * NW + warp] = ball;
            }
            if (!dry && lane < nsmon) {                      // monitored spikes of the warp
                const BatchSmon &M = N.smon[lane];
                const int lo = min(max(M.origin - wbase, 0), 32), hi = min(max(M.origin + M.n - wbase, 0), 32);
                const uint32_t range = (hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u)) & ~(lo >= 32 ? 0xffffffffu : ((1u << lo) - 1u));
                const int c = __popc(ball & range);
                if (c) atomicAdd(&stepcnt[slot][lane], c);
            }
#pragma unroll
            for (int c = 0; c < kBatchMaxConn; ++c) {
                if (c >= nconn) break;
                const BatchConn<T> &q = N.conn[c];
                const uint32_t *rows = bsm + q.smem_rows;
                const uint32_t *pk0 = q.packed;
                uint32_t *sring = q.smem_ring >= 0 ? bsm + q.smem_ring : nullptr;
                // spike k of the word goes to lane group k % G
                uint32_t m = ball;
                for (int k = 0; m; ++k) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    if (k % G != grp) continue;
                    const int j = wbase + b - q.so;
                    if (j < 0 || j >= q.sn) continue;
                    const uint32_t k0 = rows[j], k1 = rows[j + 1];
                    if (gl == 0 && k1 > k0) atomicAdd(&bcount[1 + c], (unsigned long long)(k1 - k0));
                    for (uint32_t e = k0 + gl; e < k1; e += 4u * lanes) {
                        uint32_t w4[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) w4[i] = e + i * lanes < k1 ? __ldg(pk0 + e + i * lanes) : 0xffffffffu;
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
        }
        // the step's pushes, spike words and counts are complete; the only
        // barrier of the step
        __syncthreads();
        if (tid == 0) {
#pragma unroll
            for (int m = 0; m < kBatchMaxSmon; ++m) stepcnt[(st + 2) % 3][m] = 0;   // slot of step st-1, read by all
        }
        // ---- spike-monitor records, ascending: warp q writes the spikes of
        // words 32q..32q+31 after those of the words before it
        if (!dry && nsmon && warp < NQ) {
            const int wi = warp * 32 + lane;
            const uint32_t wv = wi < NWORDS ? words[slot][wi] : 0u;
            // the words of step st-1 were read before this step's barrier:
            // clear them for step st+2
            if (wi < NWORDS) words[(st + 2) % 3][wi] = 0u;
#pragma unroll
            for (int m = 0; m < kBatchMaxSmon; ++m) {
                if (m >= nsmon) break;
                const BatchSmon &M = N.smon[m];
                auto in_range = [&](int word, uint32_t v) {
                    const int lo = min(max(M.origin - word * 32, 0), 32), hi = min(max(M.origin + M.n - word * 32, 0), 32);
                    const uint32_t r = (hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u)) & ~(lo >= 32 ? 0xffffffffu : ((1u << lo) - 1u));
                    return v & r;
                };
                uint32_t w = in_range(wi, wv);
                int before = 0;
                for (int q = 0; q < warp; ++q) {
                    const int wq = q * 32 + lane;
                    if (wq < NWORDS) before += __popc(in_range(wq, words[slot][wq]));
                }
                before = __reduce_add_sync(0xffffffffu, before);
                const int c = __popc(w);
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += v; }
                int pos = scnt[m] + before + incl - c;
                while (w) {
                    const int b = __ffs(w) - 1;
                    w &= w - 1;
                    M.idx[pos] = wi * 32 + b - M.origin;
                    M.step[pos] = st;
                    ++pos;
                }
            }
        }
#pragma unroll
        for (int m = 0; m < kBatchMaxSmon; ++m)
            if (m < nsmon) scnt[m] += stepcnt[slot][m];
        // ---- delivery of the rows due at step t, in the reference's order
#pragma unroll
        for (int di = 0; di < kBatchMaxConn; ++di) {
            if (di >= ndeliv) break;
            const BatchConn<T> &q = N.conn[N.deliv[di]];
            const int row = dcur[di];
            uint16_t *sr = q.smem_ring >= 0 ? reinterpret_cast<uint16_t *>(bsm + q.smem_ring) + row * q.tnp : nullptr;
            uint16_t *gr = q.ring ? q.ring + (int64_t)row * q.tnp : nullptr;
            const T w = q.w;
            const int to = q.to, direct = q.direct;
            const uint32_t dm = dmask[di];
            on_var<NV>(q.var, [&](auto K) {
                constexpr int k = decltype(K)::value;
#pragma unroll
                for (int u = 0; u < NPT; ++u) {
                    if (!((dm >> u) & 1u)) continue;
                    const int e = u * TH + tid - to;
                    const int cnt = sr ? sr[e] : __ldcg(gr + e);
                    if (!cnt) continue;
                    if (sr) sr[e] = 0; else gr[e] = 0;
                    if (direct) {
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
            if (c < nconn) cur[c] = cur[c] + 1 == N.conn[c].md ? 0 : cur[c] + 1;
            if (c < ndeliv) dcur[c] = dcur[c] + 1 == N.conn[N.deliv[c]].md ? 0 : dcur[c] + 1;
        }
        // ---- reset
        if (reset_kind == BG_RESET_CONST) {
            on_var<NV>(reset_var, [&](auto K) {
                constexpr int k = decltype(K)::value;
#pragma unroll
                for (int u = 0; u < NPT; ++u)
                    if ((spk >> u) & 1u) s[u][k] = reset_val;
            });
        } else if (reset_kind == BG_RESET_VAR) {
#pragma unroll
            for (int u = 0; u < NPT; ++u)
                if ((spk >> u) & 1u) uset<T, NV>(s[u], reset_var, uget<T, NV>(s[u], reset_var2));
        }
        // ---- StateMonitors ('end' slot): each thread writes its recorded neurons
        if (!dry) {
#pragma unroll
            for (int r = 0; r < kBatchMaxRec; ++r) {
                if (r >= nrec) break;
                const BatchRec &R = N.rec[r];
                if (rnext[r]) { --rnext[r]; continue; }          // uniform
                rnext[r] = R.timestep - 1;
                T *dst = (T *)R.buf + (int64_t)rrows[r] * R.nidx;
                on_var<NV>(R.var, [&](auto K) {
                    constexpr int k = decltype(K)::value;
#pragma unroll
                    for (int u = 0; u < NPT; ++u) {
                        const int li = u * TH + tid;
                        const int p = li < n ? posmap[r * pstride + li] : -1;
                        if (p >= 0) dst[p] = s[u][k];
                    }
                });
                ++rrows[r];
            }
        }
    }
    __syncthreads();                                         // the last step's shared ring rows and records
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
    for (int c = 0; c < nconn; ++c) {
        const BatchConn<T> &q = N.conn[c];
        if (q.smem_ring < 0 || q.direct) continue;
        const uint32_t *r = bsm + q.smem_ring;
        uint32_t *g = reinterpret_cast<uint32_t *>(q.ring);
        for (int k = tid; k < q.md * q.tnp / 2; k += TH) g[k] = r[k];
    }
    if (tid == 0) {
        if (bcount[0]) atomicAdd(N.counters, bcount[0]);
        for (int c = 0; c < nconn; ++c)
            if (bcount[1 + c]) atomicAdd(N.counters + 1 + c, bcount[1 + c]);
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
constexpr BatchShape kBatchShapes[] = {{128, 4}, {256, 4}, {512, 4}, {512, 8}, {1024, 4}, {768, 6}};
constexpr int kBatchNumShapes = (int)(sizeof(kBatchShapes) / sizeof(kBatchShapes[0]));

}  // namespace bg

// Launches k_batch<T, nvar, shape> over `blocks` networks (bg_batch.cu).
cudaError_t bg_batch_launch(int precision, int nvar, int shape, const void *nets, const int32_t *order, int blocks,
                            int lanes, int dry, size_t smem, cudaStream_t s);
// Largest dynamic shared memory of the instance (after raising its limit to `smem`); 0 when unavailable.
int bg_batch_prepare_shape(int precision, int nvar, int shape, size_t smem);
