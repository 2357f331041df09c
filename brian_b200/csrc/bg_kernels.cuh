// bg_kernels.cuh -- sm_100a kernels of the clock-driven loop.
//
// Spike history layout: one bit per neuron and step.  hist[slot][word] holds
// the spikes of neurons 32*word .. 32*word+31 emitted at the step whose
// counter is congruent to `slot` modulo `depth`.  The warp ballot of the
// threshold test IS the history word, so compaction needs no scan, and
// ascending neuron order (threshold.py:191) is the natural bit order.
#pragma once
#include "bg_common.cuh"

namespace bg {

constexpr int kHeadThreads = 256;
constexpr int kNPT = 4;                                  // neurons per thread
constexpr int kBlockNeurons = kHeadThreads * kNPT;       // neurons per block
constexpr int kPushBatch = 64;                           // spikes per push batch
constexpr int kPushUnroll = 4;                           // elements per thread per pass
constexpr int kMaxVars = 8;
constexpr int kMaxDeliv = 4;
constexpr int kMaxRec = 4;

// DelayConnection ring delivered into this group.  With one shared weight w
// the ring holds event COUNTS (uint16, rows of tnp = tn rounded up to even
// entries) and delivery adds table[k], where table[k] = table[k-1] + w with
// table[0] = 0: exactly the value the reference's ring entry reaches after k
// additions of w (delayconnection.py:152-153), in any order.
template <typename T> struct Deliv {
    T *ring; int64_t tn, to; int md; int var;
    uint16_t *cring; int64_t tnp; const T *table;
    int tablen;    // valid table entries (largest count + 1); 0 when unknown
};

// Count-ring helpers: entry col of a row is the low/high half of a 32-bit word.
__device__ __forceinline__ void cring_add(uint16_t *row, int32_t col) {
    atomicAdd(reinterpret_cast<unsigned int *>(row + (col & ~1)), 1u << ((col & 1) << 4));
}

// Value delivered to target neuron i (group index) from ring row ps % md,
// which is then cleared.  CG: read through L2 only (the persistent kernel
// reads rows that other blocks of the same launch incremented).
template <typename T, bool CG>
__device__ __forceinline__ T deliver(const Deliv<T> &dv, int ps, int64_t i) {
    const int64_t r = ps % dv.md;
    if (dv.cring) {
        uint16_t *p = dv.cring + r * dv.tnp + (i - dv.to);
        const uint16_t c = CG ? __ldcg(p) : *p;
        if (c) { *p = 0; return __ldg(dv.table + c); }
        return T(0);
    }
    T *p = dv.ring + r * dv.tn + (i - dv.to);
    const T v = CG ? __ldcg(p) : *p;
    if (v != T(0)) *p = T(0);
    return v;
}
// DelayConnection whose spikes are pushed by the SOURCE group's head kernel
// right after the threshold (shared-weight / atomic path).  The ring has
// md >= max delay + 2 rows, so the rows written at step t, (t + d) mod md with
// d <= max delay, never include row (t - 1) mod md that the tail of this
// same kernel delivers and clears: no grid-wide ordering is needed.
template <typename T> struct Push {
    T *ring; int md; int64_t so, sn, tn;
    const int64_t *rowptr; const int32_t *cols; const void *w; int w_bits; const uint8_t *d;
    unsigned long long *events;
    uint16_t *cring; int64_t tnp;      // count ring (shared weight), else null
    const uint32_t *packed;            // persistent path: target | delay << 24 per synapse, else null
};
constexpr int kMaxPush = 4;

struct RecDev {                        // StateMonitor recorded in this group
    int var; int nidx; const int32_t *idx; const int32_t *pos; const int32_t *blk_lo;
    void *buf; const long long *row_base; int timestep; long long start;
};

// TimedArraySetter (timedarray.py:238-303): at the start of a step, before
// the update, S[var][origin + k] (k < count) takes row r of vals[nrows][ncols]
// (ncols 1: one value for all).  mode 0 (array on a clock): r = rint((cs*dt -
// t_init) / adt) clamped to the rows; mode 1 (explicit times): r = the number
// of breakpoint steps bp[0..nrows-1) <= cs.  Nothing before clock step first.
constexpr int kMaxSet = 4;
template <typename T> struct SetDev {
    int var, mode; int64_t origin, count, nrows, ncols;
    double t_init, adt; long long first;
    const T *vals; const int64_t *bp;
};

template <typename T> struct HeadArgs {
    DevCtl *ctl;
    T *S; int64_t n, npad; int nvar;
    int linear, useC;
    T A[kMaxVars * kMaxVars]; T C[kMaxVars];
    uint64_t anz; uint32_t cnz;    // nonzero masks of A and C
    int thr_kind, thr_var, thr_var2; T thr_val; double dt;
    uint64_t seed; int rate_var;
    const int64_t *gen_steps; const int32_t *gen_idx; int64_t gen_n;
    int reset_kind, reset_var, reset_var2; T reset_val;
    int refr; double refr_time; int period; int clamp_var; T clamp_val;
    int emp_steps;                 // EmpiricalThreshold: no spike within this many steps of the last one (0: off)
    double *next_allowed; int32_t *last_spike;
    uint32_t *hist; int depth; int64_t nwords;
    int ndeliv; Deliv<T> deliv[kMaxDeliv];
    int nrec; RecDev rec[kMaxRec];
    int npush; Push<T> push[kMaxPush];
    int nset; SetDev<T> set[kMaxSet];
    unsigned long long *spikes;    // running spike count of the group
    int tail, update, last;
};

// Row of a setter's array at clock step cs (the reference's
// int(rint((t - t_init) / dt)) clamped, or the count of breakpoints <= cs).
template <typename T>
__device__ __forceinline__ int64_t setter_row(const SetDev<T> &st, long long cs, double dt) {
    if (st.mode == 0) {
        const double x = __ddiv_rn(__dsub_rn(__dmul_rn((double)cs, dt), st.t_init), st.adt);
        if (!(x > 0.0)) return 0;
        if (x >= (double)(st.nrows - 1)) return st.nrows - 1;
        return (int64_t)rint(x);
    }
    int64_t lo = 0, hi = st.nrows - 1;                   // first breakpoint > cs
    while (lo < hi) { const int64_t m = (lo + hi) >> 1; if (st.bp[m] <= cs) lo = m + 1; else hi = m; }
    return lo;
}

// Row j of the exact linear update: ((0 + A[j][k0] s_k0) + A[j][k1] s_k1) +
// ... over the nonzero coefficients (bit j*NV+k of anz), left to right, then
// + C[j] when nonzero (bit j of cnz).  Exact zeros are skipped: only the sign
// of an exact-zero result can differ from summing them (x + 0*y equals x
// for every finite x except -0), and the CPU restatement uses the same rule.  The masks are kernel parameters,
// so every test is uniform across the grid.
template <typename T, int NV>
__device__ __forceinline__ T linear_row(const T *A, const T *C, uint64_t anz, uint32_t cnz, const T (&s)[NV], int j) {
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < NV; ++k)
        if (anz & (1ull << (j * NV + k))) acc = rn<T>::add(acc, rn<T>::mul(A[j * NV + k], s[k]));
    if (cnz & (1u << j)) acc = rn<T>::add(acc, C[j]);
    return acc;
}

#ifndef __CUDACC_RTC__
// Host side: nonzero masks of the coefficients a kernel argument block holds.
template <typename Args>
inline void set_linear_masks(Args &a, int nvar) {
    a.anz = 0; a.cnz = 0;
    for (int j = 0; j < nvar; ++j) {
        for (int k = 0; k < nvar; ++k)
            if (a.A[j * nvar + k] != 0) a.anz |= 1ull << (j * nvar + k);
        if (a.useC && a.C[j] != 0) a.cnz |= 1u << j;
    }
}
#endif

// Block-aggregated counter update (one global atomic per block).
__device__ __forceinline__ void block_count(unsigned long long *g, unsigned long long v) {
    __shared__ unsigned long long acc;
    if (threadIdx.x == 0) acc = 0ull;
    __syncthreads();
    if (v) atomicAdd(&acc, v);
    __syncthreads();
    if (threadIdx.x == 0 && acc && g) atomicAdd(g, acc);
}

// Block-uniform variable access without runtime-indexed register arrays:
// `var` is a kernel parameter, so the switch is a uniform branch.
template <typename T, int NV>
__device__ __forceinline__ T uget(const T (&s)[NV], int var) {
    switch (var) {
    case 0: return s[0];
    case 1: if (NV > 1) return s[NV > 1 ? 1 : 0]; break;
    case 2: if (NV > 2) return s[NV > 2 ? 2 : 0]; break;
    default: if (NV > 3) return s[NV > 3 ? 3 : 0]; break;
    }
    return T(0);
}
template <typename T, int NV>
__device__ __forceinline__ void uset(T (&s)[NV], int var, T v) {
    switch (var) {
    case 0: s[0] = v; break;
    case 1: if (NV > 1) s[NV > 1 ? 1 : 0] = v; break;
    case 2: if (NV > 2) s[NV > 2 ? 2 : 0] = v; break;
    default: if (NV > 3) s[NV > 3 ? 3 : 0] = v; break;
    }
}

// Uniform dispatch on a state-variable index hoisted out of the per-neuron
// loops: f receives the index as a compile-time constant, so the neuron loop
// inside it indexes registers directly and the branch runs once per thread.
template <int K> struct VarIdx { static constexpr int value = K; };
template <int NV, typename F>
__device__ __forceinline__ void on_var(int var, F &&f) {
    switch (var) {
    case 0: f(VarIdx<0>()); break;
    case 1: if constexpr (NV > 1) f(VarIdx<1>()); break;
    case 2: if constexpr (NV > 2) f(VarIdx<2>()); break;
    default: if constexpr (NV > 3) f(VarIdx<3>()); break;
    }
}

template <typename T, int NV>
__device__ __forceinline__ void set_var(T (&s)[NV], int var, T v) {
#pragma unroll
    for (int k = 0; k < NV; ++k) if (k == var) s[k] = v;
}
template <typename T, int NV>
__device__ __forceinline__ T get_var(const T (&s)[NV], int var) {
    T r = T(0);
#pragma unroll
    for (int k = 0; k < NV; ++k) if (k == var) r = s[k];
    return r;
}

// scatter_batch for count rings whose synapses are packed as one word each
// (target in the low 24 bits, delay in the high 8): one load per synapse.
template <int TH>
__device__ __forceinline__ void scatter_batch_packed(const uint32_t *packed, uint16_t *cring, int64_t tnp, int md,
                                                     int cur, const int64_t *srow, const int32_t *spref, int nb,
                                                     int total) {
    const int tid = threadIdx.x;
    for (int e0 = 0; e0 < total; e0 += TH * kPushUnroll) {
        uint32_t pk[kPushUnroll];
#pragma unroll
        for (int u = 0; u < kPushUnroll; ++u) {
            const int e = e0 + u * TH + tid;
            pk[u] = 0xffffffffu;
            if (e < total) {
                int lo = 0, hi = nb;             // last s with spref[s] <= e
                while (hi - lo > 1) { const int m = (lo + hi) >> 1; if (spref[m] <= e) lo = m; else hi = m; }
                pk[u] = __ldg(packed + srow[lo] + (e - spref[lo]));
            }
        }
#pragma unroll
        for (int u = 0; u < kPushUnroll; ++u) {
            if (pk[u] == 0xffffffffu) continue;
            const int sl2 = cur + (int)(pk[u] >> 24);
            cring_add(cring + (int64_t)(sl2 >= md ? sl2 - md : sl2) * tnp, (int32_t)(pk[u] & 0xffffffu));
        }
    }
}

// Push the spikes of one block (ascending, from the history words in shared
// memory) into the rings of its outgoing delayed connections.  The
// (spike, synapse) pairs of a batch of spikes are flattened over the block's
// threads; each thread first loads kPushUnroll independent synapses, then
// issues their atomic adds, so a batch costs two dependent memory latencies
// (row pointers, then synapses) however many spikes it holds.
// Scatter the (spike, synapse) pairs of one batch: pair e belongs to spike
// s with spref[s] <= e < spref[s+1] and is synapse srow[s] + e - spref[s].
// Each thread loads kPushUnroll independent synapses before issuing their
// atomics.  Count rings need no weight.
template <typename T, int TH = kHeadThreads>
__device__ __forceinline__ void scatter_batch(const Push<T> &q, int cur, const int64_t *srow, const int32_t *spref,
                                              int nb, int total) {
    const int tid = threadIdx.x;
    for (int e0 = 0; e0 < total; e0 += TH * kPushUnroll) {
        int32_t col[kPushUnroll]; T wv[kPushUnroll]; int slot[kPushUnroll];
#pragma unroll
        for (int u = 0; u < kPushUnroll; ++u) {
            const int e = e0 + u * TH + tid;
            col[u] = -1;
            wv[u] = T(0);
            slot[u] = 0;
            if (e < total) {
                int lo = 0, hi = nb;             // last s with spref[s] <= e
                while (hi - lo > 1) { const int m = (lo + hi) >> 1; if (spref[m] <= e) lo = m; else hi = m; }
                const int64_t k = srow[lo] + (e - spref[lo]);
                col[u] = __ldg(q.cols + k);
                if (!q.cring) wv[u] = q.w_bits == 32 ? (T)__ldg((const float *)q.w + k) : (T)__ldg((const double *)q.w + k);
                const int sl2 = cur + (int)__ldg(q.d + k);
                slot[u] = sl2 >= q.md ? sl2 - q.md : sl2;
            }
        }
#pragma unroll
        for (int u = 0; u < kPushUnroll; ++u) {
            if (col[u] < 0) continue;
            if (q.cring) cring_add(q.cring + (int64_t)slot[u] * q.tnp, col[u]);
            else atomicAdd(&q.ring[(int64_t)slot[u] * q.tn + col[u]], wv[u]);
        }
    }
}

template <typename T, typename HA>
__device__ __forceinline__ void push_block_spikes(const HA &a, const uint32_t *words, int64_t base, int nstep) {
    __shared__ int32_t sl[kBlockNeurons];
    __shared__ int64_t srow[kPushBatch];
    __shared__ int32_t spref[kPushBatch + 1];
    __shared__ int nsp;
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < 32) {
        uint32_t w = words[lane];
        const int c = __popc(w);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += v; }
        int off = incl - c;
        while (w) { const int b = __ffs(w) - 1; w &= w - 1; sl[off++] = lane * 32 + b; }
        if (lane == 31) nsp = incl;
    }
    __syncthreads();
    const int n = nsp;
    if (n == 0) return;                      // block-uniform
    for (int p = 0; p < a.npush; ++p) {
        const Push<T> &q = a.push[p];
        const int cur = nstep % q.md;
        unsigned long long ev = 0;
        for (int b0 = 0; b0 < n; b0 += kPushBatch) {
            const int nb = min(kPushBatch, n - b0);
            if (tid < nb) {
                const int64_t gi = base + sl[b0 + tid];
                int64_t r0 = 0, len = 0;
                if (gi >= q.so && gi < q.so + q.sn) { r0 = __ldg(q.rowptr + (gi - q.so)); len = __ldg(q.rowptr + (gi - q.so) + 1) - r0; }
                srow[tid] = r0;
                spref[tid + 1] = (int32_t)len;
            }
            __syncthreads();
            if (tid == 0) { spref[0] = 0; for (int k = 1; k <= nb; ++k) spref[k] += spref[k - 1]; }
            __syncthreads();
            const int total = spref[nb];
            ev += (unsigned long long)total;
            scatter_batch<T>(q, cur, srow, spref, nb, total);
            __syncthreads();
        }
        if (tid == 0 && ev && q.events) atomicAdd(q.events, ev);
    }
}

// Step counters are below 2^31 (checked by the host), so slot arithmetic
// runs in 32 bits.
//
// One block = kBlockNeurons consecutive neurons, kNPT per thread (neuron
// base + u*kHeadThreads + tid), so every warp instruction touches one
// 32-neuron history word and a 262k-neuron group fits in one wave.
//   tail:   finish the previous step -- delayed-ring delivery
//           ('after_connections'), reset / refractory clamp ('resets') and
//           state monitors ('end');
//   update: this step's 'groups' slot -- state update, threshold, refractory
//           filter, history push -- then the pushes of this block's spikes
//           into the rings of outgoing delayed connections.
//
// The model hooks come from M: BuiltinModel runs the exact linear update and
// the threshold/reset kinds of HeadArgs; a generated model (compiled at run
// time by NVRTC for a nonlinear model or a general string threshold/reset)
// supplies any of update(s, t), threshold(s, t) and reset(s, t) itself.
struct BuiltinModel {
    static constexpr bool custom_update = false, custom_threshold = false, custom_reset = false;
    template <typename T, int NV> static __device__ void update(T (&)[NV], double) {}
    template <typename T, int NV> static __device__ bool threshold(const T (&)[NV], double) { return false; }
    template <typename T, int NV> static __device__ void reset(T (&)[NV], double) {}
};

template <typename T, int NV, class M>
__device__ __forceinline__ void head_body(const HeadArgs<T> &a) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t base = (int64_t)blockIdx.x * kBlockNeurons;
    const long long nstep = a.ctl->nstep;
    const long long cs = nstep + a.ctl->clock_off;
    T s[kNPT][NV];
#pragma unroll
    for (int u = 0; u < kNPT; ++u) {
        const int64_t i = base + u * kHeadThreads + tid;
#pragma unroll
        for (int k = 0; k < NV; ++k) s[u][k] = i < a.n ? a.S[k * a.npad + i] : T(0);
    }

    if (a.tail) {
        const int ps = (int)(nstep - 1);
        for (int d = 0; d < a.ndeliv; ++d) {
            const Deliv<T> &dv = a.deliv[d];
#pragma unroll
            for (int u = 0; u < kNPT; ++u) {
                const int64_t i = base + u * kHeadThreads + tid;
                if (i < a.n && i >= dv.to && i < dv.to + dv.tn)
                    set_var<T, NV>(s[u], dv.var, rn<T>::add(get_var<T, NV>(s[u], dv.var), deliver<T, false>(dv, ps, i)));
            }
        }
        if (a.period > 0) {
#pragma unroll
            for (int u = 0; u < kNPT; ++u) {
                const int64_t i = base + u * kHeadThreads + tid;
                if (i < a.n && (long long)ps - (long long)a.last_spike[i] < a.period)
                    set_var<T, NV>(s[u], a.clamp_var, a.clamp_val);
            }
        } else if (M::custom_reset || a.reset_kind) {
            const uint32_t *H = a.hist + (int64_t)(ps % a.depth) * a.nwords;
            const double tp = __dmul_rn((double)(cs - 1), a.dt);    // time of the step being finished
#pragma unroll
            for (int u = 0; u < kNPT; ++u) {
                const int64_t i = base + u * kHeadThreads + tid;
                const uint32_t w = H[i >> 5];
                if (i < a.n && ((w >> lane) & 1u)) {
                    if constexpr (M::custom_reset) M::template reset<T, NV>(s[u], tp);
                    else if (a.reset_kind == 1) set_var<T, NV>(s[u], a.reset_var, a.reset_val);
                    else set_var<T, NV>(s[u], a.reset_var, get_var<T, NV>(s[u], a.reset_var2));
                }
            }
        }
        if (a.nrec) {
            __shared__ T stash[kBlockNeurons];
            for (int r = 0; r < a.nrec; ++r) {
                const RecDev &m = a.rec[r];
                const long long rel = (long long)ps - m.start;
                if (rel < 0 || rel % m.timestep) continue;    // block-uniform
#pragma unroll
                for (int u = 0; u < kNPT; ++u) stash[u * kHeadThreads + tid] = get_var<T, NV>(s[u], m.var);
                __syncthreads();
                const long long row = rel / m.timestep - *m.row_base;
                const int e0 = m.blk_lo[blockIdx.x], e1 = m.blk_lo[blockIdx.x + 1];
                for (int e = e0 + tid; e < e1; e += kHeadThreads)
                    ((T *)m.buf)[row * m.nidx + m.pos[e]] = stash[m.idx[e] - (int)base];
                __syncthreads();
            }
        }
    }

    if (a.update) {
        // TimedArraySetters ('start' slot)
        for (int q = 0; q < a.nset; ++q) {
            const SetDev<T> &st = a.set[q];
            if (cs < st.first) continue;                       // uniform
            const int64_t r = setter_row<T>(st, cs, a.dt);
            const T *row = st.vals + r * st.ncols;
#pragma unroll
            for (int u = 0; u < kNPT; ++u) {
                const int64_t i = base + u * kHeadThreads + tid;
                if (i >= st.origin && i < st.origin + st.count)
                    set_var<T, NV>(s[u], st.var, row[st.ncols == 1 ? 0 : i - st.origin]);
            }
        }
        __shared__ uint32_t words[kBlockNeurons / 32];
        uint32_t nspk = 0;
#pragma unroll
        for (int u = 0; u < kNPT; ++u) {
            const int64_t i = base + u * kHeadThreads + tid;
            const bool act = i < a.n;
            if constexpr (M::custom_update) {
                M::template update<T, NV>(s[u], __dmul_rn((double)cs, a.dt));
            } else if (a.linear) {
                T x[NV];
#pragma unroll
                for (int j = 0; j < NV; ++j) x[j] = linear_row<T, NV>(a.A, a.C, a.anz, a.cnz, s[u], j);
#pragma unroll
                for (int j = 0; j < NV; ++j) s[u][j] = x[j];
            }
            bool spk = false;
            if (act && M::custom_threshold) {
                spk = M::template threshold<T, NV>(s[u], __dmul_rn((double)cs, a.dt));
            } else if (act) {
                switch (a.thr_kind) {
                case 1: spk = get_var<T, NV>(s[u], a.thr_var) > a.thr_val; break;
                case 2: spk = get_var<T, NV>(s[u], a.thr_var) > get_var<T, NV>(s[u], a.thr_var2); break;
                case 3: {
                    const double rate = (double)get_var<T, NV>(s[u], a.rate_var);
                    spk = bg_philox_uniform(a.seed, cs, i) < __dmul_rn(rate, a.dt);
                    break;
                }
                case 4: {
                    // spikes of this clock step: [lo, e) of the (step, index)-sorted list
                    int64_t lo = 0, hi = a.gen_n;
                    while (lo < hi) { int64_t m = (lo + hi) >> 1; if (a.gen_steps[m] < cs) lo = m + 1; else hi = m; }
                    int64_t e = lo, hi2 = a.gen_n;
                    while (e < hi2) { int64_t m = (e + hi2) >> 1; if (a.gen_steps[m] <= cs) e = m + 1; else hi2 = m; }
                    int64_t l2 = lo, h2 = e;
                    while (l2 < h2) { int64_t m = (l2 + h2) >> 1; if (a.gen_idx[m] < i) l2 = m + 1; else h2 = m; }
                    spk = l2 < e && a.gen_idx[l2] == i;
                    break;
                }
                default: break;
                }
            }
            if (act) {
                // EmpiricalThreshold (threshold.py:449-457): no spike while the
                // neuron is among the spikes of the last emp_steps steps
                if (spk && a.emp_steps > 0 && (long long)nstep - (long long)a.last_spike[i] <= a.emp_steps) spk = false;
                if (spk && a.refr) {
                    const double t = __dmul_rn((double)cs, a.dt);
                    if (a.next_allowed[i] <= t) a.next_allowed[i] = __dadd_rn(t, a.refr_time);
                    else spk = false;
                }
                if (spk && (a.period > 0 || a.emp_steps > 0)) a.last_spike[i] = (int32_t)nstep;
            }
            const uint32_t ball = __ballot_sync(0xffffffffu, spk);
            if (lane == 0) {
                a.hist[(int64_t)((int)nstep % a.depth) * a.nwords + ((base + u * kHeadThreads) >> 5) + warp] = ball;
                words[u * (kHeadThreads / 32) + warp] = ball;
                nspk += __popc(ball);
            }
        }
        block_count(a.spikes, nspk);       // contains __syncthreads: words[] is complete
        if (a.npush) push_block_spikes<T>(a, words, base, (int)nstep);
    }
    if (a.update || a.tail) {
#pragma unroll
        for (int u = 0; u < kNPT; ++u) {
            const int64_t i = base + u * kHeadThreads + tid;
            if (i < a.n) {
#pragma unroll
                for (int k = 0; k < NV; ++k) a.S[k * a.npad + i] = s[u][k];
            }
        }
    }
    bg_finish_step(a.ctl, a.last);
}

template <typename T, int NV>
__global__ void __launch_bounds__(kHeadThreads, 2) k_head(const HeadArgs<T> a) {
    head_body<T, NV, BuiltinModel>(a);
}

// ---------------------------------------------------------------------------
// Spike iteration over a history slot restricted to [origin, origin+cnt).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t masked_word(const uint32_t *H, int64_t wi, int64_t origin, int64_t end) {
    uint32_t w = H[wi];
    const int64_t base = wi << 5;
    if (base < origin) { const int sh = (int)(origin - base); w = sh >= 32 ? 0u : (w & (0xffffffffu << sh)); }
    if (base + 32 > end) { const int keep = (int)(end - base); w = keep <= 0 ? 0u : (keep >= 32 ? w : (w & ((1u << keep) - 1u))); }
    return w;
}

template <typename T> struct PropArgs {
    DevCtl *ctl;
    const uint32_t *hist; int depth; int64_t nwords; int delay;
    int64_t so, sn;                 // source range in the source group
    int64_t to, tn;                 // target range in the target group
    T *sv;                          // target state row + to (zero-delay path)
    T *ring; int md;                // DelayConnection ring [md][tn]
    const int64_t *rowptr; const int32_t *cols; const void *w; const uint8_t *d;
    int dense;
    const T *mod;                   // source modulation row + so, or null
    int parts;                      // row split for the atomic path
    // fused presynaptic STDP (stdp.py:370-414): w[i,:] += A_post; clip
    int stdp; double *A_pre; const double *A_post; double Ap; int pre_set; double wmin, wmax;
    int wmode; double wx;           // update form of the presynaptic w line (stdp_w)
    unsigned long long *events;     // running count of synaptic events
    int last;
};

// w (+)= the rule's change, then clip (stdp.py:395-408).  mode 0: w + a;
// mode 1: w * (1 + a); mode 2: w + (wx - w) * a, wx the exact maximum
// weight of the code string (stdp.py:510-533); modes 1 and 2 on FP64
// weights only.
template <typename WT>
__device__ __forceinline__ WT stdp_w_val(WT w, double add, double wmin, double wmax, int mode = 0, double wx = 0.0) {
    if (sizeof(WT) == 4) {
        float x = __double2float_rn(__dadd_rn((double)w, add));
        const float lo = __double2float_rn(wmin), hi = __double2float_rn(wmax);
        x = x < lo ? lo : (x > hi ? hi : x);
        return (WT)x;
    } else {
        const double w0 = (double)w;
        double x;
        if (mode == 1) x = __dmul_rn(w0, __dadd_rn(1.0, add));
        else if (mode == 2) x = __dadd_rn(w0, __dmul_rn(__dsub_rn(wx, w0), add));
        else x = __dadd_rn(w0, add);
        x = x < wmin ? wmin : (x > wmax ? wmax : x);
        return (WT)x;
    }
}
template <typename T, typename WT>
__device__ __forceinline__ void stdp_w(WT *w, int64_t k, double add, double wmin, double wmax, int mode = 0,
                                       double wx = 0.0) {
    w[k] = stdp_w_val<WT>(w[k], add, wmin, wmax, mode, wx);
}

// Shared-weight path (every addend of one accumulator is the same number, so
// the order of the atomic adds cannot change the result): warp items are
// (32 history words, row part).
template <typename T, typename WT, bool RING>
__global__ void __launch_bounds__(256) k_prop_atomic(const PropArgs<T> a) {
    const long long nstep = a.ctl->nstep;
    if (nstep >= a.delay) {
        const int lane = threadIdx.x & 31;
        const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
        const uint32_t *H = a.hist + (int64_t)((int)(nstep - a.delay) % a.depth) * a.nwords;
        const int64_t end = a.so + a.sn;
        const int64_t w0 = a.so >> 5, w1 = (end + 31) >> 5;
        const int64_t nch = (w1 - w0 + 31) >> 5;
        const int P = a.parts;
        const int cur = RING ? (int)nstep % a.md : 0;
        const WT *W = (const WT *)a.w;
        unsigned long long ev = 0;
        for (int64_t item = warp; item < nch * P; item += nwarps) {
            const int64_t c = item / P; const int p = (int)(item - c * P);
            const int64_t wi = w0 + c * 32 + lane;
            const uint32_t word = wi < w1 ? masked_word(H, wi, a.so, end) : 0u;
            uint32_t nz = __ballot_sync(0xffffffffu, word != 0u);
            while (nz) {
                const int l = __ffs(nz) - 1; nz &= nz - 1;
                uint32_t wd = __shfl_sync(0xffffffffu, word, l);
                const int64_t base = (w0 + c * 32 + l) << 5;
                while (wd) {
                    const int b = __ffs(wd) - 1; wd &= wd - 1;
                    const int64_t i = base + b - a.so;
                    const int64_t r0 = a.rowptr[i], r1 = a.rowptr[i + 1], len = r1 - r0;
                    const int64_t q0 = r0 + len * p / P, q1 = r0 + len * (p + 1) / P;
                    if (p == 0 && lane == 0) ev += (unsigned long long)len;
                    for (int64_t k = q0 + lane; k < q1; k += 32) {
                        const int32_t j = a.cols[k];
                        const T wv = (T)W[k];
                        if (RING) atomicAdd(&a.ring[(int64_t)((cur + a.d[k]) % a.md) * a.tn + j], wv);
                        else atomicAdd(&a.sv[j], wv);
                        if (a.stdp) stdp_w<T, WT>((WT *)a.w, k, a.A_post[j], a.wmin, a.wmax, a.wmode, a.wx);
                    }
                    if (a.stdp && p == 0 && lane == 0)
                        a.A_pre[i] = a.pre_set ? a.Ap : __dadd_rn(a.A_pre[i], a.Ap);
                }
            }
        }
        block_count(a.events, ev);
    }
    bg_finish_step(a.ctl, a.last);
}

// Ordered path (general weights): block b owns targets [b*TB, b*TB+TB) and
// walks the spikes in ascending order, so every accumulator sees its addends
// in the reference order (connection.py:239-241, delayconnection.py:152-153).
constexpr int kOrdThreads = 256;
constexpr int kOrdTB = 1024;
constexpr int kOrdBatch = 1024;

template <typename T, typename WT, bool RING>
__global__ void __launch_bounds__(kOrdThreads) k_prop_ordered(const PropArgs<T> a) {
    __shared__ int32_t sp[kOrdBatch];
    __shared__ int32_t slo[kOrdBatch], shi[kOrdBatch];
    __shared__ int32_t wcnt[kOrdThreads + 1];
    __shared__ int nb;
    const long long nstep = a.ctl->nstep;
    const int64_t t0 = (int64_t)blockIdx.x * kOrdTB, t1 = min(t0 + (int64_t)kOrdTB, a.tn);
    if (nstep >= a.delay && t0 < a.tn) {
        const uint32_t *H = a.hist + (int64_t)((int)(nstep - a.delay) % a.depth) * a.nwords;
        const int64_t end = a.so + a.sn;
        const int64_t w0 = a.so >> 5, w1 = (end + 31) >> 5;
        const int cur = RING ? (int)nstep % a.md : 0;
        WT *W = (WT *)a.w;
        const int tid = threadIdx.x;
        unsigned long long ev = 0;
        // process the source range in chunks of kOrdThreads words
        for (int64_t cw = w0; cw < w1; cw += kOrdThreads) {
            const int64_t wi = cw + tid;
            const uint32_t word = wi < w1 ? masked_word(H, wi, a.so, end) : 0u;
            // exclusive scan of popcounts (simple two-level scan)
            const int pc = __popc(word);
            int incl = pc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) { int v = __shfl_up_sync(0xffffffffu, incl, o); if ((tid & 31) >= o) incl += v; }
            if ((tid & 31) == 31) wcnt[tid >> 5] = incl;
            __syncthreads();
            if (tid == 0) { int acc = 0; for (int q = 0; q < kOrdThreads / 32; ++q) { int v = wcnt[q]; wcnt[q] = acc; acc += v; } wcnt[kOrdThreads / 32] = acc; }
            __syncthreads();
            const int total = wcnt[kOrdThreads / 32];
            int off = wcnt[tid >> 5] + incl - pc;
            // emit in batches of kOrdBatch spikes
            for (int bstart = 0; bstart < total; bstart += kOrdBatch) {
                {
                    uint32_t wd = word; int o = off;
                    while (wd) {
                        const int b = __ffs(wd) - 1; wd &= wd - 1;
                        if (o >= bstart && o < bstart + kOrdBatch) sp[o - bstart] = (int32_t)(((wi << 5) + b) - a.so);
                        ++o;
                    }
                }
                if (tid == 0) nb = min(kOrdBatch, total - bstart);
                __syncthreads();
                const int n = nb;
                // locate each spike's sub-range of targets in [t0, t1)
                for (int s = tid; s < n; s += kOrdThreads) {
                    const int64_t i = sp[s];
                    if (a.dense) { slo[s] = (int32_t)t0; shi[s] = (int32_t)t1; continue; }
                    const int64_t r0 = a.rowptr[i], r1 = a.rowptr[i + 1];
                    int64_t lo = r0, hi = r1;
                    while (lo < hi) { int64_t m = (lo + hi) >> 1; if (a.cols[m] < t0) lo = m + 1; else hi = m; }
                    int64_t lo2 = lo, hi2 = r1;
                    while (lo2 < hi2) { int64_t m = (lo2 + hi2) >> 1; if (a.cols[m] < t1) lo2 = m + 1; else hi2 = m; }
                    slo[s] = (int32_t)(lo - r0); shi[s] = (int32_t)(lo2 - r0);
                }
                __syncthreads();
                for (int s = 0; s < n; ++s) {
                    const int64_t i = sp[s];
                    const int64_t r0 = a.dense ? i * a.tn : a.rowptr[i];
                    const T mul = a.mod ? a.mod[i] : T(1);
                    for (int64_t q = slo[s] + tid; q < shi[s]; q += kOrdThreads) {
                        const int64_t k = a.dense ? r0 + q : r0 + q;
                        const int64_t j = a.dense ? q : a.cols[k];
                        T wv = (T)W[k];
                        if (a.mod) wv = rn<T>::mul(wv, mul);
                        if (RING) {
                            T *r = &a.ring[(int64_t)((cur + a.d[k]) % a.md) * a.tn + j];
                            *r = rn<T>::add(*r, wv);
                        } else {
                            a.sv[j] = rn<T>::add(a.sv[j], wv);
                        }
                        if (a.stdp) stdp_w<T, WT>(W, k, a.A_post[j], a.wmin, a.wmax, a.wmode, a.wx);
                    }
                    if (blockIdx.x == 0 && tid == 0) {
                        if (a.stdp) a.A_pre[i] = a.pre_set ? a.Ap : __dadd_rn(a.A_pre[i], a.Ap);
                        ev += (unsigned long long)(a.dense ? a.tn : a.rowptr[i + 1] - a.rowptr[i]);
                    }
                    __syncthreads();
                }
            }
            __syncthreads();
        }
        block_count(a.events, ev);
    }
    bg_finish_step(a.ctl, a.last);
}

// Dense connection, one thread per target column, spikes in ascending order
// from a shared-memory list (connection.py:256-262: sv += row).
constexpr int kDenseThreads = 256;
constexpr int kDenseList = 4096;
// TH threads per block (one target column each): 64 when the columns would
// otherwise fill few SMs
template <typename T, typename WT, int TH = kDenseThreads>
__global__ void __launch_bounds__(TH) k_prop_dense(const PropArgs<T> a) {
    __shared__ int32_t sp[kDenseList];
    __shared__ int32_t wcnt[TH / 32 + 1];
    const long long nstep = a.ctl->nstep;
    const int64_t j = (int64_t)blockIdx.x * TH + threadIdx.x;
    if (nstep >= a.delay) {
        const uint32_t *H = a.hist + (int64_t)((int)(nstep - a.delay) % a.depth) * a.nwords;
        const int64_t end = a.so + a.sn;
        const int64_t w0 = a.so >> 5, w1 = (end + 31) >> 5;
        WT *W = (WT *)a.w;
        const int tid = threadIdx.x;
        T acc = j < a.tn ? a.sv[j] : T(0);
        const double apost = (a.stdp && j < a.tn) ? a.A_post[j] : 0.0;
        unsigned long long ev = 0;
        for (int64_t cw = w0; cw < w1; cw += TH) {
            const int64_t wi = cw + tid;
            const uint32_t word = wi < w1 ? masked_word(H, wi, a.so, end) : 0u;
            const int pc = __popc(word);
            int incl = pc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) { int v = __shfl_up_sync(0xffffffffu, incl, o); if ((tid & 31) >= o) incl += v; }
            if ((tid & 31) == 31) wcnt[tid >> 5] = incl;
            __syncthreads();
            if (tid == 0) { int s = 0; for (int q = 0; q < TH / 32; ++q) { int v = wcnt[q]; wcnt[q] = s; s += v; } wcnt[TH / 32] = s; }
            __syncthreads();
            const int total = wcnt[TH / 32];
            const int off = wcnt[tid >> 5] + incl - pc;
            for (int bstart = 0; bstart < total; bstart += kDenseList) {
                { uint32_t wd = word; int o = off;
                  while (wd) { const int b = __ffs(wd) - 1; wd &= wd - 1;
                               if (o >= bstart && o < bstart + kDenseList) sp[o - bstart] = (int32_t)(((wi << 5) + b) - a.so);
                               ++o; } }
                __syncthreads();
                const int n = min(kDenseList, total - bstart);
                if (j < a.tn) {
                    // eight rows' weights loaded before any is used (the rows
                    // are distinct, so the stores below never feed a load)
                    constexpr int kB = 8;
                    int s = 0;
                    for (; s + kB <= n; s += kB) {
                        WT wl[kB];
#pragma unroll
                        for (int u = 0; u < kB; ++u) wl[u] = W[(int64_t)sp[s + u] * a.tn + j];
#pragma unroll
                        for (int u = 0; u < kB; ++u) {
                            const int64_t i = sp[s + u];
                            T wv = (T)wl[u];
                            if (a.mod) wv = rn<T>::mul(wv, a.mod[i]);
                            acc = rn<T>::add(acc, wv);
                            if (a.stdp) W[i * a.tn + j] = stdp_w_val<WT>(wl[u], apost, a.wmin, a.wmax, a.wmode, a.wx);
                        }
                    }
                    for (; s < n; ++s) {
                        const int64_t i = sp[s];
                        const int64_t k = i * a.tn + j;
                        const WT w0 = W[k];
                        T wv = (T)w0;
                        if (a.mod) wv = rn<T>::mul(wv, a.mod[i]);
                        acc = rn<T>::add(acc, wv);
                        if (a.stdp) W[k] = stdp_w_val<WT>(w0, apost, a.wmin, a.wmax, a.wmode, a.wx);
                    }
                }
                if (a.stdp && blockIdx.x == 0)
                    for (int s = tid; s < n; s += TH) {
                        const int64_t i = sp[s];
                        a.A_pre[i] = a.pre_set ? a.Ap : __dadd_rn(a.A_pre[i], a.Ap);
                    }
                if (blockIdx.x == 0 && tid == 0) ev += (unsigned long long)n * (unsigned long long)a.tn;
                __syncthreads();
            }
        }
        if (j < a.tn) a.sv[j] = acc;
        block_count(a.events, ev);
    }
    bg_finish_step(a.ctl, a.last);
}

// STDP trace decay (the G_pre/G_post groups' 1x1 linear updaters).
// On a DelayConnection the traces are also kept for `hlen` steps, as the
// RecentStateMonitors recording them at the end of each step do
// (monitor.py:1036-1049): the record of step s-1 is the trace before the
// decay of step s, so this kernel writes it into slot (s-1) mod hlen first.
struct DecayArgs {
    double *A_pre; int64_t npre; double a_pre, c_pre; double *A_post; int64_t npost; double a_post, c_post;
    double *H_pre, *H_post; int hlen;     // trace histories [hlen][n], or null
    DevCtl *ctl; int last;
};
static __global__ void k_stdp_decay(const DecayArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nstep = a.ctl->nstep;
    const bool rec = a.H_pre != nullptr && nstep > 0;
    const int64_t slot = rec ? (int64_t)((nstep - 1) % a.hlen) : 0;
    if (i < a.npre) {
        const double x = a.A_pre[i];
        if (rec) a.H_pre[slot * a.npre + i] = x;
        a.A_pre[i] = __dadd_rn(__dmul_rn(a.a_pre, x), a.c_pre);
    } else if (i < a.npre + a.npost) {
        const int64_t j = i - a.npre;
        const double x = a.A_post[j];
        if (rec) a.H_post[slot * a.npost + j] = x;
        a.A_post[j] = __dadd_rn(__dmul_rn(a.a_post, x), a.c_post);
    }
    bg_finish_step(a.ctl, a.last);
}

// Slot of the trace record `lag` records before the last one
// (monitor.py:1092: (current_time_index - 1 - lag) mod M, one record per
// step; lag < hlen); last = (nstep - 1) mod hlen, taken once per thread.
__device__ __forceinline__ int64_t hist_slot(int last, int lag, int hlen) {
    const int s = last - lag;
    return (int64_t)(s < 0 ? s + hlen : s);
}
__device__ __forceinline__ int hist_last(long long nstep, int hlen) {
    return (int)((nstep + hlen - 1) % hlen);
}

// Presynaptic rule on a DelayConnection (stdp.py:296-352): the immediate
// part, A_pre[i] (+)= Ap for this step's spikes, and the delayed part for
// the spikes of `delay` (the connection's max_delay) steps ago:
// w[i,k] += A_post[cols[k]] as recorded lag[k] records back; clip.
struct DelayedPreArgs {
    DevCtl *ctl;
    const uint32_t *hist; int depth; int64_t nwords; int delay;
    int64_t so, sn, tn;
    const int64_t *rowptr; const int32_t *cols; void *w;
    double *A_pre; double Ap; int pre_set;
    const double *H_post; int hlen; const uint8_t *lag;
    double wmin, wmax;
    int wmode; double wx;
    int last;
};
template <typename WT>
__global__ void __launch_bounds__(256) k_dstdp_pre(const DelayedPreArgs a) {
    const long long nstep = a.ctl->nstep;
    const int lane = threadIdx.x & 31;
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    const int64_t end = a.so + a.sn;
    const int64_t w0 = a.so >> 5, w1 = (end + 31) >> 5;
    {   // immediate: one thread per history word of this step
        const uint32_t *H = a.hist + (int64_t)((int)(nstep % a.depth)) * a.nwords;
        for (int64_t wi = w0 + gtid; wi < w1; wi += nthreads) {
            uint32_t wd = masked_word(H, wi, a.so, end);
            while (wd) {
                const int b = __ffs(wd) - 1; wd &= wd - 1;
                const int64_t i = (wi << 5) + b - a.so;
                a.A_pre[i] = a.pre_set ? a.Ap : __dadd_rn(a.A_pre[i], a.Ap);
            }
        }
    }
    if (nstep >= a.delay) {   // delayed: one warp per spike, lanes over the row
        const int64_t warp = gtid >> 5, nwarps = nthreads >> 5;
        const int hlast = hist_last(nstep, a.hlen);
        const uint32_t *H = a.hist + (int64_t)((int)((nstep - a.delay) % a.depth)) * a.nwords;
        WT *W = (WT *)a.w;
        for (int64_t wi0 = w0 + warp * 32; wi0 < w1; wi0 += nwarps * 32) {
            const int64_t wi = wi0 + lane;
            const uint32_t word = wi < w1 ? masked_word(H, wi, a.so, end) : 0u;
            uint32_t nz = __ballot_sync(0xffffffffu, word != 0u);
            while (nz) {
                const int l = __ffs(nz) - 1; nz &= nz - 1;
                uint32_t wd = __shfl_sync(0xffffffffu, word, l);
                const int64_t base = (wi0 + l) << 5;
                while (wd) {
                    const int b = __ffs(wd) - 1; wd &= wd - 1;
                    const int64_t i = base + b - a.so;
                    for (int64_t k = a.rowptr[i] + lane; k < a.rowptr[i + 1]; k += 32) {
                        const int64_t s = hist_slot(hlast, a.lag[k], a.hlen);
                        stdp_w<double, WT>(W, k, a.H_post[s * a.tn + a.cols[k]], a.wmin, a.wmax, a.wmode, a.wx);
                    }
                }
            }
        }
    }
    bg_finish_step(a.ctl, a.last);
}

// Standalone presynaptic STDP update (used when it cannot ride on the
// connection's propagation kernel).
template <typename WT>
__global__ void __launch_bounds__(256) k_stdp_pre(const PropArgs<double> a) {
    const long long nstep = a.ctl->nstep;
    if (nstep >= a.delay) {
        const int lane = threadIdx.x & 31;
        const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
        const uint32_t *H = a.hist + (int64_t)((int)(nstep - a.delay) % a.depth) * a.nwords;
        const int64_t end = a.so + a.sn;
        const int64_t w0 = a.so >> 5, w1 = (end + 31) >> 5;
        WT *W = (WT *)a.w;
        for (int64_t wi0 = w0 + warp * 32; wi0 < w1; wi0 += nwarps * 32) {
            const int64_t wi = wi0 + lane;
            const uint32_t word = wi < w1 ? masked_word(H, wi, a.so, end) : 0u;
            uint32_t nz = __ballot_sync(0xffffffffu, word != 0u);
            while (nz) {
                const int l = __ffs(nz) - 1; nz &= nz - 1;
                uint32_t wd = __shfl_sync(0xffffffffu, word, l);
                const int64_t base = (wi0 + l) << 5;
                while (wd) {
                    const int b = __ffs(wd) - 1; wd &= wd - 1;
                    const int64_t i = base + b - a.so;
                    const int64_t r0 = a.dense ? i * a.tn : a.rowptr[i];
                    const int64_t r1 = a.dense ? r0 + a.tn : a.rowptr[i + 1];
                    for (int64_t k = r0 + lane; k < r1; k += 32) {
                        const int64_t j = a.dense ? k - r0 : a.cols[k];
                        stdp_w<double, WT>(W, k, a.A_post[j], a.wmin, a.wmax, a.wmode, a.wx);
                    }
                    if (lane == 0) a.A_pre[i] = a.pre_set ? a.Ap : __dadd_rn(a.A_pre[i], a.Ap);
                }
            }
        }
    }
    bg_finish_step(a.ctl, a.last);
}

// Postsynaptic STDP update: for each target spike j, A_post[j] (+)= Am and
// w[:,j] += A_pre, clipped.  Columns of different spikes are disjoint.
struct PostArgs {
    DevCtl *ctl;
    const uint32_t *hist; int depth; int64_t nwords; int delay;
    int64_t to, tn, sn;
    void *w; int dense;
    const int64_t *colptr; const int64_t *colk; const int32_t *colsrc;
    double *A_post; const double *A_pre; double Am; int post_set; double wmin, wmax;
    // DelayConnection (stdp.py:296-368): w[:,j] += A_pre as recorded lag[p]
    // records back, lag in column order; null on a plain Connection
    const double *H_pre; int hlen; const uint8_t *lagc;
    int wmode; double wx;           // update form of the postsynaptic w line (stdp_w)
    int last;
};
template <typename WT>
__global__ void __launch_bounds__(256) k_stdp_post(const PostArgs a) {
    __shared__ int32_t sp[1024];
    __shared__ int ns;
    const long long nstep = a.ctl->nstep;
    const int hlast = a.H_pre ? hist_last(nstep, a.hlen) : 0;
    if (nstep >= a.delay) {
        const uint32_t *H = a.hist + (int64_t)((int)(nstep - a.delay) % a.depth) * a.nwords;
        const int64_t end = a.to + a.tn;
        const int64_t w0 = a.to >> 5, w1 = (end + 31) >> 5;
        WT *W = (WT *)a.w;
        for (int64_t cw = w0; cw < w1; cw += 32) {
            if (threadIdx.x == 0) ns = 0;
            __syncthreads();
            if (threadIdx.x < 32) {
                const int64_t wi = cw + threadIdx.x;
                uint32_t word = wi < w1 ? masked_word(H, wi, a.to, end) : 0u;
                const int pc = __popc(word);
                int incl = pc;
                for (int o = 1; o < 32; o <<= 1) { int v = __shfl_up_sync(0xffffffffu, incl, o); if ((int)threadIdx.x >= o) incl += v; }
                int o = incl - pc;
                while (word) { const int b = __ffs(word) - 1; word &= word - 1; sp[o++] = (int32_t)(((wi << 5) + b) - a.to); }
                if (threadIdx.x == 31) ns = incl;
            }
            __syncthreads();
            const int n = ns;
            for (int s = 0; s < n; ++s) {
                const int64_t j = sp[s];
                if (a.dense) {
                    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.sn; i += (int64_t)gridDim.x * blockDim.x)
                        stdp_w<double, WT>(W, i * a.tn + j, a.A_pre[i], a.wmin, a.wmax, a.wmode, a.wx);
                } else {
                    for (int64_t p = a.colptr[j] + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.colptr[j + 1];
                         p += (int64_t)gridDim.x * blockDim.x) {
                        const double add = a.H_pre ? a.H_pre[hist_slot(hlast, a.lagc[p], a.hlen) * a.sn + a.colsrc[p]]
                                                   : a.A_pre[a.colsrc[p]];
                        stdp_w<double, WT>(W, a.colk[p], add, a.wmin, a.wmax, a.wmode, a.wx);
                    }
                }
            }
            if (blockIdx.x == 0)
                for (int s = threadIdx.x; s < n; s += blockDim.x) {
                    const int64_t j = sp[s];
                    a.A_post[j] = a.post_set ? a.Am : __dadd_rn(a.A_post[j], a.Am);
                }
            __syncthreads();
        }
    }
    bg_finish_step(a.ctl, a.last);
}

// Postsynaptic STDP on a dense connection as a sweep over the rows:
// w[i,j] (+)= A_pre[i], clipped, for every target j that spiked this step
// (stdp.py:395-408; the column updates of different spikes touch disjoint
// elements, so one pass over the matrix applies all of them).  Each block
// takes bands of kPostRows rows; the spike bits of the step sit in shared
// memory and a group of 4 columns (one 16-byte vector of f32 weights) is
// loaded and stored only when one of its targets spiked.  Odd steps walk the
// bands from the end of the matrix, so the part of the previous step's sweep
// still in L2 is read first (measured on a 10 000 x 4096 matrix: 45 us a
// sweep against 56 us one way; L2 evict-last/evict-first hints on a leading
// part of the rows were slower still).  Block 0 also applies A_post[j] (+)= Am.
constexpr int kPostThreads = 256;
constexpr int kPostRows = 8;
constexpr int kPostVec = 4;                 // 16-byte groups per thread and row in flight
constexpr int kPostMaskWords = 2048;        // targets per pass: 65 536
// the lanes of one 16-byte group of f32 weights whose targets spiked
__device__ __forceinline__ void post_vec(float4 &v, uint32_t nib, double add, const PostArgs &a) {
    if (nib & 1u) v.x = stdp_w_val<float>(v.x, add, a.wmin, a.wmax, a.wmode, a.wx);
    if (nib & 2u) v.y = stdp_w_val<float>(v.y, add, a.wmin, a.wmax, a.wmode, a.wx);
    if (nib & 4u) v.z = stdp_w_val<float>(v.z, add, a.wmin, a.wmax, a.wmode, a.wx);
    if (nib & 8u) v.w = stdp_w_val<float>(v.w, add, a.wmin, a.wmax, a.wmode, a.wx);
}
template <typename WT>
__global__ void __launch_bounds__(kPostThreads) k_stdp_post_rows(const PostArgs a) {
    __shared__ uint32_t mask[kPostMaskWords];
    __shared__ int any;
    const long long nstep = a.ctl->nstep;
    if (nstep >= a.delay) {
        const uint32_t *H = a.hist + (int64_t)((int)(nstep - a.delay) % a.depth) * a.nwords;
        const int sh = (int)(a.to & 31);
        const int64_t wbase = a.to >> 5;
        const int64_t hend = a.nwords;
        WT *W = (WT *)a.w;
        const int64_t nb = (a.sn + kPostRows - 1) / kPostRows;
        for (int64_t c0 = 0; c0 < a.tn; c0 += (int64_t)kPostMaskWords * 32) {
            const int64_t cn = min((int64_t)kPostMaskWords * 32, a.tn - c0);
            const int nw = (int)((cn + 31) >> 5);
            if (threadIdx.x == 0) any = 0;
            __syncthreads();
            int mine = 0;
            for (int q = threadIdx.x; q < nw; q += kPostThreads) {
                // bits of targets to + c0 + 32q .. +31, shifted out of the history words
                const int64_t hw = wbase + ((c0 >> 5) + q);
                uint32_t lo = H[hw], hi = (sh && hw + 1 < hend) ? H[hw + 1] : 0u;
                uint32_t m = sh ? ((lo >> sh) | (hi << (32 - sh))) : lo;
                const int64_t left = cn - ((int64_t)q << 5);
                if (left < 32) m &= (1u << left) - 1u;
                mask[q] = m;
                mine |= (m != 0u);
            }
            if (mine) any = 1;
            __syncthreads();
            if (any) {
                if (blockIdx.x == 0)
                    for (int q = threadIdx.x; q < nw; q += kPostThreads) {
                        uint32_t m = mask[q];
                        while (m) {
                            const int b = __ffs(m) - 1; m &= m - 1;
                            const int64_t j = c0 + ((int64_t)q << 5) + b;
                            a.A_post[j] = a.post_set ? a.Am : __dadd_rn(a.A_post[j], a.Am);
                        }
                    }
                const bool vec = sizeof(WT) == 4 && (a.tn & 3) == 0 && (c0 & 3) == 0 &&
                                 (((uintptr_t)W) & 15) == 0;
                for (int64_t bb = blockIdx.x; bb < nb; bb += gridDim.x) {
                    const int64_t band = (nstep & 1) ? nb - 1 - bb : bb;
                    const int64_t r0 = band * kPostRows, r1 = min(a.sn, r0 + kPostRows);
                    if (vec) {
                        // two rows at a time, every 16-byte group of both
                        // loaded before any is updated and stored
                        for (int64_t i = r0; i < r1; i += 2) {
                            const bool two = i + 1 < r1;
                            const double add0 = a.A_pre[i], add1 = two ? a.A_pre[i + 1] : 0.0;
                            float4 *row0 = reinterpret_cast<float4 *>(W + i * a.tn + c0);
                            float4 *row1 = reinterpret_cast<float4 *>(W + (two ? i + 1 : i) * a.tn + c0);
                            for (int64_t cc = 0; cc < cn; cc += 4 * kPostThreads * kPostVec) {
                                float4 v0[kPostVec], v1[kPostVec];
                                uint32_t nib[kPostVec];
#pragma unroll
                                for (int u = 0; u < kPostVec; ++u) {
                                    const int64_t g = (cc >> 2) + threadIdx.x + u * kPostThreads;
                                    nib[u] = 4 * g < cn ? (mask[g >> 3] >> ((g & 7) * 4)) & 15u : 0u;
                                    if (nib[u]) { v0[u] = row0[g]; if (two) v1[u] = row1[g]; }
                                }
#pragma unroll
                                for (int u = 0; u < kPostVec; ++u) {
                                    if (!nib[u]) continue;
                                    const int64_t g = (cc >> 2) + threadIdx.x + u * kPostThreads;
                                    post_vec(v0[u], nib[u], add0, a);
                                    row0[g] = v0[u];
                                    if (two) { post_vec(v1[u], nib[u], add1, a); row1[g] = v1[u]; }
                                }
                            }
                        }
                    } else {
                        for (int64_t i = r0; i < r1; ++i) {
                            const double add = a.A_pre[i];
                            WT *row = W + i * a.tn + c0;
                            for (int64_t c = threadIdx.x; c < cn; c += kPostThreads)
                                if ((mask[c >> 5] >> (c & 31)) & 1u) stdp_w<double, WT>(row, c, add, a.wmin, a.wmax, a.wmode, a.wx);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    bg_finish_step(a.ctl, a.last);
}

// Synapses delivery (synapses.py:808-827, SpikeQueue of spikequeue.py:
// 69-330).  An event of a spike at step s through a synapse of delay d is
// applied at step s + d in the 'synapses' slot (after the connections,
// before the resets, network.py:365-380); the events reaching one target
// are applied in queue order.  Each target's incoming synapses are stored
// in that order (delay descending, then source, then synapse index) as
// words source | (d + 1) << 24 (a zero word is padding).  A block takes a tile of
// kSynTile consecutive targets: phase A tests the tile's words (all
// threads, kSynUnroll independent loads in flight each) against the
// sources' spike history and leaves one hit bit per synapse in shared
// memory; phase B gives each target a thread that applies its hits in
// order, statement by statement: x = x + term or x = x - term.  Tiles whose
// synapses exceed kSynChunk words are processed in chunks, each target
// keeping its values in registers across chunks.
constexpr int kSynMaxOps = 4;
constexpr int kSynThreads = 256;
constexpr int kSynTile = 32;
constexpr int kSynChunk = 8192;
constexpr int kSynUnroll = 8;
struct SynArgs {
    DevCtl *ctl;
    const uint32_t *hist; int depth; int64_t nwords;
    int64_t so, to, tn;
    const int64_t *colptr; const uint32_t *word;
    const double *term; int64_t nsyn;                      // [nops][nsyn], column order
    int nops, nslots;
    int slot_of[kSynMaxOps], sub[kSynMaxOps], slot_var[kSynMaxOps];
    double *S; int64_t npad;
    const int *use_pull;            // event path present: [step parity] 1 = the pull delivers this step
    int last;
};
static __global__ void __launch_bounds__(kSynThreads) k_syn_deliver(const SynArgs a) {
    __shared__ uint32_t mask[kSynChunk / 32];
    const long long nstep = a.ctl->nstep;
    if (a.use_pull && a.use_pull[nstep & 1] == 0) {   // the event bins deliver this step
        bg_finish_step(a.ctl, a.last);
        return;
    }
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int kWarps = kSynThreads / 32;
    const int64_t ntiles = (a.tn + kSynTile - 1) / kSynTile;
    // history row of step nstep - lag: (nstep mod depth) - lag, wrapped once
    // (lag <= depth - 1); no 64-bit modulo per synapse
    const int row0 = (int)nstep % a.depth;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t j0 = tile * kSynTile, j1 = min(a.tn, j0 + kSynTile);
        const int64_t P0 = a.colptr[j0], P1 = a.colptr[j1];
        const int64_t j = j0 + tid;
        const bool own = tid < kSynTile && j < j1;
        const int64_t q0 = own ? a.colptr[j] : 0, q1 = own ? a.colptr[j + 1] : 0;
        double x[kSynMaxOps];
#pragma unroll
        for (int s = 0; s < kSynMaxOps; ++s)
            x[s] = (own && q0 < q1 && s < a.nslots) ? a.S[(int64_t)a.slot_var[s] * a.npad + a.to + j] : 0.0;
        bool any = false;
        for (int64_t c0 = P0; c0 < P1; c0 += kSynChunk) {
            const int64_t c1 = min(P1, c0 + (int64_t)kSynChunk);
            const int nw = (int)((c1 - c0 + 31) >> 5);
            // phase A: word w of the chunk's mask is tested by warp w % kWarps
            for (int w0 = wid; w0 < nw; w0 += kWarps * kSynUnroll) {
                uint32_t wd[kSynUnroll];
#pragma unroll
                for (int u = 0; u < kSynUnroll; ++u) {
                    const int64_t p = c0 + (int64_t)(w0 + u * kWarps) * 32 + lane;
                    wd[u] = (w0 + u * kWarps < nw && p < c1) ? a.word[p] : 0u;
                }
                uint32_t hb[kSynUnroll];
#pragma unroll
                for (int u = 0; u < kSynUnroll; ++u) {
                    const int lag = (int)(wd[u] >> 24) - 1;
                    hb[u] = 0u;
                    if (lag >= 0 && nstep >= lag) {
                        const int64_t src = a.so + (int64_t)(wd[u] & 0xFFFFFFu);
                        int row = row0 - lag;
                        row += row < 0 ? a.depth : 0;
                        hb[u] = (a.hist[(int64_t)row * a.nwords + (src >> 5)] >> (src & 31)) & 1u;
                    }
                }
#pragma unroll
                for (int u = 0; u < kSynUnroll; ++u) {
                    const uint32_t m = __ballot_sync(0xffffffffu, hb[u] != 0u);
                    if (lane == 0 && w0 + u * kWarps < nw) mask[w0 + u * kWarps] = m;
                }
            }
            __syncthreads();
            // phase B: each target's hits within the chunk, in order
            if (own) {
                const int64_t lo = max(q0, c0), hi = min(q1, c1);
                for (int64_t p = lo; p < hi;) {
                    const int w = (int)((p - c0) >> 5), b = (int)((p - c0) & 31);
                    const int64_t wend = min(hi, c0 + (int64_t)(w + 1) * 32);
                    uint32_t m = mask[w] >> b;
                    const int nb = (int)(wend - p);
                    if (nb < 32) m &= (1u << nb) - 1u;
                    while (m) {
                        const int l = __ffs(m) - 1; m &= m - 1;
                        const int64_t q = p + l;
                        any = true;
#pragma unroll
                        for (int k = 0; k < kSynMaxOps; ++k) {
                            if (k >= a.nops) break;
                            const double t = a.term[(int64_t)k * a.nsyn + q];
#pragma unroll
                            for (int s = 0; s < kSynMaxOps; ++s)
                                if (s == a.slot_of[k]) x[s] = a.sub[k] ? __dsub_rn(x[s], t) : __dadd_rn(x[s], t);
                        }
                    }
                    p = wend;
                }
            }
            __syncthreads();
        }
        if (own && any) {
#pragma unroll
            for (int s = 0; s < kSynMaxOps; ++s)
                if (s < a.nslots) a.S[(int64_t)a.slot_var[s] * a.npad + a.to + j] = x[s];
        }
    }
    bg_finish_step(a.ctl, a.last);
}

// Synapses with code (plastic synapses, synapses.py:149-330, 400-510): per
// synapse variables in column order, the presynaptic code run for each event
// of a target in queue order (the reference's rounds over repeated targets
// run the whole code for one event of each target per round, so a target
// sees its events one by one in that order), then the postsynaptic code for
// every synapse of a target that spiked in this step (the post queue is read
// after the pre queues).  C is the generated policy: C::pre(x, sv, q, t, pre)
// and C::post(x, sv, q, t) with x the target's variables (slots), sv the
// synaptic arrays, q the synapse's column position, pre the source's
// variables that the code reads.
constexpr int kSynMaxVars = 8;
struct SynCodeArgs {
    DevCtl *ctl;
    const uint32_t *hist; int depth; int64_t nwords;        // source group's spike history
    const uint32_t *thist; int tdepth; int64_t tnwords;     // target group's (postsynaptic spikes)
    int64_t so, to, tn;
    const int64_t *colptr; const uint32_t *word;
    double *sv[kSynMaxVars];
    int nslots; int slot_var[kSynMaxOps];
    double *S; int64_t npad;                                 // target group state
    const double *Ssrc; int64_t snpad; int npre; int pre_var[kSynMaxOps];
    double dt;
    int has_post;
    int last;
};
template <typename C>
__device__ __forceinline__ void syn_code_body(const SynCodeArgs &a) {
    __shared__ uint32_t mask[kSynChunk / 32];
    const long long nstep = a.ctl->nstep;
    const double t = (double)(nstep + a.ctl->clock_off) * a.dt;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int kWarps = kSynThreads / 32;
    const int64_t ntiles = (a.tn + kSynTile - 1) / kSynTile;
    const int row0 = (int)nstep % a.depth;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t j0 = tile * kSynTile, j1 = min(a.tn, j0 + kSynTile);
        const int64_t P0 = a.colptr[j0], P1 = a.colptr[j1];
        const int64_t j = j0 + tid;
        const bool own = tid < kSynTile && j < j1;
        const int64_t q0 = own ? a.colptr[j] : 0, q1 = own ? a.colptr[j + 1] : 0;
        double x[kSynMaxOps];
#pragma unroll
        for (int s = 0; s < kSynMaxOps; ++s)
            x[s] = (own && q0 < q1 && s < a.nslots) ? a.S[(int64_t)a.slot_var[s] * a.npad + a.to + j] : 0.0;
        bool any = false;
        for (int64_t c0 = P0; c0 < P1; c0 += kSynChunk) {
            const int64_t c1 = min(P1, c0 + (int64_t)kSynChunk);
            const int nw = (int)((c1 - c0 + 31) >> 5);
            // hit bits of the chunk's synapses: kSynUnroll words in flight per warp
            for (int w0 = wid; w0 < nw; w0 += kWarps * kSynUnroll) {
                uint32_t wd[kSynUnroll];
#pragma unroll
                for (int u = 0; u < kSynUnroll; ++u) {
                    const int64_t p = c0 + (int64_t)(w0 + u * kWarps) * 32 + lane;
                    wd[u] = (w0 + u * kWarps < nw && p < c1) ? a.word[p] : 0u;
                }
#pragma unroll
                for (int u = 0; u < kSynUnroll; ++u) {
                    const int lag = (int)(wd[u] >> 24) - 1;
                    uint32_t hb = 0u;
                    if (lag >= 0 && nstep >= lag) {
                        const int64_t src = a.so + (int64_t)(wd[u] & 0xFFFFFFu);
                        int row = row0 - lag;
                        row += row < 0 ? a.depth : 0;
                        hb = (a.hist[(int64_t)row * a.nwords + (src >> 5)] >> (src & 31)) & 1u;
                    }
                    const uint32_t m = __ballot_sync(0xffffffffu, hb != 0u);
                    if (lane == 0 && w0 + u * kWarps < nw) mask[w0 + u * kWarps] = m;
                }
            }
            __syncthreads();
            if (own) {
                const int64_t lo = max(q0, c0), hi = min(q1, c1);
                for (int64_t p = lo; p < hi;) {
                    const int w = (int)((p - c0) >> 5), b = (int)((p - c0) & 31);
                    const int64_t wend = min(hi, c0 + (int64_t)(w + 1) * 32);
                    uint32_t m = mask[w] >> b;
                    const int nb = (int)(wend - p);
                    if (nb < 32) m &= (1u << nb) - 1u;
                    while (m) {
                        const int l = __ffs(m) - 1; m &= m - 1;
                        const int64_t q = p + l;
                        any = true;
                        double pv[kSynMaxOps];
#pragma unroll
                        for (int k = 0; k < kSynMaxOps; ++k) {
                            pv[k] = 0.0;
                            if (k < a.npre)
                                pv[k] = a.Ssrc[(int64_t)a.pre_var[k] * a.snpad + a.so + (int64_t)(a.word[q] & 0xFFFFFFu)];
                        }
                        C::pre(x, a.sv, q, t, pv);
                    }
                    p = wend;
                }
            }
            __syncthreads();
        }
        if (own && a.has_post && q0 < q1) {
            const int64_t tj = a.to + j;
            const int trow = (int)nstep % a.tdepth;
            if ((a.thist[(int64_t)trow * a.tnwords + (tj >> 5)] >> (tj & 31)) & 1u)
                for (int64_t q = q0; q < q1; ++q) C::post(x, a.sv, q, t);
        }
        if (own && any) {
#pragma unroll
            for (int s = 0; s < kSynMaxOps; ++s)
                if (s < a.nslots) a.S[(int64_t)a.slot_var[s] * a.npad + a.to + j] = x[s];
        }
    }
    bg_finish_step(a.ctl, a.last);
}

// Event-driven Synapses delivery.  The events of step t are the synapses of
// delay d of the sources that spiked at step t - d.  Each object keeps a
// ring of spike lists, one row per step (the sources that spiked then, in
// no particular order).  k_syn_gather appends this step's spikes to the
// ring (from the spike-history words) and walks, for every delay d >= 1,
// the list of step t - d (the delay-0 synapses come straight from the
// words), appending each event to the bin of its target's block of kSynBin
// targets, with a 64-bit key that sorts into the queue order of the pull
// above: target, then delay descending, then source, then the synapse's
// rank among the source's synapses of that delay (synapse index order).
// k_syn_bins gives each bin a block that sorts its events by key in shared
// memory and applies every target's events in that order -- the same
// additions in the same order as the pull, so the result is bit for bit the
// same.  A step whose events overflow a bin (or whose keys do not fit) is
// delivered by the pull's test instead, by the same blocks (use_pull), so
// the path is exact whatever the activity.
constexpr int kSynBin = 1024;          // targets per bin (one block)
constexpr int kSynBinCap = 4096;       // events per bin and step
struct SynEvArgs {
    DevCtl *ctl;
    const uint32_t *hist; int depth; int64_t nwords;
    int64_t so, sn, tn; int dmax;
    const int64_t *srcptr; const uint8_t *sd; const int32_t *stgt; const int32_t *sq;   // rows by source, (delay, synapse)
    const int32_t *doff;            // [sn][dmax + 2]: start of each delay within a source's row (or null)
    const int64_t *colptr; const uint32_t *word;                                         // the pull's columns
    int *bin_cnt; unsigned long long *bin_key; int32_t *bin_q; int nbins;
    int *use_pull;                  // [2] by step parity
    // spike lists: row (step % sdepth) holds scnt[row] source indices; with
    // sdepth >= dmax + 2 the row a step fills, the row it clears (the next
    // step's) and the rows it reads (steps t-1 .. t-dmax) are all different
    int32_t *slist; int *scnt; int sdepth;
    const double *term; int64_t nsyn;
    int nops, nslots;
    int slot_of[kSynMaxOps], sub[kSynMaxOps], slot_var[kSynMaxOps];
    double *S; int64_t npad; int64_t to;
    int last;
};

// Events of several Synapses objects gathered and applied by the same two
// launches (objects whose targets' variables do not overlap, so their
// order does not matter).  Gather: blocks [0, npair * nparts) walk the
// spike lists, (object, delay) pair p = block / nparts (object k owns pairs
// [pair0[k], pair0[k+1]), delays 1 .. dmax), each list split over nparts
// blocks; the blocks after them walk the history words of this step,
// object k owning words [item0[k], item0[k+1]).  Bins: object k owns bins
// [bin0[k], bin0[k+1]).
constexpr int kSynEvMerge = 4;
struct SynEvGroup {
    int nobj;
    SynEvArgs o[kSynEvMerge];
    int64_t item0[kSynEvMerge + 1];
    int pair0[kSynEvMerge + 1];
    int nparts;
    int bin0[kSynEvMerge + 1];
    DevCtl *ctl;
    int last;
};

// the synapses of source i (relative to the object's source range) with
// delay d: rows [r0, r1) of the by-source arrays
__device__ __forceinline__ void syn_src_range(const SynEvArgs &a, int64_t i, int d, int64_t &r0, int64_t &r1) {
    const int64_t lo = __ldg(a.srcptr + i);
    if (a.doff) {
        const int32_t *o = a.doff + i * (int64_t)(a.dmax + 2) + d;
        r0 = lo + __ldg(o);
        r1 = lo + __ldg(o + 1);
    } else {
        const int64_t hi = __ldg(a.srcptr + i + 1);
        int64_t l = lo, h = hi;
        while (l < h) { const int64_t m = (l + h) >> 1; if (a.sd[m] < d) l = m + 1; else h = m; }
        r0 = l;
        h = hi;
        while (l < h) { const int64_t m = (l + h) >> 1; if (a.sd[m] <= d) l = m + 1; else h = m; }
        r1 = l;
    }
}

// the events of source i's synapses of delay d, into the bins (bin_cnt,
// bin_key, bin_q: the object's bins or one parity of them)
__device__ __forceinline__ void syn_push_events(const SynEvArgs &a, int64_t i, int d, int *flag, int *bin_cnt,
                                                unsigned long long *bin_key, int32_t *bin_q) {
    int64_t r0, r1;
    syn_src_range(a, i, d, r0, r1);
    if (r1 - r0 > 256) { atomicExch(flag, 1); return; }
    // eight synapses at a time: their targets loaded, then their bin slots
    // taken, then their events written (one memory round trip per stage
    // instead of per synapse)
    for (int64_t p0 = r0; p0 < r1; p0 += 8) {
        const int m = r1 - p0 < 8 ? (int)(r1 - p0) : 8;
        int32_t tg[8], qs[8], slot[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (u < m) { tg[u] = __ldg(a.stgt + p0 + u); qs[u] = __ldg(a.sq + p0 + u); }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (u < m) slot[u] = atomicAdd(bin_cnt + tg[u] / kSynBin, 1);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (u >= m) break;
            if (slot[u] >= kSynBinCap) { atomicExch(flag, 1); continue; }
            const int64_t j = tg[u];
            const int64_t e = (j / kSynBin) * kSynBinCap + slot[u];
            bin_key[e] = ((unsigned long long)j << 40) | ((unsigned long long)(255 - d) << 32) |
                         ((unsigned long long)i << 8) | (unsigned long long)(p0 + u - r0);
            bin_q[e] = qs[u];
        }
    }
}

// history word x (of the object's source range) of step nstep: its spikes
// appended to the step's list, and their delay-0 events
__device__ __forceinline__ void syn_gather_word(const SynEvArgs &a, long long nstep, int64_t x) {
    const int64_t wi = (a.so >> 5) + x;
    uint32_t word = masked_word(a.hist + (int64_t)((int)nstep % a.depth) * a.nwords, wi, a.so, a.so + a.sn);
    if (!word) return;
    const int row = (int)nstep % a.sdepth;
    int pos = atomicAdd(a.scnt + row, __popc(word));
    int32_t *L = a.slist + (int64_t)row * a.sn;
    int *flag = a.use_pull + (nstep & 1);
    while (word) {
        const int b = __ffs(word) - 1; word &= word - 1;
        const int64_t i = (wi << 5) + b - a.so;
        L[pos++] = (int32_t)i;
        syn_push_events(a, i, 0, flag, a.bin_cnt, a.bin_key, a.bin_q);
    }
}

static __global__ void __launch_bounds__(256) k_syn_gather(const __grid_constant__ SynEvGroup g) {
    const long long nstep = g.ctl->nstep;
    const int nlist = g.pair0[g.nobj] * g.nparts;
    if (blockIdx.x == 0 && threadIdx.x < g.nobj) {
        // the next step's list row starts empty (no one reads it this step)
        const SynEvArgs &a = g.o[threadIdx.x];
        a.scnt[((int)nstep + 1) % a.sdepth] = 0;
    }
    if ((int)blockIdx.x < nlist) {
        const int pair = (int)blockIdx.x / g.nparts, part = (int)blockIdx.x % g.nparts;
        int k = 0;
        while (k + 1 < g.nobj && pair >= g.pair0[k + 1]) ++k;
        const SynEvArgs &a = g.o[k];
        const int d = 1 + pair - g.pair0[k];
        const int row = ((int)nstep - d + a.sdepth) % a.sdepth;
        const int cnt = nstep < d ? 0 : a.scnt[row];
        const int32_t *L = a.slist + (int64_t)row * a.sn;
        int *flag = a.use_pull + (nstep & 1);
        for (int e = part * blockDim.x + threadIdx.x; e < cnt; e += g.nparts * blockDim.x)
            syn_push_events(a, L[e], d, flag, a.bin_cnt, a.bin_key, a.bin_q);
    } else {
        const int64_t total = g.item0[g.nobj];
        for (int64_t x = ((int64_t)blockIdx.x - nlist) * blockDim.x + threadIdx.x; x < total;
             x += (int64_t)(gridDim.x - nlist) * blockDim.x) {
            int k = 0;
            while (k + 1 < g.nobj && x >= g.item0[k + 1]) ++k;
            syn_gather_word(g.o[k], nstep, x - g.item0[k]);
        }
    }
    bg_finish_step(g.ctl, g.last);
}

// The spike lists of steps t-1 .. t-dmax rebuilt from the spike history
// (before a run whose history did not come from the gather: a new or
// reinitialised network, a loaded state); the rows' counts are zero.
static __global__ void __launch_bounds__(256) k_syn_lists(const SynEvArgs a) {
    const long long nstep = a.ctl->nstep;
    const int64_t w0 = a.so >> 5, nw = ((a.so + a.sn + 31) >> 5) - w0;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < nw * a.dmax; x += (int64_t)gridDim.x * blockDim.x) {
        const int d = 1 + (int)(x / nw);
        const int64_t wi = w0 + x % nw;
        if (nstep < d) continue;
        uint32_t word = masked_word(a.hist + (int64_t)(((int)nstep - d) % a.depth) * a.nwords, wi, a.so, a.so + a.sn);
        if (!word) continue;
        const int row = (int)((nstep - d) % a.sdepth);
        int pos = atomicAdd(a.scnt + row, __popc(word));
        while (word) {
            const int b = __ffs(word) - 1; word &= word - 1;
            a.slist[(int64_t)row * a.sn + pos++] = (int32_t)((wi << 5) + b - a.so);
        }
    }
}

constexpr int kSynBinThreads = 512;
constexpr int kSynTPT = kSynBin / kSynBinThreads;       // targets per thread
constexpr int kSynSegMax = 64;                          // events of one target per step sorted by its thread
static_assert(kSynTPT == 2, "two targets per thread of a bin block");

// The events of one bin (step nstep, n events in gkey/gq) applied per target
// in key order -- the pull's order -- or, when `pull` (the step overflowed),
// the pull's test for every target of the bin.  Thread t serves the bin's
// targets t and t + kSynBinThreads (u = 0, 1): f.begin(u, j) before the
// first event of its target u (bin target index j), f.add(u, q) per event
// (synapse column q), f.end(u, j) after the last.  The block's
// kSynBinThreads threads all call it (it synchronises); dynamic shared memory
// holds kSynBinCap keys and positions.
template <class F>
__device__ __forceinline__ void syn_bin_apply(const SynEvArgs &a, long long nstep, int bin, bool pull, int n,
                                              const unsigned long long *gkey, const int32_t *gq, F &f) {
    extern __shared__ unsigned char syn_smem[];
    unsigned long long *key = reinterpret_cast<unsigned long long *>(syn_smem);
    int32_t *qv = reinterpret_cast<int32_t *>(key + kSynBinCap);
    const int tid = threadIdx.x;
    const int64_t jb = (int64_t)bin * kSynBin;                  // the bin's first target
    if (pull) {
        // every target of the bin walks its incoming synapses in queue order
        // and applies those whose source spiked d steps ago (the pull's test)
        const int row0 = (int)nstep % a.depth;
#pragma unroll
        for (int u = 0; u < kSynTPT; ++u) {
            const int64_t j = jb + u * kSynBinThreads + tid;
            if (j >= a.tn) continue;
            bool any = false;
            for (int64_t q = a.colptr[j]; q < a.colptr[j + 1]; ++q) {
                const uint32_t wd = a.word[q];
                const int lag = (int)(wd >> 24) - 1;
                if (lag < 0 || nstep < lag) continue;
                const int64_t src = a.so + (int64_t)(wd & 0xFFFFFFu);
                int row = row0 - lag;
                row += row < 0 ? a.depth : 0;
                if (!((__ldcg(a.hist + (int64_t)row * a.nwords + (src >> 5)) >> (src & 31)) & 1u)) continue;
                if (!any) f.begin(u, j);
                any = true;
                f.add(u, q);
            }
            if (any) f.end(u, j);
        }
        return;
    }
    if (n <= 0) return;
    // events per target (a counting sort by target): each target's events go
    // to its own segment, which its thread then orders by key (insertion
    // sort: a target's events in one step are few); a bin with a target of
    // more than kSynSegMax events takes the bitonic sort of the whole bin
    __shared__ int tcnt[kSynBin];
    __shared__ int wsum[kSynBinThreads / 32], maxc;
    const int lane = tid & 31, warp = tid >> 5;
    // the bin's first kSynBinThreads events stay in registers between the
    // count and the placement
    unsigned long long k0 = 0;
    int32_t q0 = 0;
    if (tid < n) { k0 = __ldcg(gkey + tid); q0 = __ldcg(gq + tid); }
#pragma unroll
    for (int u = 0; u < kSynTPT; ++u) tcnt[u * kSynBinThreads + tid] = 0;
    if (tid == 0) maxc = 0;
    __syncthreads();
    if (tid < n) atomicAdd(&tcnt[(int)((k0 >> 40) - (unsigned long long)jb)], 1);
    for (int e = tid + kSynBinThreads; e < n; e += kSynBinThreads)
        atomicAdd(&tcnt[(int)((__ldcg(gkey + e) >> 40) - (unsigned long long)jb)], 1);
    __syncthreads();
    int cu[kSynTPT], c = 0, cmax = 0;
#pragma unroll
    for (int u = 0; u < kSynTPT; ++u) { cu[u] = tcnt[u * kSynBinThreads + tid]; c += cu[u]; cmax = max(cmax, cu[u]); }
    if (cmax) atomicMax(&maxc, cmax);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += v; }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int v = lane < kSynBinThreads / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { const int u = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v += u; }
        if (lane < kSynBinThreads / 32) wsum[lane] = v;
    }
    __syncthreads();
    const int beg = (warp ? wsum[warp - 1] : 0) + incl - c;    // the thread's segments, u = 0 then 1
    if (maxc <= kSynSegMax) {                                    // uniform
        {
            int b = beg;                                         // the segments' fill cursors
#pragma unroll
            for (int u = 0; u < kSynTPT; ++u) { tcnt[u * kSynBinThreads + tid] = b; b += cu[u]; }
        }
        __syncthreads();
        if (tid < n) {
            const int pos = atomicAdd(&tcnt[(int)((k0 >> 40) - (unsigned long long)jb)], 1);
            key[pos] = k0;
            qv[pos] = q0;
        }
        for (int e = tid + kSynBinThreads; e < n; e += kSynBinThreads) {
            const unsigned long long k = __ldcg(gkey + e);
            const int pos = atomicAdd(&tcnt[(int)((k >> 40) - (unsigned long long)jb)], 1);
            key[pos] = k;
            qv[pos] = __ldcg(gq + e);
        }
        __syncthreads();
        int sb = beg;
#pragma unroll
        for (int u = 0; u < kSynTPT; ++u) {
            const int64_t j = jb + u * kSynBinThreads + tid;
            const int cc = cu[u];
            if (cc && j < a.tn) {
                for (int v = sb + 1; v < sb + cc; ++v) {
                    const unsigned long long kk = key[v];
                    const int32_t qq = qv[v];
                    int w = v - 1;
                    while (w >= sb && key[w] > kk) { key[w + 1] = key[w]; qv[w + 1] = qv[w]; --w; }
                    key[w + 1] = kk;
                    qv[w + 1] = qq;
                }
                f.begin(u, j);
                for (int e = sb; e < sb + cc; ++e) f.add(u, qv[e]);
                f.end(u, j);
            }
            sb += cc;
        }
    } else {
        int m = 1;
        while (m < n) m <<= 1;
        for (int e = tid; e < m; e += kSynBinThreads) {
            if (e < n) { key[e] = __ldcg(gkey + e); qv[e] = __ldcg(gq + e); }
            else { key[e] = ~0ull; qv[e] = 0; }
        }
        __syncthreads();
        // bitonic sort of (key, q) by key (keys are distinct)
        for (int k = 2; k <= m; k <<= 1) {
            for (int jj = k >> 1; jj > 0; jj >>= 1) {
                for (int e = tid; e < m; e += kSynBinThreads) {
                    const int o = e ^ jj;
                    if (o > e) {
                        const bool up = (e & k) == 0;
                        const unsigned long long ka = key[e], kb = key[o];
                        if ((ka > kb) == up) {
                            key[e] = kb; key[o] = ka;
                            const int32_t t = qv[e]; qv[e] = qv[o]; qv[o] = t;
                        }
                    }
                }
                __syncthreads();
            }
        }
        // each target of the thread: its events, in key order
#pragma unroll
        for (int u = 0; u < kSynTPT; ++u) {
            const int64_t j = jb + u * kSynBinThreads + tid;
            if (j >= a.tn || !cu[u]) continue;
            const unsigned long long want = (unsigned long long)j;
            int l = 0, h = n;
            while (l < h) { const int mm = (l + h) >> 1; if ((key[mm] >> 40) < want) l = mm + 1; else h = mm; }
            f.begin(u, j);
            for (int e = l; e < n && (key[e] >> 40) == want; ++e) f.add(u, qv[e]);
            f.end(u, j);
        }
    }
    __syncthreads();                                             // shared memory free for the next bin
}

// the stepped path's target access: the target's slots loaded from the
// group state, the statements applied, stored back
struct SynSlotsF {
    const SynEvArgs &a;
    double x[kSynTPT][kSynMaxOps];
    __device__ void begin(int u, int64_t j) {
#pragma unroll
        for (int s = 0; s < kSynMaxOps; ++s) x[u][s] = s < a.nslots ? a.S[(int64_t)a.slot_var[s] * a.npad + a.to + j] : 0.0;
    }
    __device__ void add(int u, int64_t q) {
#pragma unroll
        for (int k = 0; k < kSynMaxOps; ++k) {
            if (k >= a.nops) break;
            const double t = a.term[(int64_t)k * a.nsyn + q];
#pragma unroll
            for (int s = 0; s < kSynMaxOps; ++s)
                if (s == a.slot_of[k]) x[u][s] = a.sub[k] ? __dsub_rn(x[u][s], t) : __dadd_rn(x[u][s], t);
        }
    }
    __device__ void end(int u, int64_t j) {
#pragma unroll
        for (int s = 0; s < kSynMaxOps; ++s)
            if (s < a.nslots) a.S[(int64_t)a.slot_var[s] * a.npad + a.to + j] = x[u][s];
    }
};

// one bin of one object on the stepped path, then the bin emptied for the
// next step
__device__ __forceinline__ void syn_bins_block(const SynEvArgs &a, long long nstep, int bin) {
    const int n = min(a.bin_cnt[bin], kSynBinCap);
    const bool pull = a.use_pull[nstep & 1] != 0;
    __syncthreads();   // every thread has read the bin's count before thread 0 clears it
    SynSlotsF f{a};
    syn_bin_apply(a, nstep, bin, pull, n, a.bin_key + (int64_t)bin * kSynBinCap, a.bin_q + (int64_t)bin * kSynBinCap, f);
    if (threadIdx.x == 0) {
        a.bin_cnt[bin] = 0;                             // empty for the next step
        if (bin == 0) a.use_pull[(nstep + 1) & 1] = 0;  // next step's flag (nobody reads it this step)
    }
}

static __global__ void __launch_bounds__(kSynBinThreads, 4) k_syn_bins(const __grid_constant__ SynEvGroup g) {
    int k = 0;
    while (k + 1 < g.nobj && (int)blockIdx.x >= g.bin0[k + 1]) ++k;
    syn_bins_block(g.o[k], g.ctl->nstep, (int)blockIdx.x - g.bin0[k]);
    bg_finish_step(g.ctl, g.last);
}

// SpikeMonitor (monitor.py:156-166): one block appends the step's spikes in
// ascending order.  A pass covers kMonThreads * kMonWords history words: they
// are loaded at once (coalesced, into shared memory), thread t then owns the
// kMonWords consecutive words from t * kMonWords, and one block-wide prefix
// sum of the threads' spike counts gives every spike its slot.
struct MonArgs {
    DevCtl *ctl;
    const uint32_t *hist; int depth; int64_t nwords; int delay;
    int64_t origin, n;
    long long *cnt; int64_t cap; int32_t *idx; int32_t *steps;   // steps relative to the chunk base
    const long long *step_base;
    int last;
};
constexpr int kMonThreads = 1024;
constexpr int kMonWords = 8;
static __global__ void __launch_bounds__(kMonThreads) k_spikemon(const MonArgs a) {
    __shared__ uint32_t sw[kMonThreads * kMonWords + kMonThreads * kMonWords / 32];   // one pad word per 32: no bank conflicts either way
    __shared__ int wcnt[kMonThreads / 32];
    const long long nstep = a.ctl->nstep;
    if (nstep >= a.delay && blockIdx.x == 0) {
        const long long cs = nstep + a.ctl->clock_off;
        const int32_t srel = (int32_t)(cs - *a.step_base);
        const uint32_t *H = a.hist + (int64_t)((int)(nstep - a.delay) % a.depth) * a.nwords;
        const int64_t end = a.origin + a.n;
        const int64_t w0 = a.origin >> 5, w1 = (end + 31) >> 5;
        long long base = *a.cnt;
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        for (int64_t cw = w0; cw < w1; cw += kMonThreads * kMonWords) {
#pragma unroll
            for (int u = 0; u < kMonWords; ++u) {
                const int e = u * kMonThreads + tid;
                const int64_t wi = cw + e;
                sw[e + (e >> 5)] = wi < w1 ? masked_word(H, wi, a.origin, end) : 0u;
            }
            __syncthreads();
            uint32_t wd[kMonWords];
            int pc = 0;
#pragma unroll
            for (int u = 0; u < kMonWords; ++u) {
                const int e = tid * kMonWords + u;
                wd[u] = sw[e + (e >> 5)];
                pc += __popc(wd[u]);
            }
            int incl = pc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += v; }
            if (lane == 31) wcnt[warp] = incl;
            __syncthreads();
            int wpre = 0, tot = 0;
            {
                const int v = wcnt[lane];
                int sc = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) { const int x = __shfl_up_sync(0xffffffffu, sc, o); if (lane >= o) sc += x; }
                wpre = __shfl_sync(0xffffffffu, sc - v, warp);
                tot = __shfl_sync(0xffffffffu, sc, 31);
            }
            long long o = base + wpre + incl - pc;
#pragma unroll
            for (int u = 0; u < kMonWords; ++u) {
                uint32_t word = wd[u];
                const int64_t wi = cw + tid * kMonWords + u;
                while (word) {
                    const int b = __ffs(word) - 1; word &= word - 1;
                    if (o < a.cap) { a.idx[o] = (int32_t)(((wi << 5) + b) - a.origin); a.steps[o] = srel; }
                    else bg_raise(a.ctl, BG_DERR_MONITOR_OVERFLOW, o);
                    ++o;
                }
            }
            base += tot;
            __syncthreads();
        }
        if (tid == 0) *a.cnt = base;
    }
    bg_finish_step(a.ctl, a.last);
}

}  // namespace bg
