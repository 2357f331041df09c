// bg_persist.cuh -- one cooperative launch runs many steps of a single
// linear group whose outgoing connections are shared-weight DelayConnections
// or zero-delay Connections onto itself: the CUBA topology of Brian's
// benchmarks (CUBA-4000 with its StateMonitor, CUBA-262k with delays).
//
// Each block owns TH x NPT neurons for the whole launch and keeps their state
// in registers; the row pointers of those neurons are staged in shared memory
// once.  A step is: [wait] -> ring delivery + reset of the previous step ->
// linear update + threshold -> push of this block's spikes into the rings ->
// arrive.  Ring row r is delivered at step t+1 when r = t mod md and receives
// pushes from steps t-d (d >= 1), so delivering at step t+1 needs the pushes
// of steps <= t-1 of every block, i.e. the arrivals of step t-1: blocks may
// drift one step apart and the wait is nearly always already satisfied.
// (With a zero delay the wait is for step t.)  The two spare ring rows keep a
// block that is one step ahead from pushing into a row that a lagging block
// is still delivering.  Thread 0 publishes the arrival (a release: one L2
// round trip) while warp 1 polls for the next step's wait (an acquire: one
// more), so the two overlap.  Every wait is bounded; on timeout the block
// raises BG_DERR_TIMEOUT and leaves the loop.
#pragma once
#include "bg_kernels.cuh"

namespace bg {

constexpr int kPersistMaxPush = 2;
constexpr int kPersistMaxDeliv = 2;     // every connection targets the group itself
constexpr int kPersistTable = 2048;     // shared-memory entries for count tables

template <typename T> struct PersistArgs {
    DevCtl *ctl;
    T *S; int64_t n, npad;
    T A[kMaxVars * kMaxVars]; T C[kMaxVars]; int useC;
    uint64_t anz; uint32_t cnz;    // nonzero masks of A and C
    int thr_kind, thr_var, thr_var2; T thr_val;
    int reset_kind, reset_var, reset_var2; T reset_val;
    uint32_t *hist; int depth; int64_t nwords;
    int ndeliv; Deliv<T> deliv[kMaxDeliv];
    int npush; Push<T> push[kPersistMaxPush];
    unsigned long long *spikes;
    unsigned int *arrived;      // [4] arrivals per step mod 4 (zeroed before the launch)
    int nsteps;
    int lag;                    // 1 when some delay is zero, else 2
    uint32_t *mon_words;        // spike monitors: spike words of each step of the launch, else null
    int64_t mon_stride;         // words per step in mon_words
    unsigned int spin_limit;    // polls of a wait before it gives up (BG_DERR_TIMEOUT)
    int hold_block;             // test hook: this block never publishes its arrivals (-1: none)
    // zero-delay Connections (connection.py:224-256): bit d set when delivery
    // d adds the shared weight once per event, sv = sv + w, k times in a row
    // (the reference's additions), instead of the k-fold sum of a ring entry
    uint32_t direct_mask;
    int nrec; RecDev rec[kMaxRec];   // StateMonitors of the group ('end' slot, after the resets);
                                     // blk_lo holds the ranges of this kernel's blocks
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_add(unsigned int *p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// DIAG: the host found A's nonzeros to be exactly its first row and its
// diagonal, and C's to be at most its first entry (a potential driven by
// decaying synaptic variables, as in CUBA), so the update needs no mask tests.
template <typename T, int NV, int TH, int NPT, bool DIAG>
__global__ void __launch_bounds__(TH, TH <= 512 ? 2 : 1) k_persist(const PersistArgs<T> a) {
    constexpr int BN = TH * NPT;                                // neurons per block
    static_assert(TH >= 64 && TH % 32 == 0, "thread 0 arrives while warp 1 polls");
    // row pointers of the block's neurons, relative to the first one (the
    // host keeps the persistent path to blocks whose rows span < 2^32)
    __shared__ uint32_t srp[kPersistMaxPush][BN + 1];
    __shared__ int64_t srp0[kPersistMaxPush];
    __shared__ uint32_t words[BN / 32];
    __shared__ int32_t sl[BN];
    __shared__ int64_t srow[kPushBatch];
    __shared__ int32_t spref[kPushBatch + 1];
    __shared__ int64_t srow1[kPersistMaxPush][kPushBatch];      // first batch, per connection
    __shared__ int32_t spref1[kPersistMaxPush][kPushBatch + 1];
    __shared__ int nsp, abort_flag;
    __shared__ T stash[BN];                      // StateMonitor values of the block's neurons
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int base = blockIdx.x * BN;               // neuron counts < 2^31
    const int nvalid = (int)min((int64_t)BN, a.n - (int64_t)base);
    const unsigned int G = gridDim.x;
    const long long t0 = a.ctl->nstep;
    for (int p = 0; p < a.npush; ++p) {
        const Push<T> &q = a.push[p];
        const int64_t r0 = min(max((int64_t)base - q.so, (int64_t)0), q.sn);
        for (int j = tid; j <= BN; j += TH) {
            int64_t r = (int64_t)base + j - q.so;
            r = r < 0 ? 0 : (r > q.sn ? q.sn : r);
            srp[p][j] = (uint32_t)(q.rowptr[r] - q.rowptr[r0]);
        }
        if (tid == 0) srp0[p] = q.rowptr[r0];
    }
    if (tid == 0) abort_flag = 0;
    // deliveries: which of this thread's neurons each one targets (bit u),
    // the thread's column in ring row 0, and the row delivered next (ring
    // rows advance by one per step: no division in the loop)
    uint32_t dm[kPersistMaxDeliv];
    int drow[kPersistMaxDeliv];
    int64_t dcol[kPersistMaxDeliv];
#pragma unroll
    for (int d = 0; d < kPersistMaxDeliv; ++d) {
        dm[d] = 0; drow[d] = 0; dcol[d] = 0;
        if (d < a.ndeliv) {
            const Deliv<T> &dv = a.deliv[d];
#pragma unroll
            for (int u = 0; u < NPT; ++u) {
                const int li = u * TH + tid;
                const int64_t gi = (int64_t)base + li;
                if (li < nvalid && gi >= dv.to && gi < dv.to + dv.tn) dm[d] |= 1u << u;
            }
            drow[d] = (int)(t0 % dv.md);         // row of the first delivery (step t0)
            dcol[d] = (int64_t)base - dv.to + tid;
        }
    }
    // count tables staged in shared memory when they fit (uniform decision)
    __shared__ T stab[kPersistTable];
    int toff[kPersistMaxDeliv];
    bool staged = true;
    {
        int o = 0;
#pragma unroll
        for (int d = 0; d < kPersistMaxDeliv; ++d) {
            toff[d] = o;
            if (d < a.ndeliv && a.deliv[d].cring) {
                if (a.deliv[d].tablen <= 0) staged = false;
                o += a.deliv[d].tablen;
            }
        }
        if (o > kPersistTable) staged = false;
        if (staged)
            for (int d = 0; d < a.ndeliv; ++d)
                if (a.deliv[d].cring)
                    for (int k = tid; k < a.deliv[d].tablen; k += TH) stab[toff[d] + k] = a.deliv[d].table[k];
    }
    // pushes whose source range meets this block (uniform)
    bool pact[kPersistMaxPush];
#pragma unroll
    for (int p = 0; p < kPersistMaxPush; ++p)
        pact[p] = p < a.npush && a.push[p].so < (int64_t)base + BN && a.push[p].so + a.push[p].sn > base;
    T s[NPT][NV];
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
        const int li = u * TH + tid;
#pragma unroll
        for (int k = 0; k < NV; ++k) s[u][k] = li < nvalid ? a.S[k * a.npad + base + li] : T(0);
    }
    int pcur[kPersistMaxPush];                  // ring row of the current step, per push
#pragma unroll
    for (int p = 0; p < kPersistMaxPush; ++p) pcur[p] = p < a.npush ? (int)(t0 % a.push[p].md) : 0;
    unsigned int prev_spk = 0;                  // bit u: neuron u spiked last step
    unsigned long long my_spikes = 0, my_events[kPersistMaxPush] = {0, 0};
    __syncthreads();

    for (int st = 0; st <= a.nsteps; ++st) {    // st == nsteps: tail of the last step only
        const long long t = t0 + st;
        if (st > 0) {
            // local step whose pushes must be complete in every block
            const long long le = (t - 1 - (a.lag == 2 ? 1 : 0)) - t0;
            if (le >= 0) {
                // warp 1 polls while thread 0 may still be in the release of
                // the previous step's arrival: the two round trips overlap
                if (tid == 32) {
                    // arrivals are counted per step (slot le % 4): a running sum
                    // would also count blocks that are already one step ahead
                    const unsigned int *ctr = a.arrived + (le & 3);
                    const unsigned int target = (unsigned int)((le >> 2) + 1) * G;
                    unsigned int it = 0;
                    while (ld_acquire_u32(ctr) < target) {
                        if (++it > a.spin_limit) { abort_flag = 1; bg_raise(a.ctl, BG_DERR_TIMEOUT, t); break; }
                        __nanosleep(32);
                    }
                }
                __syncthreads();
                if (abort_flag) break;
            }
            // issue every count-ring load of every delivery first: one L2
            // latency for all of them
            uint16_t cnt[kPersistMaxDeliv][NPT];
            uint16_t *crow[kPersistMaxDeliv];
#pragma unroll
            for (int d = 0; d < kPersistMaxDeliv; ++d) {
                crow[d] = nullptr;
#pragma unroll
                for (int u = 0; u < NPT; ++u) cnt[d][u] = 0;
                if (d < a.ndeliv && a.deliv[d].cring) {
                    const Deliv<T> &dv = a.deliv[d];
                    crow[d] = dv.cring + (int64_t)drow[d] * dv.tnp + dcol[d];
#pragma unroll
                    for (int u = 0; u < NPT; ++u)
                        if ((dm[d] >> u) & 1u) cnt[d][u] = __ldcg(crow[d] + u * TH);
                }
            }
            // then add in connection order (the reference's delivery order)
#pragma unroll
            for (int d = 0; d < kPersistMaxDeliv; ++d) {
                if (d >= a.ndeliv) break;
                const Deliv<T> &dv = a.deliv[d];
                if (dv.cring && ((a.direct_mask >> d) & 1u)) {
                    // table[1] = 0 + w = w: one addition of the weight per event
                    const T w = staged ? stab[toff[d] + 1] : __ldg(dv.table + 1);
                    on_var<NV>(dv.var, [&](auto K) {
                        constexpr int k = decltype(K)::value;
#pragma unroll
                        for (int u = 0; u < NPT; ++u) {
                            const int c = cnt[d][u];
                            if (c) crow[d][u * TH] = 0;
                            for (int q = 0; q < c; ++q) s[u][k] = rn<T>::add(s[u][k], w);
                        }
                    });
                } else if (dv.cring) {
                    T v[NPT];
#pragma unroll
                    for (int u = 0; u < NPT; ++u) {
                        const int c = cnt[d][u];
                        if (c) crow[d][u * TH] = 0;
                        v[u] = c ? (staged ? stab[toff[d] + c] : __ldg(dv.table + c)) : T(0);
                    }
                    on_var<NV>(dv.var, [&](auto K) {
                        constexpr int k = decltype(K)::value;
#pragma unroll
                        for (int u = 0; u < NPT; ++u) s[u][k] = rn<T>::add(s[u][k], v[u]);
                    });
                } else {
                    T *row = dv.ring + (int64_t)drow[d] * dv.tn + dcol[d];
#pragma unroll
                    for (int u = 0; u < NPT; ++u) {
                        if ((dm[d] >> u) & 1u) {
                            const T v = __ldcg(row + u * TH);
                            if (v != T(0)) row[u * TH] = T(0);
                            uset<T, NV>(s[u], dv.var, rn<T>::add(uget<T, NV>(s[u], dv.var), v));
                        }
                    }
                }
                drow[d] = drow[d] + 1 == dv.md ? 0 : drow[d] + 1;
            }
            if (a.reset_kind == 1) {
                on_var<NV>(a.reset_var, [&](auto K) {
                    constexpr int k = decltype(K)::value;
#pragma unroll
                    for (int u = 0; u < NPT; ++u)
                        if ((prev_spk >> u) & 1u) s[u][k] = a.reset_val;
                });
            } else if (a.reset_kind) {
#pragma unroll
                for (int u = 0; u < NPT; ++u)
                    if ((prev_spk >> u) & 1u) uset<T, NV>(s[u], a.reset_var, uget<T, NV>(s[u], a.reset_var2));
            }
            // StateMonitors ('end' slot, after the resets) of the step just
            // finished: the block's recorded neurons through shared memory
            for (int r = 0; r < a.nrec; ++r) {
                const RecDev &m = a.rec[r];
                const long long rel = (t - 1) - m.start;
                if (rel < 0 || rel % m.timestep) continue;       // block-uniform
#pragma unroll
                for (int u = 0; u < NPT; ++u) stash[u * TH + tid] = uget<T, NV>(s[u], m.var);
                __syncthreads();
                const long long row = rel / m.timestep - *m.row_base;
                const int e0 = m.blk_lo[blockIdx.x], e1 = m.blk_lo[blockIdx.x + 1];
                for (int e = e0 + tid; e < e1; e += TH) ((T *)m.buf)[row * m.nidx + m.pos[e]] = stash[m.idx[e] - base];
                __syncthreads();
            }
        }
        if (st == a.nsteps) break;
        // ---- update, threshold, history
        prev_spk = 0;
        {
            // x = A s (+ C), each row summed over k in ascending order with the
            // zero coefficients skipped (the order of linear_row); the mask
            // tests are uniform and run once per thread, not per neuron
            T x[NPT][NV];
            if constexpr (DIAG) {
                // the same sums as below with the zero terms already left out
#pragma unroll
                for (int u = 0; u < NPT; ++u) {
                    T acc = T(0);
#pragma unroll
                    for (int k = 0; k < NV; ++k) acc = rn<T>::add(acc, rn<T>::mul(a.A[k], s[u][k]));
                    x[u][0] = acc;
#pragma unroll
                    for (int j = 1; j < NV; ++j) x[u][j] = rn<T>::add(T(0), rn<T>::mul(a.A[j * NV + j], s[u][j]));
                }
                if (a.cnz & 1u) {
#pragma unroll
                    for (int u = 0; u < NPT; ++u) x[u][0] = rn<T>::add(x[u][0], a.C[0]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < NV; ++j) {
#pragma unroll
                    for (int u = 0; u < NPT; ++u) x[u][j] = T(0);
#pragma unroll
                    for (int k = 0; k < NV; ++k)
                        if (a.anz & (1ull << (j * NV + k))) {
                            const T c = a.A[j * NV + k];
#pragma unroll
                            for (int u = 0; u < NPT; ++u) x[u][j] = rn<T>::add(x[u][j], rn<T>::mul(c, s[u][k]));
                        }
                    if (a.cnz & (1u << j)) {
#pragma unroll
                        for (int u = 0; u < NPT; ++u) x[u][j] = rn<T>::add(x[u][j], a.C[j]);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < NPT; ++u)
#pragma unroll
                for (int j = 0; j < NV; ++j) s[u][j] = x[u][j];
        }
        bool spk[NPT];
#pragma unroll
        for (int u = 0; u < NPT; ++u) spk[u] = false;
        if (a.thr_kind == 1) {
            on_var<NV>(a.thr_var, [&](auto K) {
                constexpr int k = decltype(K)::value;
#pragma unroll
                for (int u = 0; u < NPT; ++u) spk[u] = s[u][k] > a.thr_val;
            });
        } else if (a.thr_kind == 2) {
#pragma unroll
            for (int u = 0; u < NPT; ++u) spk[u] = uget<T, NV>(s[u], a.thr_var) > uget<T, NV>(s[u], a.thr_var2);
        }
#pragma unroll
        for (int u = 0; u < NPT; ++u) {
            const int li = u * TH + tid;
            spk[u] = spk[u] && li < nvalid;
            prev_spk |= (spk[u] ? 1u : 0u) << u;
            const uint32_t ball = __ballot_sync(0xffffffffu, spk[u]);
            // (no history words: nothing reads them on this path)
            if (lane == 0) {
                words[u * (TH / 32) + warp] = ball;
                my_spikes += __popc(ball);
            }
        }
        // the barrier also tells every thread whether the block spiked
        const int any_spike = __syncthreads_or(prev_spk != 0);
        // spike monitors: the block's words of this step, one coalesced row
        if (a.mon_words && tid < BN / 32) a.mon_words[(int64_t)st * a.mon_stride + (base >> 5) + tid] = words[tid];
        // ---- push this block's spikes: one flattened scatter over every
        // (connection, spike) pair of the block
        if (a.npush && any_spike) {
            // warp 0: the spike list, then for every connection the row starts
            // and an inclusive scan of the row lengths of a batch of spikes
            // (the first batch here, before the barrier; later ones below)
            auto batch_rows = [&](int p, int b0, int nb, int64_t *rows, int32_t *pref) {
                int len0 = 0, len1 = 0;
                if (lane < nb) { const int j = sl[b0 + lane]; rows[lane] = srp0[p] + srp[p][j]; len0 = (int)(srp[p][j + 1] - srp[p][j]); }
                if (lane + 32 < nb) { const int j = sl[b0 + lane + 32]; rows[lane + 32] = srp0[p] + srp[p][j]; len1 = (int)(srp[p][j + 1] - srp[p][j]); }
                int i0 = len0, i1 = len1;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v0 = __shfl_up_sync(0xffffffffu, i0, o), v1 = __shfl_up_sync(0xffffffffu, i1, o);
                    if (lane >= o) { i0 += v0; i1 += v1; }
                }
                const int tot0 = __shfl_sync(0xffffffffu, i0, 31);
                pref[lane + 1] = i0;
                pref[lane + 33] = tot0 + i1;
                if (lane == 0) pref[0] = 0;
            };
            if (tid < 32) {
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
                const int nb = min(kPushBatch, acc);
#pragma unroll
                for (int p = 0; p < kPersistMaxPush; ++p)
                    if (p < a.npush && pact[p]) batch_rows(p, 0, nb, srow1[p], spref1[p]);
                if (lane == 0) nsp = acc;
            }
            __syncthreads();
            const int n = nsp;
            // unrolled over the push slots: pcur, pact and my_events stay in registers
#pragma unroll
            for (int p = 0; p < kPersistMaxPush; ++p) {
                if (p >= a.npush) break;
                if (!pact[p]) continue;              // block-uniform
                const Push<T> &q = a.push[p];
                const int cur = pcur[p];
                for (int b0 = 0; b0 < n; b0 += kPushBatch) {
                    const int nb = min(kPushBatch, n - b0);
                    const int64_t *rows = srow1[p];
                    const int32_t *pref = spref1[p];
                    if (b0 > 0) {
                        __syncthreads();             // the previous batch is scattered
                        if (tid < 32) batch_rows(p, b0, nb, srow, spref);
                        __syncthreads();
                        rows = srow;
                        pref = spref;
                    }
                    const int total = pref[nb];
                    if (tid == 0) my_events[p] += (unsigned long long)total;
                    if (q.packed) scatter_batch_packed<TH>(q.packed, q.cring, q.tnp, q.md, cur, rows, pref, nb, total);
                    else scatter_batch<T, TH>(q, cur, rows, pref, nb, total);
                }
            }
        }
#pragma unroll
        for (int p = 0; p < kPersistMaxPush; ++p)
            if (p < a.npush) pcur[p] = pcur[p] + 1 == a.push[p].md ? 0 : pcur[p] + 1;
        // ---- arrive: this block's pushes and ring clears of step t are
        // ordered before the arrival (release reduction, cumulative over the
        // block's writes through the barrier)
        __syncthreads();
        if (tid == 0 && (int)blockIdx.x != a.hold_block) red_release_add(a.arrived + (st & 3), 1u);
    }
#pragma unroll
    for (int u = 0; u < NPT; ++u) {
        const int li = u * TH + tid;
        if (li < nvalid) {
#pragma unroll
            for (int k = 0; k < NV; ++k) a.S[k * a.npad + base + li] = s[u][k];
        }
    }
    block_count(a.spikes, my_spikes);
    if (tid == 0)
        for (int p = 0; p < a.npush; ++p)
            if (my_events[p] && a.push[p].events) atomicAdd(a.push[p].events, my_events[p]);
}

// ---- spike monitors of the persistent path ---------------------------------
// After a launch of nsteps steps, the words it wrote become the monitor's
// (step, index) records in the order of k_spikemon (steps ascending, indices
// ascending within a step): per-step counts, one scan over the steps, then
// one block per step writes its records at its offset.
struct MonWordsArgs {
    DevCtl *ctl;
    const uint32_t *words; int64_t stride; int nsteps;
    int s0;                               // launch-relative step of words[0] (records carry s0 + s)
    int64_t origin, n;                    // monitored range of the group
    long long *cnt; int64_t cap; int32_t *idx; int32_t *steps;
    long long *off;                       // [nsteps] per-step record offsets (scratch)
};
constexpr int kMonWordsThreads = 1024;

__global__ void __launch_bounds__(kMonWordsThreads) k_monw_count(const MonWordsArgs a) {
    __shared__ int wsum[kMonWordsThreads / 32];
    const int s = blockIdx.x, tid = threadIdx.x;
    const uint32_t *H = a.words + (int64_t)s * a.stride;
    const int64_t end = a.origin + a.n, w0 = a.origin >> 5, w1 = (end + 31) >> 5;
    int c = 0;
    for (int64_t wi = w0 + tid; wi < w1; wi += kMonWordsThreads) c += __popc(masked_word(H, wi, a.origin, end));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((tid & 31) == 0) wsum[tid >> 5] = c;
    __syncthreads();
    if (tid < 32) {
        int v = wsum[tid];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (tid == 0) a.off[s] = v;
    }
}

// one block: exclusive scan of the per-step counts from the buffer's fill
// level; advances the fill level (nsteps <= kMonWordsThreads)
__global__ void __launch_bounds__(kMonWordsThreads) k_monw_scan(const MonWordsArgs a) {
    __shared__ long long wsum[kMonWordsThreads / 32 + 1];
    const int tid = threadIdx.x, lane = tid & 31;
    const long long v = tid < a.nsteps ? a.off[tid] : 0;
    long long incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { const long long x = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += x; }
    if (lane == 31) wsum[tid >> 5] = incl;
    __syncthreads();
    if (tid == 0) {
        long long r = *a.cnt;
        for (int q = 0; q < kMonWordsThreads / 32; ++q) { const long long x = wsum[q]; wsum[q] = r; r += x; }
        wsum[kMonWordsThreads / 32] = r;
    }
    __syncthreads();
    if (tid < a.nsteps) a.off[tid] = wsum[tid >> 5] + incl - v;
    if (tid == 0) *a.cnt = wsum[kMonWordsThreads / 32];
}

__global__ void __launch_bounds__(kMonWordsThreads) k_monw_write(const MonWordsArgs a) {
    __shared__ int wcnt[kMonWordsThreads / 32 + 1];
    const int s = blockIdx.x, tid = threadIdx.x;
    const uint32_t *H = a.words + (int64_t)s * a.stride;
    const int64_t end = a.origin + a.n, w0 = a.origin >> 5, w1 = (end + 31) >> 5;
    long long base = a.off[s];
    for (int64_t cw = w0; cw < w1; cw += kMonWordsThreads) {
        const int64_t wi = cw + tid;
        uint32_t word = wi < w1 ? masked_word(H, wi, a.origin, end) : 0u;
        const int pc = __popc(word);
        int incl = pc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, o); if ((tid & 31) >= o) incl += v; }
        if ((tid & 31) == 31) wcnt[tid >> 5] = incl;
        __syncthreads();
        if (tid == 0) { int r = 0; for (int q = 0; q < kMonWordsThreads / 32; ++q) { const int v = wcnt[q]; wcnt[q] = r; r += v; } wcnt[kMonWordsThreads / 32] = r; }
        __syncthreads();
        long long o = base + wcnt[tid >> 5] + incl - pc;
        while (word) {
            const int b = __ffs(word) - 1; word &= word - 1;
            if (o < a.cap) { a.idx[o] = (int32_t)(((wi << 5) + b) - a.origin); a.steps[o] = a.s0 + s; }
            else bg_raise(a.ctl, BG_DERR_MONITOR_OVERFLOW, o);
            ++o;
        }
        base += wcnt[kMonWordsThreads / 32];
        __syncthreads();
    }
}

}  // namespace bg
