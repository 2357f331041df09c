// bg_synpersist.cuh -- one cooperative launch runs many steps of a single
// linear group whose Synapses (event path, static variables, one additive
// presynaptic statement each, one common target range) connect it to
// itself: CUBA through Synapses.
//
// Block b owns neurons [1024 b, 1024 b + 1024) for the whole launch, state in
// registers (512 threads, neurons tid and tid + 512), and bin b: the events
// of every object that reach those neurons.  A step t is
//   A: update + threshold; the block's spike words into the history (and the
//      monitor words); the last 32 x nobj threads append the block's spikes
//      to each object's spike list of step t and push their delay-0 events,
//      while the other threads push the events of the spike lists of steps
//      t-1 .. t-dmax ((object, delay) lists dealt out over the blocks) into
//      the bins of parity t: a key in the pull's order -- target, object,
//      delay descending, source, rank -- and the statement's term, read in
//      by-source order beside the target;
//   arrive at step t (release), wait for every block's arrival (acquire);
//   C: bin b of parity t ordered (counting sort by target, insertion sort of
//      each target's few events by key) and applied to the registers in that
//      order -- the additions of the pull, in its order -- the bin emptied;
//      the resets of step t; StateMonitors ('end').
// One wait per step: a block in A(t+1) has passed the wait of step t, so
// every block has finished C(t-1) (the bins of parity t+1 it pushes into are
// empty) and A(t) (the lists of step t are complete).  The overflow flags
// form a ring of three (set in A(t), read in C(t), cleared by block 0 in
// A(t+2)); the spike-list count of step t+1 is cleared by block 0 in A(t).
// A step whose events overflow a bin is delivered by the pull's test for
// every target, object by object.  Every wait is bounded; on timeout the
// block raises BG_DERR_TIMEOUT and leaves the loop.
#pragma once
#include "bg_persist.cuh"

namespace bg {

constexpr int kSPTh = kSynBinThreads;            // threads per block
constexpr int kSPNpt = kSynTPT;                  // neurons per thread
constexpr int kSPBn = kSPTh * kSPNpt;            // neurons per block
static_assert(kSPBn == kSynBin, "a block's neurons are one bin of targets");
constexpr int kSynSub = 4;                       // threads per listed source on the spike lists

struct SynPersistObj {
    SynEvArgs e;                                 // lists, rows by source, pull columns, terms
    const double *term_src;                      // the statement's term per synapse, by-source order
    int var, sub;                                // the statement: var += term (sub: var -= term)
};

struct SynPersistArgs {
    DevCtl *ctl;
    double *S; int64_t n, npad;
    double A[kMaxVars * kMaxVars]; double C[kMaxVars];
    uint64_t anz; uint32_t cnz;
    int thr_kind, thr_var, thr_var2; double thr_val;
    int reset_kind, reset_var, reset_var2; double reset_val;
    uint32_t *hist; int depth; int64_t nwords;
    int nobj; SynPersistObj o[kSynEvMerge];
    int pair0[kSynEvMerge + 1]; int nparts;      // (object, delay >= 1) lists dealt out: block / nparts
    // the objects' common bins by step parity: [2][nbins], [2][nbins][cap]
    int *bin_cnt; unsigned long long *bin_key; double *bin_t;
    int nbins, blk0; int64_t tn;                 // bin 0 is block blk0's; targets of the range
    int *use_pull;                               // [3] overflow flags by step mod 3
    unsigned long long *spikes;
    unsigned int *arrived;                       // [4] arrivals per step mod 4 (zeroed before the launch)
    int nsteps;
    uint32_t *mon_words; int64_t mon_stride;     // spike monitors: the words of each step of the launch
    unsigned int spin_limit;
    int hold_block;                              // test hook: this block never publishes its arrivals (-1: none)
    int nrec; RecDev rec[kMaxRec];               // StateMonitors; blk_lo holds this kernel's block ranges
};

// the events of source i's synapses of delay d of object k into the bins of
// one parity (key and term): this thread's share, synapses sub, sub + nsub,
// ... of the source's row of that delay, four at a time (loads, then slots,
// then stores)
__device__ __forceinline__ void synp_push(const SynPersistObj &ob, int k, int64_t i, int d, int sub, int nsub,
                                          int *flag, int *cnt, unsigned long long *key, double *tv) {
    const SynEvArgs &a = ob.e;
    int64_t r0, r1;
    syn_src_range(a, i, d, r0, r1);
    if (r1 - r0 > 256) { if (sub == 0) atomicExch(flag, 1); return; }
    for (int64_t p0 = r0 + sub; p0 < r1; p0 += 4 * nsub) {
        int32_t tg[4], slot[4];
        double tt[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (p0 + u * nsub < r1) { tg[u] = __ldg(a.stgt + p0 + u * nsub); tt[u] = __ldg(ob.term_src + p0 + u * nsub); }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (p0 + u * nsub < r1) slot[u] = atomicAdd(cnt + tg[u] / kSynBin, 1);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t p = p0 + u * nsub;
            if (p >= r1) break;
            if (slot[u] >= kSynBinCap) { atomicExch(flag, 1); continue; }
            const int64_t j = tg[u];
            const int64_t e = (j / kSynBin) * kSynBinCap + slot[u];
            key[e] = ((unsigned long long)(j * 4 + k) << 40) | ((unsigned long long)(255 - d) << 32) |
                     ((unsigned long long)i << 8) | (unsigned long long)(p - r0);
            tv[e] = tt[u];
        }
    }
}

template <int NV>
__device__ __forceinline__ void synp_apply(const SynPersistArgs &a, double (&s)[kSPNpt][NV], int u, int k, double t) {
    const int v = a.o[k].var;
    const bool sub = a.o[k].sub != 0;
#pragma unroll
    for (int uu = 0; uu < kSPNpt; ++uu)
        if (uu == u) uset<double, NV>(s[uu], v, sub ? __dsub_rn(uget<double, NV>(s[uu], v), t) : __dadd_rn(uget<double, NV>(s[uu], v), t));
}

// C(t) for this block's bin (block-uniform call; synchronises)
template <int NV>
__device__ __forceinline__ void synp_bins(const SynPersistArgs &a, long long t, int par, bool pull,
                                          double (&s)[kSPNpt][NV]) {
    extern __shared__ unsigned char syn_smem[];
    unsigned long long *key = reinterpret_cast<unsigned long long *>(syn_smem);
    double *tv = reinterpret_cast<double *>(key + kSynBinCap);
    __shared__ int tcnt[kSynBin];
    __shared__ int wsum[kSPTh / 32], maxc;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int bin = (int)blockIdx.x - a.blk0;
    if (bin < 0 || bin >= a.nbins) return;
    const int64_t jb = (int64_t)bin * kSynBin;
    int *cnt = a.bin_cnt + (int64_t)par * a.nbins + bin;
    const unsigned long long *gkey = a.bin_key + ((int64_t)par * a.nbins + bin) * kSynBinCap;
    const double *gt = a.bin_t + ((int64_t)par * a.nbins + bin) * kSynBinCap;
    // the first kSPTh entries loaded beside the count (those beyond it unused)
    const unsigned long long k0 = __ldcg(gkey + tid);
    const double t0v = __ldcg(gt + tid);
    const int n = min(__ldcg(cnt), kSynBinCap);
    if (pull) {
        // the pull's test for every target of the bin, object by object
        const int row0 = (int)t % a.depth;
#pragma unroll
        for (int u = 0; u < kSPNpt; ++u) {
            const int64_t j = jb + u * kSPTh + tid;
            if (j >= a.tn) continue;
            for (int k = 0; k < a.nobj; ++k) {
                const SynEvArgs &e = a.o[k].e;
                for (int64_t q = e.colptr[j]; q < e.colptr[j + 1]; ++q) {
                    const uint32_t wd = e.word[q];
                    const int lag = (int)(wd >> 24) - 1;
                    if (lag < 0 || t < lag) continue;
                    const int64_t src = e.so + (int64_t)(wd & 0xFFFFFFu);
                    int row = row0 - lag;
                    row += row < 0 ? a.depth : 0;
                    if (!((__ldcg(a.hist + (int64_t)row * a.nwords + (src >> 5)) >> (src & 31)) & 1u)) continue;
                    synp_apply<NV>(a, s, u, k, e.term[q]);
                }
            }
        }
    } else if (n > 0) {
#pragma unroll
        for (int u = 0; u < kSPNpt; ++u) tcnt[u * kSPTh + tid] = 0;
        if (tid == 0) maxc = 0;
        __syncthreads();
        if (tid < n) atomicAdd(&tcnt[(int)((k0 >> 42) - (unsigned long long)jb)], 1);
        for (int e = tid + kSPTh; e < n; e += kSPTh)
            atomicAdd(&tcnt[(int)((__ldcg(gkey + e) >> 42) - (unsigned long long)jb)], 1);
        __syncthreads();
        int cu[kSPNpt], c = 0, cmax = 0;
#pragma unroll
        for (int u = 0; u < kSPNpt; ++u) { cu[u] = tcnt[u * kSPTh + tid]; c += cu[u]; cmax = max(cmax, cu[u]); }
        if (cmax) atomicMax(&maxc, cmax);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += v; }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int v = lane < kSPTh / 32 ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) { const int x = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v += x; }
            if (lane < kSPTh / 32) wsum[lane] = v;
        }
        __syncthreads();
        const int beg = (warp ? wsum[warp - 1] : 0) + incl - c;
        if (maxc <= kSynSegMax) {                                // uniform
            {
                int b = beg;
#pragma unroll
                for (int u = 0; u < kSPNpt; ++u) { tcnt[u * kSPTh + tid] = b; b += cu[u]; }
            }
            __syncthreads();
            if (tid < n) {
                const int pos = atomicAdd(&tcnt[(int)((k0 >> 42) - (unsigned long long)jb)], 1);
                key[pos] = k0;
                tv[pos] = t0v;
            }
            for (int e = tid + kSPTh; e < n; e += kSPTh) {
                const unsigned long long kk = __ldcg(gkey + e);
                const int pos = atomicAdd(&tcnt[(int)((kk >> 42) - (unsigned long long)jb)], 1);
                key[pos] = kk;
                tv[pos] = __ldcg(gt + e);
            }
            __syncthreads();
            int sb = beg;
#pragma unroll
            for (int u = 0; u < kSPNpt; ++u) {
                const int cc = cu[u];
                if (cc) {
                    for (int v = sb + 1; v < sb + cc; ++v) {
                        const unsigned long long kk = key[v];
                        const double tt = tv[v];
                        int w = v - 1;
                        while (w >= sb && key[w] > kk) { key[w + 1] = key[w]; tv[w + 1] = tv[w]; --w; }
                        key[w + 1] = kk;
                        tv[w + 1] = tt;
                    }
                    for (int e = sb; e < sb + cc; ++e) synp_apply<NV>(a, s, u, (int)((key[e] >> 40) & 3u), tv[e]);
                }
                sb += cc;
            }
        } else {
            int m = 1;
            while (m < n) m <<= 1;
            for (int e = tid; e < m; e += kSPTh) {
                if (e < n) { key[e] = __ldcg(gkey + e); tv[e] = __ldcg(gt + e); }
                else { key[e] = ~0ull; tv[e] = 0.0; }
            }
            __syncthreads();
            for (int k = 2; k <= m; k <<= 1) {
                for (int jj = k >> 1; jj > 0; jj >>= 1) {
                    for (int e = tid; e < m; e += kSPTh) {
                        const int o = e ^ jj;
                        if (o > e) {
                            const bool up = (e & k) == 0;
                            const unsigned long long ka = key[e], kb = key[o];
                            if ((ka > kb) == up) {
                                key[e] = kb; key[o] = ka;
                                const double x = tv[e]; tv[e] = tv[o]; tv[o] = x;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
#pragma unroll
            for (int u = 0; u < kSPNpt; ++u) {
                if (!cu[u]) continue;
                const unsigned long long want = (unsigned long long)(jb + u * kSPTh + tid);
                int l = 0, h = n;
                while (l < h) { const int mm = (l + h) >> 1; if ((key[mm] >> 42) < want) l = mm + 1; else h = mm; }
                for (int e = l; e < n && (key[e] >> 42) == want; ++e)
                    synp_apply<NV>(a, s, u, (int)((key[e] >> 40) & 3u), tv[e]);
            }
        }
    }
    __syncthreads();                     // every thread has read the count; shared memory free
    if (tid == 0) *cnt = 0;              // pushed into again in A(t+2)
}

template <int NV, bool DIAG>
__global__ void __launch_bounds__(kSPTh, 2) k_syn_persist(const __grid_constant__ SynPersistArgs a) {
    __shared__ uint32_t words[kSPBn / 32];
    __shared__ int abort_flag, pull_s;
    __shared__ double stash[kSPBn];              // StateMonitor values of the block's neurons
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int base = blockIdx.x * kSPBn;         // neuron counts < 2^31
    const int nvalid = (int)min((int64_t)kSPBn, a.n - (int64_t)base);
    const unsigned int G = gridDim.x;
    const long long t0 = a.ctl->nstep;          // step counters are below 2^31 (checked by the host)
    const int nl = kSPTh - 32 * a.nobj;          // threads on the spike lists; the rest on this step's words
    if (tid == 0) abort_flag = 0;
    double s[kSPNpt][NV];
#pragma unroll
    for (int u = 0; u < kSPNpt; ++u) {
        const int li = u * kSPTh + tid;
#pragma unroll
        for (int k = 0; k < NV; ++k) s[u][k] = li < nvalid ? a.S[k * a.npad + base + li] : 0.0;
    }
    unsigned long long my_spikes = 0;
    __syncthreads();

    for (int st = 0; st < a.nsteps; ++st) {
        const long long t = t0 + st;
        const int par = (int)(t & 1);
        // ---- A(t): update (x = A s + C, the order of linear_row), threshold
        {
            double x[kSPNpt][NV];
            if constexpr (DIAG) {
#pragma unroll
                for (int u = 0; u < kSPNpt; ++u) {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < NV; ++k) acc = __dadd_rn(acc, __dmul_rn(a.A[k], s[u][k]));
                    x[u][0] = acc;
#pragma unroll
                    for (int j = 1; j < NV; ++j) x[u][j] = __dadd_rn(0.0, __dmul_rn(a.A[j * NV + j], s[u][j]));
                }
                if (a.cnz & 1u) {
#pragma unroll
                    for (int u = 0; u < kSPNpt; ++u) x[u][0] = __dadd_rn(x[u][0], a.C[0]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < NV; ++j) {
#pragma unroll
                    for (int u = 0; u < kSPNpt; ++u) x[u][j] = 0.0;
#pragma unroll
                    for (int k = 0; k < NV; ++k)
                        if (a.anz & (1ull << (j * NV + k))) {
                            const double c = a.A[j * NV + k];
#pragma unroll
                            for (int u = 0; u < kSPNpt; ++u) x[u][j] = __dadd_rn(x[u][j], __dmul_rn(c, s[u][k]));
                        }
                    if (a.cnz & (1u << j)) {
#pragma unroll
                        for (int u = 0; u < kSPNpt; ++u) x[u][j] = __dadd_rn(x[u][j], a.C[j]);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kSPNpt; ++u)
#pragma unroll
                for (int j = 0; j < NV; ++j) s[u][j] = x[u][j];
        }
        unsigned int spk_bits = 0;
#pragma unroll
        for (int u = 0; u < kSPNpt; ++u) {
            const int li = u * kSPTh + tid;
            bool spk = false;
            if (a.thr_kind == 1) spk = uget<double, NV>(s[u], a.thr_var) > a.thr_val;
            else if (a.thr_kind == 2) spk = uget<double, NV>(s[u], a.thr_var) > uget<double, NV>(s[u], a.thr_var2);
            spk = spk && li < nvalid;
            spk_bits |= (spk ? 1u : 0u) << u;
            const uint32_t ball = __ballot_sync(0xffffffffu, spk);
            if (lane == 0) {
                const int w = u * (kSPTh / 32) + warp;
                words[w] = ball;
                a.hist[(int64_t)((int)t % a.depth) * a.nwords + (base >> 5) + w] = ball;
                if (a.mon_words) a.mon_words[(int64_t)st * a.mon_stride + (base >> 5) + w] = ball;
                my_spikes += __popc(ball);
            }
        }
        __syncthreads();
        if (blockIdx.x == 0) {
            if (tid < a.nobj) {
                const SynEvArgs &e = a.o[tid].e;
                e.scnt[((int)t + 1) % e.sdepth] = 0;              // step t+1's list starts empty
            }
            if (tid == 32) a.use_pull[((int)t + 1) % 3] = 0;     // step t+1's overflow flag (last read in C(t-2))
        }
        int *flag = a.use_pull + (int)t % 3;
        int *bcnt = a.bin_cnt + (int64_t)par * a.nbins;
        unsigned long long *bkey = a.bin_key + (int64_t)par * a.nbins * kSynBinCap;
        double *bt = a.bin_t + (int64_t)par * a.nbins * kSynBinCap;
        if (tid >= nl) {
            // this block's spikes: into object k's list of step t (when they
            // are its sources), with their delay-0 events
            const int k = (tid - nl) >> 5, w = tid & 31;
            const SynPersistObj &ob = a.o[k];
            const SynEvArgs &e = ob.e;
            const int64_t wb = (int64_t)((base >> 5) + w) << 5;
            uint32_t word = words[w];
            if (wb < e.so) { const int sh = (int)(e.so - wb); word = sh >= 32 ? 0u : (word & (0xffffffffu << sh)); }
            if (wb + 32 > e.so + e.sn) { const int keep = (int)(e.so + e.sn - wb); word = keep <= 0 ? 0u : (keep >= 32 ? word : (word & ((1u << keep) - 1u))); }
            if (word) {
                const int row = (int)t % e.sdepth;
                const int pos = atomicAdd(e.scnt + row, __popc(word));   // used after the pushes
                for (uint32_t wv = word; wv; wv &= wv - 1)
                    synp_push(ob, k, wb + (__ffs(wv) - 1) - e.so, 0, 0, 1, flag, bcnt, bkey, bt);
                int32_t *L = e.slist + (int64_t)row * e.sn + pos;
                for (uint32_t wv = word; wv; wv &= wv - 1) *L++ = (int32_t)(wb + (__ffs(wv) - 1) - e.so);
            }
        } else {
            // the spike lists of steps t-1 .. t-dmax dealt out over the blocks
            for (int pr = blockIdx.x; pr < a.pair0[a.nobj] * a.nparts; pr += G) {
                const int pair = pr / a.nparts, part = pr % a.nparts;
                int k = 0;
                while (k + 1 < a.nobj && pair >= a.pair0[k + 1]) ++k;
                const SynPersistObj &ob = a.o[k];
                const SynEvArgs &e = ob.e;
                const int d = 1 + pair - a.pair0[k];
                if (t < d) continue;
                const int row = ((int)t - d) % e.sdepth;
                const int32_t *L = e.slist + (int64_t)row * e.sn;
                // kSynSub threads per listed source, each with a share of its synapses
                const int q0 = (part * nl + tid) / kSynSub, sub = tid % kSynSub;
                const int32_t first = q0 < e.sn ? __ldcg(L + q0) : 0;   // loaded beside the count
                const int cnt = __ldcg(e.scnt + row);
                for (int q = q0; q < cnt; q += a.nparts * nl / kSynSub)
                    synp_push(ob, k, q == q0 ? first : __ldcg(L + q), d, sub, kSynSub, flag, bcnt, bkey, bt);
            }
        }
        // ---- arrive at step t; wait for every block's arrival
        __syncthreads();
        if (tid == 0 && (int)blockIdx.x != a.hold_block) red_release_add(a.arrived + (st & 3), 1u);
        if (tid == 32) {
            const unsigned int *ctr = a.arrived + (st & 3);
            const unsigned int target = (unsigned int)((st >> 2) + 1) * G;
            unsigned int it = 0;
            while (ld_acquire_u32(ctr) < target) {
                if (++it > a.spin_limit) { abort_flag = 1; bg_raise(a.ctl, BG_DERR_TIMEOUT, t); break; }
                __nanosleep(32);
            }
            // the step's overflow flag, read once per block (every warp of
            // every block reading one address queues at one L2 slice)
            pull_s = __ldcg(flag);
        }
        __syncthreads();
        if (abort_flag) break;
        // ---- C(t): this block's bin, then the resets of step t
        synp_bins<NV>(a, t, par, pull_s != 0, s);
        if (a.reset_kind == 1) {
#pragma unroll
            for (int u = 0; u < kSPNpt; ++u)
                if ((spk_bits >> u) & 1u) uset<double, NV>(s[u], a.reset_var, a.reset_val);
        } else if (a.reset_kind) {
#pragma unroll
            for (int u = 0; u < kSPNpt; ++u)
                if ((spk_bits >> u) & 1u) uset<double, NV>(s[u], a.reset_var, uget<double, NV>(s[u], a.reset_var2));
        }
        // StateMonitors ('end' slot, after the resets)
        for (int r = 0; r < a.nrec; ++r) {
            const RecDev &m = a.rec[r];
            const long long rel = t - m.start;
            if (rel < 0 || rel % m.timestep) continue;           // block-uniform
#pragma unroll
            for (int u = 0; u < kSPNpt; ++u) stash[u * kSPTh + tid] = uget<double, NV>(s[u], m.var);
            __syncthreads();
            const long long row = rel / m.timestep - *m.row_base;
            const int e0 = m.blk_lo[blockIdx.x], e1 = m.blk_lo[blockIdx.x + 1];
            for (int e = e0 + tid; e < e1; e += kSPTh) ((double *)m.buf)[row * m.nidx + m.pos[e]] = stash[m.idx[e] - base];
            __syncthreads();
        }
    }
#pragma unroll
    for (int u = 0; u < kSPNpt; ++u) {
        const int li = u * kSPTh + tid;
        if (li < nvalid) {
#pragma unroll
            for (int k = 0; k < NV; ++k) a.S[k * a.npad + base + li] = s[u][k];
        }
    }
    block_count(a.spikes, my_spikes);
}

// the statement's term per synapse in by-source order: out[p] = term[sq[p]]
static __global__ void k_syn_term_src(const int32_t *sq, const double *term, int64_t nsyn, double *out) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nsyn; p += (int64_t)gridDim.x * blockDim.x)
        out[p] = term[sq[p]];
}

}  // namespace bg
