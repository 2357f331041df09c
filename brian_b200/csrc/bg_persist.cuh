// bg_persist.cuh -- one cooperative launch runs many steps of a single
// linear group whose outgoing connections are DelayConnections on the
// shared-weight (atomic) path: the CUBA topology of Brian's benchmarks.
//
// Each block owns kBlockNeurons neurons for the whole launch and keeps their
// state in registers; the row pointers of those neurons are staged in shared
// memory once.  A step is: [wait] -> ring delivery + reset of the previous
// step -> linear update + threshold -> push of this block's spikes into the
// rings -> arrive.  Ring row r is delivered at step t+1 when r = t mod md and
// receives pushes from steps t-d (d >= 1), so delivering at step t+1 needs
// the pushes of steps <= t-1 of every block, i.e. the arrivals of step t-1:
// blocks may drift one step apart and the wait is nearly always already
// satisfied.  (With a zero delay the wait is for step t.)  The two spare ring
// rows keep a block that is one step ahead from pushing into a row that a
// lagging block is still delivering.  Every wait is bounded; on timeout the
// block raises BG_DERR_TIMEOUT and leaves the loop.
#pragma once
#include "bg_kernels.cuh"

namespace bg {

constexpr int kPersistMaxPush = 2;

template <typename T> struct PersistArgs {
    DevCtl *ctl;
    T *S; int64_t n, npad;
    T A[kMaxVars * kMaxVars]; T C[kMaxVars]; int useC;
    int thr_kind, thr_var, thr_var2; T thr_val;
    int reset_kind, reset_var, reset_var2; T reset_val;
    uint32_t *hist; int depth; int64_t nwords;
    int ndeliv; Deliv<T> deliv[kMaxDeliv];
    int npush; Push<T> push[kPersistMaxPush];
    unsigned long long *spikes;
    unsigned int *arrived;      // [4] arrivals per step mod 4 (zeroed before the launch)
    int nsteps;
    int lag;                    // 1 when some delay is zero, else 2
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename T, int NV>
__global__ void __launch_bounds__(kHeadThreads, 2) k_persist(const PersistArgs<T> a) {
    __shared__ int64_t srp[kPersistMaxPush][kBlockNeurons + 1];
    __shared__ uint32_t words[kBlockNeurons / 32];
    __shared__ int32_t sl[kBlockNeurons];
    __shared__ int64_t srow[kPushBatch];
    __shared__ int32_t spref[kPushBatch + 1];
    __shared__ int nsp, abort_flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t base = (int64_t)blockIdx.x * kBlockNeurons;
    const unsigned int G = gridDim.x;
    const long long t0 = a.ctl->nstep;
    // row pointers of this block's neurons (clamped: outside the source range
    // a row is empty)
    for (int p = 0; p < a.npush; ++p) {
        const Push<T> &q = a.push[p];
        for (int j = tid; j <= kBlockNeurons; j += kHeadThreads) {
            int64_t r = base + j - q.so;
            r = r < 0 ? 0 : (r > q.sn ? q.sn : r);
            srp[p][j] = q.rowptr[r];
        }
    }
    if (tid == 0) abort_flag = 0;
    T s[kNPT][NV];
#pragma unroll
    for (int u = 0; u < kNPT; ++u) {
        const int64_t i = base + u * kHeadThreads + tid;
#pragma unroll
        for (int k = 0; k < NV; ++k) s[u][k] = i < a.n ? a.S[k * a.npad + i] : T(0);
    }
    unsigned int prev_spk = 0;                  // bit u: neuron u spiked last step
    unsigned long long my_spikes = 0, my_events[kPersistMaxPush] = {0, 0};
    __syncthreads();

    for (int st = 0; st <= a.nsteps; ++st) {    // st == nsteps: tail of the last step only
        const long long t = t0 + st;
        if (st > 0) {
            // local step whose pushes must be complete in every block
            const long long le = (t - 1 - (a.lag == 2 ? 1 : 0)) - t0;
            if (le >= 0) {
                if (tid == 0) {
                    // arrivals are counted per step (slot le % 4): a running sum
                    // would also count blocks that are already one step ahead
                    const unsigned int *ctr = a.arrived + (le & 3);
                    const unsigned int target = (unsigned int)((le >> 2) + 1) * G;
                    unsigned int it = 0;
                    while (ld_acquire_u32(ctr) < target) {
                        if (++it > BG_SPIN_LIMIT) { abort_flag = 1; bg_raise(a.ctl, BG_DERR_TIMEOUT, t); break; }
                        __nanosleep(64);
                    }
                }
                __syncthreads();
                if (abort_flag) break;
            }
            const int ps = (int)(t - 1);
            for (int d = 0; d < a.ndeliv; ++d) {
                const Deliv<T> &dv = a.deliv[d];
                T *row = dv.ring + (int64_t)(ps % dv.md) * dv.tn - dv.to;
#pragma unroll
                for (int u = 0; u < kNPT; ++u) {
                    const int64_t i = base + u * kHeadThreads + tid;
                    if (i < a.n && i >= dv.to && i < dv.to + dv.tn) {
                        const T v = __ldcg(row + i);
                        set_var<T, NV>(s[u], dv.var, rn<T>::add(get_var<T, NV>(s[u], dv.var), v));
                        if (v != T(0)) row[i] = T(0);
                    }
                }
            }
            if (a.reset_kind) {
#pragma unroll
                for (int u = 0; u < kNPT; ++u)
                    if ((prev_spk >> u) & 1u) {
                        if (a.reset_kind == 1) set_var<T, NV>(s[u], a.reset_var, a.reset_val);
                        else set_var<T, NV>(s[u], a.reset_var, get_var<T, NV>(s[u], a.reset_var2));
                    }
            }
        }
        if (st == a.nsteps) break;
        // ---- update, threshold, history
        prev_spk = 0;
#pragma unroll
        for (int u = 0; u < kNPT; ++u) {
            const int64_t i = base + u * kHeadThreads + tid;
            T x[NV];
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                T acc = rn<T>::mul(a.A[j * NV + 0], s[u][0]);
#pragma unroll
                for (int k = 1; k < NV; ++k) acc = rn<T>::add(acc, rn<T>::mul(a.A[j * NV + k], s[u][k]));
                if (a.useC) acc = rn<T>::add(acc, a.C[j]);
                x[j] = acc;
            }
#pragma unroll
            for (int j = 0; j < NV; ++j) s[u][j] = x[j];
            bool spk = false;
            if (i < a.n) {
                if (a.thr_kind == 1) spk = get_var<T, NV>(s[u], a.thr_var) > a.thr_val;
                else if (a.thr_kind == 2) spk = get_var<T, NV>(s[u], a.thr_var) > get_var<T, NV>(s[u], a.thr_var2);
            }
            prev_spk |= (spk ? 1u : 0u) << u;
            const uint32_t ball = __ballot_sync(0xffffffffu, spk);
            if (lane == 0) {
                a.hist[(int64_t)((int)t % a.depth) * a.nwords + ((base + u * kHeadThreads) >> 5) + warp] = ball;
                words[u * (kHeadThreads / 32) + warp] = ball;
                my_spikes += __popc(ball);
            }
        }
        __syncthreads();
        // ---- push this block's spikes
        if (a.npush) {
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
            for (int p = 0; p < a.npush && n > 0; ++p) {
                const Push<T> &q = a.push[p];
                const int cur = (int)t % q.md;
                for (int b0 = 0; b0 < n; b0 += kPushBatch) {
                    const int nb = min(kPushBatch, n - b0);
                    if (tid < nb) {
                        const int j = sl[b0 + tid];
                        srow[tid] = srp[p][j];
                        spref[tid + 1] = (int32_t)(srp[p][j + 1] - srp[p][j]);
                    }
                    __syncthreads();
                    if (tid == 0) { spref[0] = 0; for (int k = 1; k <= nb; ++k) spref[k] += spref[k - 1]; my_events[p] += spref[nb]; }
                    __syncthreads();
                    const int total = spref[nb];
                    for (int e0 = 0; e0 < total; e0 += kHeadThreads * kPushUnroll) {
                        int32_t col[kPushUnroll]; T wv[kPushUnroll]; int slot[kPushUnroll];
#pragma unroll
                        for (int u = 0; u < kPushUnroll; ++u) {
                            const int e = e0 + u * kHeadThreads + tid;
                            col[u] = -1;
                            if (e < total) {
                                int lo = 0, hi = nb;
                                while (hi - lo > 1) { const int m = (lo + hi) >> 1; if (spref[m] <= e) lo = m; else hi = m; }
                                const int64_t k = srow[lo] + (e - spref[lo]);
                                col[u] = __ldg(q.cols + k);
                                wv[u] = q.w_bits == 32 ? (T)__ldg((const float *)q.w + k) : (T)__ldg((const double *)q.w + k);
                                const int sl2 = cur + (int)__ldg(q.d + k);
                                slot[u] = sl2 >= q.md ? sl2 - q.md : sl2;
                            }
                        }
#pragma unroll
                        for (int u = 0; u < kPushUnroll; ++u)
                            if (col[u] >= 0) atomicAdd(&q.ring[(int64_t)slot[u] * q.tn + col[u]], wv[u]);
                    }
                    __syncthreads();
                }
            }
        }
        // ---- arrive: this block's pushes of step t are performed
        __syncthreads();
        if (tid == 0) { __threadfence(); atomicAdd(a.arrived + (st & 3), 1u); }
    }
#pragma unroll
    for (int u = 0; u < kNPT; ++u) {
        const int64_t i = base + u * kHeadThreads + tid;
        if (i < a.n) {
#pragma unroll
            for (int k = 0; k < NV; ++k) a.S[k * a.npad + i] = s[u][k];
        }
    }
    block_count(a.spikes, my_spikes);
    if (tid == 0)
        for (int p = 0; p < a.npush; ++p)
            if (my_events[p] && a.push[p].events) atomicAdd(a.push[p].events, my_events[p]);
}

}  // namespace bg
