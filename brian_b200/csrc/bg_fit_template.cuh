// bg_fit_template.cuh -- source of the batched fitting kernel, compiled at
// run time by NVRTC for sm_100a once the model is known.
//
// One thread simulates one candidate (particle x target x slice) over its own
// duration and counts coincidences with its target spike train online: the
// semantics of the reference's `runsim` template
// (library/modelfitting/gpu_modelfitting.py:39-116) and its exclusive and
// inclusive coincidence algorithms (gpu_modelfitting.py:118-156):
//
//   I = input[T + I_offset]; state update; is_refractory = T <= next_allowed;
//   has_spiked = threshold && !is_refractory; spikes counted from `onset`;
//   reset while spiking or refractory; next_allowed = T + refractory;
//   the coincidence test uses Tspike = T + spike delay against the last and
//   next target spikes, then the target pointer moves on once Tspike has
//   reached the next target spike.
//
// Differences from the reference template, all by design:
//   * each simulation has its own number of steps (uneven durations);
//   * the target pointer stops at the train's final sentinel instead of
//     reading past the end of the train;
//   * candidates are visited in `order` (longest first, candidates of one
//     target side by side) so a warp shares its input row and its length;
//   * every simulation's state, pointer and flags are loaded once and stored
//     once per launch (the whole run is normally one launch).
//
// Scheduling: simulations are grouped into warp tasks of 32 consecutive
// entries of `order` (longest first, one target's candidates together, so a
// task shares its length and its input row).  A fixed number of resident
// warps pull tasks from an atomic counter, longest first: the long
// simulations start at once and the short ones fill the gaps (greedy
// longest-processing-time scheduling).  No warp waits on another.
//
// Latency: the state update is a chain of dependent operations per step, so
// the hot loop carries nothing else: per step it integrates, tests the
// threshold and refractoriness, applies the reset as selects and shifts the
// spike into a 32-bit word.  Everything that only changes at a model spike or
// at a target-pointer move -- the coincidence test, the spike count from
// onset, the record, the pointer itself -- is replayed once per block of 32
// steps, in step order, from that word and the next target time: per step T
// the spike's coincidence test comes first, then the pointer moves at most
// once, exactly as in the reference's per-step loop.  The input of step T+1
// is loaded while step T computes.
//
// The host prepends `typedef <float|double> scalar;`, BG_DT (double),
// BG_DELTA (steps), BG_EXCLUSIVE (0/1) and a `struct Model`
// holding the state registers with load/store/update/threshold/reset members.
#pragma once

// Division by a divisor fixed for the whole run, given its reciprocal y:
//  * float: RN32(RN64(a * RN64(1/b))) equals RN32(a/b) whenever a is normal
//    and a/b is neither subnormal nor zero-divided: the double product is
//    within 2^-52 (relative) of a/b, while a/b lies at least 2^-49 away from
//    every rounding midpoint of binary32 (a midpoint m with a = m*b would need
//    a 25-bit odd significand inside a 24-bit one);
//  * double: Markstein's correction (P. Markstein, IBM J. Res. Dev. 34(1),
//    1990): q = RN(a*y), r = a - b*q (exact with one FMA), RN(q + r*y) is
//    RN(a/b) when y = RN(1/b) and nothing under- or overflows; a = 0 returns
//    q, which carries the sign IEEE division gives.
// Outside those ranges `suspect` is set and the kernel redoes the block with
// IEEE division.
static const char kFitHelperSource[] = R"BGFIT(
__device__ __forceinline__ float bg_div_fast(const float a, const float b, const double y, const float thr,
                                             bool &suspect) {
    suspect |= (fabsf(a) < thr) && (a != 0.0f);
    return __double2float_rn(__dmul_rn((double)a, y));
}
__device__ __forceinline__ double bg_div_fast(const double a, const double b, const double y, const double thr,
                                              bool &suspect) {
    const double m = fabs(a);
    suspect |= !(m >= thr && m <= 0x1p+900) && (a != 0.0);
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-b, q, a);
    const double q1 = __fma_rn(r, y, q);
    return a == 0.0 ? q : q1;
}
)BGFIT";

static const char kFitKernelSource[] = R"BGFIT(
struct FitArgs {
    scalar *S;                  // [nstate][ns] state, SoA
    const scalar *I;            // concatenated input traces
    const long long *I_off;     // first input sample of each simulation
    const int *nsteps;          // length of each simulation (steps)
    const int *spk;             // concatenated target trains (steps), sentinel-framed
    const long long *spk_end;   // one past the last entry of each simulation's train
    long long *spk_idx;         // current position in the train
    const int *delay;           // spike delay (steps)
    const int *refr;            // refractory period (steps)
    int *next_allowed;          // last refractory step
    int *ncoinc;
    int *nspikes;
    unsigned char *flags;       // bit 0 last_spike_allowed, bit 1 next_spike_allowed
    const int *order;           // thread -> simulation
    int *rec;                   // optional spike record [ns][rec_cap]
    int *rec_n;
    int *next_task;             // task counter, zero at launch
    long long ns;
    int Tstart, Tend, onset, rec_cap;
};

#define BG_NO_SPIKE 0x7fffffff

struct Sim {
    Model m;
    const int *spk;
    long long idx, last_idx;
    int last_spike, next_spike, next2_spike;
    bool last_allowed, next_allowed;
    int ncoinc, nspikes, spikedelay, refractory, next_allowed_T, onset;
    int *rec;
    int nrec, rec_cap;

    __device__ __forceinline__ int train_at(long long k) const {
        return k <= last_idx ? __ldg(spk + k) : BG_NO_SPIKE;
    }

    // update, threshold, refractoriness and reset of step T; true on a spike.
    // FAST selects the update with reciprocal divisions (sets `suspect` when
    // one of them may differ from IEEE division).
    template <bool FAST>
    __device__ __forceinline__ bool step(const int T, const scalar I_in, bool &suspect) {
        const scalar t = (scalar)((double)T * BG_DT);
        if (FAST) m.update_fast(I_in, t, suspect);
        else m.update(I_in, t);
        const bool is_refractory = (T <= next_allowed_T);
        const bool has_spiked = m.threshold(I_in, t) && !is_refractory;
        m.reset(I_in, t, has_spiked || is_refractory);
        next_allowed_T = has_spiked ? T + refractory : next_allowed_T;
        return has_spiked;
    }

    // Steps T0 .. T0+n-1 have run; bit k of `bits` is the spike of step T0+k.
    __device__ __forceinline__ void replay(const int T0, const int n, unsigned bits) {
        const int Tn = T0 + n;
        if (bits) {
            const int c = onset - T0;
            const unsigned counted = c <= 0 ? 0xffffffffu : (c >= 32 ? 0u : (0xffffffffu << c));
            nspikes += __popc(bits & counted);
            if (rec) {
                for (unsigned b = bits; b; b &= b - 1) {
                    if (nrec < rec_cap) rec[nrec] = T0 + __ffs(b) - 1;
                    ++nrec;
                }
            }
        }
        int Tc = T0;                        // first step whose pointer test is pending
        for (;;) {
            const long long ta = (long long)next_spike - spikedelay;
            const int Tadv = ta <= Tc ? Tc : (ta >= Tn ? Tn : (int)ta);
            const int Tsp = bits ? T0 + __ffs(bits) - 1 : Tn;
            const int Te = min(Tadv, Tsp);
            if (Te >= Tn) break;
            const int Tspike = Te + spikedelay;
            if (Te == Tsp) {
                bits &= bits - 1;
#if BG_EXCLUSIVE
                const bool near_last = last_spike + BG_DELTA >= Tspike;
                const bool near_next = next_spike - BG_DELTA <= Tspike;
                const bool ml = near_last && last_allowed, mn = near_next && next_allowed;
                ncoinc += (ml || mn) ? 1 : 0;
                last_allowed = last_allowed && !near_last;
                next_allowed = (next_allowed && !near_next) || (ml && mn);
#else
                ncoinc += ((last_spike + BG_DELTA >= Tspike) || (next_spike - BG_DELTA <= Tspike)) ? 1 : 0;
#endif
            }
            if (Tspike >= next_spike) {
                ++idx;
                last_spike = next_spike;
                next_spike = next2_spike;
                next2_spike = train_at(idx + 2);
#if BG_EXCLUSIVE
                last_allowed = next_allowed;
                next_allowed = true;
#endif
            }
            Tc = Te + 1;
        }
    }
};

__device__ __forceinline__ void run_sim(const FitArgs &a, const long long i)
{
    Sim s;
    s.m.load(a.S, a.ns, i);
    const scalar *Iin = a.I + a.I_off[i];
    s.spk = a.spk;
    s.idx = a.spk_idx[i];
    s.last_idx = a.spk_end[i] - 1;
    s.last_spike = s.train_at(s.idx);
    s.next_spike = s.train_at(s.idx + 1);
    s.next2_spike = s.train_at(s.idx + 2);
    const unsigned char fl = a.flags[i];
    s.last_allowed = (fl & 1) != 0;
    s.next_allowed = (fl & 2) != 0;
    s.ncoinc = a.ncoinc[i];
    s.nspikes = a.nspikes[i];
    s.spikedelay = a.delay[i];
    s.refractory = a.refr[i];
    s.next_allowed_T = a.next_allowed[i];
    s.onset = a.onset;
    s.rec = a.rec ? a.rec + i * (long long)a.rec_cap : (int *)0;
    s.nrec = a.rec ? a.rec_n[i] : 0;
    s.rec_cap = a.rec_cap;
    const int Tend = min(a.Tend, a.nsteps[i]);
    if (a.Tstart < Tend) {
        // loads clamp to the last step, so every address stays inside this
        // simulation's input
        const int Tlast = Tend - 1;
        scalar Icur = __ldg(Iin + a.Tstart);
        int T0 = a.Tstart;
        const bool fast_ok = !s.m.bg_exact;
        while (T0 < Tend) {
            const int n = min(32, Tend - T0);
            // checkpoint: a block with a suspect division runs again exactly
            const Model m0 = s.m;
            const int na0 = s.next_allowed_T;
            unsigned bits = 0;
            bool suspect = !fast_ok;
            if (fast_ok) {
                if (n == 32) {
#pragma unroll 4
                    for (int k = 0; k < 32; ++k) {
                        const scalar Inext = __ldg(Iin + min(T0 + k + 1, Tlast));
                        bits = (bits >> 1) | (s.template step<true>(T0 + k, Icur, suspect) ? 0x80000000u : 0u);
                        Icur = Inext;
                    }
                } else {
                    for (int k = 0; k < n; ++k) {
                        const scalar Inext = __ldg(Iin + min(T0 + k + 1, Tlast));
                        bits |= (s.template step<true>(T0 + k, Icur, suspect) ? 1u : 0u) << k;
                        Icur = Inext;
                    }
                }
            }
            if (suspect) {
                s.m = m0;
                s.next_allowed_T = na0;
                bits = 0;
                bool unused = false;
                for (int k = 0; k < n; ++k)
                    bits |= (s.template step<false>(T0 + k, __ldg(Iin + T0 + k), unused) ? 1u : 0u) << k;
                Icur = __ldg(Iin + min(T0 + n, Tlast));
            }
            s.replay(T0, n, bits);
            T0 += n;
        }
    }
    s.m.store(a.S, a.ns, i);
    a.spk_idx[i] = s.idx;
    a.flags[i] = (unsigned char)((s.last_allowed ? 1 : 0) | (s.next_allowed ? 2 : 0));
    a.ncoinc[i] = s.ncoinc;
    a.nspikes[i] = s.nspikes;
    a.next_allowed[i] = s.next_allowed_T;
    if (a.rec) a.rec_n[i] = s.nrec;
}

extern "C" __global__ void __launch_bounds__(128) bg_fit_sim(const FitArgs a)
{
    const int lane = threadIdx.x & 31;
    const long long ntasks = (a.ns + 31) / 32;
    for (;;) {
        int task = 0;
        if (lane == 0) task = atomicAdd(a.next_task, 1);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= ntasks) break;
        const long long g = (long long)task * 32 + lane;
        if (g < a.ns) run_sim(a, a.order[g]);
        __syncwarp();
    }
}
)BGFIT";
