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
// The host prepends `typedef <float|double> scalar;`, BG_DT (double),
// BG_DELTA (steps), BG_EXCLUSIVE (0/1) and a `struct Model` holding the
// state registers with load/store/update/threshold/reset members.
#pragma once

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
    long long ns;
    int Tstart, Tend, onset, rec_cap;
};

extern "C" __global__ void __launch_bounds__(128) bg_fit_sim(const FitArgs a)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.ns) return;
    const long long i = a.order[g];
    Model m;
    m.load(a.S, a.ns, i);
    const scalar *Iin = a.I + a.I_off[i];
    const int *spk = a.spk;
    long long idx = a.spk_idx[i];
    const long long last_idx = a.spk_end[i] - 1;
    int last_spike = spk[idx];
    int next_spike = idx < last_idx ? spk[idx + 1] : 0x7fffffff;
    const unsigned char fl = a.flags[i];
    bool last_allowed = (fl & 1) != 0;
    bool next_allowed = (fl & 2) != 0;
    int ncoinc = a.ncoinc[i];
    int nspikes = a.nspikes[i];
    const int spikedelay = a.delay[i];
    const int refractory = a.refr[i];
    int next_allowed_T = a.next_allowed[i];
    const int Tend = min(a.Tend, a.nsteps[i]);
    int *rec = a.rec ? a.rec + i * (long long)a.rec_cap : (int *)0;
    int nrec = a.rec ? a.rec_n[i] : 0;
    for (int T = a.Tstart; T < Tend; ++T) {
        const scalar t = (scalar)((double)T * BG_DT);
        const scalar I_in = Iin[T];
        m.update(I_in, t);
        const bool is_refractory = (T <= next_allowed_T);
        const bool has_spiked = m.threshold(I_in, t) && !is_refractory;
        nspikes += (has_spiked && T >= a.onset) ? 1 : 0;
        if (has_spiked || is_refractory) m.reset(I_in, t);
        if (has_spiked) {
            next_allowed_T = T + refractory;
            if (rec) {
                if (nrec < a.rec_cap) rec[nrec] = T;
                ++nrec;
            }
        }
        const int Tspike = T + spikedelay;
#if BG_EXCLUSIVE
        const bool near_last = has_spiked && (last_spike + BG_DELTA >= Tspike);
        const bool near_next = has_spiked && (next_spike - BG_DELTA <= Tspike);
        const bool ml = near_last && last_allowed, mn = near_next && next_allowed;
        ncoinc += (ml || mn) ? 1 : 0;
        last_allowed = last_allowed && !near_last;
        next_allowed = (next_allowed && !near_next) || (ml && mn);
#else
        ncoinc += (has_spiked && ((last_spike + BG_DELTA >= Tspike) || (next_spike - BG_DELTA <= Tspike))) ? 1 : 0;
#endif
        if (Tspike >= next_spike) {
            ++idx;
            last_spike = next_spike;
            next_spike = idx < last_idx ? spk[idx + 1] : 0x7fffffff;
#if BG_EXCLUSIVE
            last_allowed = next_allowed;
            next_allowed = true;
#endif
        }
    }
    m.store(a.S, a.ns, i);
    a.spk_idx[i] = idx;
    a.flags[i] = (unsigned char)((last_allowed ? 1 : 0) | (next_allowed ? 2 : 0));
    a.ncoinc[i] = ncoinc;
    a.nspikes[i] = nspikes;
    a.next_allowed[i] = next_allowed_T;
    if (a.rec) a.rec_n[i] = nrec;
}
)BGFIT";
