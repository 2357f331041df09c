/*
 * oracle.cpp -- CPU restatement of Brian 1.4.4's clock-driven loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine
 * in brian_b200/csrc: tests, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it; the product never does.
 *
 * It exports the same C ABI as include/brian_b200.h with the prefix
 * `or_` instead of `bg_`, so one network description can be replayed into
 * both.  Single-threaded, compiled with -O2 -ffp-contract=off: every
 * floating-point operation is one IEEE rounding in the order written.
 *
 * Semantics followed (file:line in the Brian 1.4.4 tree):
 *   step loop / schedule ......... network.py:365-380, 516-586; clock.py:162-212
 *   linear update S <- A.S + C ... stateupdater.py:404-417 (sum fixed left to
 *                                   right over columns, no FMA)
 *   threshold ..................... threshold.py:160-191 (v > Vt, ascending)
 *   variable threshold ............ threshold.py:373-396
 *   Poisson threshold ............. threshold.py:461-471 (u < rate*dt)
 *   spike generator ............... directcontrol.py:231-268
 *   refractory filter ............. neurongroup.py:495-516
 *   spike history ring ............ utils/circular.py:171-250
 *   reset / variable reset ........ reset.py:139-147, 241-254
 *   Refractoriness clamp .......... reset.py:311-332 (LS[0:period])
 *   sparse propagation ............ connection.py:224-256
 *   dense propagation ............. connection.py:256-262
 *   delayed propagation ........... delayconnection.py:132-206 (ring row
 *                                   (cur + d) % md), delivery :112-121
 *   STDP pre/post updaters ........ stdp.py:31-54, 370-414, 452-539
 *   STDP on a DelayConnection ..... stdp.py:57-89, 296-368; RecentStateMonitor
 *                                   monitor.py:991-1099
 *   Synapses / SpikeQueue ......... synapses/synapses.py:808-827;
 *                                   synapses/spikequeue.py:209-216, 270-363
 *   SpikeMonitor .................. monitor.py:156-166
 *   StateMonitor .................. monitor.py:824-842
 *   EmpiricalThreshold ............ threshold.py:449-457 (LS[0:refractory])
 *   nonlinear model / StringThreshold / StringReset: the generated C snippets
 *   of the model (the engine compiles the same text with NVRTC) are compiled
 *   here with gcc -O2 -ffp-contract=off and applied neuron by neuron in the
 *   slots above; the numpy evaluation of the equations (oracle/fitting.py)
 *   checks the snippets themselves.
 */
#include <cstdint>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <deque>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <dlfcn.h>

#define OR_OK 0
#define OR_EINVAL (-1)
#define OR_ESTATE (-6)
#define OR_ENOSYS (-7)

static thread_local std::string g_err;
#include <unistd.h>
static long getpid_or() { return (long)getpid(); }
static int fail(int code, const std::string &m) { g_err = m; return code; }

/* ---------------- Philox4x32-10 (Salmon et al., SC'11) ------------------ */
static inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}
/* uniform double in [0,1) with 53 random bits, keyed by (seed, step, i) */
static inline double philox_uniform(uint64_t seed, int64_t step, int64_t i) {
    uint32_t c[4] = {(uint32_t)step, (uint32_t)((uint64_t)step >> 32),
                     (uint32_t)i, (uint32_t)((uint64_t)i >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint64_t a = c[0] >> 5, b = c[1] >> 6;
    return (double)(a * 67108864ull + b) * (1.0 / 9007199254740992.0);
}

/* ---------------- data ---------------------------------------------------- */
struct Group {
    int64_t n = 0; int nvar = 0;
    std::vector<double> S;           /* [nvar][n] */
    std::vector<double> S0;
    bool linear = false, useC = false;
    std::vector<double> A, C;
    int thr_kind = 0, thr_var = 0, thr_var2 = 0; double thr_val = 0;
    int rate_var = 0; uint64_t seed = 0;
    std::vector<int64_t> gen_steps; std::vector<int32_t> gen_idx;
    int reset_kind = 0, reset_var = 0, reset_var2 = 0; double reset_val = 0;
    bool refr = false; double refr_time = 0; int32_t period = 0; int clamp_var = 0; double clamp_val = 0;
    std::vector<double> next_allowed;
    std::deque<std::vector<int32_t>> hist;   /* hist[0] = current step */
    int32_t depth = 1;
    int64_t nspikes = 0;
    int32_t emp_steps = 0; std::vector<int64_t> last_spike;
    /* TimedArraySetters (timedarray.py:238-303): see or_group_set_timed_array */
    struct Setter {
        int var, mode; int64_t origin, count, nrows, ncols; double t_init, adt; int64_t first;
        std::vector<double> vals; std::vector<int64_t> bp;
    };
    std::vector<Setter> setters;
    /* generated model: one neuron at a time over S[var * n + i] */
    void (*gen_update)(double *, int64_t, int64_t, double) = nullptr;
    int (*gen_threshold)(const double *, int64_t, int64_t, double) = nullptr;
    void (*gen_reset)(double *, int64_t, int64_t, double) = nullptr;
};
struct Conn {
    int32_t src, tgt; int64_t so, sn, to, tn; int var;
    bool dense = false;
    std::vector<int64_t> rowptr; std::vector<int32_t> cols;
    int w_bits = 64; std::vector<double> w64; std::vector<float> w32;
    int32_t delay = 0; bool hetero = false; std::vector<uint8_t> d;
    int32_t md = 0, cur = 0; std::vector<double> ring;
    int mod_var = -1;
    /* column index (built at prepare when STDP needs it) */
    std::vector<int64_t> colptr; std::vector<int64_t> colk; std::vector<int32_t> colsrc;
    int64_t events = 0;
    double getw(int64_t k) const { return w_bits == 64 ? w64[k] : (double)w32[k]; }
};
struct Stdp {
    int32_t cid; double a_pre, c_pre, a_post, c_post, Ap, Am, wmin, wmax;
    int inter; int32_t pre_delay, post_delay;
    std::vector<double> A_pre, A_post;
    /* update forms of the w lines: 0 w += a, 1 w *= (1 + a), 2 w += (wx - w)*a
     * (ExponentialSTDP update='multiplicative'/'mixed', stdp.py:510-533) */
    int pre_mode = 0, post_mode = 0; double wx = 0.0;
    /* DelayConnection (stdp.py:296-368): RecentStateMonitors of both traces
     * (monitor.py:991-1099): M slots [M][n], written at the end of each step
     * at current_time_index, which then advances modulo M */
    bool delayed = false; int32_t M = 0; int64_t cur = 0;
    std::vector<uint8_t> lag_pre, lag_post;
    std::vector<double> H_pre, H_post;
};
/* Synapses (synapses/synapses.py:43-1058) with static synaptic variables
 * and presynaptic statements x (+|-)= term on the target; SpikeQueue
 * (synapses/spikequeue.py:69-330): L rows of synapse indices, filled in the
 * connections slot at row (cur + delay) % L, read and cleared at row cur in
 * the 'synapses' slot of the same step (after 'after_connections', before
 * the resets, network.py:365-380, 472-483), which then advances cur. */
struct Syn {
    int32_t src, tgt; int64_t so, sn, to, tn; int64_t nsyn;
    std::vector<int32_t> pre, post, delay;
    int nops; std::vector<int32_t> op_var, op_sub; std::vector<double> terms;   /* [nops][nsyn] */
    std::vector<std::vector<int32_t>> syn_of_pre;                               /* ascending */
    int32_t L = 1; int64_t cur = 0; std::vector<std::vector<int32_t>> X;
    /* synapses with code (or_synapses_set_code): synaptic variables
     * [nsv][nsyn] in synapse order, the compiled pre/post codes, the target
     * variables they use (slots) and the source variables they read */
    bool coded = false; int nsv = 0; std::vector<double> sv;
    std::vector<int32_t> slot_var, pre_var; std::vector<std::vector<int32_t>> syn_of_post;
    void (*sc_pre)(double *, double *const *, int64_t, double, const double *) = nullptr;
    void (*sc_post)(double *, double *const *, int64_t, double) = nullptr;
};
struct SpikeMon { int32_t gid; int64_t origin, n; int32_t delay; std::vector<int64_t> steps; std::vector<int32_t> idx; };
struct StateMon { int32_t gid; int var; std::vector<int32_t> idx; int32_t timestep; int64_t start;
                  std::vector<double> vals; std::vector<int64_t> steps; };
enum { IT_CONN = 0, IT_SPIKEMON = 1, IT_STDP_PRE = 2, IT_STDP_POST = 3, IT_SYN = 4 };
struct Item { int kind; int32_t id; };

struct or_net {
    double dt; int precision;
    std::vector<Group> groups; std::vector<Conn> conns; std::vector<Stdp> stdps;
    std::vector<SpikeMon> smons; std::vector<StateMon> stmons; std::vector<Item> items;
    std::vector<Syn> syns;
    std::vector<int32_t> mon_kind;   /* monitor id -> 0 spike, 1 state (index into vector in mon_idx) */
    std::vector<int32_t> mon_idx;
    bool prepared = false; int64_t nstep = 0;
};

extern "C" {

int or_version(void) { return 1; }
int or_last_error(char *buf, int64_t len) {
    if (!buf || len <= 0) return OR_EINVAL;
    std::strncpy(buf, g_err.c_str(), (size_t)len - 1); buf[len - 1] = 0; return OR_OK;
}
int or_net_create(int device, int precision, int deterministic, double dt, or_net **out) {
    (void)device; (void)deterministic;
    if (!out || !(dt > 0)) return fail(OR_EINVAL, "bad dt/out");
    if (precision != 64) return fail(OR_ENOSYS, "oracle runs the FP64 path only");
    or_net *n = new or_net(); n->dt = dt; n->precision = precision; *out = n; return OR_OK;
}
int or_net_destroy(or_net *n) { delete n; return OR_OK; }

static bool gid_ok(or_net *n, int32_t g) { return n && g >= 0 && g < (int32_t)n->groups.size(); }

int or_group_add(or_net *n, int64_t N, int nvar, const double *S0, int32_t *gid) {
    if (!n || N < 0 || nvar < 0 || (N > 0 && nvar > 0 && !S0)) return fail(OR_EINVAL, "group_add");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    Group g; g.n = N; g.nvar = nvar;
    g.S.assign(S0, S0 + (size_t)N * nvar); g.S0 = g.S;
    n->groups.push_back(std::move(g)); *gid = (int32_t)n->groups.size() - 1; return OR_OK;
}
int or_group_set_linear(or_net *n, int32_t gid, const double *A, const double *C) {
    if (!gid_ok(n, gid) || !A) return fail(OR_EINVAL, "set_linear");
    Group &g = n->groups[gid]; int m = g.nvar;
    g.linear = true; g.A.assign(A, A + m * m);
    g.useC = C != nullptr; if (C) g.C.assign(C, C + m);
    return OR_OK;
}
/* TimedArraySetter: at the start of the step (before every group's update)
 * S[var][origin + k] = values[r][ncols == 1 ? 0 : k] with r the row of
 * TimedArray.__call__ (timedarray.py:209-235: int(rint((t - t_init)/dt))
 * clamped) for an array on a clock (mode 0), or the row the setter's walk
 * through ascending times reaches (timedarray.py:280-292: the last i with
 * times[i] <= t), given as the clock steps bp[i-1] at which row i starts
 * (mode 1). */
int or_group_set_timed_array(or_net *n, int32_t gid, int var, int64_t origin, int64_t count, const double *values,
                             int64_t nrows, int64_t ncols, int mode, double t_init, double adt, int64_t first_step,
                             const int64_t *bp) {
    if (!gid_ok(n, gid) || !values) return fail(OR_EINVAL, "set_timed_array");
    Group &g = n->groups[gid];
    if (var < 0 || var >= g.nvar || origin < 0 || count < 1 || origin + count > g.n || nrows < 1 ||
        (ncols != 1 && ncols != count) || (mode != 0 && mode != 1) || (mode == 0 && !(adt > 0)) ||
        (mode == 1 && nrows > 1 && !bp))
        return fail(OR_EINVAL, "set_timed_array");
    Group::Setter h;
    h.var = var; h.mode = mode; h.origin = origin; h.count = count; h.nrows = nrows; h.ncols = ncols;
    h.t_init = t_init; h.adt = adt; h.first = first_step;
    h.vals.assign(values, values + nrows * ncols);
    if (mode == 1 && nrows > 1) h.bp.assign(bp, bp + (nrows - 1));
    g.setters.push_back(std::move(h));
    return OR_OK;
}

static int64_t setter_row(const Group::Setter &h, int64_t cs, double dt) {
    if (h.mode == 0) {
        const double x = ((double)cs * dt - h.t_init) / h.adt;
        if (!(x > 0.0)) return 0;
        if (x >= (double)(h.nrows - 1)) return h.nrows - 1;
        return (int64_t)std::nearbyint(x);      /* round half to even, as numpy.rint */
    }
    return (int64_t)(std::upper_bound(h.bp.begin(), h.bp.end(), cs) - h.bp.begin());
}

int or_group_set_threshold(or_net *n, int32_t gid, int kind, int var, double value, int var2) {
    if (!gid_ok(n, gid)) return fail(OR_EINVAL, "set_threshold");
    Group &g = n->groups[gid];
    if ((kind == 1 || kind == 2) && (var < 0 || var >= g.nvar)) return fail(OR_EINVAL, "threshold var");
    if (kind == 2 && (var2 < 0 || var2 >= g.nvar)) return fail(OR_EINVAL, "threshold var2");
    g.thr_kind = kind; g.thr_var = var; g.thr_val = value; g.thr_var2 = var2; return OR_OK;
}
int or_group_set_poisson(or_net *n, int32_t gid, int rate_var, uint64_t seed) {
    if (!gid_ok(n, gid)) return fail(OR_EINVAL, "set_poisson");
    Group &g = n->groups[gid];
    if (rate_var < 0 || rate_var >= g.nvar) return fail(OR_EINVAL, "rate var");
    g.thr_kind = 3; g.rate_var = rate_var; g.seed = seed; return OR_OK;
}
int or_group_set_generator(or_net *n, int32_t gid, int64_t ns, const int64_t *steps, const int32_t *idx) {
    if (!gid_ok(n, gid) || ns < 0) return fail(OR_EINVAL, "set_generator");
    Group &g = n->groups[gid]; g.thr_kind = 4;
    g.gen_steps.assign(steps, steps + ns); g.gen_idx.assign(idx, idx + ns);
    for (int64_t k = 0; k < ns; ++k) {
        if (idx[k] < 0 || idx[k] >= g.n) return fail(OR_EINVAL, "generator index");
        if (k && (steps[k] < steps[k - 1] || (steps[k] == steps[k - 1] && idx[k] < idx[k - 1])))
            return fail(OR_EINVAL, "generator spikes not sorted by (step, index)");
    }
    return OR_OK;
}
int or_group_set_reset(or_net *n, int32_t gid, int kind, int var, double value, int var2) {
    if (!gid_ok(n, gid)) return fail(OR_EINVAL, "set_reset");
    Group &g = n->groups[gid];
    if (kind && (var < 0 || var >= g.nvar)) return fail(OR_EINVAL, "reset var");
    if (kind == 2 && (var2 < 0 || var2 >= g.nvar)) return fail(OR_EINVAL, "reset var2");
    g.reset_kind = kind; g.reset_var = var; g.reset_val = value; g.reset_var2 = var2; return OR_OK;
}
int or_group_set_empirical(or_net *n, int32_t gid, int32_t steps) {
    if (!gid_ok(n, gid) || steps < 0) return fail(OR_EINVAL, "set_empirical");
    n->groups[gid].emp_steps = steps;
    return OR_OK;
}

/* Same layout as bg_fit_model: state names (comma separated), update,
 * update with reciprocals (unused here), threshold, reset, aux decl, setup. */
struct or_model {
    const char *state_names, *update_code, *update_fast_code, *threshold_code, *reset_code, *aux_decl, *setup_code;
};

int or_group_set_model(or_net *n, int32_t gid, const or_model *m) {
    if (!gid_ok(n, gid) || !m || !m->state_names) return fail(OR_EINVAL, "set_model");
    Group &g = n->groups[gid];
    std::vector<std::string> names;
    std::string cur;
    for (const char *p = m->state_names;; ++p) {
        if (*p == ',' || *p == 0) { names.push_back(cur); cur.clear(); if (!*p) break; }
        else if (*p != ' ') cur += *p;
    }
    if ((int)names.size() != g.nvar) return fail(OR_EINVAL, "model names do not match the group");
    auto s = [](const char *x) { return std::string(x ? x : ""); };
    const std::string upd = s(m->update_code), thr = s(m->threshold_code), rst = s(m->reset_code);
    std::string c = "#include <math.h>\ntypedef double scalar;\n"
                    "static inline double __longlong_as_double(long long x) { union { long long i; double d; } u; u.i = x; return u.d; }\n";
    auto load = [&]() {
        std::string o;
        for (size_t k = 0; k < names.size(); ++k)
            o += "    scalar s_" + names[k] + " = S[" + std::to_string(k) + "LL * N + i];\n";
        return o;
    };
    auto store = [&]() {
        std::string o;
        for (size_t k = 0; k < names.size(); ++k) o += "    S[" + std::to_string(k) + "LL * N + i] = s_" + names[k] + ";\n";
        return o;
    };
    const std::string pre = "    const scalar t = (scalar)t_; const scalar I_in = 0; (void)t; (void)I_in;\n";
    c += "void gm_update(double *S, long long N, long long i, double t_) {\n" + pre + load() + upd + "\n" + store() + "}\n";
    c += "int gm_threshold(const double *S, long long N, long long i, double t_) {\n" + pre + load() + "    return (" +
         (thr.empty() ? std::string("0") : thr) + ") ? 1 : 0;\n}\n";
    c += "void gm_reset(double *S, long long N, long long i, double t_) {\n" + pre +
         "    const int reset_on = 1; (void)reset_on;\n" + load() + rst + "\n" + store() + "}\n";
    /* compile next to this library (_ref/gen under the oracle's directory) */
    Dl_info info;
    if (!dladdr((void *)&or_group_set_model, &info) || !info.dli_fname) return fail(OR_ESTATE, "dladdr");
    std::string dir = info.dli_fname;
    dir = dir.substr(0, dir.find_last_of('/')) + "/_ref/gen";
    static int counter = 0;
    const std::string stem = dir + "/model_" + std::to_string((long long)getpid_or()) + "_" + std::to_string(counter++);
    if (std::system(("mkdir -p '" + dir + "'").c_str()) != 0) return fail(OR_ESTATE, "mkdir " + dir);
    FILE *f = std::fopen((stem + ".c").c_str(), "w");
    if (!f) return fail(OR_ESTATE, "cannot write " + stem + ".c");
    std::fputs(c.c_str(), f);
    std::fclose(f);
    const std::string cmd = "gcc -O2 -ffp-contract=off -fno-fast-math -shared -fPIC -w -o '" + stem + ".so' '" + stem + ".c' -lm";
    if (std::system(cmd.c_str()) != 0) return fail(OR_ESTATE, "gcc failed on the generated model: " + stem + ".c");
    void *h = dlopen((stem + ".so").c_str(), RTLD_NOW | RTLD_LOCAL);
    std::remove((stem + ".c").c_str());     /* the loaded image stays mapped */
    std::remove((stem + ".so").c_str());
    if (!h) return fail(OR_ESTATE, std::string("dlopen: ") + dlerror());
    if (!upd.empty()) { g.gen_update = (void (*)(double *, int64_t, int64_t, double))dlsym(h, "gm_update"); g.linear = false; }
    if (!thr.empty()) g.gen_threshold = (int (*)(const double *, int64_t, int64_t, double))dlsym(h, "gm_threshold");
    if (!rst.empty()) g.gen_reset = (void (*)(double *, int64_t, int64_t, double))dlsym(h, "gm_reset");
    return OR_OK;
}

int or_group_set_refractory(or_net *n, int32_t gid, double rt, int32_t period, int var, double value) {
    if (!gid_ok(n, gid) || period < 0) return fail(OR_EINVAL, "set_refractory");
    Group &g = n->groups[gid];
    if (period > 0 && (var < 0 || var >= g.nvar)) return fail(OR_EINVAL, "clamp var");
    /* rt <= 0: no spike filter (refractory < 0.9*dt), clamp only */
    g.refr = rt > 0; g.refr_time = rt; g.period = period; g.clamp_var = var; g.clamp_val = value; return OR_OK;
}

static int add_conn_common(or_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to,
                           int64_t tn, int var, int32_t delay, int mod_var, Conn &c) {
    if (!gid_ok(n, src) || !gid_ok(n, tgt)) return fail(OR_EINVAL, "conn groups");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    const Group &gs = n->groups[src], &gt = n->groups[tgt];
    if (so < 0 || sn < 0 || so + sn > gs.n || to < 0 || tn < 0 || to + tn > gt.n) return fail(OR_EINVAL, "conn ranges");
    if (var < 0 || var >= gt.nvar) return fail(OR_EINVAL, "conn target var");
    if (delay < 0) return fail(OR_EINVAL, "conn delay");
    if (mod_var >= gs.nvar) return fail(OR_EINVAL, "modulation var");
    c.src = src; c.tgt = tgt; c.so = so; c.sn = sn; c.to = to; c.tn = tn; c.var = var;
    c.delay = delay; c.mod_var = mod_var;
    return OR_OK;
}
int or_conn_add(or_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to, int64_t tn,
                int var, int64_t nnz, const int64_t *rowptr, const int32_t *cols, const void *w, int w_bits,
                int32_t delay, const uint8_t *delays, int32_t ring_depth, int mod_var, int32_t *cid) {
    Conn c; int st = add_conn_common(n, src, so, sn, tgt, to, tn, var, delay, mod_var, c);
    if (st) return st;
    if (w_bits != 32 && w_bits != 64) return fail(OR_EINVAL, "w_bits");
    if (!rowptr || nnz < 0 || (nnz > 0 && (!cols || !w))) return fail(OR_EINVAL, "csr arrays");
    if (rowptr[0] != 0 || rowptr[sn] != nnz) return fail(OR_EINVAL, "rowptr bounds");
    c.rowptr.assign(rowptr, rowptr + sn + 1); c.cols.assign(cols, cols + nnz);
    for (int64_t i = 0; i < sn; ++i) {
        if (rowptr[i + 1] < rowptr[i]) return fail(OR_EINVAL, "rowptr not monotone");
        for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            if (cols[k] < 0 || cols[k] >= tn) return fail(OR_EINVAL, "column index out of range");
            if (k > rowptr[i] && cols[k] <= cols[k - 1]) return fail(OR_EINVAL, "columns not strictly ascending in a row");
        }
    }
    c.w_bits = w_bits;
    if (w_bits == 64) c.w64.assign((const double *)w, (const double *)w + nnz);
    else c.w32.assign((const float *)w, (const float *)w + nnz);
    if (delays) {
        if (ring_depth < 1 || ring_depth > 255) return fail(OR_EINVAL, "ring depth");
        c.hetero = true; c.d.assign(delays, delays + nnz); c.md = ring_depth;
        for (int64_t k = 0; k < nnz; ++k) if (delays[k] >= ring_depth) return fail(OR_EINVAL, "delay >= ring depth");
        c.ring.assign((size_t)ring_depth * tn, 0.0);
    }
    n->conns.push_back(std::move(c)); *cid = (int32_t)n->conns.size() - 1;
    n->items.push_back({IT_CONN, *cid});
    return OR_OK;
}
int or_conn_add_dense(or_net *n, int32_t src, int64_t so, int64_t sn, int32_t tgt, int64_t to, int64_t tn,
                      int var, const void *W, int w_bits, int32_t delay, int mod_var, int32_t *cid) {
    Conn c; int st = add_conn_common(n, src, so, sn, tgt, to, tn, var, delay, mod_var, c);
    if (st) return st;
    if ((w_bits != 32 && w_bits != 64) || (!W && sn * tn > 0)) return fail(OR_EINVAL, "dense weights");
    c.dense = true; c.w_bits = w_bits;
    size_t nn = (size_t)sn * tn;
    if (w_bits == 64) c.w64.assign((const double *)W, (const double *)W + nn);
    else c.w32.assign((const float *)W, (const float *)W + nn);
    n->conns.push_back(std::move(c)); *cid = (int32_t)n->conns.size() - 1;
    n->items.push_back({IT_CONN, *cid});
    return OR_OK;
}
static size_t conn_size(const Conn &c) { return c.w_bits == 64 ? c.w64.size() : c.w32.size(); }
int or_conn_get_weights(or_net *n, int32_t cid, double *out) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !out) return fail(OR_EINVAL, "get_weights");
    const Conn &c = n->conns[cid];
    for (size_t k = 0; k < conn_size(c); ++k) out[k] = c.getw((int64_t)k);
    return OR_OK;
}
int or_conn_set_weights(or_net *n, int32_t cid, const double *in) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !in) return fail(OR_EINVAL, "set_weights");
    Conn &c = n->conns[cid];
    for (size_t k = 0; k < conn_size(c); ++k) { if (c.w_bits == 64) c.w64[k] = in[k]; else c.w32[k] = (float)in[k]; }
    return OR_OK;
}
int or_stdp_add(or_net *n, int32_t cid, const double *decay, double Ap, double Am, double wmin, double wmax,
                int inter, int32_t pre_delay, int32_t post_delay, int32_t *sid) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !decay) return fail(OR_EINVAL, "stdp_add");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    Conn &c = n->conns[cid];
    if (c.hetero) return fail(OR_ENOSYS, "STDP on a DelayConnection is not supported");
    if (pre_delay < 0 || post_delay < 0) return fail(OR_EINVAL, "stdp delays");
    Stdp s; s.cid = cid; s.a_pre = decay[0]; s.c_pre = decay[1]; s.a_post = decay[2]; s.c_post = decay[3];
    s.Ap = Ap; s.Am = Am; s.wmin = wmin; s.wmax = wmax; s.inter = inter;
    s.pre_delay = pre_delay; s.post_delay = post_delay;
    s.A_pre.assign(c.sn, 0.0); s.A_post.assign(c.tn, 0.0);
    n->stdps.push_back(std::move(s)); *sid = (int32_t)n->stdps.size() - 1;
    n->items.push_back({IT_STDP_PRE, *sid}); n->items.push_back({IT_STDP_POST, *sid});
    return OR_OK;
}
/* ExponentialSTDP on a DelayConnection: the presynaptic code splits into an
 * immediate updater (delay 0) and a delayed one (delay = pre_delay, the
 * connection's max_delay), the postsynaptic code runs at delay 0; the w
 * lines read past trace values (stdp.py:296-352, DelayedSTDPUpdater
 * stdp.py:57-89). */
int or_stdp_add_delayed(or_net *n, int32_t cid, const double *decay, double Ap, double Am, double wmin, double wmax,
                        int inter, int32_t pre_delay, int32_t hist_len, const uint8_t *lag_pre, const uint8_t *lag_post,
                        int32_t *sid) {
    if (!n || cid < 0 || cid >= (int32_t)n->conns.size() || !decay) return fail(OR_EINVAL, "stdp_add_delayed");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    Conn &c = n->conns[cid];
    if (!c.hetero || c.dense) return fail(OR_EINVAL, "delayed STDP needs a sparse DelayConnection");
    if (pre_delay < 0 || hist_len < 1 || hist_len > 256) return fail(OR_EINVAL, "stdp parameters");
    const size_t nnz = c.cols.size();
    for (size_t k = 0; k < nnz; ++k)
        if (lag_pre[k] >= hist_len || lag_post[k] >= hist_len) return fail(OR_EINVAL, "stdp lags");
    Stdp s; s.cid = cid; s.a_pre = decay[0]; s.c_pre = decay[1]; s.a_post = decay[2]; s.c_post = decay[3];
    s.Ap = Ap; s.Am = Am; s.wmin = wmin; s.wmax = wmax; s.inter = inter;
    s.pre_delay = pre_delay; s.post_delay = 0;
    s.A_pre.assign(c.sn, 0.0); s.A_post.assign(c.tn, 0.0);
    s.delayed = true; s.M = hist_len; s.cur = 0;
    s.lag_pre.assign(lag_pre, lag_pre + nnz); s.lag_post.assign(lag_post, lag_post + nnz);
    s.H_pre.assign((size_t)hist_len * c.sn, 0.0); s.H_post.assign((size_t)hist_len * c.tn, 0.0);
    n->stdps.push_back(std::move(s)); *sid = (int32_t)n->stdps.size() - 1;
    n->items.push_back({IT_STDP_PRE, *sid}); n->items.push_back({IT_STDP_POST, *sid});
    return OR_OK;
}
int or_synapses_add(or_net *n, int32_t src_gid, int64_t src_origin, int64_t src_n, int32_t tgt_gid, int64_t tgt_origin,
                    int64_t tgt_n, int64_t nsyn, const int32_t *pre, const int32_t *post, const int32_t *delay, int nops,
                    const int32_t *op_var, const int32_t *op_sub, const double *terms, int32_t *sid) {
    if (!gid_ok(n, src_gid) || !gid_ok(n, tgt_gid) || nsyn < 0 || nops < 0 || nops > 4 || !sid)
        return fail(OR_EINVAL, "synapses_add");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    const Group &gs = n->groups[src_gid], &gt = n->groups[tgt_gid];
    if (src_origin < 0 || src_n < 0 || src_origin + src_n > gs.n || tgt_origin < 0 || tgt_n < 0 || tgt_origin + tgt_n > gt.n)
        return fail(OR_EINVAL, "synapses ranges");
    Syn y; y.src = src_gid; y.tgt = tgt_gid; y.so = src_origin; y.sn = src_n; y.to = tgt_origin; y.tn = tgt_n;
    y.nsyn = nsyn; y.nops = nops;
    y.pre.assign(pre, pre + nsyn); y.post.assign(post, post + nsyn); y.delay.assign(delay, delay + nsyn);
    y.op_var.assign(op_var, op_var + nops); y.op_sub.assign(op_sub, op_sub + nops);
    y.terms.assign(terms, terms + (size_t)nops * nsyn);
    int32_t dmax = 0;
    for (int64_t k = 0; k < nsyn; ++k) {
        if (pre[k] < 0 || pre[k] >= src_n || post[k] < 0 || post[k] >= tgt_n || delay[k] < 0) return fail(OR_EINVAL, "synapse");
        dmax = std::max(dmax, delay[k]);
    }
    for (int k = 0; k < nops; ++k) if (op_var[k] < 0 || op_var[k] >= gt.nvar) return fail(OR_EINVAL, "synaptic statement");
    y.syn_of_pre.assign(src_n, std::vector<int32_t>());
    for (int64_t k = 0; k < nsyn; ++k) y.syn_of_pre[pre[k]].push_back((int32_t)k);
    y.L = dmax + 1; y.cur = 0; y.X.assign(y.L, std::vector<int32_t>());
    n->syns.push_back(std::move(y)); *sid = (int32_t)n->syns.size() - 1;
    n->items.push_back({IT_SYN, *sid});
    return OR_OK;
}
int or_synapses_set_terms(or_net *n, int32_t sid, const double *terms) {
    if (!n || sid < 0 || sid >= (int32_t)n->syns.size() || !terms) return fail(OR_EINVAL, "synapses_set_terms");
    Syn &y = n->syns[sid];
    std::copy(terms, terms + (size_t)y.nops * y.nsyn, y.terms.begin());
    return OR_OK;
}
/* Synapses with code: the codes are C statements over X(s), SV(k), PRE(k)
 * and T (the engine compiles the same text for the GPU), compiled here with
 * gcc (no contraction) next to the library and loaded.  bg_exp / bg_clip
 * come from the engine's bg_expfn.h so both sides run the same operations. */
int or_synapses_set_code(or_net *n, int32_t sid, int32_t nsv, const double *sv, const char *pre_code,
                         const char *post_code, int32_t nslots, const int32_t *slot_var, int32_t nwrites,
                         const int32_t *writes, int32_t npre, const int32_t *pre_var) {
    (void)writes;
    if (!n || sid < 0 || sid >= (int32_t)n->syns.size() || nsv < 0 || nsv > 8 || nslots < 0 || nslots > 4 ||
        npre < 0 || npre > 4 || nwrites < 0 || nwrites > nslots)
        return fail(OR_EINVAL, "synapses_set_code");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    Syn &y = n->syns[sid];
    if (y.nops) return fail(OR_EINVAL, "Synapses with code take no separate statements");
    y.coded = true; y.nsv = nsv;
    if (sv) y.sv.assign(sv, sv + (size_t)nsv * y.nsyn); else y.sv.assign((size_t)nsv * y.nsyn, 0.0);
    y.slot_var.assign(slot_var, slot_var + nslots); y.pre_var.assign(pre_var, pre_var + npre);
    y.syn_of_post.assign(y.tn, std::vector<int32_t>());
    for (int64_t k = 0; k < y.nsyn; ++k) y.syn_of_post[y.post[k]].push_back((int32_t)k);
    Dl_info info;
    if (!dladdr((void *)&or_synapses_set_code, &info) || !info.dli_fname) return fail(OR_ESTATE, "dladdr");
    std::string here = info.dli_fname;
    here = here.substr(0, here.find_last_of('/'));
    const std::string dir = here + "/_ref/gen";
    std::string c = "#include <math.h>\n#include <stdint.h>\n#include \"" + here + "/../brian_b200/csrc/bg_expfn.h\"\n"
                    "#define X(s) x_[s]\n#define SV(k) sv_[k][q_]\n#define PRE(k) pre_[k]\n#define T t_\n"
                    "void sc_pre(double *x_, double *const *sv_, int64_t q_, double t_, const double *pre_) {\n"
                    "    (void)x_; (void)sv_; (void)q_; (void)t_; (void)pre_;\n" + std::string(pre_code ? pre_code : "") +
                    "\n}\nvoid sc_post(double *x_, double *const *sv_, int64_t q_, double t_) {\n"
                    "    (void)x_; (void)sv_; (void)q_; (void)t_;\n" + std::string(post_code ? post_code : "") + "\n}\n";
    static int counter = 0;
    const std::string stem = dir + "/syn_" + std::to_string((long long)getpid_or()) + "_" + std::to_string(counter++);
    if (std::system(("mkdir -p '" + dir + "'").c_str()) != 0) return fail(OR_ESTATE, "mkdir " + dir);
    FILE *f = std::fopen((stem + ".c").c_str(), "w");
    if (!f) return fail(OR_ESTATE, "cannot write " + stem + ".c");
    std::fputs(c.c_str(), f);
    std::fclose(f);
    const std::string cmd = "gcc -O2 -ffp-contract=off -fno-fast-math -shared -fPIC -w -o '" + stem + ".so' '" + stem + ".c' -lm";
    if (std::system(cmd.c_str()) != 0) return fail(OR_ESTATE, "gcc failed on the synaptic code: " + stem + ".c");
    void *h = dlopen((stem + ".so").c_str(), RTLD_NOW | RTLD_LOCAL);
    std::remove((stem + ".c").c_str());
    std::remove((stem + ".so").c_str());
    if (!h) return fail(OR_ESTATE, std::string("dlopen: ") + dlerror());
    y.sc_pre = (void (*)(double *, double *const *, int64_t, double, const double *))dlsym(h, "sc_pre");
    y.sc_post = (void (*)(double *, double *const *, int64_t, double))dlsym(h, "sc_post");
    if (!y.sc_pre || !y.sc_post) return fail(OR_ESTATE, "synaptic code symbols");
    if (!post_code || !*post_code) y.sc_post = nullptr;
    return OR_OK;
}
int or_synapses_get_var(or_net *n, int32_t sid, int32_t k, double *out) {
    if (!n || sid < 0 || sid >= (int32_t)n->syns.size() || !out) return fail(OR_EINVAL, "synapses_get_var");
    const Syn &y = n->syns[sid];
    if (!y.coded || k < 0 || k >= y.nsv) return fail(OR_EINVAL, "synaptic variable");
    std::copy(y.sv.begin() + (size_t)k * y.nsyn, y.sv.begin() + (size_t)(k + 1) * y.nsyn, out);
    return OR_OK;
}
int or_synapses_set_var(or_net *n, int32_t sid, int32_t k, const double *in) {
    if (!n || sid < 0 || sid >= (int32_t)n->syns.size() || !in) return fail(OR_EINVAL, "synapses_set_var");
    Syn &y = n->syns[sid];
    if (!y.coded || k < 0 || k >= y.nsv) return fail(OR_EINVAL, "synaptic variable");
    std::copy(in, in + y.nsyn, y.sv.begin() + (size_t)k * y.nsyn);
    return OR_OK;
}

/* Synapses.update (synapses.py:808-827) in the 'synapses' slot: the events
 * of this step, in queue order, applied statement by statement (with code:
 * the whole presynaptic code per event, a target's events in queue order,
 * then the postsynaptic code for each synapse of a target that spiked in
 * this step); then next(). */
static void synapses_deliver(or_net *n, double t) {
    for (auto &y : n->syns) {
        Group &g = n->groups[y.tgt];
        if (y.coded) {
            const Group &gs = n->groups[y.src];
            std::vector<double *> svp(8, nullptr);
            for (int v = 0; v < y.nsv; ++v) svp[v] = &y.sv[(size_t)v * y.nsyn];
            double x[4] = {0, 0, 0, 0}, pv[4] = {0, 0, 0, 0};
            for (int32_t e : y.X[y.cur]) {
                const int64_t j = y.to + y.post[e];
                for (size_t s2 = 0; s2 < y.slot_var.size(); ++s2) x[s2] = g.S[(size_t)y.slot_var[s2] * g.n + j];
                for (size_t k = 0; k < y.pre_var.size(); ++k) pv[k] = gs.S[(size_t)y.pre_var[k] * gs.n + y.so + y.pre[e]];
                y.sc_pre(x, svp.data(), e, t, pv);
                for (size_t s2 = 0; s2 < y.slot_var.size(); ++s2) g.S[(size_t)y.slot_var[s2] * g.n + j] = x[s2];
            }
            if (y.sc_post)
                for (int32_t i : g.hist[0]) {
                    if (i < y.to || i >= y.to + y.tn) continue;
                    for (size_t s2 = 0; s2 < y.slot_var.size(); ++s2) x[s2] = g.S[(size_t)y.slot_var[s2] * g.n + i];
                    for (int32_t e : y.syn_of_post[i - y.to]) y.sc_post(x, svp.data(), e, t);
                }
            y.X[y.cur].clear();
            y.cur = (y.cur + 1) % y.L;
            continue;
        }
        for (int32_t e : y.X[y.cur]) {
            const int64_t j = y.to + y.post[e];
            for (int k = 0; k < y.nops; ++k) {
                double &x = g.S[(size_t)y.op_var[k] * g.n + j];
                const double term = y.terms[(size_t)k * y.nsyn + e];
                x = y.op_sub[k] ? x - term : x + term;
            }
        }
        y.X[y.cur].clear();
        y.cur = (y.cur + 1) % y.L;
    }
}
int or_stdp_set_update(or_net *n, int32_t sid, int pre_mode, int post_mode, double wmax_exact) {
    if (!n || sid < 0 || sid >= (int32_t)n->stdps.size() || pre_mode < 0 || pre_mode > 2 || post_mode < 0 ||
        post_mode > 2)
        return fail(OR_EINVAL, "stdp_set_update");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    Stdp &s = n->stdps[sid];
    if ((pre_mode || post_mode) && n->conns[s.cid].w_bits != 64) return fail(OR_ENOSYS, "multiplicative STDP on FP32 weights");
    s.pre_mode = pre_mode; s.post_mode = post_mode; s.wx = wmax_exact;
    return OR_OK;
}
/* the w line of an STDP code string, as numpy evaluates it */
static inline double wupd(double w, double a, int mode, double wx) {
    if (mode == 1) return w * (1.0 + a);
    if (mode == 2) return w + (wx - w) * a;
    return w + a;
}
/* get_past_values_sequence (monitor.py:1088-1096): the slot of the value
 * recorded `lag` records before the last one */
static inline size_t past_slot(const Stdp &s, int lag) {
    int64_t q = (s.cur - 1 - lag) % s.M; if (q < 0) q += s.M; return (size_t)q;
}
int or_stdp_get_traces(or_net *n, int32_t sid, double *a_pre, double *a_post) {
    if (!n || sid < 0 || sid >= (int32_t)n->stdps.size()) return fail(OR_EINVAL, "stdp id");
    const Stdp &s = n->stdps[sid];
    if (a_pre) std::copy(s.A_pre.begin(), s.A_pre.end(), a_pre);
    if (a_post) std::copy(s.A_post.begin(), s.A_post.end(), a_post);
    return OR_OK;
}
int or_spikemon_add(or_net *n, int32_t gid, int64_t origin, int64_t cnt, int32_t delay, int32_t *mid) {
    if (!gid_ok(n, gid) || origin < 0 || cnt < 0 || origin + cnt > n->groups[gid].n || delay < 0)
        return fail(OR_EINVAL, "spikemon_add");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    SpikeMon m; m.gid = gid; m.origin = origin; m.n = cnt; m.delay = delay;
    n->smons.push_back(m);
    n->items.push_back({IT_SPIKEMON, (int32_t)n->smons.size() - 1});
    n->mon_kind.push_back(0); n->mon_idx.push_back((int32_t)n->smons.size() - 1);
    *mid = (int32_t)n->mon_kind.size() - 1; return OR_OK;
}
int or_statemon_add(or_net *n, int32_t gid, int var, int64_t nidx, const int32_t *idx, int32_t timestep, int32_t *mid) {
    if (!gid_ok(n, gid) || var < 0 || var >= n->groups[gid].nvar || timestep < 1 || nidx < 0)
        return fail(OR_EINVAL, "statemon_add");
    if (n->prepared) return fail(OR_ESTATE, "network already prepared");
    StateMon m; m.gid = gid; m.var = var; m.timestep = timestep; m.start = 0;
    if (idx) m.idx.assign(idx, idx + nidx);
    else { m.idx.resize(n->groups[gid].n); for (int64_t i = 0; i < n->groups[gid].n; ++i) m.idx[i] = (int32_t)i; }
    for (int32_t i : m.idx) if (i < 0 || i >= n->groups[gid].n) return fail(OR_EINVAL, "statemon index");
    n->stmons.push_back(std::move(m));
    n->mon_kind.push_back(1); n->mon_idx.push_back((int32_t)n->stmons.size() - 1);
    *mid = (int32_t)n->mon_kind.size() - 1; return OR_OK;
}
static bool mon_ok(or_net *n, int32_t mid, int kind) {
    return n && mid >= 0 && mid < (int32_t)n->mon_kind.size() && n->mon_kind[mid] == kind;
}
int or_spikemon_count(or_net *n, int32_t mid, int64_t *cnt) {
    if (!mon_ok(n, mid, 0)) return fail(OR_EINVAL, "spikemon id");
    *cnt = (int64_t)n->smons[n->mon_idx[mid]].idx.size(); return OR_OK;
}
int or_spikemon_read(or_net *n, int32_t mid, int64_t *steps, int32_t *idx, int64_t cap, int64_t *cnt) {
    if (!mon_ok(n, mid, 0)) return fail(OR_EINVAL, "spikemon id");
    const SpikeMon &m = n->smons[n->mon_idx[mid]];
    int64_t k = std::min<int64_t>(cap, (int64_t)m.idx.size());
    for (int64_t i = 0; i < k; ++i) { steps[i] = m.steps[i]; idx[i] = m.idx[i]; }
    *cnt = k; return OR_OK;
}
int or_statemon_count(or_net *n, int32_t mid, int64_t *rows) {
    if (!mon_ok(n, mid, 1)) return fail(OR_EINVAL, "statemon id");
    *rows = (int64_t)n->stmons[n->mon_idx[mid]].steps.size(); return OR_OK;
}
int or_statemon_read(or_net *n, int32_t mid, double *vals, int64_t *steps, int64_t cap, int64_t *rows) {
    if (!mon_ok(n, mid, 1)) return fail(OR_EINVAL, "statemon id");
    const StateMon &m = n->stmons[n->mon_idx[mid]];
    int64_t r = std::min<int64_t>(cap, (int64_t)m.steps.size()), w = (int64_t)m.idx.size();
    for (int64_t i = 0; i < r; ++i) {
        steps[i] = m.steps[i];
        for (int64_t j = 0; j < w; ++j) vals[i * w + j] = m.vals[i * w + j];
    }
    *rows = r; return OR_OK;
}
int or_monitor_clear(or_net *n, int32_t mid) {
    if (!n || mid < 0 || mid >= (int32_t)n->mon_kind.size()) return fail(OR_EINVAL, "monitor id");
    if (n->mon_kind[mid] == 0) { SpikeMon &m = n->smons[n->mon_idx[mid]]; m.steps.clear(); m.idx.clear(); }
    else { StateMon &m = n->stmons[n->mon_idx[mid]]; m.steps.clear(); m.vals.clear(); m.start = n->nstep; }
    return OR_OK;
}

int or_net_prepare(or_net *n) {
    if (!n) return fail(OR_EINVAL, "net");
    if (n->prepared) return OR_OK;
    /* history depth: max delay read from each group, + 1 for the current bin,
     * and the refractory period (neurongroup.py:459-473). */
    for (auto &g : n->groups) g.depth = std::max<int32_t>(1, g.period);
    for (auto &c : n->conns) {
        Group &g = n->groups[c.src]; g.depth = std::max(g.depth, c.delay + 1);
    }
    for (auto &s : n->stdps) {
        Conn &c = n->conns[s.cid];
        n->groups[c.src].depth = std::max(n->groups[c.src].depth, s.pre_delay + 1);
        n->groups[c.tgt].depth = std::max(n->groups[c.tgt].depth, s.post_delay + 1);
        if (!c.dense && c.colptr.empty()) {
            /* column access order: ascending source within each target column
             * (connectionmatrix.py:317-333 coldataindices) */
            c.colptr.assign(c.tn + 1, 0);
            for (int32_t j : c.cols) c.colptr[j + 1]++;
            for (int64_t j = 0; j < c.tn; ++j) c.colptr[j + 1] += c.colptr[j];
            std::vector<int64_t> fill(c.colptr.begin(), c.colptr.end() - 1);
            c.colk.resize(c.cols.size()); c.colsrc.resize(c.cols.size());
            for (int64_t i = 0; i < c.sn; ++i)
                for (int64_t k = c.rowptr[i]; k < c.rowptr[i + 1]; ++k) {
                    int64_t p = fill[c.cols[k]]++; c.colk[p] = k; c.colsrc[p] = (int32_t)i;
                }
        }
    }
    for (auto &m : n->smons) { Group &g = n->groups[m.gid]; g.depth = std::max(g.depth, m.delay + 1); }
    for (auto &g : n->groups) {
        g.hist.assign(g.depth, std::vector<int32_t>());
        if (g.refr) g.next_allowed.assign(g.n, -1.0);
        if (g.emp_steps > 0) g.last_spike.assign(g.n, -(1ll << 40));
    }
    n->prepared = true; return OR_OK;
}

int or_net_reinit(or_net *n) {
    if (!n) return fail(OR_EINVAL, "net");
    for (auto &g : n->groups) {
        for (auto &h : g.hist) h.clear();
        if (g.refr) std::fill(g.next_allowed.begin(), g.next_allowed.end(), -1.0);
        std::fill(g.last_spike.begin(), g.last_spike.end(), -(1ll << 40));
    }
    for (auto &c : n->conns) std::fill(c.ring.begin(), c.ring.end(), 0.0);
    for (auto &y : n->syns) { for (auto &r : y.X) r.clear(); y.cur = 0; }
    for (auto &s : n->stdps) {
        std::fill(s.A_pre.begin(), s.A_pre.end(), 0.0); std::fill(s.A_post.begin(), s.A_post.end(), 0.0);
        std::fill(s.H_pre.begin(), s.H_pre.end(), 0.0); std::fill(s.H_post.begin(), s.H_post.end(), 0.0); s.cur = 0;
    }
    return OR_OK;
}

/* spikes of group g `delay` bins back, restricted to [origin, origin+cnt),
 * returned relative to origin (utils/circular.py:232-238 get_spikes). */
static void get_spikes(const Group &g, int32_t delay, int64_t origin, int64_t cnt, std::vector<int32_t> &out) {
    out.clear();
    for (int32_t i : g.hist[delay]) if (i >= origin && i < origin + cnt) out.push_back((int32_t)(i - origin));
}

static inline float clipf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
static inline double clipd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

static void step(or_net *n, int64_t cs) {
    const double dt = n->dt;
    const double t = (double)cs * dt;
    std::vector<int32_t> spk;
    /* ---- start slot: TimedArraySetters ---- */
    for (auto &g : n->groups)
        for (const auto &h : g.setters) {
            if (cs < h.first) continue;
            const double *row = &h.vals[(size_t)(setter_row(h, cs, dt) * h.ncols)];
            double *sv = &g.S[(size_t)h.var * g.n + h.origin];
            for (int64_t k = 0; k < h.count; ++k) sv[k] = row[h.ncols == 1 ? 0 : k];
        }
    /* ---- groups slot ---- */
    for (size_t gi = 0; gi < n->groups.size(); ++gi) {
        Group &g = n->groups[gi];
        const int64_t N = g.n; const int m = g.nvar;
        if (g.gen_update) {
            for (int64_t i = 0; i < N; ++i) g.gen_update(g.S.data(), N, i, t);
        } else if (g.linear) {
            std::vector<double> x(m), s(m);
            for (int64_t i = 0; i < N; ++i) {
                for (int k = 0; k < m; ++k) s[k] = g.S[(size_t)k * N + i];
                /* x_j = ((0 + A[j][k0] s_k0) + A[j][k1] s_k1) + ... over the
                 * nonzero A[j][k] left to right, then + C[j] when nonzero.
                 * Skipping exact zeros of A and C (the reference's dot product
                 * adds them) and starting from +0 change nothing but the sign
                 * of an exact-zero result. */
                for (int j = 0; j < m; ++j) {
                    double acc = 0.0;
                    for (int k = 0; k < m; ++k) {
                        if (g.A[j * m + k] == 0.0) continue;
                        acc = acc + g.A[j * m + k] * s[k];
                    }
                    if (g.useC && g.C[j] != 0.0) acc = acc + g.C[j];
                    x[j] = acc;
                }
                for (int k = 0; k < m; ++k) g.S[(size_t)k * N + i] = x[k];
            }
        }
        std::vector<int32_t> spikes;
        if (g.gen_threshold) {
            for (int64_t i = 0; i < N; ++i) if (g.gen_threshold(g.S.data(), N, i, t)) spikes.push_back((int32_t)i);
        } else
        switch (g.thr_kind) {
        case 1: { const double *v = &g.S[(size_t)g.thr_var * N];
                  for (int64_t i = 0; i < N; ++i) if (v[i] > g.thr_val) spikes.push_back((int32_t)i); break; }
        case 2: { const double *v = &g.S[(size_t)g.thr_var * N], *vt = &g.S[(size_t)g.thr_var2 * N];
                  for (int64_t i = 0; i < N; ++i) if (v[i] > vt[i]) spikes.push_back((int32_t)i); break; }
        case 3: { const double *r = &g.S[(size_t)g.rate_var * N];
                  for (int64_t i = 0; i < N; ++i) if (philox_uniform(g.seed, cs, i) < r[i] * dt) spikes.push_back((int32_t)i); break; }
        case 4: { auto lo = std::lower_bound(g.gen_steps.begin(), g.gen_steps.end(), cs);
                  for (auto it = lo; it != g.gen_steps.end() && *it == cs; ++it) {
                      int32_t i = g.gen_idx[it - g.gen_steps.begin()];
                      if (spikes.empty() || spikes.back() != i) spikes.push_back(i);
                  } break; }
        default: break;
        }
        if (g.emp_steps > 0) {   /* not among the spikes of the last emp_steps steps */
            if (g.last_spike.empty()) g.last_spike.assign(N, -(1ll << 40));
            std::vector<int32_t> kept;
            for (int32_t i : spikes) if (n->nstep - g.last_spike[i] > g.emp_steps) kept.push_back(i);
            for (int32_t i : kept) g.last_spike[i] = n->nstep;
            spikes.swap(kept);
        }
        if (g.refr) {
            std::vector<int32_t> kept;
            for (int32_t i : spikes) if (g.next_allowed[i] <= t) kept.push_back(i);
            for (int32_t i : kept) g.next_allowed[i] = t + g.refr_time;
            spikes.swap(kept);
        }
        g.nspikes += (int64_t)spikes.size();
        g.hist.pop_back(); g.hist.push_front(std::move(spikes));
    }
    for (auto &s : n->stdps) {   /* trace groups G_pre / G_post (stdp.py:282-293) */
        for (auto &a : s.A_pre) a = s.a_pre * a + s.c_pre;
        for (auto &a : s.A_post) a = s.a_post * a + s.c_post;
    }
    /* ---- connections slot ---- */
    for (const Item &it : n->items) {
        if (it.kind == IT_CONN) {
            Conn &c = n->conns[it.id];
            const Group &gs = n->groups[c.src]; Group &gt = n->groups[c.tgt];
            get_spikes(gs, c.hetero ? 0 : c.delay, c.so, c.sn, spk);
            double *sv = &gt.S[(size_t)c.var * gt.n + c.to];
            const double *mod = c.mod_var >= 0 ? &gs.S[(size_t)c.mod_var * gs.n + c.so] : nullptr;
            for (int32_t i : spk) {
                c.events += c.dense ? c.tn : c.rowptr[i + 1] - c.rowptr[i];
                if (c.dense) {
                    for (int64_t j = 0; j < c.tn; ++j) {
                        double w = c.getw((int64_t)i * c.tn + j);
                        if (mod) w = w * mod[i];
                        sv[j] = sv[j] + w;
                    }
                } else if (!c.hetero) {
                    for (int64_t k = c.rowptr[i]; k < c.rowptr[i + 1]; ++k) {
                        double w = c.getw(k); if (mod) w = w * mod[i];
                        sv[c.cols[k]] = sv[c.cols[k]] + w;
                    }
                } else {
                    for (int64_t k = c.rowptr[i]; k < c.rowptr[i + 1]; ++k) {
                        double w = c.getw(k); if (mod) w = w * mod[i];
                        size_t slot = (size_t)((c.cur + c.d[k]) % c.md);
                        double &r = c.ring[slot * c.tn + c.cols[k]];
                        r = r + w;
                    }
                }
            }
        } else if (it.kind == IT_SYN) {
            Syn &y = n->syns[it.id];
            get_spikes(n->groups[y.src], 0, y.so, y.sn, spk);
            for (int32_t i : spk)
                for (int32_t e : y.syn_of_pre[i]) y.X[(size_t)((y.cur + y.delay[e]) % y.L)].push_back(e);
        } else if (it.kind == IT_SPIKEMON) {
            SpikeMon &m = n->smons[it.id];
            get_spikes(n->groups[m.gid], m.delay, m.origin, m.n, spk);
            for (int32_t i : spk) { m.steps.push_back(cs); m.idx.push_back(i); }
        } else if (it.kind == IT_STDP_PRE && n->stdps[it.id].delayed) {
            Stdp &s = n->stdps[it.id]; Conn &c = n->conns[s.cid];
            /* immediate updater: spikes of this step */
            get_spikes(n->groups[c.src], 0, c.so, c.sn, spk);
            for (int32_t i : spk) {
                if (s.inter == 0 || s.inter == 3) s.A_pre[i] = s.A_pre[i] + s.Ap; else s.A_pre[i] = s.Ap;
            }
            /* delayed updater: spikes of max_delay ago, w[i,:] += A_post past values */
            get_spikes(n->groups[c.src], s.pre_delay, c.so, c.sn, spk);
            for (int32_t i : spk)
                for (int64_t k = c.rowptr[i]; k < c.rowptr[i + 1]; ++k) {
                    const double add = s.H_post[past_slot(s, s.lag_pre[k]) * c.tn + c.cols[k]];
                    if (c.w_bits == 64) c.w64[k] = clipd(wupd(c.w64[k], add, s.pre_mode, s.wx), s.wmin, s.wmax);
                    else c.w32[k] = clipf((float)((double)c.w32[k] + add), (float)s.wmin, (float)s.wmax);
                }
        } else if (it.kind == IT_STDP_POST && n->stdps[it.id].delayed) {
            Stdp &s = n->stdps[it.id]; Conn &c = n->conns[s.cid];
            get_spikes(n->groups[c.tgt], 0, c.to, c.tn, spk);
            for (int32_t j : spk) {
                if (s.inter == 0) s.A_post[j] = s.A_post[j] + s.Am; else s.A_post[j] = s.Am;
            }
            for (int32_t j : spk)
                for (int64_t p = c.colptr[j]; p < c.colptr[j + 1]; ++p) {
                    const int64_t k = c.colk[p]; const int32_t i = c.colsrc[p];
                    const double add = s.H_pre[past_slot(s, s.lag_post[k]) * c.sn + i];
                    if (c.w_bits == 64) c.w64[k] = clipd(wupd(c.w64[k], add, s.post_mode, s.wx), s.wmin, s.wmax);
                    else c.w32[k] = clipf((float)((double)c.w32[k] + add), (float)s.wmin, (float)s.wmax);
                }
        } else if (it.kind == IT_STDP_PRE) {
            Stdp &s = n->stdps[it.id]; Conn &c = n->conns[s.cid];
            get_spikes(n->groups[c.src], s.pre_delay, c.so, c.sn, spk);
            for (int32_t i : spk) {
                if (s.inter == 0 || s.inter == 3) s.A_pre[i] = s.A_pre[i] + s.Ap; else s.A_pre[i] = s.Ap;
                if (c.dense) {
                    for (int64_t j = 0; j < c.tn; ++j) {
                        size_t k = (size_t)i * c.tn + j;
                        if (c.w_bits == 64) c.w64[k] = clipd(wupd(c.w64[k], s.A_post[j], s.pre_mode, s.wx), s.wmin, s.wmax);
                        else c.w32[k] = clipf((float)((double)c.w32[k] + s.A_post[j]), (float)s.wmin, (float)s.wmax);
                    }
                } else {
                    for (int64_t k = c.rowptr[i]; k < c.rowptr[i + 1]; ++k) {
                        int32_t j = c.cols[k];
                        if (c.w_bits == 64) c.w64[k] = clipd(wupd(c.w64[k], s.A_post[j], s.pre_mode, s.wx), s.wmin, s.wmax);
                        else c.w32[k] = clipf((float)((double)c.w32[k] + s.A_post[j]), (float)s.wmin, (float)s.wmax);
                    }
                }
            }
        } else if (it.kind == IT_STDP_POST) {
            Stdp &s = n->stdps[it.id]; Conn &c = n->conns[s.cid];
            get_spikes(n->groups[c.tgt], s.post_delay, c.to, c.tn, spk);
            if (c.dense) {
                /* w[:, j] += A_pre for every spiking j: the columns are
                 * disjoint, so the matrix is walked row by row (one update
                 * of each element, as column by column) */
                for (int32_t j : spk) {
                    if (s.inter == 0) s.A_post[j] = s.A_post[j] + s.Am; else s.A_post[j] = s.Am;
                }
                for (int64_t i = 0; i < c.sn && !spk.empty(); ++i) {
                    const double add = s.A_pre[i];
                    for (int32_t j : spk) {
                        size_t k = (size_t)i * c.tn + j;
                        if (c.w_bits == 64) c.w64[k] = clipd(wupd(c.w64[k], add, s.post_mode, s.wx), s.wmin, s.wmax);
                        else c.w32[k] = clipf((float)((double)c.w32[k] + add), (float)s.wmin, (float)s.wmax);
                    }
                }
                continue;
            }
            for (int32_t j : spk) {
                if (s.inter == 0) s.A_post[j] = s.A_post[j] + s.Am; else s.A_post[j] = s.Am;   /* 'nearest_pre' is A_post=+Am */
                {
                    for (int64_t p = c.colptr[j]; p < c.colptr[j + 1]; ++p) {
                        int64_t k = c.colk[p]; int32_t i = c.colsrc[p];
                        if (c.w_bits == 64) c.w64[k] = clipd(wupd(c.w64[k], s.A_pre[i], s.post_mode, s.wx), s.wmin, s.wmax);
                        else c.w32[k] = clipf((float)((double)c.w32[k] + s.A_pre[i]), (float)s.wmin, (float)s.wmax);
                    }
                }
            }
        }
    }
    /* ---- after_connections: DelayConnection.delayed_propagate ---- */
    for (auto &c : n->conns) {
        if (!c.hetero) continue;
        Group &gt = n->groups[c.tgt];
        double *sv = &gt.S[(size_t)c.var * gt.n + c.to];
        double *row = &c.ring[(size_t)c.cur * c.tn];
        for (int64_t j = 0; j < c.tn; ++j) { sv[j] = sv[j] + row[j]; row[j] = 0.0; }
        c.cur = (c.cur + 1) % c.md;
    }
    /* ---- synapses ---- */
    synapses_deliver(n, t);
    /* ---- resets ---- */
    for (auto &g : n->groups) {
        const int64_t N = g.n;
        if (g.refr && g.period > 0) {
            double *v = &g.S[(size_t)g.clamp_var * N];
            for (int32_t b = 0; b < g.period && b < g.depth; ++b)
                for (int32_t i : g.hist[b]) v[i] = g.clamp_val;
        } else if (g.gen_reset) {
            for (int32_t i : g.hist[0]) g.gen_reset(g.S.data(), N, i, t);
        } else if (g.reset_kind == 1) {
            double *v = &g.S[(size_t)g.reset_var * N];
            for (int32_t i : g.hist[0]) v[i] = g.reset_val;
        } else if (g.reset_kind == 2) {
            double *v = &g.S[(size_t)g.reset_var * N]; const double *r = &g.S[(size_t)g.reset_var2 * N];
            for (int32_t i : g.hist[0]) v[i] = r[i];
        }
    }
    /* ---- end: state monitors ---- */
    for (auto &m : n->stmons) {
        if ((n->nstep - m.start) % m.timestep != 0) continue;
        const Group &g = n->groups[m.gid];
        const double *v = &g.S[(size_t)m.var * g.n];
        for (int32_t i : m.idx) m.vals.push_back(v[i]);
        m.steps.push_back(cs);
    }
    /* ---- end: the STDP trace RecentStateMonitors (monitor.py:1036-1049) ---- */
    for (auto &s : n->stdps) {
        if (!s.delayed) continue;
        std::copy(s.A_pre.begin(), s.A_pre.end(), s.H_pre.begin() + (size_t)s.cur * s.A_pre.size());
        std::copy(s.A_post.begin(), s.A_post.end(), s.H_post.begin() + (size_t)s.cur * s.A_post.size());
        s.cur = (s.cur + 1) % s.M;
    }
    n->nstep++;
}

int or_net_run(or_net *n, int64_t nsteps, int64_t cs0) {
    if (!n || nsteps < 0) return fail(OR_EINVAL, "run");
    if (!n->prepared) { int st = or_net_prepare(n); if (st) return st; }
    for (int64_t k = 0; k < nsteps; ++k) step(n, cs0 + k);
    return OR_OK;
}
int or_group_get_state(or_net *n, int32_t gid, int var, double *out) {
    if (!gid_ok(n, gid) || var < 0 || var >= n->groups[gid].nvar || !out) return fail(OR_EINVAL, "get_state");
    const Group &g = n->groups[gid];
    std::copy(g.S.begin() + (size_t)var * g.n, g.S.begin() + (size_t)(var + 1) * g.n, out); return OR_OK;
}
int or_group_set_state(or_net *n, int32_t gid, int var, const double *in) {
    if (!gid_ok(n, gid) || var < 0 || var >= n->groups[gid].nvar || !in) return fail(OR_EINVAL, "set_state");
    Group &g = n->groups[gid];
    std::copy(in, in + g.n, g.S.begin() + (size_t)var * g.n); return OR_OK;
}
int or_net_counters(or_net *n, int64_t *group_spikes, int64_t *conn_events) {
    if (!n) return fail(OR_EINVAL, "net");
    for (size_t g = 0; g < n->groups.size(); ++g) if (group_spikes) group_spikes[g] = n->groups[g].nspikes;
    for (size_t c = 0; c < n->conns.size(); ++c) if (conn_events) conn_events[c] = n->conns[c].events;
    return OR_OK;
}
int or_net_stats(or_net *n, int64_t *steps, int64_t *launches, double *ms) {
    if (!n) return fail(OR_EINVAL, "net");
    if (steps) *steps = n->nstep; if (launches) *launches = 0; if (ms) *ms = 0; return OR_OK;
}

}  /* extern "C" */

/* Checkpoint / resume of the oracle's dynamic state (the engine's
 * bg_net_save_state/bg_net_load_state; the reference pickles the network,
 * network.py:652, utils/circular.py:249-269): step counter, states, spike
 * histories, refractory bookkeeping, weights, rings and cursors, traces and
 * their records, SpikeQueue rows, counters and monitor records, loaded into
 * a network built the same way (sizes checked). */
namespace {
struct OW { std::vector<char> b;
    void raw(const void *p, size_t k) { const char *c = (const char *)p; b.insert(b.end(), c, c + k); }
    template <typename V> void val(const V &v) { raw(&v, sizeof(v)); }
    template <typename V> void vec(const std::vector<V> &v) { val((uint64_t)v.size()); raw(v.data(), v.size() * sizeof(V)); } };
struct OR_ { const char *p; size_t left; bool ok = true;
    void raw(void *d, size_t k) { if (!ok || k > left) { ok = false; return; } std::memcpy(d, p, k); p += k; left -= k; }
    template <typename V> void val(V &v) { raw(&v, sizeof(v)); }
    template <typename V> void vec(std::vector<V> &v) { uint64_t k = 0; val(k); if (!ok || k * sizeof(V) > left) { ok = false; return; } v.resize(k); raw(v.data(), k * sizeof(V)); }
    /* a vector whose size the network fixes */
    template <typename V> void same(std::vector<V> &v) { const size_t want = v.size(); std::vector<V> t; vec(t); if (ok && t.size() != want) ok = false; if (ok) v.swap(t); } };
template <typename IO> void or_visit(or_net *n, IO &io) {
    for (auto &g : n->groups) {
        io.same(g.S); io.same(g.next_allowed); io.same(g.last_spike); io.val(g.nspikes);
        uint64_t d = g.hist.size(); io.val(d);
        if (d != g.hist.size()) { io.ok = false; return; }
        for (auto &h : g.hist) io.vec(h);
    }
    for (auto &c : n->conns) { io.same(c.w64); io.same(c.w32); io.same(c.ring); io.val(c.cur); io.val(c.events); }
    for (auto &s : n->stdps) { io.same(s.A_pre); io.same(s.A_post); io.same(s.H_pre); io.same(s.H_post); io.val(s.cur); }
    for (auto &y : n->syns) {
        io.val(y.cur);
        uint64_t L = y.X.size(); io.val(L);
        if (L != y.X.size()) { io.ok = false; return; }
        for (auto &x : y.X) io.vec(x);
        io.same(y.sv);
    }
    for (auto &m : n->smons) { io.vec(m.steps); io.vec(m.idx); }
    for (auto &m : n->stmons) { io.vec(m.vals); io.vec(m.steps); }
}
/* the writer has no size check: `same` is `vec` */
struct OWv : OW { bool ok = true; template <typename V> void same(const std::vector<V> &v) { vec(v); } };
const uint64_t kOrMagic = 0x31534f4e47425242ull;
}

extern "C" {

int or_net_state_bytes(or_net *n, int64_t *bytes) {
    if (!n || !bytes) return fail(OR_EINVAL, "state_bytes");
    if (!n->prepared) { int st = or_net_prepare(n); if (st) return st; }
    OWv w; w.val(kOrMagic); w.val(n->nstep); or_visit(n, w);
    *bytes = (int64_t)w.b.size(); return OR_OK;
}
int or_net_save_state(or_net *n, void *buf, int64_t cap, int64_t *written) {
    if (!n || (!buf && cap > 0)) return fail(OR_EINVAL, "save_state");
    if (!n->prepared) { int st = or_net_prepare(n); if (st) return st; }
    OWv w; w.val(kOrMagic); w.val(n->nstep); or_visit(n, w);
    if ((int64_t)w.b.size() > cap) return fail(OR_EINVAL, "buffer too small for the state");
    std::memcpy(buf, w.b.data(), w.b.size());
    if (written) *written = (int64_t)w.b.size();
    return OR_OK;
}
int or_net_load_state(or_net *n, const void *buf, int64_t bytes) {
    if (!n || !buf || bytes < 0) return fail(OR_EINVAL, "load_state");
    if (!n->prepared) { int st = or_net_prepare(n); if (st) return st; }
    OR_ r{(const char *)buf, (size_t)bytes};
    uint64_t magic = 0; int64_t nstep = 0;
    r.val(magic); r.val(nstep);
    if (!r.ok || magic != kOrMagic) return fail(OR_EINVAL, "not a saved network state");
    or_visit(n, r);
    if (!r.ok || r.left) return fail(OR_EINVAL, "state does not match this network");
    n->nstep = nstep;
    return OR_OK;
}
int or_net_save(or_net *n, const char *path) {
    int64_t b = 0; int st = or_net_state_bytes(n, &b); if (st) return st;
    std::vector<char> buf((size_t)b); int64_t w = 0;
    st = or_net_save_state(n, buf.data(), b, &w); if (st) return st;
    FILE *f = std::fopen(path, "wb"); if (!f) return fail(OR_EINVAL, "open");
    const bool good = std::fwrite(buf.data(), 1, (size_t)w, f) == (size_t)w;
    if (std::fclose(f) != 0 || !good) return fail(OR_EINVAL, "write");
    return OR_OK;
}
int or_net_load(or_net *n, const char *path) {
    FILE *f = std::fopen(path, "rb"); if (!f) return fail(OR_EINVAL, "open");
    std::vector<char> buf; char tmp[1 << 16]; size_t k;
    while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
    std::fclose(f);
    return or_net_load_state(n, buf.data(), (int64_t)buf.size());
}

/* Uniform draw shared with the device Poisson source; exported so tests can
 * pin the stream against known answers. */
double or_philox_uniform(uint64_t seed, int64_t step, int64_t i) { return philox_uniform(seed, step, i); }

/* Fixed in-degree connectivity (random_matrix_fixed_column,
 * construction.py:149-177: every target receives k distinct sources drawn
 * uniformly), the draws of the engine's bg_fixed_indegree_csr: per target j,
 * Philox4x32-10 blocks keyed by the seed with counter (j, attempt) give two
 * sources each (high half of word * n_src); the row is sorted, duplicates
 * dropped and the missing entries drawn again after the kept ones.  CSR rows
 * over sources with ascending targets.  Single-threaded, so the CPU side of
 * a benchmark builds its network without the engine library. */
int or_fixed_indegree_csr(int64_t n_src, int64_t n_tgt, int64_t k, uint64_t seed, int64_t *rowptr, int32_t *cols) {
    if (n_src <= 0 || n_tgt < 0 || k < 0 || k > n_src || !rowptr || (n_tgt * k > 0 && !cols))
        return fail(OR_EINVAL, "fixed_indegree_csr arguments");
    std::vector<int32_t> s((size_t)k);
    std::memset(rowptr, 0, sizeof(int64_t) * (size_t)(n_src + 1));
    std::vector<int32_t> src((size_t)(n_tgt * k));
    for (int64_t j = 0; j < n_tgt; ++j) {
        int64_t have = 0; uint64_t attempt = 0;
        while (have < k) {
            for (int64_t r = have; r < k; r += 2) {
                uint32_t c[4] = {(uint32_t)j, (uint32_t)((uint64_t)j >> 32), (uint32_t)attempt, (uint32_t)(attempt >> 32)};
                philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
                ++attempt;
                s[r] = (int32_t)(((uint64_t)c[0] * (uint64_t)n_src) >> 32);
                if (r + 1 < k) s[r + 1] = (int32_t)(((uint64_t)c[1] * (uint64_t)n_src) >> 32);
            }
            std::sort(s.begin(), s.end());
            have = std::unique(s.begin(), s.end()) - s.begin();
        }
        for (int64_t r = 0; r < k; ++r) { src[(size_t)(j * k + r)] = s[r]; rowptr[s[r] + 1]++; }
    }
    for (int64_t i = 0; i < n_src; ++i) rowptr[i + 1] += rowptr[i];
    std::vector<int64_t> fill(rowptr, rowptr + n_src);
    for (int64_t j = 0; j < n_tgt; ++j)
        for (int64_t r = 0; r < k; ++r) cols[fill[src[(size_t)(j * k + r)]]++] = (int32_t)j;
    return OR_OK;
}

}  /* extern "C" */
