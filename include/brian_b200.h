/*
 * brian_b200.h -- C ABI of the B200 clock-driven spiking-network engine.
 *
 * The engine replaces Brian 1.4.4's clock-driven simulation loop
 * (NeuronGroup.update / Connection.propagate / DelayConnection /
 * ExponentialSTDP / SpikeMonitor / StateMonitor / Network.run) and the GPU
 * model-fitting kernel (GPUModelFitting).  Every entry point is plain C:
 * pointers, sizes, and an int status.  Nothing here throws; a negative
 * status carries an error class and bg_last_error() returns the message
 * of the calling thread's last failure.
 *
 * Ownership: handles (bg_net, bg_fit) own every device buffer they
 * allocate and free them in bg_*_destroy.  Host arrays passed in are
 * copied before the call returns.  One handle = one CUDA stream; calls on
 * different handles may come from different threads, calls on one handle
 * must be serialised by the caller.
 *
 * Units: all values are SI floats (volt, second, ...), the same numbers
 * Brian holds in its state matrix when units are stripped.
 */
#ifndef BRIAN_B200_H
#define BRIAN_B200_H

#include <stdint.h>
#include <stddef.h>

#if defined(__GNUC__)
#define BG_API __attribute__((visibility("default")))
#else
#define BG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define BG_OK        0
#define BG_EINVAL   (-1)   /* bad argument (size, index, kind)              */
#define BG_ENOMEM   (-2)   /* device or host allocation failed              */
#define BG_ECUDA    (-3)   /* a CUDA runtime/driver call failed             */
#define BG_ETIMEOUT (-4)   /* a bounded device-side wait gave up            */
#define BG_ENUMERIC (-5)   /* non-finite value detected                     */
#define BG_ESTATE   (-6)   /* call not valid in the handle's current state  */
#define BG_ENOSYS   (-7)   /* feature combination not implemented           */
#define BG_ECOMPILE (-8)   /* runtime compilation of generated code failed  */

/* threshold kinds: Threshold (threshold.py:129-200), VariableThreshold
 * (threshold.py:337-406), PoissonThreshold (threshold.py:461-471),
 * SpikeGeneratorGroup (directcontrol.py:63-217). */
#define BG_THR_NONE      0
#define BG_THR_CONST     1   /* S[var] >  value                                */
#define BG_THR_VAR       2   /* S[var] >  S[var2]                              */
#define BG_THR_POISSON   3   /* u(seed,step,i) < S[var]*dt  (Philox4x32-10)    */
#define BG_THR_GENERATOR 4   /* explicit (step, index) list                    */

/* reset kinds: Reset (reset.py:115-152), VariableReset (reset.py:220-257) */
#define BG_RESET_NONE  0
#define BG_RESET_CONST 1     /* S[var] = value                                 */
#define BG_RESET_VAR   2     /* S[var] = S[var2]                               */

/* STDP interaction kinds (stdp.py:495-509) */
#define BG_STDP_ALL          0
#define BG_STDP_NEAREST      1
#define BG_STDP_NEAREST_PRE  2
#define BG_STDP_NEAREST_POST 3

typedef struct bg_net bg_net;
typedef struct bg_fit bg_fit;

/* ---- library ----------------------------------------------------------- */
BG_API int bg_version(void);
/* Copies the calling thread's last error message (NUL-terminated). */
BG_API int bg_last_error(char *buf, int64_t len);

/* ---- network handle ------------------------------------------------------
 * Replaces Network (network.py:62-679): groups, connections and monitors are
 * registered, bg_net_prepare freezes the schedule, bg_net_run advances it.
 * precision: 64 (bit-exact FP64 path) or 32 (FP32 state/accumulation).
 * deterministic: 1 = accumulation order of the reference for every
 * connection; 0 = atomics allowed where the result may then differ in the
 * last bit (FP32 studies).  Connections with one shared weight use atomics
 * in both modes, which is exact because every addend is identical. */
BG_API int bg_net_create(int device, int precision, int deterministic, double dt,
                  bg_net **out);
BG_API int bg_net_destroy(bg_net *net);

/* ---- neuron groups --------------------------------------------------------
 * NeuronGroup.__init__ (neurongroup.py:258-456): state matrix _S of shape
 * (nvar, n), row-major, rows in the model's variable order. */
BG_API int bg_group_add(bg_net *net, int64_t n, int nvar, const double *S0,
                 int32_t *gid);
/* LinearStateUpdater (stateupdater.py:328-417): S <- A.S (+ C when C is not
 * NULL).  A is nvar x nvar row-major; the sum runs left to right over the
 * columns without fused multiply-add. */
BG_API int bg_group_set_linear(bg_net *net, int32_t gid, const double *A,
                        const double *C);
/* TimedArraySetter (timedarray.py:238-303; TimedArray.__call__ 209-235):
 * at the start of every step (clock step cs >= first_step), before the
 * update, S[var][origin + k] for k < count takes row r of
 * values[nrows][ncols] (ncols 1: the same value for all, else ncols =
 * count).  mode 0, an array on a clock grid: r = rint((cs*dt - t_init) /
 * adt) clamped to [0, nrows); mode 1, an array on explicit ascending times:
 * r = the number of the nrows-1 breakpoint clock steps bp[] (ascending; bp[i-1]
 * the first step whose time reaches times[i]) that are <= cs.  At most 4 per
 * group; groups with one run on the per-step kernels. */
BG_API int bg_group_set_timed_array(bg_net *net, int32_t gid, int var, int64_t origin, int64_t count,
                                    const double *values, int64_t nrows, int64_t ncols, int mode,
                                    double t_init, double adt, int64_t first_step, const int64_t *bp);
/* Threshold / VariableThreshold (threshold.py:160-191, 373-396). */
BG_API int bg_group_set_threshold(bg_net *net, int32_t gid, int kind, int var,
                           double value, int var2);
/* PoissonGroup (directcontrol.py:406-447) + PoissonThreshold
 * (threshold.py:461-471): spike when u < S[rate_var]*dt, u from a
 * counter-based Philox4x32-10 stream keyed by (seed, clock step, index). */
BG_API int bg_group_set_poisson(bg_net *net, int32_t gid, int rate_var,
                         uint64_t seed);
/* SpikeGeneratorGroup (directcontrol.py:63-217): spikes given as clock
 * steps, sorted by (step, index). */
BG_API int bg_group_set_generator(bg_net *net, int32_t gid, int64_t nspikes,
                           const int64_t *steps, const int32_t *idx);
/* Reset / VariableReset (reset.py:139-147, 241-254), applied in the
 * 'resets' slot to the neurons that spiked in this step. */
BG_API int bg_group_set_reset(bg_net *net, int32_t gid, int kind, int var,
                       double value, int var2);
/* Refractoriness (neurongroup.py:506-515, reset.py:311-332).
 * refractory_time = T - dt/2 (next allowed spike time offset; <= 0 turns
 * the spike filter off, as for T < 0.9*dt);
 * period = int(T/dt)+1 bins during which S[var] is clamped to value
 * (period 0: no clamp, only the spike filter). */
/* EmpiricalThreshold (threshold.py:409-457): a neuron that spiked in the
 * last `steps` steps does not spike (steps = the threshold's refractory in
 * steps); 0 turns it off. */
BG_API int bg_group_set_empirical(bg_net *net, int32_t gid, int32_t steps);
BG_API int bg_group_set_refractory(bg_net *net, int32_t gid, double refractory_time,
                            int32_t period, int var, double value);

/* ---- connections ----------------------------------------------------------
 * Connection (connection.py:224-296) with SparseConnectionMatrix rows
 * (connectionmatrix.py:196-387) and, when delays != NULL, DelayConnection
 * (delayconnection.py:132-206): emission-time scatter into a ring of
 * ring_depth rows, delivered in the 'after_connections' slot.
 * rowptr has src_n+1 entries; cols are target indices (relative to
 * tgt_origin), ascending within a row; w has w_bits 32 or 64.
 * delay_steps is the homogeneous presynaptic delay of a plain Connection
 * (spikes read from the source history delay_steps bins back).
 * mod_var >= 0 multiplies each weight by the source's S[mod_var][i]. */
BG_API int bg_conn_add(bg_net *net, int32_t src_gid, int64_t src_origin,
                int64_t src_n, int32_t tgt_gid, int64_t tgt_origin,
                int64_t tgt_n, int tgt_var, int64_t nnz,
                const int64_t *rowptr, const int32_t *cols, const void *w,
                int w_bits, int32_t delay_steps, const uint8_t *delays,
                int32_t ring_depth, int mod_var, int32_t *cid);
/* bg_conn_add for a connection whose synapses all carry one weight (the
 * scalar `weight` argument of Connection.connect*, connection.py:354-475,
 * stored as w_bits 32 or 64): no per-synapse weight array is passed. */
BG_API int bg_conn_add_shared(bg_net *net, int32_t src_gid, int64_t src_origin,
                int64_t src_n, int32_t tgt_gid, int64_t tgt_origin,
                int64_t tgt_n, int tgt_var, int64_t nnz,
                const int64_t *rowptr, const int32_t *cols, double weight,
                int w_bits, int32_t delay_steps, const uint8_t *delays,
                int32_t ring_depth, int mod_var, int32_t *cid);
/* DenseConnectionMatrix (connectionmatrix.py:141-193): W[src_n][tgt_n]. */
BG_API int bg_conn_add_dense(bg_net *net, int32_t src_gid, int64_t src_origin,
                      int64_t src_n, int32_t tgt_gid, int64_t tgt_origin,
                      int64_t tgt_n, int tgt_var, const void *W, int w_bits,
                      int32_t delay_steps, int mod_var, int32_t *cid);
/* Weights in the connection's own order (CSR data order, or row-major for
 * dense), widened to double. */
BG_API int bg_conn_get_weights(bg_net *net, int32_t cid, double *out);
BG_API int bg_conn_set_weights(bg_net *net, int32_t cid, const double *in);

/* ExponentialSTDP / STDP (stdp.py:181-539) on a non-delayed connection.
 * decay = {a_pre, c_pre, a_post, c_post}: the 1x1 linear updaters of the
 * separated trace groups (A <- a*A + c).  Pre spike i: A_pre[i] (+)= Ap;
 * w[i,:] += A_post; clip.  Post spike j: A_post[j] (+)= Am; w[:,j] +=
 * A_pre; clip.  pre_delay/post_delay in bins.  Two items are appended to
 * the connections slot: the presynaptic then the postsynaptic updater. */
BG_API int bg_stdp_add(bg_net *net, int32_t cid, const double *decay, double Ap,
                double Am, double wmin, double wmax, int interactions,
                int32_t pre_delay, int32_t post_delay, int32_t *sid);
/* Synapses (synapses/synapses.py:43-1058) with static synaptic variables and
 * presynaptic code of `nops` (<= 4) statements x (+|-)= term, replacing
 * Synapses.__init__/create_synapses and the SpikeQueue
 * (synapses/spikequeue.py:69-330).  Synapse k joins source pre[k] (relative
 * to src_origin) to target post[k] (relative to tgt_origin) with a delay of
 * delay[k] bins (<= 253).  Statement q sets target variable op_var[q] to
 * x - terms[q][k] when op_sub[q], else x + terms[q][k], terms [nops][nsyn]
 * in synapse order.  A spike of step s is applied at step s + delay, in
 * the 'synapses' slot after the connections and before the resets
 * (network.py:365-380); the events reaching one target in one step are
 * applied in queue order (insertion step, then source index, then synapse
 * index).  FP64 networks only; a target variable also fed by a
 * DelayConnection on the same neurons is refused at prepare (BG_ENOSYS). */
BG_API int bg_synapses_add(bg_net *net, int32_t src_gid, int64_t src_origin,
                int64_t src_n, int32_t tgt_gid, int64_t tgt_origin, int64_t tgt_n,
                int64_t nsyn, const int32_t *pre, const int32_t *post,
                const int32_t *delay, int nops, const int32_t *op_var,
                const int32_t *op_sub, const double *terms, int32_t *sid);
/* New statement terms ([nops][nsyn], synapse order), e.g. after S.w[:] = ...
 * (synapticvariable.py __setitem__) between runs. */
BG_API int bg_synapses_set_terms(bg_net *net, int32_t sid, const double *terms);
/* Synapses with code (synapses.py:149-330, 400-510): nsv synaptic
 * variables (initial values sv[nsv][nsyn], synapse order; NULL: zeros), a
 * presynaptic code run for every event of a target in queue order and a
 * postsynaptic code run for every synapse of a target that spiked in the
 * step, after the events (the post queue, delay 0), both in the 'synapses'
 * slot.  The codes are C statement lists over X(s) (target variable
 * slot_var[s]), SV(k) (synaptic variable k), PRE(k) (source variable
 * pre_var[k], read only), T (the time), bg_exp and bg_clip (identical on
 * the GPU and in the CPU restatement); `writes` lists the target variables
 * the codes assign.  Replaces the statement terms of bg_synapses_add (nops
 * must be 0); before prepare. */
BG_API int bg_synapses_set_code(bg_net *net, int32_t sid, int32_t nsv, const double *sv, const char *pre_code,
                                const char *post_code, int32_t nslots, const int32_t *slot_var, int32_t nwrites,
                                const int32_t *writes, int32_t npre, const int32_t *pre_var);
/* Synaptic variable k of a Synapses with code, in synapse order. */
BG_API int bg_synapses_get_var(bg_net *net, int32_t sid, int32_t k, double *out);
BG_API int bg_synapses_set_var(bg_net *net, int32_t sid, int32_t k, const double *in);

/* ExponentialSTDP on a sparse DelayConnection (stdp.py:296-368, replacing
 * the STDPUpdater / DelayedSTDPUpdater pair and the two RecentStateMonitors
 * of monitor.py:991-1099).  Three items run in the connections slot, after
 * the connection: a spike of source i now does A_pre[i] (+)= Ap; a spike of
 * source i `pre_delay` bins ago (the connection's max_delay) does
 * w[k] += A_post[cols[k]] as recorded lag_pre[k] steps back, clip, for each
 * synapse k of row i; a spike of target j now does A_post[j] (+)= Am, then
 * w[k] += A_pre[src(k)] as recorded lag_post[k] steps back, clip, for each
 * synapse k of column j.  The traces are recorded once per step, at the end
 * of the step, into `hist_len` slots; lag L at step t reads the record of
 * step t-1-L, zero before the first record.  lag_pre / lag_post are per
 * synapse in CSR order, each in [0, hist_len): the reference's
 * int((1/dt) * (max_delay - d)) and int((1/dt) * d) modulo hist_len, d the
 * synapse's delay in seconds.  hist_len <= 256. */
BG_API int bg_stdp_add_delayed(bg_net *net, int32_t cid, const double *decay,
                double Ap, double Am, double wmin, double wmax,
                int interactions, int32_t pre_delay, int32_t hist_len,
                const uint8_t *lag_pre, const uint8_t *lag_post,
                int32_t *sid);
/* Update forms of the rule's w lines (ExponentialSTDP update='multiplicative'
 * or 'mixed', stdp.py:510-533): mode 0 w += a (the default), mode 1
 * w *= (1 + a), mode 2 w += (wmax_exact - w) * a, then the clip; pre_mode
 * for the presynaptic line (a = A_post), post_mode for the postsynaptic one
 * (a = A_pre).  Modes 1 and 2 need FP64 weights. */
BG_API int bg_stdp_set_update(bg_net *net, int32_t sid, int pre_mode, int post_mode,
                double wmax_exact);
BG_API int bg_stdp_get_traces(bg_net *net, int32_t sid, double *a_pre,
                       double *a_post);

/* ---- monitors ------------------------------------------------------------
 * SpikeMonitor (monitor.py:84-218): appends (clock step, index - origin) in
 * the connections slot; StateMonitor (monitor.py:683-989): records S[var] at
 * idx every `timestep` steps after the resets (when='end'). */
BG_API int bg_spikemon_add(bg_net *net, int32_t gid, int64_t origin, int64_t n,
                    int32_t delay, int32_t *mid);
BG_API int bg_statemon_add(bg_net *net, int32_t gid, int var, int64_t nidx,
                    const int32_t *idx, int32_t timestep, int32_t *mid);
/* Number of spikes recorded so far. */
BG_API int bg_spikemon_count(bg_net *net, int32_t mid, int64_t *n);
/* Copies up to cap recorded spikes; *n receives the number copied. */
BG_API int bg_spikemon_read(bg_net *net, int32_t mid, int64_t *steps, int32_t *idx,
                     int64_t cap, int64_t *n);
BG_API int bg_statemon_count(bg_net *net, int32_t mid, int64_t *nrows);
/* values: row-major [row][nidx]; steps: clock step of each row. */
BG_API int bg_statemon_read(bg_net *net, int32_t mid, double *values,
                     int64_t *steps, int64_t cap_rows, int64_t *nrows);
/* Clears a monitor's records (SpikeMonitor.reinit / StateMonitor.reinit). */
BG_API int bg_monitor_clear(bg_net *net, int32_t mid);

/* ---- schedule -------------------------------------------------------------
 * Network.prepare + Network.run (network.py:313-363, 541-586): each step is
 * groups -> connections slot (items in registration order) ->
 * after_connections (ring delivery) -> resets -> end (state monitors). */
BG_API int bg_net_prepare(bg_net *net);
BG_API int bg_net_run(bg_net *net, int64_t nsteps, int64_t clock_step0);
BG_API int bg_group_get_state(bg_net *net, int32_t gid, int var, double *out);
BG_API int bg_group_set_state(bg_net *net, int32_t gid, int var, const double *in);
/* Clears spike history, rings, refractory state and trace variables
 * (NeuronGroup.reinit / Connection.reinit); states are set by the caller. */
BG_API int bg_net_reinit(bg_net *net);
/* Running totals since prepare: spikes emitted per group (index = group id)
 * and synaptic events (sum over spiking sources of their row length) per
 * connection (index = connection id).  No counterpart in the reference;
 * its benchmark derives events as spikes x out-degree. */
BG_API int bg_net_counters(bg_net *net, int64_t *group_spikes,
                           int64_t *conn_events);
/* Runs nsteps steps launching each kernel of the step separately with CUDA
 * events in between and writes the mean device milliseconds of every
 * launch of the step (in schedule order) to ms[0..*nitems).  The steps
 * are real simulation steps.  Networks with monitors are rejected. */
BG_API int bg_net_profile(bg_net *net, int64_t nsteps, int64_t clock_step0,
                          double *ms, int64_t cap, int64_t *nitems);
/* Name of the idx-th launch of a step, e.g. "head[g0]", "prop_ring_atomic[c1]". */
BG_API int bg_net_item_name(bg_net *net, int64_t idx, char *buf, int64_t len);
/* Connectivity of random_matrix_fixed_column (construction.py:149-177):
 * each of n_tgt targets gets k distinct sources drawn uniformly from
 * [0, n_src); CSR over sources (rowptr n_src+1, cols n_tgt*k) with
 * ascending targets.  Counter-based draws keyed by (seed, target). */
BG_API int bg_fixed_indegree_csr(int64_t n_src, int64_t n_tgt, int64_t k,
                                 uint64_t seed, int64_t *rowptr,
                                 int32_t *cols);
/* Allow (1, default) or forbid (0) the persistent single-launch step loop
 * for networks of its shape; call before bg_net_prepare.  256 or 512 allow
 * it with that many threads per block (256 x 4 or 512 x 2 neurons per
 * block) instead of the automatic choice, when the blocks fit co-resident.
 * All paths and block shapes give identical results. */
BG_API int bg_net_set_persistent(bg_net *net, int enable);
/* Threads per block of the persistent kernel the prepared network runs
 * with, or 0 when it runs the general per-step launches. */
BG_API int bg_net_persistent_threads(bg_net *net, int32_t *threads);
/* ---- borrowed device buffers --------------------------------------------
 * Device memory the caller owns (a torch tensor, another library's buffer)
 * registered with the network; the library never frees it.  bytes >= what
 * its use needs, 256-byte aligned, on the network's device.  No counterpart
 * in the reference (its state arrays are numpy arrays the updaters mutate in
 * place, stateupdater.py:175-221; here a group's state can likewise be an
 * array the caller holds). */
#define BG_DTYPE_F64 0
#define BG_DTYPE_F32 1
BG_API int bg_import_device_ptr(bg_net *net, void *ptr, int64_t bytes,
                                int dtype, int32_t *buf_id);
/* The group's state lives in the borrowed buffer: [nvar][npad] rows of the
 * network's precision (npad from bg_group_padded_size, a multiple of 1024;
 * entries past the group's size are scratch).  bg_net_prepare writes the
 * initial state into it; between runs (after the call returns) the caller
 * may read and write it directly, as bg_group_get_state/set_state do.  Set
 * before bg_net_prepare. */
BG_API int bg_group_use_buffer(bg_net *net, int32_t gid, int32_t buf_id);
BG_API int bg_group_padded_size(bg_net *net, int32_t gid, int64_t *npad);
/* Synapses delivery: mode 0 (default) takes the event path (the events of
 * the spiking sources, binned by target block and applied in queue order)
 * when the synapse words exceed half of L2 or the network has the shape of
 * the persistent kernel for Synapses (one linear group, its Synapses onto
 * itself with one statement each), the pull over every synapse otherwise;
 * mode 1 takes the event path whatever the size, mode 2 the pull.  All give
 * identical results.  Set before bg_net_prepare. */
BG_API int bg_net_set_synapse_events(bg_net *net, int mode);
/* ---- checkpoint / resume (Network.__reduce__, network.py:652;
 * SpikeContainer.__reduce__, utils/circular.py:249-269;
 * LinearStateUpdater.__getstate__, stateupdater.py:469-481) ----------------
 * The dynamic state of a prepared network -- step counter, group states,
 * spike histories, refractory bookkeeping, delay and count rings, plastic
 * weights, STDP traces and trace records, counters and monitor records --
 * as one byte string.  It is loaded into a network built the same way
 * (same objects, sizes and precision; every section's size is checked,
 * BG_EINVAL on a mismatch).  Ring cursors and Poisson draws follow from the
 * step counter, so run(T1); save; load into a rebuilt network; run(T2)
 * equals run(T1 + T2).  bg_net_save/bg_net_load write and read a file. */
BG_API int bg_net_state_bytes(bg_net *net, int64_t *bytes);
BG_API int bg_net_save_state(bg_net *net, void *buf, int64_t cap,
                             int64_t *written);
BG_API int bg_net_load_state(bg_net *net, const void *buf, int64_t bytes);
BG_API int bg_net_save(bg_net *net, const char *path);
BG_API int bg_net_load(bg_net *net, const char *path);
/* ---- failure detection (no counterpart in the reference, where a stalled
 * or diverging simulation just runs on) -------------------------------------
 * Polls of the persistent kernel's bounded inter-block wait before it gives
 * up (default 2^22, a few seconds): every block then leaves its step loop,
 * bg_net_run returns BG_ETIMEOUT with no kernel left running, and the
 * network refuses further runs (BG_ESTATE).  Set before bg_net_prepare. */
BG_API int bg_net_set_spin_limit(bg_net *net, int64_t polls);
/* Test hook for the bounded waits: block `block` of the persistent kernel
 * never publishes its step arrivals, so the other blocks' waits run out
 * (-1, the default: off).  Set before bg_net_prepare. */
BG_API int bg_net_debug_hold_arrival(bg_net *net, int32_t block);
/* With enable = 1, every bg_net_run ends with a scan of all state
 * variables; a NaN or infinity returns BG_ENUMERIC naming the group,
 * variable and neuron, and the network refuses further runs. */
BG_API int bg_net_set_check_finite(bg_net *net, int enable);
/* ---- allocation-free entry point ------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (code inside another framework's caching allocator, which owns the
 * device memory, or a process that reserved all device memory up front):
 * runs one linear group with up to 4
 * shared-weight DelayConnections onto itself for nsteps steps, like a fresh
 * bg_net with those objects and bg_net_run(nsteps, 0), with identical
 * results.  It calls no cudaMalloc/cudaFree; its scratch is a file-scope
 * device array of bg_noalloc_scratch_bytes() bytes (32 MiB) that every GPU
 * loading the library holds until the process exits.  Networks needing more
 * scratch are rejected with BG_EINVAL.
 *   S      device, [nvar][n] row-major (stride n), updated in place
 *   A, C   host, the linear propagator (C may be NULL)
 *   connection c: sources [src_origin[c], +src_n[c]) of the group, target
 *   variable tgt_var[c]; rowptr[c] (device, src_n+1 entries, rowptr[0] >= 0,
 *   non-decreasing), cols[c] (device, targets in [0,n), ascending per row),
 *   delays[c] (device, steps below ring_depth[c] = int(max_delay/dt)+1,
 *   ring_depth in [1, 255]), shared weight weight[c].  Row pointers, targets
 *   and delays are checked on the device before the step loop (BG_EINVAL).
 * All calls share the scratch and each one clears what must start at zero,
 * so calls that overlap on the GPU (different streams or threads) race.  The
 * first call on a device looks up the scratch address for that device; make
 * that first call before any stream capture, and do not call the entry point
 * on a device after a cudaDeviceReset of it.  The call synchronises the
 * stream (it reads the checks and the spike count back to the host).
 * *spikes_out receives the number of spikes emitted (may be NULL); stream
 * may be NULL. */
BG_API int bg_delay_group_run_noalloc(
    int64_t n, int nvar, double *S, const double *A, const double *C,
    int thr_var, double thr_val, int reset_var, double reset_val, int nconn,
    const int64_t *src_origin, const int64_t *src_n, const int *tgt_var,
    const int64_t *const *rowptr, const int32_t *const *cols,
    const uint8_t *const *delays, const double *weight,
    const int32_t *ring_depth, int64_t nsteps, void *stream,
    int64_t *spikes_out);
/* Size in bytes of the allocation-free entry point's scratch array. */
BG_API int bg_noalloc_scratch_bytes(int64_t *bytes);
/* steps run, kernel launches issued, device milliseconds of the last run. */
BG_API int bg_net_stats(bg_net *net, int64_t *steps, int64_t *launches,
                 double *last_run_ms);

/* ---- batched model fitting ------------------------------------------------
 * Replaces GPUModelFitting (library/modelfitting/gpu_modelfitting.py:
 * 202-401) and the fitness loop of ModelFitting (modelfitting.py:26-227).
 * A handle holds ns independent simulations (particles x targets x slices)
 * of one generated model; each has its own input row, length, target train,
 * spike delay and refractory period.  The kernel follows the reference's
 * runsim template (gpu_modelfitting.py:39-156).
 *
 * The model is C code over the state registers s_<name>, the input I_in
 * and the time t (bg_fit_model below).  precision 32 or 64 selects the
 * scalar type; delta_steps = rint(delta/dt); exclusive = 1 for the
 * 'exclusive' coincidence algorithm, 0 for 'inclusive'.  The kernel is
 * compiled by NVRTC for sm_100a; BG_ECOMPILE carries the compiler log in
 * bg_last_error. */
typedef struct bg_fit_model {
    const char *state_names;      /* state rows in storage order, comma-separated */
    const char *update_code;      /* statements of one step                       */
    const char *update_fast_code; /* the same step with divisions by run-constant
                                     divisors written bg_div_fast(a, b, y, thr,
                                     suspect); NULL/"" = update_code            */
    const char *threshold_code;   /* bool expression                              */
    const char *reset_code;       /* statements run every step; the bool reset_on
                                     is true on a spike and while refractory, so
                                     write x = reset_on ? v : x                   */
    const char *aux_decl;         /* extra Model members (reciprocals), or NULL   */
    const char *setup_code;       /* statements run once after the state is
                                     loaded (may set bool bg_exact), or NULL      */
} bg_fit_model;

/* A group's model as generated C (the snippets of bg_fit_model over the
 * registers s_<name>, names in the group's variable order): any of the
 * update of one step, the threshold condition and the reset statements
 * (selects on `reset_on`) replaces the built-in linear update, threshold
 * kind and reset kind of that group.  The group's head kernel is compiled
 * with them by NVRTC at bg_net_prepare.  Replaces the state updater,
 * StringThreshold and StringReset of a nonlinear NeuronGroup
 * (stateupdater.py:70-172, threshold.py:203-242, reset.py:155-217). */
BG_API int bg_group_set_model(bg_net *net, int32_t gid, const bg_fit_model *model);
/* Compile only (no device needed); the log is copied to `log`. */
BG_API int bg_fit_compile_check(int precision, const bg_fit_model *model, double dt,
                                int delta_steps, int exclusive, char *log, int64_t log_len);
/* GPUModelFitting.__init__ (gpu_modelfitting.py:266-331). */
BG_API int bg_fit_create(bg_fit **out, int device, int precision, const bg_fit_model *model,
                         double dt, int delta_steps, int exclusive);
BG_API int bg_fit_destroy(bg_fit *h);
/* I (the reference's I_arr): all input traces concatenated; converted to
 * the scalar type on upload (gpu_modelfitting.py:353). */
BG_API int bg_fit_set_input(bg_fit *h, const double *I, int64_t n);
/* All target trains concatenated, in steps (rint(t/dt)), each framed by a
 * leading sentinel before 0 and a trailing one after its simulation ends
 * (gpu_modelfitting.py:255-263, 356). */
BG_API int bg_fit_set_targets(bg_fit *h, const int32_t *spiketimes, int64_t n);
/* reinit_vars (gpu_modelfitting.py:333-379): S0 is the initial state
 * [nstate][nsims]; simulation i reads input[I_offset[i] + T] for
 * T < nsteps[i] and its train spiketimes[spk_offset[i] .. spk_end[i]);
 * delay/refractory in steps (NULL = 0); spikes before step `onset` are not
 * counted.  Resets every simulation to S0. */
BG_API int bg_fit_set_sims(bg_fit *h, int64_t nsims, const double *S0,
                           const int64_t *I_offset, const int32_t *nsteps,
                           const int64_t *spk_offset, const int64_t *spk_end,
                           const int32_t *delay, const int32_t *refractory,
                           int32_t onset);
/* Record the first `cap` spike steps of every simulation (0 = off). */
BG_API int bg_fit_set_record(bg_fit *h, int32_t cap);
/* State back to S0, counters and train pointers to the start. */
BG_API int bg_fit_reinit(bg_fit *h);
/* launch (gpu_modelfitting.py:381-393): steps [Tstart, min(Tend, nsteps[i]))
 * of every simulation, continuing from the current state. */
BG_API int bg_fit_run(bg_fit *h, int32_t Tstart, int32_t Tend);
/* coincidence_count / spike_count (gpu_modelfitting.py:395-401) and,
 * optionally, the state [nstate][nsims] as doubles.  NULL skips an output. */
BG_API int bg_fit_read(bg_fit *h, int32_t *coinc, int32_t *nspikes, double *state);
/* Recorded spikes: counts[nsims] (may exceed cap), steps[nsims][cap]. */
BG_API int bg_fit_read_spikes(bg_fit *h, int32_t *counts, int32_t *steps);
/* Features of every simulation's recorded spikes and its input, out
 * [nsims][64] (the learned proposal's input): 32-bin log-ISI histogram over
 * [1 ms, 2 s), firing rate (statistics.py:15-21), CV (statistics.py:23-30)
 * and a 30-bin spike-triggered average of the input in nA over 30 ms
 * (statistics.py:125-153).  Needs bg_fit_set_record. */
BG_API int bg_fit_features(bg_fit *h, float *out);
/* The same features for given trains: steps[offsets[i] .. offsets[i+1]) of
 * train i (clock steps), its input I[I_offset[i] + T] (amperes); out
 * [ntrains][64].  Every spike's window must lie inside the input. */
BG_API int bg_spike_features(int device, int64_t ntrains, const int32_t *steps,
                             const int64_t *offsets, const double *I, const int64_t *I_offset,
                             int64_t ninput, double dt, float *out);
/* The same features for given trains whose inputs are already in the
 * handle: train i's input starts at I_offset[i] of the handle's input array;
 * gpu_ms (nullable) receives the device time including the copies. */
BG_API int bg_fit_train_features(bg_fit *h, int64_t ntrains, const int32_t *steps,
                                 const int64_t *offsets, const int64_t *I_offset, float *out,
                                 float *gpu_ms);
/* Gamma factor inputs (ModelFitting.prepare_data, modelfitting.py:117-173):
 * nparticles x slices = nsims (simulation i is particle i % nparticles),
 * per particle the target train's length and rate (firing_rate), delta in
 * seconds. */
BG_API int bg_fit_set_gamma(bg_fit *h, int64_t nparticles, int32_t slices,
                            const int32_t *target_length, const double *target_rate,
                            double delta);
/* Fitted parameter d writes state row dim_var[d]; -1 = spike delay,
 * -2 = refractory period (both rint(x/dt) steps). */
BG_API int bg_fit_set_params(bg_fit *h, int32_t ndim, const int32_t *dim_var);
/* ModelFitting.evaluate (modelfitting.py:175-227): X is [ndim][nparticles];
 * resets, simulates every particle over its full length and writes the
 * gamma factor (FP64, get_gamma_factor, statistics.py:236-240). */
BG_API int bg_fit_evaluate(bg_fit *h, const double *X, double *gamma_out);
/* Launch shape of the simulation kernel: resident 128-thread blocks per SM
 * (1..16, default 2).  Results never depend on it. */
BG_API int bg_fit_set_blocks_per_sm(bg_fit *h, int32_t blocks_per_sm);
/* Time one full run per candidate launch shape (1, 2, 3, 4, 6, 8 blocks per
 * SM) with parameters X ([ndim][nparticles], NULL = the initial state), keep
 * the fastest; ms_out[6] (nullable) receives each candidate's time.  Leaves
 * the simulations reset with X. */
BG_API int bg_fit_autotune(bg_fit *h, const double *X, int32_t *blocks_per_sm, float *ms_out);
/* Grouped particle swarm on the device (particle_swarm.py:6-111): groups of
 * group_size consecutive particles optimise independently (one target
 * each); X0 [ndim][nparticles] is clipped into [xmin, xmax]. */
BG_API int bg_fit_pso_init(bg_fit *h, int32_t group_size, const double *X0,
                           const double *xmin, const double *xmax, double omega,
                           double c1, double c2, uint64_t seed);
/* Evaluate the current positions and fold them into the local and group
 * bests without moving (the initial swarm's scores; the reference's loop
 * moves before its first evaluation, particle_swarm.py:65-84). */
BG_API int bg_fit_pso_evaluate_initial(bg_fit *h);
/* `iterations` swarm iterations (move, evaluate, best updates) queued
 * without host synchronisation; trace [iterations][ngroups] receives the
 * group best fitness after each, iter_ms the GPU time of each (NULL = off). */
BG_API int bg_fit_pso_run(bg_fit *h, int32_t iterations, double *trace, float *iter_ms);
/* Group bests: X_gbest [ndim][ngroups], fit_gbest [ngroups]. */
BG_API int bg_fit_pso_best(bg_fit *h, double *X_gbest, double *fit_gbest);
/* Swarm state: X, V, X_lbest [ndim][nparticles], fit_lbest [nparticles]. */
BG_API int bg_fit_pso_state(bg_fit *h, double *X, double *V, double *X_lbest,
                            double *fit_lbest);
/* out[0..n): last simulation launch (GPU ms), launches, neuron-steps of one
 * full run, longest simulation (steps), last whole evaluation (GPU ms). */
BG_API int bg_fit_stats(bg_fit *h, double *out, int n);

/* ---- learned proposal network ----------------------------------------------
 * A 4-layer MLP (64 -> 512 -> 512 -> 512 -> 2*ydim, ReLU) whose output is a
 * diagonal Gaussian (ydim means, ydim log standard deviations) over the
 * normalised fitted parameters; it proposes starting points for the swarm
 * (no reference counterpart: the reference starts its optimisers from
 * uniform draws, modelfitting.py:479-516).  Matrix products run on the
 * tensor cores (tcgen05, BF16 operands, FP32 accumulation); the loss is the
 * Gaussian negative log-likelihood, the optimiser Adam. */
typedef struct bg_mlp bg_mlp;
BG_API int bg_mlp_create(bg_mlp **out, int device, int ydim);
BG_API int bg_mlp_destroy(bg_mlp *h);
/* Layer l (0..3) parameters, fp32 row-major W[rows][cols], b[rows]; rows =
 * 512, 512, 512, 64 (the output layer padded with zero rows), cols = 64,
 * 512, 512, 512.  Setting resets the optimiser state of the layer. */
BG_API int bg_mlp_set_params(bg_mlp *h, int layer, const float *W, const float *b);
BG_API int bg_mlp_get_params(bg_mlp *h, int layer, float *W, float *b);
/* out[n][2*ydim] = network(X[n][64]). */
BG_API int bg_mlp_forward(bg_mlp *h, const float *X, int64_t n, float *out);
/* Device time (ms) of the last bg_mlp_forward, copies included. */
BG_API int bg_mlp_last_forward_ms(bg_mlp *h, float *ms);
/* Training set: X[n][64] features, Y[n][ydim] targets (already normalised). */
BG_API int bg_mlp_set_data(bg_mlp *h, const float *X, const float *Y, int64_t n);
/* `epochs` passes of mini-batch Adam (batch a multiple of 512); the batch
 * order of each epoch comes from Philox keyed (seed, epoch).  epoch_loss
 * [epochs] and gpu_ms (nullable) report the mean loss and device time. */
BG_API int bg_mlp_train(bg_mlp *h, int epochs, int batch, float lr, uint64_t seed,
                        float *epoch_loss, float *gpu_ms);
/* Data-parallel training (one bg_mlp per rank, the same training set and
 * seed on every rank).  bg_mlp_epoch_order draws the epoch's row order
 * (the order bg_mlp_train uses).  bg_mlp_step_gradients runs forward and
 * backward on rows [row0, row0 + batch) of that order (row0 a multiple of
 * batch; batch a multiple of 512) and returns the mean loss and the flat
 * FP32 gradient of every tensor (W0, b0, W1, b1, ... row-major) as a device
 * pointer into the handle (*ngrad floats, valid until the next call), for
 * the caller's all-reduce.  bg_mlp_apply_gradients takes one Adam step from
 * a device gradient of that layout multiplied by `scale` (1/ranks after a
 * summing all-reduce).  With one rank these steps equal bg_mlp_train's bit
 * for bit. */
BG_API int bg_mlp_epoch_order(bg_mlp *h, uint64_t seed, int64_t epoch);
BG_API int bg_mlp_step_gradients(bg_mlp *h, int batch, int64_t row0, float *loss, void **grad, int64_t *ngrad);
BG_API int bg_mlp_apply_gradients(bg_mlp *h, const void *grad, float lr, float scale);
/* Loss and gradients on the first `batch` training rows without an update
 * (dW[l] [rows][cols], db[l] [rows]; entries may be NULL). */
BG_API int bg_mlp_gradients(bg_mlp *h, int batch, float *loss, float *const *dW,
                            float *const *db);
/* C[M][N] = A[M][K] . B[N][K]^T on device buffers: A, B bf16 row-major, C
 * fp32, K a multiple of 64; runs on `stream` (a cudaStream_t, NULL =
 * default) and returns when done. */
BG_API int bg_gemm_bf16(int64_t M, int64_t N, int64_t K, const void *A, const void *B,
                        float *C, void *stream);

/* ---- batches of independent networks ----------------------------------
 * Many small networks simulated side by side in one kernel launch, one
 * thread block per network (no counterpart in the reference, which runs one
 * Network per process: network.py:403-430 is the step each block repeats).
 * A network qualifies when it is what the persistent kernel runs -- one
 * linear group of 1-4 variables and at most 4096 neurons, no
 * refractoriness, at most 2 connections onto the group that are zero-delay
 * shared-weight Connections or shared-weight DelayConnections, at most 2
 * undelayed spike monitors and 4 StateMonitors, no STDP or Synapses -- and
 * the networks of a batch share the device, the precision and the number of
 * state variables.  Each network keeps its own parameters, connectivity,
 * weights, thresholds and durations; its results are those of bg_net_run on
 * it alone, bit for bit: its state, rings, counters and monitor records
 * advance as if it had.  The networks (prepared by this call if needed) must
 * outlive the batch and are not run alone while a batch call is in flight. */
typedef struct bg_batch bg_batch;
BG_API int bg_batch_create(bg_net *const *nets, int32_t count, bg_batch **out);
BG_API int bg_batch_free(bg_batch *b);
/* Runs network i for nsteps[i] steps (uneven durations allowed); cs0[i] is
 * its clock step at the start (as for bg_net_run).  Monitor records are
 * drained into the networks' host records between launches. */
BG_API int bg_batch_run(bg_batch *b, const int64_t *nsteps, const int64_t *cs0);
/* Block shape (an index into the kernel's shapes: 128x4, 256x4, 512x4,
 * 512x8, 1024x4, 768x6 threads x neurons per thread; the block must hold
 * the largest network) and lanes per spike row in the push (4, 8, 16, 32). */
BG_API int bg_batch_set_shape(bg_batch *b, int32_t shape, int32_t lanes);
BG_API int bg_batch_get_shape(bg_batch *b, int32_t *shape, int32_t *threads, int32_t *npt, int32_t *lanes);
/* Times `steps` steps of every valid (shape, lanes) pair on the batch
 * without changing any network (state, rings and records are left as they
 * were) and keeps the fastest; best_ms (nullable) is its time. */
BG_API int bg_batch_autotune(bg_batch *b, int32_t steps, double *best_ms);
/* Kernel launches so far and device time (ms) of the last bg_batch_run. */
BG_API int bg_batch_stats(bg_batch *b, int64_t *launches, double *ms);

#ifdef __cplusplus
}
#endif
#endif /* BRIAN_B200_H */
