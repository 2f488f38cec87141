/*
 * tasep.h - C ABI of the B200 TASEP master-equation integrator
 *           (libtasep_cuda.so, sm_100a).
 *
 * The reference (KilianPiochUBT/TASEP) has no plugin or FFI layer: its hot
 * path is the step loop of bin/masterEquation calling the C functions of
 * src/lib/solv.c and src/lib/matgen.c.  Each entry point below names the
 * reference code it replaces.  Plain C types only; no CUDA or torch types in
 * any signature (streams are passed as void*, i.e. a cudaStream_t).
 *
 * State convention (as in the reference): N = 2^n states, bit b of a state
 * index is lattice site n-1-b (site 0 = entry site).  Rates r[0..n]:
 * r[0] = alpha (entry into site 0), r[j] = hop rate site j-1 -> j
 * (j = 1..n-1), r[n] = beta (exit from site n-1)
 * (reference src/masterEquation.c:457-460, src/lib/matgen.c:29-67).
 *
 * Errors: every call returns a tasep_status; tasep_last_error() gives a
 * thread-local message.  Nothing prints and nothing calls exit() (the
 * reference exits with -1 through err_exit, src/lib/io.c:13-19).
 */
#ifndef TASEP_H
#define TASEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TASEP_ABI_VERSION 1
#define TASEP_MAX_N 33

typedef enum {
    TASEP_OK = 0,
    TASEP_ERR_INVALID = 1,     /* bad argument or call order */
    TASEP_ERR_NOMEM = 2,       /* device allocation failed */
    TASEP_ERR_CUDA = 3,        /* CUDA runtime error */
    TASEP_ERR_NODEV = 4,       /* no usable CUDA device */
    TASEP_ERR_TIMEOUT = 5,     /* a bounded device-side wait expired */
    TASEP_ERR_UNSUPPORTED = 6  /* combination not implemented */
} tasep_status;

/* Integrators.
 * REF: the reference's step, bit for bit.  Its four stage calls all gather
 *      from the state (src/masterEquation.c:630-636, src/lib/solv.c:13), so a
 *      step is x += (k+2k+2k+k)/6 with k = h*M*x (one generator application).
 * RK4: classical fourth-order Runge-Kutta (four generator applications). */
enum { TASEP_INTEGRATOR_REF = 0, TASEP_INTEGRATOR_RK4 = 1 };

/* FP64: every vector in double.  MIXED (RK4 with constant rates only): the
 * state, the convergence norm and the final update stay in double; the three
 * stage vectors and their generator gathers are float. */
enum { TASEP_PRECISION_FP64 = 0, TASEP_PRECISION_MIXED = 1 };

/* Initial states: UNIFORM = 2^-n everywhere (src/masterEquation.c:402-409),
 * EMPTY = empty lattice, P(state 0) = 1. */
enum { TASEP_INIT_UNIFORM = 0, TASEP_INIT_EMPTY = 1 };

/* Time-variant rate functions (src/lib/matvec.c:44-68):
 * SIN: A*sin(w*t+phi)+c, COS: A*cos(w*t+phi)+c, LIN: A*t+c; clamped at 0. */
enum { TASEP_FUN_SIN = 0, TASEP_FUN_COS = 1, TASEP_FUN_LIN = 2 };

typedef struct tasep_meq tasep_meq; /* opaque; owns all device buffers */

typedef struct {
    int n;          /* lattice length, 1..TASEP_MAX_N */
    int integrator; /* TASEP_INTEGRATOR_* */
    int precision;  /* TASEP_PRECISION_* */
    int device;     /* CUDA device ordinal; -1 = the current device */
    void *stream;   /* cudaStream_t to launch on; NULL = the handle makes one */
} tasep_meq_config;

typedef struct {
    double t0;       /* start time; time-variant rates are evaluated from it */
    double h;        /* step size, h = (T - t)/steps in the reference (:586) */
    uint64_t steps;  /* maximum number of steps (-s) */
    double stop_tol; /* exit test: L1 norm of the increment < stop_tol*h ...  */
    int stop_count;  /* ... on more than stop_count consecutive steps          */
    int exit_rule;   /* 1 = apply the rule (src/masterEquation.c:670-679);
                        0 = run every step (the reference time-var loop) */
} tasep_run_config;

typedef struct {
    uint64_t steps_done;    /* loop iterations executed */
    uint64_t steps_at_stop; /* index of the last qualifying step */
    int early_stop;         /* qualifying steps in a row at the end */
    int converged;          /* 1 if the loop ended through the exit rule */
    double last_checksum;   /* L1 norm of the last increment */
    double t_end;           /* t0 + h added steps_done times */
} tasep_run_result;

/* ---- handle lifecycle --------------------------------------------------
 * Replaces the allocations of src/masterEquation.c:354-505 (x, x1, k1..k4)
 * and, for -f, :586-616 (the CSR arrays): the generator is never stored. */
tasep_status tasep_meq_create(const tasep_meq_config *cfg, tasep_meq **out);
tasep_status tasep_meq_destroy(tasep_meq *m);

/* Rates r[0..n] (n+1 doubles).  Replaces the -i file / --alpha --beta
 * --gamma set-up of src/masterEquation.c:432-461. */
tasep_status tasep_meq_set_rates(tasep_meq *m, const double *rates);

/* Time-variant rates, n+1 entries each; evaluated on the device at every
 * stage time.  Replaces the per-step timeVariantProbs call
 * (src/masterEquation.c:886, src/lib/matvec.c:44-68).  REF evaluates all
 * of a step at its start time t, as the reference does; RK4 at t, t+h/2,
 * t+h/2, t+h. */
tasep_status tasep_meq_set_timevar(tasep_meq *m, const int *type, const double *amplitude,
                                   const double *period, const double *offset,
                                   const double *constant);
tasep_status tasep_meq_clear_timevar(tasep_meq *m);

/* Initial state.  Replaces src/masterEquation.c:402-409. */
tasep_status tasep_meq_init(tasep_meq *m, int kind);
/* Initial state from a host vector of 2^n doubles. */
tasep_status tasep_meq_load(tasep_meq *m, const double *host_x);

/* The integration loop with its exit rule.  Replaces the step loops of
 * src/masterEquation.c:628-682 (-f), :883-921 (time-var) and :929-982 (per
 * row), including rk4_step / rk4_step_reduced / gen_meq_row
 * (src/lib/solv.c:3-135).  Blocks until the loop ends. */
tasep_status tasep_meq_run(tasep_meq *m, const tasep_run_config *rc, tasep_run_result *res);

/* The same loop with snapshots, for the animation branch of the reference
 * (-a R, src/masterEquation.c:646-666, :900-918, :949-966): after every step
 * whose 0-based index is a multiple of `every`, and before that step's exit
 * test takes effect, the loop calls fn(m, step, t, user) with the state of
 * that step current on the device (t = time after the step).  The hook may
 * call tasep_meq_observables and tasep_meq_store on the handle; it must not
 * run or change the state. */
typedef void (*tasep_snapshot_fn)(tasep_meq *m, uint64_t step, double t, void *user);
tasep_status tasep_meq_run_snapshots(tasep_meq *m, const tasep_run_config *rc, uint64_t every,
                                     tasep_snapshot_fn fn, void *user, tasep_run_result *res);

/* The same snapshots without stopping the integration: each snapshot's
 * observables (and, when with_probs is set, a copy of its 2^n probabilities)
 * are taken on the device in stream order into one of two slots and copied to
 * pinned host memory on a second stream while the steps go on; the loop reads
 * its exit state one chunk behind the device.  fn gets, in step order, host
 * pointers that are valid during the call only: rho[n] (bit order), cov[n*n]
 * and mul[n*n] (site order), window4[(n-3)*16] (NULL for n < 4), as from
 * tasep_meq_observables, and probs[2^n] (NULL unless with_probs).  Snapshots
 * whose step the loop did not reach are not delivered.  fn must not call the
 * handle.  Result and final state as tasep_meq_run_snapshots. */
typedef void (*tasep_stream_fn)(tasep_meq *m, uint64_t step, double t, const double *rho, const double *cov,
                                const double *mul, const double *window4, const double *probs, void *user);
tasep_status tasep_meq_run_stream(tasep_meq *m, const tasep_run_config *rc, uint64_t every, int with_probs,
                                  tasep_stream_fn fn, void *user, tasep_run_result *res);

/* Enqueues `steps` steps on the handle's stream without the exit rule and
 * without waiting (benchmarks, CUDA-graph capture); t advances by h. */
tasep_status tasep_meq_enqueue_steps(tasep_meq *m, double t0, double h, uint64_t steps);
tasep_status tasep_meq_synchronize(tasep_meq *m);

/* Copies probabilities [offset, offset+count) of the state to host memory. */
tasep_status tasep_meq_store(const tasep_meq *m, double *host_x, uint64_t offset, uint64_t count);

/* Observables of the current state, each output optional (NULL skips it):
 *   rho[b]   - per-bit densities, bit order (condense / exp_val_eval,
 *              src/lib/matvec.c:10-42, :70-91); site j is rho[n-1-j];
 *   cov      - n*n covariance in site order, as src/masterEquation.c:1121-1139;
 *   mul      - n*n y_k*y_i + cov, as src/masterEquation.c:1289-1302;
 *   window4  - (n-3)*16 marginals of the 4-bit windows: window4[p*16+q] =
 *              sum over states whose bits p..p+3 equal q (feeds the window
 *              observables of src/masterEquation.c:32-143, :1422-1539);
 *   mass     - sum of all probabilities. */
tasep_status tasep_meq_observables(tasep_meq *m, double *rho, double *cov, double *mul,
                                   double *window4, double *mass);

/* cudaStream_t the handle launches on. */
void *tasep_meq_stream(const tasep_meq *m);

/* L2 cache policy of the generator sweep (no counterpart in the reference,
 * whose CSR product has no cache control).  A state's hop partners lie
 * 2^k states ahead; the sweep reads a tile first as a partner of an earlier
 * tile and last as its own tile.  near_bits: partner tiles of hops across
 * the lowest near_bits tile-index bits are read with L2 evict_last (they come
 * back as own tiles while L2 still holds them); farther partners follow
 * TASEP_L2_FAR_FIRST.  flags: TASEP_L2_OWN_FIRST reads own tiles evict_first,
 * TASEP_L2_DEMOTE lowers a tile's lines to evict_normal once its own read has
 * landed, TASEP_L2_FAR_FIRST reads far partners evict_first.  Only speed
 * depends on it, never the results; the default is the fastest measured. */
enum { TASEP_L2_OWN_FIRST = 1, TASEP_L2_DEMOTE = 2, TASEP_L2_FAR_FIRST = 4 };
tasep_status tasep_meq_set_cache_policy(tasep_meq *m, int near_bits, int flags);
tasep_status tasep_meq_get_cache_policy(const tasep_meq *m, int *near_bits, int *flags);

/* Per-kernel device time (CUDA events around each launch on the handle's
 * stream).  enable=1 starts recording and clears the totals. */
tasep_status tasep_meq_profile(tasep_meq *m, int enable);
/* names[i] (static strings), total milliseconds and launch counts of up to
 * `cap` kernels; returns the number of kernels in *count. */
tasep_status tasep_meq_profile_read(tasep_meq *m, const char **names, double *ms,
                                    uint64_t *launches, int cap, int *count);

/* ---- batched parameter sweeps --------------------------------------------
 * nsys independent systems of the same length n (kTileBits < n <= 24), each
 * with its own n+1 rates, integrated with classical RK4 (FP64 or MIXED) until each meets the exit rule on its own.  The reference has no
 * batching; this replaces running bin/masterEquation once per rate vector.
 * Converged systems retire: later steps skip them.  Steps run as replays of a
 * CUDA graph of a few steps; the sweep schedule (tiles interleaved over the
 * SMs, or whole systems per SM) is chosen by timing both. */
typedef struct tasep_batch tasep_batch;
tasep_status tasep_batch_create(int n, int nsys, int precision, int device, void *stream, tasep_batch **out);
tasep_status tasep_batch_destroy(tasep_batch *b);
/* rates: nsys*(n+1) doubles, system-major. */
tasep_status tasep_batch_set_rates(tasep_batch *b, const double *rates);
tasep_status tasep_batch_init(tasep_batch *b, int kind);
/* host_x: nsys*2^n doubles. */
tasep_status tasep_batch_load(tasep_batch *b, const double *host_x);
/* res: nsys results (NULL skips them).  schedule: -1 = choose, 0 = tiles
 * interleaved over the SMs, 1 = whole systems per SM, 2 = cluster-resident:
 * each system held entirely in the shared memory of one thread-block cluster
 * (2^(n-13) .. 2^(n-11) CTAs, n <= 17) and run to its exit rule there, with no
 * device-memory traffic between steps; its shape (states per CTA) is chosen
 * by timing the feasible shapes on a short run of copies of the first
 * systems.  -1 times schedules 0 and 1 and keeps the faster (re-timed each
 * time the number of running systems halves).  *schedule_used (may be NULL)
 * reports the choice. */
tasep_status tasep_batch_run(tasep_batch *b, const tasep_run_config *rc, int schedule, tasep_run_result *res,
                             int *schedule_used);
/* The configuration the last tasep_batch_run used: schedule, states per CTA
 * and CTAs per system (0 for schedules 0 and 1). */
tasep_status tasep_batch_last_config(const tasep_batch *b, int *schedule, int *states_per_cta,
                                     int *ctas_per_system);
tasep_status tasep_batch_store(const tasep_batch *b, int sys, double *host_x);
/* Per-bit densities of every system: nsys*n doubles (bit order). */
tasep_status tasep_batch_densities(tasep_batch *b, double *rho);

/* ---- learned warm start ------------------------------------------------------
 * No counterpart in the reference.  A per-site network (TASEP_MLP_IN inputs,
 * three hidden layers of 64 tanh units, 2 outputs: density and nearest-
 * neighbour covariance) trained on the GPU with the library's own forward
 * (tcgen05 tensor cores), backward and Adam kernels (BF16 weights, FP32
 * accumulation), and a device-side builder of the pair-Markov initial
 * measure from predicted profiles.  A tensor-core wait that expires returns
 * TASEP_ERR_TIMEOUT. */
#define TASEP_MLP_IN 16
#define TASEP_MLP_OUT 2
#define TASEP_MLP_PARAMS 9538
typedef struct tasep_mlp tasep_mlp;
/* Weights initialised (Glorot-uniform) from `seed`. */
tasep_status tasep_mlp_create(int device, uint64_t seed, tasep_mlp **out);
tasep_status tasep_mlp_destroy(tasep_mlp *m);
tasep_status tasep_mlp_set_params(tasep_mlp *m, const float *params);
tasep_status tasep_mlp_get_params(tasep_mlp *m, float *params);
/* Loss sum_s sum_o w[o]*(y_so - t_so)^2 / n and its gradient (host buffers;
 * x: n*TASEP_MLP_IN, t: n*TASEP_MLP_OUT). */
tasep_status tasep_mlp_loss_grad(tasep_mlp *m, const float *x, const float *t, int n, const float *out_weights,
                                 float *loss, float *grad);
/* Mini-batch Adam on (x, t); loss_per_epoch (may be NULL) gets the mean
 * training loss of each epoch.  The sample order is shuffled from `seed`. */
tasep_status tasep_mlp_train(tasep_mlp *m, const float *x, const float *t, int n, const float *out_weights,
                             int epochs, int batch, float lr, uint64_t seed, float *loss_per_epoch);
tasep_status tasep_mlp_predict(tasep_mlp *m, const float *x, int n, float *y);
/* The network's mean-field input feature, on the host: for each of `count`
 * rate vectors (n+1 doubles each, consecutive), explicit Euler on
 * d rho_i/dt = J_i - J_(i+1) (J_0 = alpha (1 - rho_0), J_i = r_i rho_(i-1)
 * (1 - rho_i), J_n = beta rho_(n-1)) from rho = 1/2 with dt = 1/(4 max rate)
 * for `steps` steps, then clipped to [1e-6, 1 - 1e-6]; rho gets count*n
 * doubles in site order.  Every operation is the one the Python driver's
 * numpy form performs, in the same order, so the results are equal bit for
 * bit.  Needs no device. */
tasep_status tasep_mean_field_profile(int n, int count, int steps, const double *rates, double *rho);
/* Initial state P(tau) = P(tau_0) prod_j P(tau_(j+1)|tau_j) from densities
 * rho[j] (site order, n values) and nearest-neighbour covariances cov[j] =
 * <tau_j tau_(j+1)> - rho_j rho_(j+1) (n-1 values).  Covariances are clipped to
 * the range a joint distribution allows; a density outside (0,1) returns
 * TASEP_ERR_INVALID and leaves the state unchanged (the caller falls back to
 * the empty lattice). */
tasep_status tasep_meq_init_pair_markov(tasep_meq *m, const double *rho, const double *cov);

/* ---- device-pointer operators ------------------------------------------
 * For callers that keep their own device vectors.  x, y: 2^n doubles in
 * device memory; rates: n+1 doubles in host memory; stream may be NULL. */

/* y = M x, each row summed in the reference's entry order (entry, diagonal,
 * exit, hops by ascending bit) with separate multiply and add, so y equals
 * the CSR product of gencrs + rk4_step's gather bit for bit
 * (src/lib/matgen.c:7-74, src/lib/solv.c:9-13). */
tasep_status tasep_apply_device(int n, const double *rates, const double *x, double *y,
                                void *stream);

/* One reference step x_out = x + (k+2k+2k+k)/6, k = h*M*x, and its L1 norm
 * written to *checksum_host (src/masterEquation.c:628-642).  x and x_out must
 * not overlap.  Scratch for the norm is allocated on the first call per
 * device and reused. */
tasep_status tasep_step_ref_device(int n, const double *rates, double h, const double *x,
                                   double *x_out, double *checksum_host, void *stream);

/* The same reference step as tasep_step_ref_device, for callers that must not
 * allocate device memory: a host program whose device memory is all handed
 * out by its own pool allocator (and which forbids plugins from calling
 * cudaMalloc, since a raw allocation fragments or escapes that pool), or a
 * loop that cannot afford the device-wide synchronisation cudaMalloc and
 * cudaFree may cause.  No counterpart in the reference.
 *
 * It allocates nothing: the scratch for the L1 norm (one partial sum per CTA,
 * a ticket counter and the step's status) is a fixed 8.3 KB array in the
 * library's device image, which every GPU that loads the library holds until
 * the process exits.  It holds at most 1024 per-CTA partial sums; the step
 * launches one CTA per SM, and a device with more SMs than that is rejected
 * with TASEP_ERR_INVALID.  The first call on a device looks up that array's
 * device address (and the device's SM count); make that first call before any
 * stream capture.  The caller passes every input and output: x and x_out
 * (2^n doubles each, device memory, not overlapping), rates (n+1 doubles,
 * host memory) and checksum_dev (one double in device memory that receives the
 * step's L1 norm; NULL skips it).  Nothing is synchronised; results are ready
 * when `stream` reaches them.  The step's status stays in the shared array,
 * so a bounded device wait that expired (TASEP_ERR_TIMEOUT for the other
 * entry points) shows here as a NaN in *checksum_dev: pass checksum_dev to
 * learn of it; x_out is then invalid.  All calls share the one array, and each call
 * clears its counter and status first, so calls that overlap on the GPU (on
 * different streams or from different threads without ordering) race and
 * must not be issued. */
tasep_status tasep_step_ref_device_noalloc(int n, const double *rates, double h, const double *x,
                                           double *x_out, double *checksum_dev, void *stream);

/* ---- misc ---------------------------------------------------------------- */
const char *tasep_last_error(void);

/* Test hook for the error path of the bounded device waits (no counterpart in
 * the reference, which has no device code).  Every later launch of the
 * generator sweep (n > 11) gives up a wait after wait_limit_ns (0 = the
 * default, about 2 s) and, if skip_partner_copy >= 0, the first CTA leaves
 * out that partner copy (counted from 0 within the launch), so a consumer
 * wait on it expires.  The kernel then flags the error, lets the copies it
 * did issue land and returns: no GPU fault, no hang.  Such steps report
 * TASEP_ERR_TIMEOUT and their results are invalid.  (0, -1) switches the
 * hook off; it is process-wide and not meant for concurrent use. */
tasep_status tasep_test_inject_wait_expiry(uint64_t wait_limit_ns, int skip_partner_copy);
/* Test entry: out[i] = in[i] / 6 as the REF and time-variant steps compute it
 * on the device (correctly rounded, without a division instruction sequence),
 * for checking against IEEE division on the host. */
tasep_status tasep_test_div6(const double *host_in, double *host_out, uint64_t count);
int tasep_abi_version(void);
/* Bytes of device memory a handle with this configuration allocates. */
uint64_t tasep_meq_footprint(int n, int integrator, int precision, int timevar);

#ifdef __cplusplus
}
#endif
#endif
