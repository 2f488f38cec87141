/*
 * me_main.c - drop-in replacement for the reference's bin/masterEquation.
 *
 * Same command line (src/masterEquation.h:45-59, src/masterEquation.c:239-336),
 * prompts for missing values (:342-429), rate set-up (:357-461), time-variant
 * rate files (:700-875), step size h = (T - t)/steps in long double (:586), exit
 * rule (:670-679), console report (:993-1017) and output files (:1019-1539).
 * The integration runs on the GPU through libtasep_cuda.so (include/tasep.h).
 *
 * Options added here (all optional):
 *   --integrator ref|rk4    ref (default): the reference's step bit for bit;
 *                           rk4: classical fourth-order Runge-Kutta
 *   --precision fp64|mixed  mixed: float stage vectors (rk4, constant rates)
 *   --init uniform|empty|learned
 *                           initial state (default uniform, as the reference);
 *                           learned: pair-Markov measure predicted by the
 *                           shipped warm-start network (empty if infeasible)
 *   --init-params <path>    network parameters for --init learned (default:
 *                           data/warmstart_params.npy beside bin/)
 *   --init-file <path>      initial state from a probability file in this
 *                           program's output format
 *   --stop-tol <x>          exit when |dP|_1 < x*h (default 1e-10)
 *   --stop-count <k>        ... on more than k consecutive steps (default 100)
 *   --device <d>            CUDA device
 */
#include <getopt.h>
#include <inttypes.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>

#include "me_host.h"
#include "tasep.h"

static void usage(const char *progname) {
    printf("Usage: %s\n-i jump rate file\n-n chain length\n-o output file name\n-t start time\n-T endtime\n"
           "-s steps\n-f fast option (accepted; the GPU path never stores the generator)\n"
           "-a space between snapshots\n"
           "--time-var sets jump rates to time variant. CAUTION: This cannot be used in combination with -f\n"
           "--function-type <char* filename with sin,cos,lin in order> sets function type of jump rate (when using "
           "<lin> --period option is not used)\n"
           "--amplitude <char* filename> reads amplitudes from given file and sets functions, when using <lin> these "
           "serve as the gradient\n"
           "--period <char* filename> reads period multipliers from given file an sets jump rate functions. (default "
           "is 1)\n"
           "--offset <char* filename> reads offsets from given file and sets jump rate functions. (default is 0)\n"
           "--constant <char* filename> reads constants from given file and sets jump rate functions. (default is "
           "0)\n"
           "--thread-num <char* number_of_threads_to_use> sets number of threads used for writing output files\n"
           "--save-select <char* shorts for what to save> shorts are: 'a': all 'e': expected values 'p': "
           "probabilities 'c': covariance Matrices 'm': multiplicative expected values\n"
           "--alpha <float> entry flow rate\n"
           "--beta <float> exit flow rate\n"
           "--gamma <float> flow rate inside lattice\n"
           "--integrator <ref|rk4> step: the reference's (default) or classical RK4\n"
           "--precision <fp64|mixed> stage vectors in double (default) or float (rk4 only)\n"
           "--init <uniform|empty|learned> initial state (default uniform); learned: warm start predicted by the "
           "shipped network\n"
           "--init-params <path> network parameters for --init learned\n"
           "--init-file <path> initial state from a probability file written by this program\n"
           "--stop-tol <float> exit when the L1 change per step stays below stop-tol*h (default 1e-10)\n"
           "--stop-count <int> ... for more than this many consecutive steps (default 100)\n"
           "--device <int> CUDA device\n"
           "-h\n",
           progname);
}

enum {
    OPT_TIMEVAR = 0, OPT_FUNTYPE, OPT_OFFSET, OPT_AMPLITUDE, OPT_PERIOD, OPT_CONSTANT, OPT_SAVESEL, OPT_THREADS,
    OPT_ALPHA, OPT_BETA, OPT_GAMMA, OPT_INTEGRATOR, OPT_PRECISION, OPT_INIT, OPT_INITFILE, OPT_STOPTOL,
    OPT_STOPCOUNT, OPT_DEVICE, OPT_INITPARAMS
};

enum { ME_INIT_LEARNED = 100 };

static struct option long_opt[] = {{"time-var", no_argument, NULL, OPT_TIMEVAR},
                                   {"function-type", required_argument, NULL, OPT_FUNTYPE},
                                   {"offset", required_argument, NULL, OPT_OFFSET},
                                   {"amplitude", required_argument, NULL, OPT_AMPLITUDE},
                                   {"period", required_argument, NULL, OPT_PERIOD},
                                   {"constant", required_argument, NULL, OPT_CONSTANT},
                                   {"save-select", required_argument, NULL, OPT_SAVESEL},
                                   {"thread-num", required_argument, NULL, OPT_THREADS},
                                   {"alpha", required_argument, NULL, OPT_ALPHA},
                                   {"beta", required_argument, NULL, OPT_BETA},
                                   {"gamma", required_argument, NULL, OPT_GAMMA},
                                   {"integrator", required_argument, NULL, OPT_INTEGRATOR},
                                   {"precision", required_argument, NULL, OPT_PRECISION},
                                   {"init", required_argument, NULL, OPT_INIT},
                                   {"init-file", required_argument, NULL, OPT_INITFILE},
                                   {"stop-tol", required_argument, NULL, OPT_STOPTOL},
                                   {"stop-count", required_argument, NULL, OPT_STOPCOUNT},
                                   {"device", required_argument, NULL, OPT_DEVICE},
                                   {"init-params", required_argument, NULL, OPT_INITPARAMS},
                                   {NULL, 0, NULL, 0}};

static void tasep_fail(const char *what) {
    char msg[1024];
    snprintf(msg, sizeof msg, "ERROR: %s: %s", what, tasep_last_error());
    me_err_exit(msg, -1);
}

/* Reads a probability file written by this program (or the reference). */
static int read_prob_file(const char *path, int n, double *x) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    const uint64_t dim = (uint64_t)1 << n;
    char bits[64];
    double v;
    uint64_t seen = 0;
    while (fscanf(f, "%63s %lf", bits, &v) == 2) {
        if ((int)strlen(bits) != n) break;
        uint64_t i = 0;
        for (int s = 0; s < n; s++) i = (i << 1) | (uint64_t)(bits[s] == '1');
        if (i < dim) {
            x[i] = v;
            seen++;
        }
    }
    fclose(f);
    return seen == dim ? 0 : -2;
}

/* Snapshot of -a (src/masterEquation.c:646-666), streamed from the device
 * while the integration goes on: densities, covariance and product matrices,
 * and the state itself for the 4-site correlations of the timed correlation
 * file and, when probabilities are saved, for the probability snapshot file. */
static void snapshot_hook(tasep_meq *m, uint64_t step, double t, const double *rho, const double *cov,
                          const double *mul, const double *window4, const double *probs, void *user) {
    (void)m;
    (void)step;
    (void)t;
    me_snaps *s = (me_snaps *)user;
    const int n = s->n, vals = n > 5 ? n - 5 : 0;
    if (s->count == s->cap) {
        s->cap = s->cap ? 2 * s->cap : 16;
        s->obs = (me_obs *)realloc(s->obs, sizeof(me_obs) * s->cap);
        s->corr = (double *)realloc(s->corr, sizeof(double) * (vals ? vals : 1) * s->cap);
        if (s->keep_probs) s->probs = (double *)realloc(s->probs, sizeof(double) * s->dim * s->cap);
        if (!s->obs || !s->corr || (s->keep_probs && !s->probs))
            me_err_exit("ERROR: Not Enough memory to allocate animation data array", -1);
    }
    me_obs *ob = &s->obs[s->count];
    memset(ob, 0, sizeof *ob);
    ob->n = n;
    memcpy(ob->y, rho, sizeof(double) * n);
    memcpy(ob->cov, cov, sizeof(double) * n * n);
    memcpy(ob->mul, mul, sizeof(double) * n * n);
    if (window4) memcpy(ob->p4, window4, sizeof(double) * (n - 3) * 16);
    for (int k = 1; k <= vals; k++) s->corr[s->count * vals + (k - 1)] = me_state_corr(probs, n, 15, 4, n - 4 - k);
    if (s->keep_probs) memcpy(s->probs + s->count * s->dim, probs, sizeof(double) * s->dim);
    s->count++;
}

static double wall(void) {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

int main(int argc, char *argv[]) {
    int opt, option_index = 0;
    int if_found = 0, of_found = 0, t_found = 0, T_found = 0, n_found = 0, s_found = 0, f_found = 0, a_found = 0;
    char *i_filename = NULL, *o_filename = NULL;
    double t = 0, T = 0;
    int n = 0;
    unsigned int steps = 0;
    int animation_resolution = 0;
    int time_var_found = 0, funtyp_found = 0, offset_found = 0, period_found = 0, amplit_found = 0,
        constf_found = 0;
    char *funTyp_filename = NULL, *offset_filename = NULL, *period_filename = NULL, *amplit_filename = NULL,
         *constf_filename = NULL;
    double alpha = 0, beta = 0, gamma_ = 0;
    int alpha_found = 0, beta_found = 0, gamma_found = 0;
    int save_select_found = 0;
    char *save_selection = NULL;
    long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    int num_threads = ncpu > 0 ? (int)ncpu : 1;
    int integrator = TASEP_INTEGRATOR_REF, precision = TASEP_PRECISION_FP64, init_kind = TASEP_INIT_UNIFORM;
    char *init_file = NULL, *init_params = NULL;
    double stop_condition = 1e-10;
    int stop_count = 100, device = -1;
    int err;

    while ((opt = getopt_long(argc, argv, "i:v:o:t:T:n:s:a:fh?", long_opt, &option_index)) != -1) {
        switch (opt) {
        case 'i': if_found = 1; i_filename = strdup(optarg); break;
        case 'o': of_found = 1; o_filename = strdup(optarg); break;
        case 't': t_found = 1; t = atof(optarg); break;
        case 'T': T_found = 1; T = atof(optarg); break;
        case 'n': n_found = 1; n = atoi(optarg); break;
        case 's': s_found = 1; steps = (unsigned int)atoi(optarg); break;
        case 'f': f_found = 1; break;
        case 'a': a_found = 1; animation_resolution = atoi(optarg); break;
        case OPT_TIMEVAR: time_var_found = 1; break;
        case OPT_FUNTYPE: funtyp_found = 1; funTyp_filename = strdup(optarg); break;
        case OPT_OFFSET: offset_found = 1; offset_filename = strdup(optarg); break;
        case OPT_AMPLITUDE: amplit_found = 1; amplit_filename = strdup(optarg); break;
        case OPT_PERIOD: period_found = 1; period_filename = strdup(optarg); break;
        case OPT_CONSTANT: constf_found = 1; constf_filename = strdup(optarg); break;
        case OPT_SAVESEL: save_select_found = 1; save_selection = strdup(optarg); break;
        case OPT_THREADS: num_threads = atoi(optarg); break;
        case OPT_ALPHA: alpha = atof(optarg); alpha_found = 1; break;
        case OPT_BETA: beta = atof(optarg); beta_found = 1; break;
        case OPT_GAMMA: gamma_ = atof(optarg); gamma_found = 1; break;
        case OPT_INTEGRATOR:
            if (!strcmp(optarg, "ref")) integrator = TASEP_INTEGRATOR_REF;
            else if (!strcmp(optarg, "rk4")) integrator = TASEP_INTEGRATOR_RK4;
            else { usage(argv[0]); exit(-1); }
            break;
        case OPT_PRECISION:
            if (!strcmp(optarg, "fp64")) precision = TASEP_PRECISION_FP64;
            else if (!strcmp(optarg, "mixed")) precision = TASEP_PRECISION_MIXED;
            else { usage(argv[0]); exit(-1); }
            break;
        case OPT_INIT:
            if (!strcmp(optarg, "uniform")) init_kind = TASEP_INIT_UNIFORM;
            else if (!strcmp(optarg, "empty")) init_kind = TASEP_INIT_EMPTY;
            else if (!strcmp(optarg, "learned")) init_kind = ME_INIT_LEARNED;
            else { usage(argv[0]); exit(-1); }
            break;
        case OPT_INITFILE: init_file = strdup(optarg); break;
        case OPT_INITPARAMS: init_params = strdup(optarg); break;
        case OPT_STOPTOL: stop_condition = atof(optarg); break;
        case OPT_STOPCOUNT: stop_count = atoi(optarg); break;
        case OPT_DEVICE: device = atoi(optarg); break;
        default:
            usage(argv[0]);
            exit(-1);
        }
    }

    if (f_found && time_var_found) me_err_exit("ERROR: -f cannot be selected in combination with --time-var", -1);

    if (!n_found) {
        printf("Enter length: ");
        err = fscanf(stdin, "%d", &n);
        if (err == EOF) me_err_exit("ERROR: Issue while reading n from stdin", err);
    }
    if (n < 1 || n > TASEP_MAX_N) {
        fprintf(stderr, "ERROR: lattice length %d outside 1..%d\n", n, TASEP_MAX_N);
        exit(-1);
    }
    const uint64_t dim = (uint64_t)1 << n;
    double *x = (double *)malloc((size_t)dim * sizeof(double));
    if (x == NULL) me_err_exit("ERROR: Not enough memory to allocate x array", -1);
    printf("Allocated result-vector\n");

    double *rates = NULL;
    if (alpha_found || beta_found || gamma_found) {
        if (!alpha_found) {
            fprintf(stderr, "ERROR: No value for alpha found. Please ammend option --alpha to command line options. "
                            "Exiting\n");
            exit(-1);
        } else {
            fprintf(stdout, "Found value for\n   alpha: %lf\n", alpha);
        }
        if (!gamma_found) {
            fprintf(stderr, "CAUTION: No value for gamma found. If you want to specify gamma, please ammend option "
                            "--gamma to command line options.\n");
            gamma_ = 1;
            gamma_found = 1;
        }
        fprintf(stdout, "   gamma: %lf\n", gamma_);
        if (!beta_found) {
            fprintf(stderr, "ERROR: No value for beta found. Please ammend option --beta to command line options. "
                            "Exiting\n");
            exit(-1);
        } else {
            fprintf(stdout, "   beta: %lf\n", beta);
        }
    } else if (!if_found && !time_var_found) {
        printf("Enter %d probabilities: ", n + 1);
        rates = (double *)malloc((size_t)(n + 1) * sizeof(double));
        for (int i = 0; i < n + 1; i++)
            if (scanf("%lf", &rates[i]) == EOF) me_err_exit("ERROR: Could not read from stdin.", EOF);
    }
    if (!T_found) {
        printf("No end time found. Please enter: ");
        err = scanf("%lf", &T);
        if (err == EOF) me_err_exit("ERROR: Issue while reading end time from stdin", err);
    }
    if (!t_found) {
        printf("No start time found. Please enter: ");
        err = scanf("%lf", &t);
        if (err == EOF) me_err_exit("ERROR: Issue while reading start time from stdin", err);
    }
    if (init_file) {
        if (read_prob_file(init_file, n, x) != 0) me_err_exit("ERROR: Could not read the initial state file", -1);
        printf("Read initial vector from '%s'\n", init_file);
    } else if (init_kind == ME_INIT_LEARNED) {
        printf("Initial vector from the learned warm start\n");
    } else if (init_kind == TASEP_INIT_EMPTY) {
        printf("Generated inital vector with empty lattice (P(0)=1)\n");
    } else {
        double d = (double)dim;
        printf("Generated inital vector with identical values(%.30g)\n", 1. / d);
    }

    if (!of_found) {
        o_filename = (char *)malloc(19);
        of_found = 1;
        printf("WARNING: No output file found. Generating default output file ('generic_output.vec').\n");
        snprintf(o_filename, 19, "generic_output.vec");
        FILE *g = fopen(o_filename, "w");
        if (g == NULL) {
            printf("ERROR: Cannot open generic output file. Check permissions.\n");
            exit(-1);
        }
        fclose(g);
    }
    if (!s_found) {
        printf("No step number found. Please Enter: ");
        err = scanf("%u", &steps);
        if (err == EOF) me_err_exit("ERROR: Issue while reading step number from stdin", err);
    }

    if (if_found) {
        rates = (double *)realloc(rates, (size_t)(n + 1) * sizeof(double));
        int rc = me_read_doubles(i_filename, n + 1, rates, "%lf");
        if (rc == -1) {
            printf("ERROR: Cannot open jump rate file '%s'\n", i_filename);
            exit(-1);
        }
        if (rc == -2) me_err_exit("ERROR: Issue while reading from jump rate file name", EOF);
        if (alpha_found || beta_found || gamma_found)
            fprintf(stdout, "CAUTION: Switch '-i' overrides values given for alpha, beta and gamma.\n");
    } else if (alpha_found && beta_found) {
        rates = (double *)realloc(rates, (size_t)(n + 1) * sizeof(double));
        rates[0] = alpha;
        rates[n] = beta;
        for (int i = 1; i < n; i++) rates[i] = gamma_;
    }
    if (rates == NULL) {
        /* the reference dereferences an unset rate array here (--time-var without -i or rates) */
        me_err_exit("ERROR: --time-var needs -i or --alpha/--beta for the initial rates", -1);
    }
    printf("Allocated calculation vectors\n");
    if (a_found) {
        if (animation_resolution < 1) me_err_exit("ERROR: -a needs a positive number of steps", -1);
        printf("Allocatng memory for animation data\n");
    }
    printf("Number of threads to be used: %d\n", num_threads);

    int save_e = 0, save_p = 0, save_c = 0, save_m = 0;
    if (save_select_found) {
        for (size_t i = 0; i < strlen(save_selection); i++) switch (save_selection[i]) {
            case 'a': save_e = save_p = save_c = 1; break;
            case 'e': save_e = 1; break;
            case 'p': save_p = 1; break;
            case 'c': save_c = 1; break;
            case 'm': save_m = 1; break;
            default: printf("Could not parse save selction\n");
            }
    } else {
        save_e = save_p = save_c = save_m = 1;
    }

    const double h = (double)((T - t) / ((long double)steps));

    /* time-variant rate functions (src/masterEquation.c:700-875) */
    int tv_type[TASEP_MAX_N + 1];
    double tv_off[TASEP_MAX_N + 1], tv_amp[TASEP_MAX_N + 1], tv_per[TASEP_MAX_N + 1], tv_cst[TASEP_MAX_N + 1];
    if (time_var_found) {
        if (funtyp_found) {
            FILE *F = fopen(funTyp_filename, "r");
            if (F == NULL) {
                printf("ERROR: Cannot open file containing function Types. Aborting\n");
                exit(-1);
            }
            char sel[256];
            for (int i = 0; i < n + 1; i++) {
                if (fscanf(F, "%255s", sel) == EOF)
                    me_err_exit("ERROR: Issue while reading function type file: Reached early EOF", EOF);
                switch (sel[0]) {
                case 's': tv_type[i] = TASEP_FUN_SIN; break;
                case 'c': tv_type[i] = TASEP_FUN_COS; break;
                case 'l': tv_type[i] = TASEP_FUN_LIN; break;
                default:
                    printf("ERROR: Non identifiable function type fonud in%s. Read %s. Aborting!\n", funTyp_filename,
                           sel);
                    tv_type[i] = -1; /* keeps the constant rate */
                }
            }
            fclose(F);
            printf("Read function types successfully\n");
        } else {
            for (int i = 0; i < n + 1; i++) tv_type[i] = TASEP_FUN_SIN;
            printf("Wrote function type array successfully\n");
        }
        struct {
            int found;
            const char *file;
            double *dst;
            double dflt;
            const char *ok_read, *ok_default, *eof_msg, *open_msg;
        } tab[4] = {
            {offset_found, offset_filename, tv_off, 0., "Read offset values successfully",
             "Wrote offset values sucessfully", "ERROR: Issue while reading offset filename",
             "ERROR: Cannot open file containing offset values. Aborting"},
            {amplit_found, amplit_filename, tv_amp, 1., "Read amplitude values correctly",
             "Wrote amplitude values correctly", "ERROR: Issue while reading amplitude-file",
             "ERROR: Cannot open file containing amplitude values. Aborting"},
            {period_found, period_filename, tv_per, 1., "Read period values correctly",
             "Wrote period values correctly", "ERROR: Issue while reading period-file",
             "ERROR: Cannot open file containing amplitude values. Aborting"},
            {constf_found, constf_filename, tv_cst, 1., "Read constant values correctly",
             "Wrote constant values correctly", "ERROR: Issue while reading const-file",
             "ERROR: Cannot open file containing amplitude values. Aborting"},
        };
        for (int k = 0; k < 4; k++) {
            if (tab[k].found) {
                int rc = me_read_doubles(tab[k].file, n + 1, tab[k].dst, "%lf, ");
                if (rc == -1) {
                    printf("%s\n", tab[k].open_msg);
                    exit(-1);
                }
                if (rc == -2) me_err_exit(tab[k].eof_msg, EOF);
                printf("%s\n", tab[k].ok_read);
            } else {
                for (int i = 0; i < n + 1; i++) tab[k].dst[i] = tab[k].dflt;
                printf("%s\n", tab[k].ok_default);
            }
        }
    }

    /* ---- the integration, on the GPU ---- */
    double start = wall();
    tasep_meq *m = NULL;
    tasep_meq_config mc = {n, integrator, precision, device, NULL};
    if (tasep_meq_create(&mc, &m) != TASEP_OK) tasep_fail("cannot set up the integrator");
    if (tasep_meq_set_rates(m, rates) != TASEP_OK) tasep_fail("rates");
    if (time_var_found && tasep_meq_set_timevar(m, tv_type, tv_amp, tv_per, tv_off, tv_cst) != TASEP_OK)
        tasep_fail("time-variant rates");
    if (init_file) {
        if (tasep_meq_load(m, x) != TASEP_OK) tasep_fail("initial state");
    } else if (init_kind == ME_INIT_LEARNED) {
        char path[4096];
        if (init_params) {
            snprintf(path, sizeof path, "%s", init_params);
        } else {  /* data/warmstart_params.npy beside the bin/ directory of this program */
            ssize_t len = readlink("/proc/self/exe", path, sizeof path - 64);
            if (len < 0) len = 0;
            path[len] = 0;
            char *slash = strrchr(path, '/');
            if (slash) *slash = 0;
            strcat(path, "/../data/warmstart_params.npy");
        }
        const int w = me_warm_start(m, n, rates, path, device);
        if (w < 0) tasep_fail("learned warm start");
        if (w == 1) {
            printf("Warm-start prediction infeasible; starting from the empty lattice\n");
            if (tasep_meq_init(m, TASEP_INIT_EMPTY) != TASEP_OK) tasep_fail("initial state");
        }
    } else if (tasep_meq_init(m, init_kind) != TASEP_OK) {
        tasep_fail("initial state");
    }
    printf(time_var_found ? "Starting Calculation\n" : "Starting Calculation!\n");
    if (f_found) printf("Generating Matrix: 100.000000%%\nTime elapsed: %f seconds\nCalculating result vector..\n\n", 0.0);

    /* run in chunks so that a progress line can be printed */
    tasep_run_result rr;
    memset(&rr, 0, sizeof rr);
    me_snaps snaps;
    memset(&snaps, 0, sizeof snaps);
    double tt = t;
    uint64_t done = 0;
    int early_stop = 0;
    uint64_t steps_at_stop = 0;
    double checksum = 0;
    {
        tasep_run_config rc = {tt, h, steps, stop_condition, stop_count, time_var_found ? 0 : 1};
        if (a_found) {
            snaps.n = n;
            snaps.dim = dim;
            snaps.keep_probs = save_p;
            if (tasep_meq_run_stream(m, &rc, (uint64_t)animation_resolution, n > 5 || save_p, snapshot_hook,
                                     &snaps, &rr) != TASEP_OK)
                tasep_fail("integration");
        } else if (tasep_meq_run(m, &rc, &rr) != TASEP_OK) {
            tasep_fail("integration");
        }
        done = rr.steps_done;
        early_stop = rr.early_stop;
        steps_at_stop = rr.steps_at_stop;
        checksum = rr.last_checksum;
        tt = rr.t_end;
        if (time_var_found)
            printf("\r%lf%%, step %" PRIu64 " of %u", 100. * (double)(done ? done - 1 : 0) / (double)steps,
                   done ? done - 1 : 0, steps);
        else if (f_found)
            printf("Sim Time: %lf ------ Delta %.5g ------ Stop condition %d%%\r", tt, checksum, early_stop);
        else
            printf("Simulation time elapsed: %lf ------ Delta %.5g ------ Stop condition reached %d%%\r", tt, checksum,
                   early_stop);
        if (time_var_found) printf("\n");
    }
    if (tasep_meq_store(m, x, 0, dim) != TASEP_OK) tasep_fail("copy of the result");
    me_obs ob;
    memset(&ob, 0, sizeof ob);
    ob.n = n;
    double mass = 0;
    if (tasep_meq_observables(m, ob.y, ob.cov, ob.mul, n >= 4 ? ob.p4 : NULL, &mass) != TASEP_OK)
        tasep_fail("observables");
    tasep_meq_destroy(m);

    double secs = wall() - start;
    FILE *F = fopen("runtimes.txt", "a");
    if (F != NULL) {
        fprintf(F, "%i %f\n", n, secs);
        fclose(F);
    }
    printf("\n####Finished Calculation####\n");
    printf("Real Time elapsed: %f\n", secs);
    printf("Simulation time elapsed: %lf\n", tt);
    if (early_stop)
        printf("Convergence after %" PRIu64 " steps\nConfidience |Δx| = %.20g\n", steps_at_stop,
               stop_condition * h);
    printf("Checksum over result vector: %lf\n", mass);

    /* ---- output files (src/masterEquation.c:1019-1539) ---- */
    const size_t olen = strlen(o_filename);
    char *name = (char *)malloc(olen + 32);
    if (save_p) {
        if (me_write_probs(o_filename, n, x, num_threads) != 0) printf("ERROR: Cant write to %s\n", o_filename);
        snprintf(name, olen + 32, "%s_prb.txt", o_filename);
        me_write_prb_txt(name, a_found ? &snaps : NULL, h * animation_resolution);
    }
    if (save_e) {
        me_write_exp_values(o_filename, &ob);
        if (a_found) me_write_exp_timed(o_filename, &snaps, h * animation_resolution);
    }
    if (save_c) {
        char *ppm = (char *)malloc(olen + 32);
        snprintf(name, olen + 32, "%s_cov.mat", o_filename);
        snprintf(ppm, olen + 32, "%s_cov.ppm", o_filename);
        me_write_cov(name, ppm, &ob);
        free(ppm);
        if (a_found) me_write_anim_dir(o_filename, 0, &ob, &snaps, h * animation_resolution);
    }
    if (save_m) {
        /* With the default selection the reference sizes this name for "_cov.ppm"
           plus one character, so both the matrix and the picture go to
           "<o>_mulExpVa" and the picture overwrites the matrix
           (src/masterEquation.c:1285-1322).  That file name is kept for that
           case; otherwise the full names are written. */
        char *ppm = (char *)malloc(olen + 32);
        if (save_c && save_p) {
            snprintf(name, olen + 32, "%s_mulExpVa", o_filename);
            snprintf(ppm, olen + 32, "%s_mulExpVa", o_filename);
        } else {
            snprintf(name, olen + 32, "%s_mulExpVal.mat", o_filename);
            snprintf(ppm, olen + 32, "%s_mulExpVal.ppm", o_filename);
        }
        me_write_mul(name, ppm, &ob);
        free(ppm);
        if (a_found) me_write_anim_dir(o_filename, 1, &ob, &snaps, h * animation_resolution);
    }
    free(name);
    if (n >= 4) me_write_windows(o_filename, &ob);
    if (a_found) {
        me_write_highcorr_timed(o_filename, &snaps, h * animation_resolution);
        free(snaps.obs);
        free(snaps.probs);
        free(snaps.corr);
    }

    free(x);
    free(rates);
    free(i_filename);
    free(o_filename);
    free(save_selection);
    free(funTyp_filename);
    free(offset_filename);
    free(period_filename);
    free(amplit_filename);
    free(constf_filename);
    free(init_file);
    free(init_params);
    return 0;
}
