/*
 * lfts_b200 -- C ABI of the B200 (sm_100a) Langevin field-theoretic simulation
 * step for AB diblock copolymers.
 *
 * The entry points replace the C++ methods the reference driver calls
 * (tmbeardsley/lfts_cpu); each declaration cites the method it stands in for.
 * All state lives on one GPU inside an opaque context; host pointers are plain
 * C arrays with the reference's layouts:
 *   fields   w = [W-(M) | w+(M) | phi-(M) | phi+(M)]       (src/lfts_simulation.h:21)
 *   mesh     r = mz*(i*my + j) + k                         (src/field_generator.h:18)
 *   spectrum k = k2 + (mz/2+1)*(K1 + my*K0), Mk entries    (src/step.cc:83)
 * Every call returns an lfts_status (0 = success).  A context is used by one
 * host thread at a time.  Calls are synchronous unless the name ends in _async.
 * There is no CPU fallback: a missing GPU or unsupported mesh is an error.
 */
#ifndef LFTS_B200_H
#define LFTS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum lfts_status {
    LFTS_OK = 0,
    LFTS_ERR_ARG = 1,          /* bad argument (null pointer, size, index) */
    LFTS_ERR_UNSUPPORTED = 2,  /* mesh size without an FFT kernel, or odd my */
    LFTS_ERR_CUDA = 3,         /* CUDA runtime error (see lfts_last_error_string) */
    LFTS_ERR_NOMEM = 4,        /* device allocation failed */
    LFTS_ERR_SINGULAR = 5,     /* Anderson least-squares matrix singular */
    LFTS_ERR_STATE = 6,        /* call out of order (e.g. fields never set) */
    LFTS_ERR_NOTCONV = 7,      /* Anderson mixing stopped at maxIter above the tolerance;
                                  the fields are updated as the reference leaves them,
                                  so a caller may carry on (the reference does, silently) */
    LFTS_ERR_NONFINITE = 8     /* a NaN or infinite Anderson residual: the mix stopped
                                  before updating w+ with it */
} lfts_status;

typedef enum lfts_precision {
    LFTS_FP64 = 0,       /* everything FP64: matches the reference to ~1e-10 */
    LFTS_FP32_MIXED = 1  /* FP32 FFTs/propagators; FP64 Q, log, Anderson, H, fields */
} lfts_precision;

/* Simulation constants after the reference's input conversion
 * (src/lfts_params.cc:87-119): XbN is the bare chi*N actually simulated. */
typedef struct lfts_params {
    int N;         /* monomers per chain */
    int NA;        /* A-block length (NB = N - NA) */
    double XbN;    /* bare chi * N */
    double C;      /* sqrt(Nbar) */
    double dt;     /* Langevin time step * N */
    int m[3];      /* mesh mx, my, mz */
    double L[3];   /* box Lx, Ly, Lz in R0 */
} lfts_params;

typedef struct lfts_ctx lfts_ctx;

const char *lfts_version(void);
const char *lfts_status_string(int status);
/* text of the last CUDA error seen by any call in this process */
const char *lfts_last_error_string(void);
/* 1 when mesh dimension n has an FFT kernel compiled into the library */
int lfts_mesh_supported(int n);

/* Allocates device state for one system: the diblock, step, anderson and
 * strFunc objects of lfts_simulation's constructor (src/lfts_simulation.cc:29-42). */
int lfts_create(const lfts_params *p, int precision, int device, lfts_ctx **out);
int lfts_destroy(lfts_ctx *ctx);
/* device bytes held by the context */
int lfts_device_bytes(const lfts_ctx *ctx, size_t *bytes);

/* Upload W- and w+ (2M doubles, host); replaces the reference's readArray /
 * generate_field into w_ (src/lfts_simulation.cc:45-49). */
int lfts_set_fields(lfts_ctx *ctx, const double *w_host);
/* Download w = [W-, w+, phi-, phi+] (4M doubles, host). */
int lfts_get_fields(lfts_ctx *ctx, double *w_host);
/* Device address of the FP64 field array (4M doubles) owned by the context. */
int lfts_fields_device(lfts_ctx *ctx, double **w_dev);

/* diblock::calc_concs (src/diblock.cc:30-60): phi-, phi+ from W-, w+; ln Q out. */
int lfts_calc_concs(lfts_ctx *ctx, double *lnQ);

/* anderson::mix (src/anderson.cc:24-93): saddle point of w+ by Anderson
 * mixing with history 10; *k_out receives the reference's return value.
 * The reference reports no failure; here the loop's end is reported:
 * LFTS_ERR_NOTCONV when it stopped at maxIter with the error above errTol
 * (fields and *k_out as the reference leaves them), LFTS_ERR_NONFINITE when
 * the residual is NaN or infinite (w+ not updated with it; *k_out = the value
 * the reference's loop returns, which ends there), LFTS_ERR_SINGULAR when the least-squares matrix
 * is exactly singular (where the reference's GSL solve aborts the program). */
int lfts_anderson_mix(lfts_ctx *ctx, int maxIter, double errTol, int *k_out);

/* langevin::langevin (src/langevin.cc:7-17): the initial "previous" noise, M
 * doubles already scaled by sigma, drawn by the caller's generator. */
int lfts_langevin_init(lfts_ctx *ctx, const double *noise_prev_host);
/* langevin::step_wm (src/langevin.cc:23-37): W- += -(phi- + 2W-/XbN) dt +
 * (eta_prev + eta_new)/2 with the caller's new noise (M doubles, host). */
int lfts_langevin_step(lfts_ctx *ctx, const double *noise_new_host);
/* same with the new noise already in device memory */
int lfts_langevin_step_device(lfts_ctx *ctx, const double *noise_new_dev);

/* One reference Langevin step (src/lfts_simulation.cc:69-76): step_wm, mix,
 * then the extra calc_concs whose ln Q the reference prints.  A mix that ends
 * with LFTS_ERR_NOTCONV still runs the extra calc_concs (the step completes,
 * as in the reference) and the call returns LFTS_ERR_NOTCONV. */
int lfts_langevin_full_step(lfts_ctx *ctx, const double *noise_new_dev, int maxIter,
                            double errTol, int *k_out, double *lnQ);

/* strFunc::sample (src/strFunc.cc:36-46): S(k) += |FFT(W-)(k)|^2 */
int lfts_sk_sample(lfts_ctx *ctx);
/* raw accumulator (Mk doubles) and the number of samples */
int lfts_sk_get(lfts_ctx *ctx, double *S_host, int *nsamples);
int lfts_sk_reset(lfts_ctx *ctx);
/* strFunc::save averaging (src/strFunc.cc:50-76): spherical average over |K|
 * with tolerance dK.  K_out and S_out hold at least Mk entries; *nbins out. */
int lfts_sk_bin(lfts_ctx *ctx, double dK, double *K_out, double *S_out, int *nbins);

/* lfts_simulation::getH (src/lfts_simulation.cc:122-135) */
int lfts_get_H(lfts_ctx *ctx, double *H);

/* step::fwd (src/step.cc:35-65): one contour step of both chains.
 * q_in, q_out, h: 2M doubles each (host); i: monomer index of q_in. */
int lfts_step_fwd(lfts_ctx *ctx, const double *q_in, double *q_out, const double *h, int i);
/* step::update_g_lookup (src/step.cc:69-89): the Mk Boltzmann weights g(k) */
int lfts_g_lookup(lfts_ctx *ctx, double *g_host);

/* ---- adjoint ------------------------------------------------------------- */
/* Gradients of the reference's H (src/lfts_simulation.cc:122-135) for the
 * current fields: dH/dL[3] (box lengths, mesh-point fields held fixed) and
 * dH/dXbN (bare chi N), plus H itself.  The reference has no such method (its
 * lfts_params.h:4-6 anticipates box-altering moves that need it).  dH/dL comes
 * from the forward and complementary propagators, the latter being the adjoint
 * chain: dQ/dL_a = (1/M) sum_i sum_k dg/dL_a Re[q_i(k) conj(q^_{i+1}(k))].
 * ckpt_every = 0 uses every stored propagator (and leaves phi of the fields);
 * ckpt_every = K > 0 keeps q only at every K-th monomer and recomputes the
 * segments in between (q^ kept in full; phi is not produced).  For an input
 * with effective chi (isXeN = 1) the caller adds dH/dXbN * dXbN/dL through
 * z_inf.  FP64 contexts only. */
int lfts_backward(lfts_ctx *ctx, int ckpt_every, double *dH_dL, double *dH_dXbN, double *H);

/* ---- allocation-free contour step ----------------------------------------- */
/* Largest spectrum the allocation-free step holds: 2*mx*my*(mz/2+1) complex
 * doubles (every mesh up to 64^3), about 4.3 MB of static device memory. */
#define LFTS_NOALLOC_MAX_SPECTRUM (2LL * 64 * 64 * 33)

/* No counterpart in the reference: the contour step of step::fwd for callers
 * that cannot allocate device memory (their device memory comes from a pool
 * or framework that owns all allocations, or they run where allocation is not
 * allowed).  Needs no context and allocates nothing: q_in, q_out, h are the
 * caller's DEVICE arrays (2M doubles each, layout of src/step.h:40-42), and the
 * step's scratch is one static device array per GPU, holding meshes up to
 * LFTS_NOALLOC_MAX_SPECTRUM (larger meshes return LFTS_ERR_ARG).  FP64 only.
 * Work is enqueued on `stream` (a cudaStream_t; 0 = legacy default stream) of
 * the current device and the call returns without waiting.  All calls on a
 * device share that array, so calls whose kernels overlap on the GPU race:
 * serialise them.  The first call on each device sets up the array's address;
 * make it before any stream capture. */
int lfts_step_fwd_noalloc(const lfts_params *p, const double *q_in, double *q_out,
                          const double *h, int i, void *stream);

/* ---- timing / integration helpers -------------------------------------- */
/* The CUDA stream every call of this context runs on (a cudaStream_t). */
void *lfts_stream(lfts_ctx *ctx);
/* Time the contour chain of one calc_concs: mean ms of a yz-plane step
 * kernel and of an x-pencil kernel (one stream, events around every launch),
 * and ms of the whole production chain (leaves the current fields' propagators). */
int lfts_profile_chain(lfts_ctx *ctx, double *ms_plane, double *ms_pencil, double *ms_chain);
/* Mean ms over `reps` back-to-back runs of each part of one Anderson
 * iteration on the current fields: the contour chain with Q (one
 * calc_concs's propagators), the concentration pass with the residual dot
 * products against a full history (10) and their reduction, and the w+
 * update over a full history.  A timing helper: the fields, phi and w+ are
 * left as they were (the update runs with lambda = 0 and zero coefficients). */
int lfts_profile_iteration(lfts_ctx *ctx, int reps, double *ms_chain, double *ms_concs, double *ms_update);
/* Number of kernels this context has launched so far. */
long long lfts_kernel_launches(const lfts_ctx *ctx);
/* The free choices of a context's contour chain.  None changes what is
 * computed: pencil_cw changes no value at all, the others change FP32-mixed
 * results only within that path's stated error (and FP64 ones not at all:
 * two_streams only reorders independent launches). */
typedef struct lfts_tiles {
    int pencil_cw;     /* x-pencil columns per CTA: 8, 16 or 32 */
    int plane_stages;  /* yz-plane transform stages per axis: 2, or 3 (FP32-mixed, 64/96/128 square planes) */
    int h_in_pencil;   /* FP32-mixed: h and the propagator stores in the x-pencil kernel and g in the
                          yz-plane kernel (1; 96- and 128-point x lines, 3 stages), or all in the yz-plane (0) */
    int two_streams;   /* FP64: each chain on its own stream (1) or both chains in every launch (0) */
    int phi_in_chain;  /* with h_in_pencil: the concentration sums formed in the x-pencil from the
                          middle of the chain on (each new slot times its already stored partner,
                          FP32 sums; the later slots are then not stored) (1), or by a separate
                          pass over all N stored slots (0) */
    int plane_split;   /* FP32-mixed 128 x 128 planes with h_in_pencil: CTAs per x-plane in the yz-plane
                          kernel, 8 (the plane split over a thread-block cluster, its transposes through
                          distributed shared memory; bitwise the same values) or 1; 0 reads as 1 */
} lfts_tiles;
/* lfts_create picks the tiles by timing the whole contour chain for every
 * valid combination on the context's own buffers and keeping the fastest,
 * once per precision and mesh in a process (the counterpart of the
 * reference's FFTW_PATIENT planning, src/step.cc:15-16).  Environment:
 * LFTS_AUTOTUNE=0 skips the timing (built-in choice); LFTS_PENCIL_CW=8|16|32,
 * LFTS_XH_CHAIN=0|1, LFTS_PHI_IN_CHAIN=0|1, LFTS_PLANE_SPLIT=1|8 and
 * LFTS_ONE_STREAM=1 fix one choice each. */
int lfts_get_tiles(const lfts_ctx *ctx, lfts_tiles *out);
/* Installs a tile choice (LFTS_ERR_ARG / LFTS_ERR_UNSUPPORTED for an
 * invalid one), e.g. to make a context compute exactly what an ensemble
 * replica with those tiles computes. */
int lfts_set_tiles(lfts_ctx *ctx, const lfts_tiles *tiles);
/* pencil_cw and plane_stages of the current tiles */
int lfts_tuning(const lfts_ctx *ctx, int *pencil_cw, int *plane_stages);
/* Mean Anderson iteration count of all lfts_anderson_mix calls so far. */
int lfts_anderson_stats(const lfts_ctx *ctx, long long *calls, long long *iterations);
/* Copy the propagators of the last calc_concs, 2(N+1)M doubles (slot 0
 * zero), layout of src/diblock.cc:19-24. */
int lfts_get_propagators(lfts_ctx *ctx, double *q_host);


/* ---- ensemble of independent replicas ------------------------------------ */
/* Many independent FP32-mixed systems (the batched configuration:
 * replicas of different meshes, each with its own parameters and noise
 * stream) advanced together.  The reference runs one system per process;
 * there is no counterpart.  Each replica is a context of its own (buffers,
 * tables), with tiles picked by timing the batched chain of its mesh group
 * (lfts_ensemble_tiles), and computes exactly what a single FP32-mixed context
 * with those tiles (lfts_set_tiles) computes when fed the same noise.  A run
 * of Langevin steps of every replica -- update, Anderson loop with the least
 * squares on the device, the extra calc_concs -- is one CUDA graph launch (up
 * to 1024 steps per launch): a WHILE node over the steps holds a WHILE node
 * over the Anderson iterations, which runs until every replica's loop has
 * ended.  Replicas share N; meshes are 16, 24, 32, 48, 64 or 96 per side
 * with square yz planes. */
typedef struct lfts_ensemble lfts_ensemble;
/* params[nrep], seeds[nrep]: the replicas' parameters and Philox streams. */
int lfts_ensemble_create(const lfts_params *params, const unsigned long long *seeds, int nrep, int device,
                         lfts_ensemble **out);
int lfts_ensemble_destroy(lfts_ensemble *ens);
/* W- and w+ of replica r (2M doubles), as lfts_set_fields. */
int lfts_ensemble_set_fields(lfts_ensemble *ens, int r, const double *w_host);
/* [W-, w+, phi-, phi+] of replica r (4M doubles), as lfts_get_fields. */
int lfts_ensemble_get_fields(lfts_ensemble *ens, int r, double *w_host);
/* Anderson mix of every replica followed by its calc_concs (the reference's
 * start of run); k_out[nrep] (may be null) the values anderson::mix returns,
 * lnQ_out[nrep] (may be null) ln Q of the mixed fields.  maxIter >= 2. */
int lfts_ensemble_mix(lfts_ensemble *ens, int maxIter, double tol, int *k_out, double *lnQ_out);
/* nsteps Langevin steps of every replica (src/lfts_simulation.cc:69-76 per
 * replica: step_wm with on-device noise, mix, calc_concs); k_out[nsteps][nrep]
 * (may be null; recorded on the device), lnQ_out[nrep] (may be null) after
 * the last step.  Every step runs: a replica whose mix fails stops its own
 * Anderson loop in that step (and, with non-finite fields, in the later ones)
 * while the others go on.  The noise of replica r at step s is
 * lfts_noise_philox(seeds[r], s, M, sigma_r); step 0 is the initial noise,
 * the first call's first step is step 1. */
int lfts_ensemble_run(lfts_ensemble *ens, int nsteps, int maxIter, double tol, int *k_out, double *lnQ_out);
/* Mix and run report the most severe status over the replicas and the mixes
 * of the call (LFTS_ERR_NONFINITE > LFTS_ERR_SINGULAR > LFTS_ERR_NOTCONV, as
 * for lfts_anderson_mix); a replica that fails stops its own Anderson loop
 * and leaves the others running.  A run goes on past a mix that stopped at
 * the cap (the reference does).  This gives replica r's own status of the last
 * mix or run call. */
int lfts_ensemble_replica_status(const lfts_ensemble *ens, int r, int *status);
/* x-pencil columns per CTA of replica r's mesh (autotuned). */
int lfts_ensemble_tuning(const lfts_ensemble *ens, int r, int *pencil_cw);
/* The tiles replica r computes with: picked per mesh group by timing the
 * group's batched contour chain (x-pencil width, yz-plane stages), once per
 * mesh, group size and N in a process.  A single FP32-mixed context given
 * these tiles (lfts_set_tiles) computes exactly what the replica computes. */
int lfts_ensemble_tiles(const lfts_ensemble *ens, int r, lfts_tiles *out);
/* The CUDA stream the ensemble's graphs run on (a cudaStream_t). */
void *lfts_ensemble_stream(lfts_ensemble *ens);
/* Kernels placed in the ensemble's graphs so far (per body iteration). */
long long lfts_ensemble_kernel_launches(const lfts_ensemble *ens);
/* sigma * z for points 0..n-1 of step s of Philox stream `seed`, computed on
 * the current device (the ensemble's noise; see lfts_cpu_b200/csrc/philox.cuh). */
int lfts_noise_philox(unsigned long long seed, long long step, long long n, double sigma, double *out_host);

/* ---- host helpers with the reference driver's semantics ------------------ */
/* Everything the reference's lfts_params derives from the 3-line input header
 * (src/lfts_params.cc:87-119). */
typedef struct lfts_input {
    int N, NA, NB;
    double XN_in;      /* XN as written in the file */
    double C, dt;
    int isXeN;
    int m[3];
    double L[3];
    int equil_its, sim_its, sample_freq, save_freq, loadType;
    /* derived */
    double XbN, XeN, V, sigma;
    long long M, Mk;
} lfts_input;

/* lfts_params::read_Input_Params + calculate_Derived_Params: step counts
 * rounded down to multiples of sample_freq, chi converted through z_inf. */
int lfts_read_input(const char *path, lfts_input *out);
/* lfts_params::z_inf_discrete (src/lfts_params.cc:122-142) */
double lfts_z_inf_discrete(const double L[3], const int m[3], int N, double Nbar, int tmax);
/* Fill the simulation constants from a parsed input. */
void lfts_params_from_input(const lfts_input *in, lfts_params *p);

/* The reference's generator: std::mt19937_64 seeded with `seed` feeding ONE
 * std::normal_distribution(0, sigma) (it keeps a cached spare deviate) and
 * uniform_real_distribution(0, 1) draws (src/langevin.cc:13-16,28;
 * src/lfts_simulation.cc:23,149-155).  Same libstdc++ => same stream. */
typedef struct lfts_rng lfts_rng;
int lfts_rng_create(unsigned long long seed, double sigma, lfts_rng **out);
int lfts_rng_destroy(lfts_rng *r);
int lfts_rng_normal(lfts_rng *r, long long n, double *out);
int lfts_rng_uniform(lfts_rng *r, long long n, double *out);
/* field_generator::create_lamellar (src/field_generator.h:11-24), W- and w+ */
int lfts_lamellar_field(double *w, double amplitude, const int m[3], int kx, int ky, int kz);
/* lfts_simulation::generate_field default branch (src/lfts_simulation.cc:149-155):
 * W- = XbN (U(0,1) - 1/2), w+ = 0, drawing M uniforms from r. */
int lfts_random_field(lfts_rng *r, double *w, double XbN, long long M);

#ifdef __cplusplus
}
#endif
#endif
