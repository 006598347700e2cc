/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the L-FTS diblock step.
 *
 * A plain-C restatement of tmbeardsley/lfts_cpu's hot path, used by tests/,
 * the smoke check and the CPU-baseline leg of bench.py as the oracle.  The
 * product (lfts_cpu_b200/) never links or calls it.  Each function cites the
 * reference lines it restates.  All arithmetic is FP64 like the reference.
 *
 * Field array w (4M doubles) = [W-, w+, phi-, phi+], mesh index
 * r = mz*(i*my + j) + k (src/field_generator.h:18); half-spectrum index
 * k2 + (mz/2+1)*(K1 + my*K0) (src/step.cc:83).
 */
#ifndef LFTS_ORACLE_H
#define LFTS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sys orc_sys;

/* diblock(NA, NB, m, L, M, Mk) + step(...) (src/diblock.cc:9-25, src/step.cc:10-28) */
orc_sys *orc_create(int NA, int NB, const int m[3], const double L[3]);
void orc_destroy(orc_sys *s);
void orc_set_threads(int nthreads);

/* g[k] = exp(-K^2/6N)/M, src/step.cc:69-89 */
void orc_g_lookup(const orc_sys *s, double *g);
/* step::fwd, src/step.cc:35-65: q_in/q_out/h are 2M each */
void orc_step_fwd(orc_sys *s, const double *q_in, double *q_out, const double *h, int i);
/* diblock::calc_concs, src/diblock.cc:30-60; returns ln Q and writes phi-/phi+ into w */
double orc_calc_concs(orc_sys *s, double *w);
/* optional: copy of all propagators of the last calc_concs, 2(N+1)M doubles (slot 0 unused) */
const double *orc_propagators(const orc_sys *s);

/* anderson(M, maxHist) + anderson::mix, src/anderson.cc:8-93 */
typedef struct orc_anderson orc_anderson;
orc_anderson *orc_anderson_create(int M, int maxHist);
void orc_anderson_destroy(orc_anderson *a);
int orc_anderson_mix(orc_anderson *a, orc_sys *s, int maxIter, double errTol, double *w);

/* langevin::step_wm update line, src/langevin.cc:31 (noise supplied by the caller) */
void orc_langevin_update(double *w, const double *noise_prev, const double *noise_new,
                         double XbN, double dt, int M);

/* strFunc::sample, src/strFunc.cc:36-46: S[k] += |FFT(W-)(k)|^2 */
void orc_sk_sample(orc_sys *s, const double *w, double *S);
/* strFunc::save binning, src/strFunc.cc:9-32,50-76,80-103.  Writes one (K, S)
 * pair per output line; returns the number of lines.  Kout/Sout hold Mk. */
int orc_sk_bin(const int m[3], const double L[3], const double *S, int nsamples,
               double CV, double chi_b, double dK, double *Kout, double *Sout);

/* lfts_simulation::getH, src/lfts_simulation.cc:122-135 */
double orc_getH(orc_sys *s, double *w, double XbN);

/* lfts_params::z_inf_discrete, src/lfts_params.cc:122-142 */
double orc_z_inf_discrete(const double L[3], const int m[3], int N, double Nbar, int tmax);

#ifdef __cplusplus
}
#endif
#endif
