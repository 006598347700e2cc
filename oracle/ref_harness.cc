/*
 * TEST INFRASTRUCTURE ONLY -- a C entry layer over the reference's own classes,
 * linked with the reference's unmodified src/*.cc (compiled against
 * oracle/shim) into oracle/_ref/libref_harness.so by oracle/Makefile.  Used
 * only to pin the oracle (tests/golden/make_golden.py) and as the "reference"
 * CPU baseline; never by the product.
 *
 * The reference exposes no API beyond its classes, and lfts_simulation keeps
 * its state private, so this file opens class access before including the
 * reference headers (all standard headers are included first, untouched;
 * the reference headers declare no templates).
 * The per-step loop body below repeats src/lfts_simulation.cc:69-83 / 93-113
 * so that K (the return of anderson::mix, discarded by the reference) and
 * ln Q can be returned at full precision.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <math.h>
#include <memory>
#include <numeric>
#include <random>
#include <sstream>
#include <stdlib.h>
#include <string>
#include <unistd.h>
#include <vector>
#include <fftw3.h>
#include <gsl/gsl_linalg.h>
#include <gsl/gsl_blas.h>

#define class struct
#define private public
#include "lfts_simulation.h"
#undef private
#undef class

extern "C" {

/* ---- component level ---------------------------------------------------- */
struct ref_sys {
    std::unique_ptr<diblock> dbc;
    std::unique_ptr<anderson> am;
    std::unique_ptr<step> stp;
    int M;
};

ref_sys *ref_sys_create(int NA, int NB, const int *m_in, const double *L_in)
{
    int m[3] = {m_in[0], m_in[1], m_in[2]};
    double L[3] = {L_in[0], L_in[1], L_in[2]};
    int M = m[0] * m[1] * m[2];
    int Mk = m[0] * m[1] * (m[2] / 2 + 1);
    ref_sys *s = new ref_sys;
    s->M = M;
    s->dbc = std::make_unique<diblock>(NA, NB, m, L, M, Mk);
    s->am = std::make_unique<anderson>(M, 10);
    s->stp = std::make_unique<step>(NA, NB, m, L, M, Mk);
    return s;
}

void ref_sys_destroy(ref_sys *s) { delete s; }

double ref_sys_calc_concs(ref_sys *s, double *w) { return s->dbc->calc_concs(w); }

int ref_sys_mix(ref_sys *s, int maxIter, double tol, double *w)
{
    return s->am->mix(s->dbc.get(), maxIter, tol, w);
}

void ref_sys_step_fwd(ref_sys *s, const double *q_in, double *q_out, const double *h, int i)
{
    std::vector<double> qi(q_in, q_in + 2 * (size_t)s->M), hh(h, h + 2 * (size_t)s->M);
    s->stp->fwd(qi.data(), q_out, hh.data(), i);
}

void ref_sys_g(ref_sys *s, double *g, int Mk) { std::memcpy(g, s->stp->g_.get(), sizeof(double) * Mk); }

/* The reference's langevin object (src/langevin.cc:7-17) on its own
 * mt19937_64 seeded with `seed`: the constructor draws the initial "previous"
 * noise.  One Langevin step below is the loop body of
 * src/lfts_simulation.cc:69-76: step_wm, mix (200, 1e-4), the extra calc_concs. */
struct ref_lgv {
    std::mt19937_64 rng;
    std::unique_ptr<langevin> lgv;
};

ref_lgv *ref_lgv_create(unsigned long long seed, double sigma, int M)
{
    ref_lgv *l = new ref_lgv;
    l->rng.seed(seed);
    l->lgv = std::make_unique<langevin>(l->rng, sigma, M);
    return l;
}

void ref_lgv_destroy(ref_lgv *l) { delete l; }

/* lfts_simulation::generate_field's default branch (src/lfts_simulation.cc:
 * 150-154), drawing from this object's generator after the langevin
 * constructor's draws, as the reference's program does: W- = XbN (U - 0.5),
 * w+ = 0, into w[0, 2M) */
void ref_lgv_uniform_field(ref_lgv *l, double XbN, int M, double *w)
{
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (int r = 0; r < M; r++) {
        w[r] = XbN * (u(l->rng) - 0.5);
        w[r + M] = 0.0;
    }
}

void ref_sys_full_step(ref_sys *s, ref_lgv *l, double XbN, double sigma, double dt, double *w, int *K,
                       double *lnQ)
{
    l->lgv->step_wm(w, l->rng, XbN, sigma, dt);
    *K = s->am->mix(s->dbc.get(), 200, 1e-4, w);
    *lnQ = s->dbc->calc_concs(w);
}

void ref_set_threads(int n)
{
    fftw_init_threads();
    fftw_plan_with_nthreads(n);
}

/* ---- whole simulation ----------------------------------------------------- */
struct ref_sim {
    std::unique_ptr<lfts_simulation> sim;
};

static std::streambuf *g_saved_cout = nullptr;
static std::ostringstream g_sink;

void ref_quiet(int on)
{
    if (on && !g_saved_cout) g_saved_cout = std::cout.rdbuf(g_sink.rdbuf());
    if (!on && g_saved_cout) { std::cout.rdbuf(g_saved_cout); g_saved_cout = nullptr; }
    g_sink.str("");
}

/* Runs the reference constructor (src/lfts_simulation.cc:8-57) on inputFile;
 * it writes w_0/phi_0 into the current directory. */
ref_sim *ref_sim_create(const char *inputFile)
{
    ref_sim *r = new ref_sim;
    r->sim = std::make_unique<lfts_simulation>(std::string(inputFile));
    return r;
}

void ref_sim_destroy(ref_sim *r) { delete r; }

int ref_sim_M(ref_sim *r) { return r->sim->M_; }

void ref_sim_params(ref_sim *r, double *out /* XbN, XeN, sigma, C*V, dt */, int *iout /* N NA m0 m1 m2 equil sim sample save loadType */)
{
    lfts_params *P = r->sim->P_.get();
    out[0] = P->XbN(); out[1] = P->XeN(); out[2] = P->sigma(); out[3] = P->n(); out[4] = P->dt();
    iout[0] = P->N(); iout[1] = P->NA(); iout[2] = P->mx(); iout[3] = P->my(); iout[4] = P->mz();
    iout[5] = P->equil_its(); iout[6] = P->sim_its(); iout[7] = P->sample_freq();
    iout[8] = P->save_freq(); iout[9] = P->loadType();
}

void ref_sim_get_w(ref_sim *r, double *out) { std::memcpy(out, r->sim->w_.get(), sizeof(double) * 4 * (size_t)r->sim->M_); }

/* noise arrays of the langevin object: prev (M) then new (M) */
void ref_sim_get_noise(ref_sim *r, double *prev, double *next)
{
    int M = r->sim->M_;
    std::memcpy(prev, r->sim->Langevin_->noise_cpu_prev_, sizeof(double) * M);
    std::memcpy(next, r->sim->Langevin_->noise_cpu_new_, sizeof(double) * M);
}

/* One Langevin step, the body of equilibrate()/statistics().  sample != 0
 * takes an S(k) sample like statistics() does on sample steps. */
void ref_sim_step(ref_sim *r, int sample, int *K, double *lnQ)
{
    lfts_simulation *S = r->sim.get();
    lfts_params *P = S->P_.get();
    S->Langevin_->step_wm(S->w_.get(), S->RNG_, P->XbN(), P->sigma(), P->dt());
    *K = S->AM_->mix(S->dbc_.get(), 200, 1e-4, S->w_.get());
    *lnQ = S->dbc_->calc_concs(S->w_.get());
    if (sample) S->Sk_->sample(S->w_.get());
}

double ref_sim_getH(ref_sim *r) { return r->sim->getH(); }

void ref_sim_sk_save(ref_sim *r, const char *fname) { r->sim->Sk_->save(std::string(fname)); }

void ref_sim_sk_raw(ref_sim *r, double *S, int *nsamples)
{
    int Mk = r->sim->P_->Mk();
    std::memcpy(S, r->sim->Sk_->S_.get(), sizeof(double) * Mk);
    *nsamples = r->sim->Sk_->nsamples_;
}

void ref_sim_equilibrate(ref_sim *r) { r->sim->equilibrate(); }
void ref_sim_statistics(ref_sim *r) { r->sim->statistics(); }

/* field_generator::create_lamellar (src/field_generator.h:11-24): the (300)
 * lamellar W- of amplitude amp, w+ = 0, into w[0, 2M) */
void ref_lamellar(double *w, double amp, const int *m_in)
{
    int m[3] = {m_in[0], m_in[1], m_in[2]};
    field_generator::create_lamellar(w, amp, m);
}

/* draws from a fresh mt19937_64(seed) + normal_distribution(0, sigma) */
void ref_normal_stream(unsigned long long seed, double sigma, int n, double *out)
{
    std::mt19937_64 rng;
    rng.seed(seed);
    std::normal_distribution<double> nd(0.0, sigma);
    for (int i = 0; i < n; i++) out[i] = nd(rng);
}

} /* extern "C" */
