// Host-side helpers of the C ABI with the reference driver's semantics:
// input parsing and chi conversion (src/lfts_params.cc), the random number
// stream (src/langevin.cc, src/lfts_simulation.cc) and the initial fields
// (src/field_generator.h).  No CUDA here.
#include <cmath>
#include <fstream>
#include <random>
#include <string>

#include "../../include/lfts_b200.h"

struct lfts_rng {
    std::mt19937_64 eng;
    std::normal_distribution<double> normal;
};

extern "C" {

// z_inf of the discrete Gaussian chain on the mesh (src/lfts_params.cc:122-142):
// the same terms in the same order and the same variable roles (R0dL, ell,
// the t-sum, the tail correction), so that chi_b N comes out bit for bit equal
// to the reference's for the same input header.
double lfts_z_inf_discrete(const double L[3], const int m[3], int N, double Nbar, int tmax)
{
    const double pi = 3.14159265358979323846;
    double R0 = std::sqrt((double)N), R0dL[3], prod = 1.0;
    for (int i = 0; i < 3; i++) {
        R0dL[i] = R0 * L[i] / m[i];
        prod *= R0dL[i];
    }
    const double ell = std::pow(prod, 1.0 / 3.0);
    double sum = 0.5, X;
    for (int t = 1; t <= tmax; t++) {
        X = (pi / ell) * std::sqrt(t / 6.0);
        double p = 1.0;
        for (int i = 0; i < 3; i++) p *= std::erf(X * ell / R0dL[i]);
        sum += std::pow(std::sqrt(pi) / (2 * X), 3.0) * p;
    }
    sum *= 2 * R0 / (std::pow(ell, 3.0) * std::sqrt(Nbar));
    X = (pi / ell) * std::sqrt((0.5 + tmax) / 6.0);
    return 1.0 - sum - 3 * R0 / (ell * std::sqrt(pi * Nbar) * X);
}

int lfts_read_input(const char *path, lfts_input *o)
{
    if (!path || !o) return LFTS_ERR_ARG;
    std::ifstream in(path);
    if (!in) return LFTS_ERR_ARG;
    lfts_input v{};
    in >> v.N >> v.NA >> v.XN_in >> v.C >> v.dt >> v.isXeN;
    in >> v.m[0] >> v.m[1] >> v.m[2] >> v.L[0] >> v.L[1] >> v.L[2];
    in >> v.equil_its >> v.sim_its >> v.sample_freq >> v.save_freq >> v.loadType;
    if (!in || v.sample_freq <= 0) return LFTS_ERR_ARG;
    v.equil_its = (v.equil_its / v.sample_freq) * v.sample_freq;
    v.sim_its = (v.sim_its / v.sample_freq) * v.sample_freq;
    const double z_inf = lfts_z_inf_discrete(v.L, v.m, v.N, v.C * v.C, 100);
    if (v.isXeN == 1) {
        v.XeN = v.XN_in;
        v.XbN = v.XN_in / z_inf;
    } else {
        v.XbN = v.XN_in;
        v.XeN = v.XN_in * z_inf;
    }
    v.M = (long long)v.m[0] * v.m[1] * v.m[2];
    v.Mk = (long long)v.m[0] * v.m[1] * (v.m[2] / 2 + 1);
    v.V = v.L[0] * v.L[1] * v.L[2];
    v.sigma = std::sqrt(2.0 * v.M * v.dt / (v.C * v.V));
    v.NB = v.N - v.NA;
    *o = v;
    return LFTS_OK;
}

void lfts_params_from_input(const lfts_input *in, lfts_params *p)
{
    p->N = in->N;
    p->NA = in->NA;
    p->XbN = in->XbN;
    p->C = in->C;
    p->dt = in->dt;
    for (int d = 0; d < 3; d++) {
        p->m[d] = in->m[d];
        p->L[d] = in->L[d];
    }
}

int lfts_rng_create(unsigned long long seed, double sigma, lfts_rng **out)
{
    if (!out) return LFTS_ERR_ARG;
    lfts_rng *r = new lfts_rng;
    r->eng.seed(seed);
    r->normal = std::normal_distribution<double>(0.0, sigma);
    *out = r;
    return LFTS_OK;
}

int lfts_rng_destroy(lfts_rng *r)
{
    delete r;
    return LFTS_OK;
}

int lfts_rng_normal(lfts_rng *r, long long n, double *out)
{
    if (!r || (!out && n > 0)) return LFTS_ERR_ARG;
    for (long long i = 0; i < n; i++) out[i] = r->normal(r->eng);
    return LFTS_OK;
}

int lfts_rng_uniform(lfts_rng *r, long long n, double *out)
{
    if (!r || (!out && n > 0)) return LFTS_ERR_ARG;
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (long long i = 0; i < n; i++) out[i] = u(r->eng);
    return LFTS_OK;
}

int lfts_lamellar_field(double *w, double amplitude, const int m[3], int kx, int ky, int kz)
{
    if (!w || !m) return LFTS_ERR_ARG;
    const long long M = (long long)m[0] * m[1] * m[2];
    const double two_pi = 2.0 * 3.14159265358979323846;
    for (int x = 0; x < m[0]; x++)
        for (int y = 0; y < m[1]; y++)
            for (int z = 0; z < m[2]; z++) {
                const long long r = (long long)m[2] * ((long long)x * m[1] + y) + z;
                w[r] = amplitude * std::cos(two_pi * (kx * ((double)x) / m[0] + ky * ((double)y) / m[1] +
                                                      kz * ((double)z) / m[2]));
                w[r + M] = 0.0;
            }
    return LFTS_OK;
}

int lfts_random_field(lfts_rng *r, double *w, double XbN, long long M)
{
    if (!r || !w) return LFTS_ERR_ARG;
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (long long i = 0; i < M; i++) {
        w[i] = XbN * (u(r->eng) - 0.5);
        w[i + M] = 0.0;
    }
    return LFTS_OK;
}

}  // extern "C"
