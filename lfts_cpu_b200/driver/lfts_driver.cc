// lfts-b200: the drop-in L-FTS program.  Same command line, input file, stdout
// and output files (w_*, phi_*, struct_st_*) as the reference program
// (src/fts_cpu.cc + src/lfts_simulation.cc), with every hot-path call going
// through the C ABI in include/lfts_b200.h to the B200 kernels.
//
//     lfts-b200 <input_file> [--fp32]
//
// --fp32 (or LFTS_PRECISION=fp32) selects the FP32-mixed path; default FP64.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

#include "lfts_b200.h"

namespace {

void die_on(int status, const char *what)
{
    if (status == LFTS_ERR_NOTCONV) {
        // the reference carries on silently when anderson::mix reaches its
        // cap; the run goes on here too, with a note on stderr (stdout and the
        // output files stay the reference program's)
        std::cerr << "lfts-b200: " << what << ": " << lfts_status_string(status) << " (continuing)" << std::endl;
        return;
    }
    if (status != LFTS_OK) {
        std::cerr << "lfts-b200: " << what << ": " << lfts_status_string(status);
        const char *e = lfts_last_error_string();
        if (e && *e) std::cerr << " (" << e << ")";
        std::cerr << std::endl;
        std::exit(2);
    }
}

// One double per line with the stream's default 6 significant digits
// (src/file_IO.h:31-37).
void write_values(const std::string &path, const double *v, long long n, bool append)
{
    std::ofstream out(path, append ? std::ios_base::app : std::ios_base::out);
    for (long long i = 0; i < n; i++) out << v[i] << '\n';
}

class Simulation {
  public:
    explicit Simulation(const std::string &input, int precision) : input_(input)
    {
        std::ifstream probe(input);
        if (input.empty() || probe.fail()) {
            std::cout << "ERROR => Cannot open one of the input files." << std::endl;
            std::exit(1);
        }
        std::cout << "Creating lfts_params object..." << std::endl;
        die_on(lfts_read_input(input.c_str(), &in_), "reading the input header");
        print_params();
        M_ = in_.M;
        w_.assign(4 * M_, 0.0);
        eta_.assign(M_, 0.0);
        die_on(lfts_rng_create(123456789ULL, in_.sigma, &rng_), "rng");

        lfts_params p;
        lfts_params_from_input(&in_, &p);
        std::cout << "Creating diblock object..." << std::endl;
        die_on(lfts_create(&p, precision, 0, &ctx_), "creating the GPU context");
        std::cout << "Creating anderson object..." << std::endl;
        std::cout << "Creating langevin object..." << std::endl;
        // the langevin constructor's M draws precede the field generation
        die_on(lfts_rng_normal(rng_, M_, eta_.data()), "rng");
        die_on(lfts_langevin_init(ctx_, eta_.data()), "langevin init");

        if (in_.loadType == 1) {
            std::cout << "Loading input field..." << std::endl;
            read_fields();
        } else if (in_.loadType == 2) {
            die_on(lfts_lamellar_field(w_.data(), in_.XbN, in_.m, 3, 0, 0), "lamellar field");
        } else {
            die_on(lfts_random_field(rng_, w_.data(), in_.XbN, M_), "random field");
        }
        die_on(lfts_set_fields(ctx_, w_.data()), "set fields");
        int k = 0;
        die_on(lfts_anderson_mix(ctx_, 200, 1e-4, &k), "anderson mix");
        fetch();
        save_fields("w_0");
        write_values("phi_0", w_.data() + 2 * M_, 2 * M_, false);
    }

    ~Simulation()
    {
        lfts_destroy(ctx_);
        lfts_rng_destroy(rng_);
    }

    void equilibrate()
    {
        int it;
        for (it = 1; it <= in_.equil_its; it++) {
            step();
            if (it % in_.save_freq == 0) save_pair("eq", it);
        }
        save_pair("eq", it - 1);
    }

    void statistics()
    {
        int it;
        for (it = 1; it <= in_.sim_its; it++) {
            step();
            if (it % in_.sample_freq == 0) die_on(lfts_sk_sample(ctx_), "S(k) sample");
            if (it % in_.save_freq == 0) {
                save_pair("st", it);
                save_struct("struct_st_" + std::to_string(it));
            }
        }
        save_pair("st", it - 1);
        save_struct("struct_st_" + std::to_string(it - 1));
    }

    double H()
    {
        double h = 0.0;
        die_on(lfts_get_H(ctx_, &h), "H");
        return h;
    }

  private:
    // step_wm, mix, then the extra calc_concs whose ln Q is printed
    // (src/lfts_simulation.cc:69-76)
    void step()
    {
        die_on(lfts_rng_normal(rng_, M_, eta_.data()), "rng");
        die_on(lfts_langevin_step(ctx_, eta_.data()), "langevin step");
        int k = 0;
        die_on(lfts_anderson_mix(ctx_, 200, 1e-4, &k), "anderson mix");
        double lnQ = 0.0;
        die_on(lfts_calc_concs(ctx_, &lnQ), "calc_concs");
        std::cout << "lnQ = " << lnQ << std::endl;
    }

    void fetch() { die_on(lfts_get_fields(ctx_, w_.data()), "get fields"); }

    void save_pair(const char *phase, int it)
    {
        fetch();
        save_fields(std::string("w_") + phase + "_" + std::to_string(it));
        write_values(std::string("phi_") + phase + "_" + std::to_string(it), w_.data() + 2 * M_, 2 * M_, false);
    }

    // a file that is again a valid input: header with loadType 1, then W-, w+
    // (src/lfts_params.cc:73-83)
    void save_fields(const std::string &path)
    {
        {
            std::ofstream out(path);
            const double xn = in_.isXeN == 1 ? in_.XeN : in_.XbN;
            out << in_.N << " " << in_.NA << " " << xn << " " << in_.C << " " << in_.dt << " " << in_.isXeN << '\n';
            out << in_.m[0] << " " << in_.m[1] << " " << in_.m[2] << " " << in_.L[0] << " " << in_.L[1] << " "
                << in_.L[2] << '\n';
            out << in_.equil_its << " " << in_.sim_its << " " << in_.sample_freq << " " << in_.save_freq << " " << 1
                << '\n';
        }
        write_values(path, w_.data(), 2 * M_, true);
    }

    // spherically averaged S(k): "K\tS" with 8 decimals (src/strFunc.cc:50-76)
    void save_struct(const std::string &path)
    {
        int ns = 0;
        die_on(lfts_sk_get(ctx_, nullptr, &ns), "S(k)");
        std::ofstream out(path);
        std::vector<double> K(in_.Mk), S(in_.Mk);
        int nb = 0;
        die_on(lfts_sk_bin(ctx_, 1e-5, K.data(), S.data(), &nb), "S(k) bins");
        out.precision(8);
        out.setf(std::ios::fixed, std::ios::floatfield);
        for (int b = 0; b < nb; b++) {
            out << K[b] << "\t";
            if (ns > 0)
                out << S[b];
            else
                out << "-nan";  // what the reference prints after 0/0 on x86
            out << '\n';
        }
    }

    void read_fields()
    {
        std::ifstream f(input_);
        for (int i = 0; i < 3; i++) f.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
        for (long long r = 0; r < 2 * M_; r++) f >> w_[r];
    }

    void print_params()
    {
        std::cout << "N = " << in_.N << std::endl;
        std::cout << "NA = " << in_.NA << std::endl;
        std::cout << "NB = " << in_.NB << std::endl;
        std::cout << "chi_b = " << in_.XbN << std::endl;
        std::cout << "C = " << in_.C << std::endl;
        std::cout << "dt = " << in_.dt << std::endl;
        std::cout << "XeN = " << in_.XeN << std::endl;
        std::cout << "isXeN = " << in_.isXeN << std::endl;
        for (int d = 0; d < 3; d++) std::cout << "m[" << d << "] = " << in_.m[d] << std::endl;
        for (int d = 0; d < 3; d++) std::cout << "L[" << d << "] = " << in_.L[d] << std::endl;
        std::cout << "equil_its = " << in_.equil_its << std::endl;
        std::cout << "sim_its = " << in_.sim_its << std::endl;
        std::cout << "sample_freq = " << in_.sample_freq << std::endl;
        std::cout << "save_freq_ = " << in_.save_freq << std::endl;
        std::cout << "loadType_ = " << in_.loadType << std::endl;
        std::cout << "M_ = " << in_.M << std::endl;
        std::cout << "Mk_ = " << in_.Mk << std::endl;
        std::cout << "V_ = " << in_.V << std::endl;
        std::cout << "sigma_ = " << in_.sigma << std::endl;
    }

    std::string input_;
    lfts_input in_{};
    long long M_ = 0;
    std::vector<double> w_, eta_;
    lfts_rng *rng_ = nullptr;
    lfts_ctx *ctx_ = nullptr;
};

}  // namespace

int main(int argc, char *argv[])
{
    int precision = LFTS_FP64;
    if (const char *e = std::getenv("LFTS_PRECISION"))
        if (std::strcmp(e, "fp32") == 0) precision = LFTS_FP32_MIXED;
    std::string input;
    int nargs = 0;
    for (int i = 1; i < argc; i++) {
        if (std::strcmp(argv[i], "--fp32") == 0)
            precision = LFTS_FP32_MIXED;
        else {
            input = argv[i];
            nargs++;
        }
    }
    if (nargs != 1) {
        std::cout << "Please supply an input file name as first command-line argument." << std::endl << std::endl;
        std::exit(1);
    }
    Simulation sim(input, precision);

    using clk = std::chrono::steady_clock;
    std::cout << "Starting Equilibration..." << std::endl;
    auto t0 = clk::now();
    sim.equilibrate();
    auto secs = std::chrono::duration_cast<std::chrono::seconds>(clk::now() - t0).count();
    std::cout << "Equlibration time = " << secs << "secs" << std::endl << std::endl;

    std::cout << "Starting Statistics..." << std::endl;
    t0 = clk::now();
    sim.statistics();
    secs = std::chrono::duration_cast<std::chrono::seconds>(clk::now() - t0).count();
    std::cout << "Statistics time = " << secs << "secs" << std::endl << std::endl;

    std::cout.precision(6);
    std::cout << sim.H() << std::endl;
    return 0;
}
