// cushg_main.cpp — command-line drop-in for the reference program (src/cuSHG.cu:27-113).
//
//   cushg <power W> <waist um> <oven temperature C> <save_only_last 0|1> <save_temperature 0|1>
//         [--nx N] [--nz NZ] [--lx um] [--ly um] [--lz um] [--focus um] [--waist-y um] [--t-inf C]
//         [--deff um/V] [--period um] [--alpha-p 1/um] [--alpha-s 1/um] [--beta-s um/W]
//         [--rho-p rad] [--rho-s rad] [--kappa W/(um K)] [--h-conv W/(um^2 K)] [--lambda um]
//         [--thermal] [--precision 32|64] [--boundary top-open|oven-surrounded]
//         [--max-outer N] [--check-every N] [--tol value] [--conv reference|maxabs]
//
// The five positional arguments are the reference's argv (src/cuSHG.cu:46-58); the options
// replace its compile-time constants (src/cuSHG.cu:11-13, src/headers/Crystal.h:19-52), with
// the reference's values as defaults.  Outputs are the reference's files in the working
// directory: Pump_out_{r,i}.dat and Signal_out_{r,i}.dat (save_only_last = 1) or
// Pump_<s>_{r,i}.dat / Signal_<s>_{r,i}.dat for every slice (save_only_last = 0), NY rows of
// NX tab-separated values at 20 significant digits (src/headers/Files.h:69-90); Tfinal_<z>.dat
// per z plane for thermal runs with save_temperature = 1 (Files.h:169-188); and the elapsed
// time appended to GPUTime_NZ_<NZ>_N_<NX>_T.txt (src/cuSHG.cu:90-107).
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "../../../include/shg.h"

namespace {

double seconds() {
    struct timeval tp;
    gettimeofday(&tp, nullptr);
    return (double)tp.tv_sec + (double)tp.tv_usec * 1.e-6;
}

template <typename C>
void save_complex(const C* a, int nx, int ny, const std::string& name) {
    for (int part = 0; part < 2; ++part) {
        std::ofstream f(name + (part ? "_i.dat" : "_r.dat"));
        for (int y = 0; y < ny; ++y) {
            for (int x = 0; x < nx; ++x) f << std::setprecision(20) << a[2 * ((size_t)y * nx + x) + part] << "\t";
            f << "\n";
        }
    }
}

template <typename R>
void save_tensor(const R* t, int nx, int ny, int nz, const std::string& name) {
    for (int z = 0; z < nz; ++z) {
        std::ofstream f(name + "_" + std::to_string(z) + ".dat");
        for (int y = 0; y < ny; ++y) {
            for (int x = 0; x < nx; ++x) f << t[((size_t)z * ny + y) * nx + x] << "\t";
            f << "\n";
        }
    }
}

int usage() {
    std::cerr << "usage: cushg <power W> <waist um> <oven temperature C> <save_only_last 0|1> "
                 "<save_temperature 0|1> [options]\n";
    return 2;
}

template <typename R>
int run(const shg_params& p, bool save_only_last, bool save_temperature) {
    const size_t plane = (size_t)p.nx * p.ny;
    const size_t planes = save_only_last ? 1 : (size_t)p.nz;
    std::vector<R> pump(2 * plane * planes), sig(2 * plane * planes);
    std::vector<R> T((p.thermal && save_temperature) ? plane * p.nz : 0);
    shg_stats st;
    void* tptr = T.empty() ? nullptr : T.data();
    shg_status rc = save_only_last ? shg_solve(&p, nullptr, pump.data(), sig.data(), tptr, &st)
                                   : shg_solve_slices(&p, nullptr, pump.data(), sig.data(), tptr, &st);
    if (rc != SHG_OK) {
        std::cerr << "cushg: " << shg_status_string(rc) << ": " << shg_last_error() << std::endl;
        return 1;
    }
    if (save_only_last) {
        save_complex(pump.data(), p.nx, p.ny, "Pump_out");
        save_complex(sig.data(), p.nx, p.ny, "Signal_out");
    } else {
        for (int s = 0; s < p.nz; ++s) {
            save_complex(pump.data() + 2 * plane * s, p.nx, p.ny, "Pump_" + std::to_string(s));
            save_complex(sig.data() + 2 * plane * s, p.nx, p.ny, "Signal_" + std::to_string(s));
        }
    }
    if (!T.empty()) save_tensor(T.data(), p.nx, p.ny, p.nz, "Tfinal");
    std::cout << "SH power = " << std::setprecision(12) << st.sh_power << " W, pump power = " << st.pump_power
              << " W, steps = " << st.steps;
    if (p.thermal) std::cout << ", Jacobi sweeps = " << st.jacobi_sweeps << ", outer iterations = " << st.outer_iterations;
    std::cout << ", device time = " << st.device_ms << " ms" << std::endl;
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 6) return usage();
    shg_params p;
    shg_default_params(&p);
    // positional argv of src/cuSHG.cu:46-58
    p.power = std::atof(argv[1]);
    p.waist = std::atof(argv[2]);
    p.temp = std::atof(argv[3]);
    p.t_peltier = std::atof(argv[3]);
    const bool save_only_last = std::atoi(argv[4]) != 0;
    const bool save_temperature = std::atoi(argv[5]) != 0;
    bool focus_given = false;
    for (int i = 6; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&](double& dst) {
            if (i + 1 >= argc) { usage(); std::exit(2); }
            dst = std::atof(argv[++i]);
        };
        auto ival = [&](int32_t& dst) {
            if (i + 1 >= argc) { usage(); std::exit(2); }
            dst = std::atoi(argv[++i]);
        };
        if (a == "--nx") { ival(p.nx); p.ny = p.nx; }
        else if (a == "--nz") ival(p.nz);
        else if (a == "--lx") val(p.lx);
        else if (a == "--ly") val(p.ly);
        else if (a == "--lz") val(p.lz);
        else if (a == "--focus") { val(p.focus); focus_given = true; }
        else if (a == "--waist-y") val(p.waist_y);
        else if (a == "--t-inf") val(p.t_inf);
        else if (a == "--deff") val(p.deff);
        else if (a == "--period") val(p.period);
        else if (a == "--alpha-p") val(p.alpha_p);
        else if (a == "--alpha-s") val(p.alpha_s);
        else if (a == "--beta-s") val(p.beta_s);
        else if (a == "--rho-p") val(p.rho_p);
        else if (a == "--rho-s") val(p.rho_s);
        else if (a == "--kappa") val(p.kappa);
        else if (a == "--h-conv") val(p.h_conv);
        else if (a == "--lambda") val(p.lambda_p);
        else if (a == "--thermal") p.thermal = 1;
        else if (a == "--precision") ival(p.precision);
        else if (a == "--max-outer") ival(p.max_outer);
        else if (a == "--check-every") ival(p.check_every);
        else if (a == "--tol") val(p.jacobi_tol);
        else if (a == "--boundary") {
            if (i + 1 >= argc) return usage();
            const std::string b = argv[++i];
            p.boundary = b == "oven-surrounded" ? SHG_BOUNDARY_OVEN_SURROUNDED : SHG_BOUNDARY_TOP_OPEN;
        } else if (a == "--conv") {
            if (i + 1 >= argc) return usage();
            const std::string b = argv[++i];
            p.conv_rule = b == "maxabs" ? SHG_CONV_MAXABS : SHG_CONV_REFERENCE;
        } else {
            std::cerr << "cushg: unknown option " << a << std::endl;
            return usage();
        }
    }
    if (!focus_given) p.focus = 0.5 * p.lz;  // src/cuSHG.cu:48
    std::cout << "Pump power = " << p.power << " W, beam waist = " << p.waist << " um, focal distance = " << p.focus
              << " um, oven temperature = " << p.temp << " C, grid = " << p.nx << " x " << p.ny << " x " << p.nz
              << (p.thermal ? ", thermal" : "") << std::endl;
    const double t0 = seconds();
    const int rc = p.precision == 32 ? run<float>(p, save_only_last, save_temperature)
                                     : run<double>(p, save_only_last, save_temperature);
    if (rc != 0) return rc;
    const double el = seconds() - t0;
    std::cout << "time elapsed " << el << " seconds" << std::endl;
    std::ofstream tf("GPUTime_NZ_" + std::to_string(p.nz) + "_N_" + std::to_string(p.nx) + "_T.txt", std::ios::app);
    if (tf.is_open()) tf << el << std::endl;
    return 0;
}
