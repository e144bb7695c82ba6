// cushg_main.cpp — command-line drop-in for the reference program (src/cuSHG.cu:27-113).
//
//   cushg <power W> <waist um> <oven temperature C> <save_only_last 0|1> <save_temperature 0|1>
//         [--nx N] [--nz NZ] [--lx um] [--ly um] [--lz um] [--focus um] [--waist-y um] [--t-inf C]
//         [--deff um/V] [--period um] [--alpha-p 1/um] [--alpha-s 1/um] [--beta-s um/W]
//         [--rho-p rad] [--rho-s rad] [--kappa W/(um K)] [--h-conv W/(um^2 K)] [--lambda um]
//         [--thermal] [--precision 32|64] [--boundary top-open|oven-surrounded] [--crystal spplt|ppln]
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
//
//   cushg --sweep <powers> <waists> <oven temperatures> <save_only_last> <save_temperature> [options]
//
// is the sweep script src/cuSHG.sh:43-105: the three comma-separated lists play ARG1, ARG2
// and ARG3, every combination is a run, and each run's files go into the script's folder
// sPPLT_P_<power>_W_T1_<temperature>_WAIST_<waist>/ with its report in <folder>/<folder>.txt.
// Runs that keep only the last slice go through one batched call: shg_solve_batch for plain
// runs, shg_thermal_batch for thermal runs (their outer iterations in lockstep; if the batch
// does not fit in device memory the points run one after another).  With every slice kept,
// the points run one after another.
#include <sys/stat.h>
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

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
                 "<save_temperature 0|1> [options]\n"
                 "       cushg --sweep <powers> <waists> <oven temperatures> <save_only_last 0|1> "
                 "<save_temperature 0|1> [options]   (comma-separated lists)\n";
    return 2;
}

// The run's report line (the stdout of the reference's run).
std::string report(const shg_params& p, const shg_stats& st) {
    std::ostringstream o;
    o << "SH power = " << std::setprecision(12) << st.sh_power << " W, pump power = " << st.pump_power
      << " W, steps = " << st.steps;
    if (p.thermal) o << ", Jacobi sweeps = " << st.jacobi_sweeps << ", outer iterations = " << st.outer_iterations;
    o << ", device time = " << st.device_ms << " ms";
    return o.str();
}

// One run; its files go to directory prefix `dir` ("" or "<folder>/").
template <typename R>
int run(const shg_params& p, bool save_only_last, bool save_temperature, const std::string& dir, std::string* line) {
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
        save_complex(pump.data(), p.nx, p.ny, dir + "Pump_out");
        save_complex(sig.data(), p.nx, p.ny, dir + "Signal_out");
    } else {
        for (int s = 0; s < p.nz; ++s) {
            save_complex(pump.data() + 2 * plane * s, p.nx, p.ny, dir + "Pump_" + std::to_string(s));
            save_complex(sig.data() + 2 * plane * s, p.nx, p.ny, dir + "Signal_" + std::to_string(s));
        }
    }
    if (!T.empty()) save_tensor(T.data(), p.nx, p.ny, p.nz, dir + "Tfinal");
    *line = report(p, st);
    return 0;
}

// The thermal points of a sweep that keeps only the last slice, as one shg_thermal_batch call
// on device buffers; each point's files as run() writes them.  Returns 0, 1 on an error, or -1
// when the batch's buffers or workspace do not fit in device memory (the caller then runs the
// points one by one).
template <typename R>
int thermal_sweep_batch(const std::vector<shg_params>& ps, const std::vector<std::string>& dirs, bool save_temperature,
                        std::vector<std::string>* lines) {
    const size_t n = ps.size();
    const shg_params& p0 = ps[0];
    const size_t plane = (size_t)p0.nx * p0.ny, vol = plane * p0.nz;
    std::vector<void*> bufs;
    auto release = [&]() {
        for (void* b : bufs) cudaFree(b);
        bufs.clear();
    };
    auto alloc = [&](size_t bytes, void** out) {
        if (cudaMalloc(out, bytes) != cudaSuccess) {
            cudaGetLastError();  // clear the allocation error; the caller falls back
            return false;
        }
        bufs.push_back(*out);
        return true;
    };
    std::vector<void*> pp(n, nullptr), sp(n, nullptr), tp(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
        if (!alloc(2 * sizeof(R) * plane, &pp[i]) || !alloc(2 * sizeof(R) * plane, &sp[i]) ||
            (save_temperature && !alloc(sizeof(R) * vol, &tp[i]))) {
            release();
            return -1;
        }
    }
    std::vector<shg_stats> st(n);
    const shg_status rc = shg_thermal_batch(ps.data(), (int32_t)n, pp.data(), sp.data(),
                                            save_temperature ? tp.data() : nullptr, st.data(), nullptr, nullptr);
    if (rc == SHG_ERR_NOMEM) {
        release();
        return -1;
    }
    if (rc != SHG_OK) {
        std::cerr << "cushg: " << shg_status_string(rc) << ": " << shg_last_error() << std::endl;
        release();
        return 1;
    }
    std::vector<R> pump(2 * plane), sig(2 * plane), T(save_temperature ? vol : 0);
    for (size_t i = 0; i < n; ++i) {
        if (cudaMemcpy(pump.data(), pp[i], 2 * sizeof(R) * plane, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(sig.data(), sp[i], 2 * sizeof(R) * plane, cudaMemcpyDeviceToHost) != cudaSuccess ||
            (save_temperature && cudaMemcpy(T.data(), tp[i], sizeof(R) * vol, cudaMemcpyDeviceToHost) != cudaSuccess)) {
            std::cerr << "cushg: copying the results back failed" << std::endl;
            release();
            return 1;
        }
        save_complex(pump.data(), p0.nx, p0.ny, dirs[i] + "Pump_out");
        save_complex(sig.data(), p0.nx, p0.ny, dirs[i] + "Signal_out");
        if (save_temperature) save_tensor(T.data(), p0.nx, p0.ny, p0.nz, dirs[i] + "Tfinal");
        (*lines)[i] = report(ps[i], st[i]) + " (batched thermal sweep of " + std::to_string(n) + " runs)";
    }
    release();
    return 0;
}

// Options after the positional arguments: the reference's compile-time constants
// (src/cuSHG.cu:11-13, src/headers/Crystal.h:19-52).  Returns 0 or the usage status.
int parse_options(int argc, char** argv, int first, shg_params& p) {
    bool focus_given = false;
    for (int i = first; i < argc; ++i) {
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
        } else if (a == "--crystal") {
            if (i + 1 >= argc) return usage();
            const std::string b = argv[++i];
            if (b != "spplt" && b != "ppln") {
                std::cerr << "cushg: --crystal takes spplt or ppln" << std::endl;
                return usage();
            }
            p.crystal = b == "ppln" ? SHG_CRYSTAL_MGO_PPLN : SHG_CRYSTAL_MGO_SPPLT;
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
    return 0;
}

std::vector<std::string> split(const std::string& s) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ','))
        if (!item.empty()) out.push_back(item);
    return out;
}

void time_record(const shg_params& p, double el) {
    std::ofstream tf("GPUTime_NZ_" + std::to_string(p.nz) + "_N_" + std::to_string(p.nx) + "_T.txt", std::ios::app);
    if (tf.is_open()) tf << el << std::endl;
}

// The sweep of src/cuSHG.sh:58-105: every (power, waist, temperature) combination, in the
// script's loop order, each run's files in its folder.
int sweep(int argc, char** argv) {
    if (argc < 7) return usage();
    const std::vector<std::string> powers = split(argv[2]), waists = split(argv[3]), temps = split(argv[4]);
    const bool save_only_last = std::atoi(argv[5]) != 0;
    const bool save_temperature = std::atoi(argv[6]) != 0;
    shg_params base;
    shg_default_params(&base);
    if (int rc = parse_options(argc, argv, 7, base)) return rc;
    struct Point { shg_params p; std::string folder; };
    std::vector<Point> pts;
    for (const auto& P : powers)
        for (const auto& W : waists)
            for (const auto& T : temps) {
                shg_params q = base;
                q.power = std::atof(P.c_str());
                q.waist = std::atof(W.c_str());
                q.temp = q.t_peltier = std::atof(T.c_str());
                pts.push_back({q, "sPPLT_P_" + P + "_W_T1_" + T + "_WAIST_" + W});  // cuSHG.sh:81
            }
    const double t0 = seconds();
    std::vector<std::string> lines(pts.size());
    if (save_only_last && !base.thermal) {
        // one batched call for the whole sweep
        const size_t n = pts.size();
        const size_t plane = 2 * (size_t)base.nx * base.ny;
        const bool f32 = base.precision == 32;
        std::vector<double> pd(f32 ? 0 : 2 * n * plane);
        std::vector<float> pf(f32 ? 2 * n * plane : 0);
        std::vector<shg_params> ps(n);
        std::vector<void*> pp(n), sp(n);
        for (size_t i = 0; i < n; ++i) {
            ps[i] = pts[i].p;
            pp[i] = f32 ? (void*)(pf.data() + 2 * i * plane) : (void*)(pd.data() + 2 * i * plane);
            sp[i] = f32 ? (void*)(pf.data() + (2 * i + 1) * plane) : (void*)(pd.data() + (2 * i + 1) * plane);
        }
        std::vector<double> power(n);
        shg_status rc = shg_solve_batch(ps.data(), (int32_t)n, pp.data(), sp.data(), power.data());
        if (rc != SHG_OK) {
            std::cerr << "cushg: " << shg_status_string(rc) << ": " << shg_last_error() << std::endl;
            return 1;
        }
        for (size_t i = 0; i < n; ++i) {
            mkdir(pts[i].folder.c_str(), 0755);
            const std::string dir = pts[i].folder + "/";
            if (f32) {
                save_complex((const float*)pp[i], base.nx, base.ny, dir + "Pump_out");
                save_complex((const float*)sp[i], base.nx, base.ny, dir + "Signal_out");
            } else {
                save_complex((const double*)pp[i], base.nx, base.ny, dir + "Pump_out");
                save_complex((const double*)sp[i], base.nx, base.ny, dir + "Signal_out");
            }
            std::ostringstream o;
            o << "SH power = " << std::setprecision(12) << power[i] << " W (batched sweep of " << n << " runs)";
            lines[i] = o.str();
        }
    } else {
        int batched = -1;
        if (save_only_last && base.thermal && !pts.empty()) {
            std::vector<shg_params> ps;
            std::vector<std::string> dirs;
            for (const Point& pt : pts) {
                mkdir(pt.folder.c_str(), 0755);
                ps.push_back(pt.p);
                dirs.push_back(pt.folder + "/");
            }
            batched = base.precision == 32 ? thermal_sweep_batch<float>(ps, dirs, save_temperature, &lines)
                                           : thermal_sweep_batch<double>(ps, dirs, save_temperature, &lines);
            if (batched > 0) return batched;
        }
        for (size_t i = 0; batched != 0 && i < pts.size(); ++i) {
            mkdir(pts[i].folder.c_str(), 0755);
            const int rc = base.precision == 32
                               ? run<float>(pts[i].p, save_only_last, save_temperature, pts[i].folder + "/", &lines[i])
                               : run<double>(pts[i].p, save_only_last, save_temperature, pts[i].folder + "/", &lines[i]);
            if (rc) return rc;
        }
    }
    const double el = seconds() - t0;
    for (size_t i = 0; i < pts.size(); ++i) {
        const Point& pt = pts[i];
        std::ofstream f(pt.folder + "/" + pt.folder + ".txt");
        f << "Power = " << pt.p.power << " W, beam waist = " << pt.p.waist << " um, oven temperature = " << pt.p.temp
          << " C\n" << lines[i] << "\n";
        std::cout << pt.folder << ": " << lines[i] << std::endl;
    }
    std::cout << "time elapsed " << el << " seconds for " << pts.size() << " runs" << std::endl;
    time_record(base, el);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc >= 2 && std::string(argv[1]) == "--sweep") return sweep(argc, argv);
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
    if (int rc = parse_options(argc, argv, 6, p)) return rc;
    std::cout << "Pump power = " << p.power << " W, beam waist = " << p.waist << " um, focal distance = " << p.focus
              << " um, oven temperature = " << p.temp << " C, grid = " << p.nx << " x " << p.ny << " x " << p.nz
              << (p.thermal ? ", thermal" : "") << std::endl;
    const double t0 = seconds();
    std::string line;
    const int rc = p.precision == 32 ? run<float>(p, save_only_last, save_temperature, "", &line)
                                     : run<double>(p, save_only_last, save_temperature, "", &line);
    if (rc != 0) return rc;
    std::cout << line << std::endl;
    const double el = seconds() - t0;
    std::cout << "time elapsed " << el << " seconds" << std::endl;
    time_record(p, el);
    return 0;
}
