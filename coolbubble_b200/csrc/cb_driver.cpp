/* cb_driver.cpp -- coolbubble_gpu: a whole run on the GPU library with the
 * reference program's command line, run folder and output files.
 *
 * Written against the behaviour of the reference's src/main.cpp (options
 * main.cpp:68-139, folder name 243-249, stability check 171-183, snapshot
 * schedule 201-223, loop 274-288) and the writers of src/bubble.cpp
 * (parameters.dat 1018-1032, EnergyDensities.dat 958-989, spectrum files
 * 642-709, FullField.dat 993-1006) and the wall tracking of bubble.cpp:535-634
 * (gamma.dat 1009-1015). The compile-time def.h values become
 * options (--dt, --nbubbles, ...) with def.h's defaults. Snapshots are
 * HDF5 files with OutField's datasets, chunking, filters and attributes
 * (bubble.cpp:887-954), written by the library's own writer (cb_out_field,
 * no libhdf5) in the background while the run steps on. Plots and videos
 * are not made.
 */
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "coolbubble_b200.h"

namespace fs = std::filesystem;

namespace {

struct Options {
    int D = 2, nGrids = 512, nt = 1000, mode = 1, snapshots = 20;
    double L = 32, c = 4.0;
    std::string out = "./";
    /* def.h values (def.h:33-76) */
    double dt = 0.004, trad = 0.2, deltar = 0.0, mpl = 200.0;
    int nbubbles = 5, test = 0, expansion = 0, alpha = 0, memorysave = 0, walltracking = 0;
    int precision = CB_FP64;
    unsigned position_seed = 42;
    unsigned long long thermal_seed = 12345;
};

const int kOutEnergyEvery = 40;    /* def.h:65 */
const int kFull1DFieldEvery = 100; /* def.h:71 */
const int kWallTrackEvery = 400;   /* def.h:73 */

void usage(const char *prog) {
    std::cout << "Usage: " << prog << " [options]\n\n"
              << "  --D <1|2|3>  --L <value>  --nGrids <n>  --nt <n>  --c <value>  --mode <1|0|-1|-2|-3>\n"
              << "  --snapshots <n>  --out <dir>  --no-plots  --python-dir <d>   (as the reference)\n"
              << "  --dt <value> (TIME_STEP, 0.004)  --nbubbles <n> (5)  --trad <T> (0.2)  --deltar <x> (0)\n"
              << "  --test <0|1>  --expansion <0|1>  --alpha <0|1>  --mpl <value> (200)  --memorysave <0|1>\n"
              << "  --wall-tracking <0|1> (WallTracking, 0)\n"
              << "  --precision <fp64|fp32c>  --position-seed <n> (42)  --thermal-seed <n> (12345)\n";
}

/* main.cpp:62-66: a number with `p` decimals, cut from std::to_string */
std::string precistr(double num, int p) {
    const std::string s = std::to_string(num);
    return s.substr(0, s.find(".") + p + 1);
}

bool parse(int argc, char **argv, Options &o) {
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-h" || a == "--help") { usage(argv[0]); std::exit(0); }
        if (a == "--no-plots") continue;
        if (i + 1 >= argc) { std::cerr << "Error: option " << a << " needs a value (see --help)\n"; return false; }
        const std::string v = argv[++i];
        try {
            if (a == "--D") o.D = std::stoi(v);
            else if (a == "--L") o.L = std::stod(v);
            else if (a == "--nGrids") o.nGrids = std::stoi(v);
            else if (a == "--nt") o.nt = std::stoi(v);
            else if (a == "--c") o.c = std::stod(v);
            else if (a == "--mode") o.mode = std::stoi(v);
            else if (a == "--snapshots") o.snapshots = std::stoi(v);
            else if (a == "--out") o.out = v;
            else if (a == "--python-dir") { /* no plots are made */ }
            else if (a == "--dt") o.dt = std::stod(v);
            else if (a == "--nbubbles") o.nbubbles = std::stoi(v);
            else if (a == "--trad") o.trad = std::stod(v);
            else if (a == "--deltar") o.deltar = std::stod(v);
            else if (a == "--test") o.test = std::stoi(v);
            else if (a == "--expansion") o.expansion = std::stoi(v);
            else if (a == "--alpha") o.alpha = std::stoi(v);
            else if (a == "--mpl") o.mpl = std::stod(v);
            else if (a == "--memorysave") o.memorysave = std::stoi(v);
            else if (a == "--wall-tracking") o.walltracking = std::stoi(v);
            else if (a == "--position-seed") o.position_seed = (unsigned)std::stoul(v);
            else if (a == "--thermal-seed") o.thermal_seed = std::stoull(v);
            else if (a == "--precision") {
                if (v == "fp64") o.precision = CB_FP64;
                else if (v == "fp32c") o.precision = CB_FP32C;
                else throw std::invalid_argument(v);
            } else {
                std::cerr << "Error: unknown option " << a << " (see --help)\n";
                return false;
            }
        } catch (const std::exception &) {
            std::cerr << "Error: cannot read the value '" << v << "' of option " << a << "\n";
            return false;
        }
    }
    if (o.D < 1 || o.D > 3) { std::cerr << "Error: --D must be 1, 2 or 3\n"; return false; }
    if (o.nGrids < 2 || o.L <= 0 || o.nt < 1) { std::cerr << "Error: --nGrids, --L and --nt must be positive\n"; return false; }
    if (o.mode < -3 || o.mode > 1) { std::cerr << "Error: --mode must be between -3 and 1\n"; return false; }
    if (o.snapshots < 1) { std::cerr << "Error: --snapshots must be at least 1\n"; return false; }
    return true;
}

/* main.cpp:201-223 with SnapshotSpacing = 0: evenly spaced in time */
std::vector<int> schedule(const Options &o) {
    const double T = o.nt * o.dt;
    std::vector<int> steps;
    for (int k = 1; k <= o.snapshots; ++k) {
        const double time = T * k / o.snapshots;
        const int step = std::min(o.nt, std::max(1, (int)std::lround(time / o.dt)));
        if (steps.empty() || step > steps.back()) steps.push_back(step);
    }
    return steps;
}

std::string four(int n) {
    char b[16];
    std::snprintf(b, sizeof b, "%04d", n);
    return b;
}

/* Wall of the tracked bubble (bubble.hpp:89-90; bubble.cpp:164-168, 309-313). */
struct Wall {
    double dini = 0, width = 0, rmin = 0, rmax = 0;
    double rn = 0, lw = 0, phi_zero = 0, phi_max = 0, mT = 0;
    int centre[3] = {0, 0, 0};
};

struct Run {
    Options o;
    std::string folder;
    cb_handle *h = nullptr;
    cb_sums line{};
    double DeltaV = 1.0;
    size_t N = 0;
    Wall wall;
    std::string writing;   /* the snapshot whose write is in flight */
    bool fail(int st, const char *what) {
        std::cerr << "Error: " << what << ": " << cb_last_error(h) << " (" << cb_status_string(st) << ")\n";
        return false;
    }
};

/* bubble.cpp:958-973 */
void init_energy_file(const Run &r) {
    FILE *fp = std::fopen((r.folder + "/EnergyDensities.dat").c_str(), "w");
    if (!fp) throw std::runtime_error("Could not open EnergyDensities.dat for writing");
    std::fprintf(fp, "# c and DeltaV are: %.2f %.4f \n", r.o.c, r.DeltaV);
    std::fprintf(fp, "# columns: 1 t, 2 a, 3 Etot, 4 Ekin, 5 Egrad, 6 Epot, 7-10 spread of Etot/Ekin/Egrad/Epot,\n");
    std::fprintf(fp, "#          11 <phi>, 12 spread of <phi>, 13 <phi'>, 14 spread of <phi'>, 15 H, 16 Hubble constraint C = H^2 - rho/(3 Mpl^2)\n");
    std::fclose(fp);
    /* bubble.cpp:967-973 */
    if (r.o.walltracking == 1) {
        fp = std::fopen((r.folder + "/gamma.dat").c_str(), "w");
        if (!fp) throw std::runtime_error("Could not open gamma.dat for writing");
        std::fprintf(fp, "#t, gamma factor, wall width, rmin, rmax\n");
        std::fclose(fp);
    }
}

/* bubble.cpp:977-989: one line of the box averages */
void energy_line(const Run &r, const cb_sums &s) {
    FILE *fp = std::fopen((r.folder + "/EnergyDensities.dat").c_str(), "a");
    if (!fp) return;
    std::fprintf(fp, "%.6e %.10e %.12e %.12e %.12e %.12e %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.8e %.8e\n", s.t, s.a,
                 s.etot, s.ekin, s.egrad, s.epot, std::sqrt(s.etot_var), std::sqrt(s.ekin_var), std::sqrt(s.egrad_var),
                 std::sqrt(s.epot_var), s.avphi, std::sqrt(s.avphi_var), s.avphip, std::sqrt(s.avphip_var), s.H, s.C);
    std::fclose(fp);
}

/* bubble.cpp:1018-1032 */
void parameters_file(const Run &r) {
    const Options &o = r.o;
    const double dx = o.L / o.nGrids;
    const double rn = o.D == 3 ? 0.823 * std::pow(o.c, 0.203) * 1.3 : 0.823 * std::pow(o.c, 0.203);
    const double kUV = std::sqrt(double(o.D)) * M_PI / dx;
    const double kIR = 2 * M_PI / double(o.L);
    const double kRStar = std::sqrt(double(o.D)) * 4 * M_PI / (double(o.L - 2 * rn));
    const double kMeff = std::sqrt(2 * (o.c + 6));
    FILE *fp = std::fopen((r.folder + "/parameters.dat").c_str(), "w");
    if (!fp) throw std::runtime_error("Could not open parameters.dat for writing");
    std::fprintf(fp, "# The data in this folder correspond to the following:\n");
    std::fprintf(fp, " D = %d , L = %.10g,  nGrids = %d , TIME_STEP = %.10g  \n", o.D, o.L, o.nGrids, o.dt);
    std::fprintf(fp, " c = %.10g , nt = %d,  readxns = %d , expansion = %d  \n", o.c, o.nt, o.mode, o.expansion);
    std::fprintf(fp, " nb = %d , FFT = %d,  ALPHAVAL = %d , WallTracking = %d  \n", o.nbubbles, 1, o.alpha,
                 o.walltracking);
    std::fprintf(fp, "Mpl = %.10g, memorysave = %d, TEST = %d  \n", o.mpl, o.memorysave, o.test);
    std::fprintf(fp, " Full1DFieldEvery = %d , Trad = %.10g , fixedseed = %d \n", kFull1DFieldEvery, o.trad, 1);
    std::fprintf(fp, " kUV = %.10g , kIR = %.10g , kRStar = %.10g , kMeff = %.10g \n", kUV, kIR, kRStar, kMeff);
    std::fclose(fp);
}

/* Collects the snapshot write in flight; a file that could not be written is
 * reported and the run carries on, as in bubble.cpp:948-952. */
bool collect_snapshot(Run &r) {
    if (r.writing.empty()) return true;
    const int st = cb_out_field_wait(r.h);
    if (st == CB_EIO) std::cerr << "Error: could not write the snapshot " << r.writing << std::endl;
    else if (st != CB_OK) return r.fail(st, "writing a snapshot");
    r.writing.clear();
    return true;
}

/* bubble.cpp:887-954: the HDF5 snapshot (datasets phi, pi and, with
 * memorysave == 0, Ekin, gradphi, potEnergy; attributes D, L, nGrids, reduc,
 * c, t, a), written by the library's own HDF5 writer in the background while
 * the run goes on (the fields are copied first) */
bool snapshot(Run &r, int n) {
    const Options &o = r.o;
    std::cout << "snapshot " << n << " at t = " << r.line.t << std::endl;
    const std::string path = r.folder + "/_phi_t=" + four(n) + ".h5";
    if (!collect_snapshot(r)) return false;
    int st = cb_out_field_async(r.h, path.c_str(), 0);
    if (st != CB_OK) return r.fail(st, "writing a snapshot");
    r.writing = path;
    /* bubble.cpp:642-709: the power spectrum file */
    const int nb = cb_nbins(o.D, o.nGrids);
    std::vector<double> pw(nb), ws(nb), ks(nb);
    st = cb_power_spectrum(r.h, pw.data(), ws.data(), ks.data(), nb);
    if (st != CB_OK) return r.fail(st, "power spectrum");
    std::fstream dat((r.folder + "/_phi_k_t=" + four(n) + ".dat").c_str(), std::ios::out);
    dat << "# t    a        (then one line per |k| bin: k_comoving  k_physical  Delta(k))" << std::endl;
    dat << r.line.t << " " << r.line.a << std::endl;
    for (int b = 0; b < nb; ++b)
        if (ws[b] > 0) {
            const double kMean = ks[b] / ws[b];
            dat << kMean << "   " << kMean / r.line.a << "   " << pw[b] / ws[b] << std::endl;
        }
    return true;
}

/* bubble.cpp:993-1006 (1-D): the whole field as one line */
bool full_field(Run &r) {
    std::vector<double> phi(r.N);
    int st = cb_get_fields(r.h, phi.data(), nullptr, nullptr, nullptr, nullptr);
    if (st != CB_OK) return r.fail(st, "downloading the field");
    FILE *fp = std::fopen((r.folder + "/FullField.dat").c_str(), "a");
    if (!fp) return true;
    for (double v : phi) std::fprintf(fp, "%.5f ", v);
    std::fprintf(fp, "\n");
    std::fclose(fp);
    return true;
}

/* ---- wall tracking (bubble.cpp:535-634) ---------------------------------- */

bool can_track_wall(const Options &o) { return o.D == 1 || o.mode == -1 || o.mode == -2; }

/* first step of the tracking: half an oscillation period in the true vacuum */
int wall_track_start(const Run &r) { return int(M_PI / r.wall.mT / r.o.dt); }

void init_wall(Run &r) {
    const Options &o = r.o;
    Wall &w = r.wall;
    w.rn = o.D == 3 ? 0.823 * std::pow(o.c, 0.203) * 1.3 : 0.823 * std::pow(o.c, 0.203);
    w.lw = 0.496 * std::pow(o.c, -0.531);
    w.phi_max = o.c / (6 + 2 * o.c);
    w.phi_zero = (2 + o.c - std::sqrt(4 + o.c)) / (3 + o.c);
    w.mT = std::sqrt(2 * (o.c + 6));
    const int mid = o.D == 3 ? o.nGrids / 2 : 0;
    if (o.mode == -2 && o.D >= 2) { w.centre[0] = o.nGrids / 2; w.centre[1] = o.nGrids / 2; w.centre[2] = mid; }
    else if (o.mode == -1 && o.D >= 2) { w.centre[0] = o.nGrids / 4; w.centre[1] = o.nGrids / 4; w.centre[2] = mid; }
}

double gamma_factor(const Run &r, double d) {
    if (r.o.walltracking == 0 || d == 0) return 0;
    return r.wall.dini / d;
}

/* WallFinder (bubble.cpp:575-617): along axis 0 from the bubble centre, Rmin
 * is the outermost radius where phi is still above its exit value, Rmax the
 * first where it has dropped to the barrier top. The line comes from the
 * device (cb_get_line); the search is the reference's, on the host. */
bool wall_finder(Run &r) {
    const Options &o = r.o;
    Wall &w = r.wall;
    const double dx = double(o.L) / o.nGrids;
    const double maximal = (o.mode == -1 && o.D >= 2) ? o.L / 4.0 - o.deltar : o.L / 2.0;
    if (w.rmax >= 0.98 * maximal || w.rmin >= 0.98 * maximal) {
        std::cout << "bubble has almost left the box" << std::endl;
        return true;
    }
    std::vector<double> line(o.nGrids);
    const int st = cb_get_line(r.h, w.centre[0], w.centre[1], w.centre[2], o.nGrids, line.data());
    if (st != CB_OK) return r.fail(st, "reading the wall line");
    auto radius = [&](int i) { return dx * std::sqrt((i + 0.5) * (i + 0.5) + 0.25 * (o.D - 1)); };
    const int istart = std::max(int((w.rmin - w.lw) / dx), int(w.rn / (2 * dx)));
    w.rmin = 0;
    w.rmax = 0;
    for (int i = istart; (w.rmax == 0 || w.rmin == 0) && radius(i) < maximal; i++) {
        const double v = line[(size_t)i % line.size()];
        if (v > w.phi_zero) w.rmin = radius(i);
        if (v <= w.phi_max && w.rmax == 0) w.rmax = radius(i);
    }
    if (w.rmax < w.rmin) {
        std::cout << "Rmax < Rmin ! Something went wrong ... " << std::endl;
        return true;
    }
    if (w.rmax * w.rmin == 0 && w.rmin + w.rmax != 0) w.rmax = w.rmin;
    w.width = w.rmax - w.rmin;
    std::cout << "WallWidth is: " << w.width << std::endl;
    return true;
}

/* bubble.cpp:1009-1015 */
void out_gamma(const Run &r) {
    FILE *fp = std::fopen((r.folder + "/gamma.dat").c_str(), "a");
    if (!fp) return;
    std::fprintf(fp, "%.3f %.4f %.3f %.3f %.3f\n ", r.line.t, gamma_factor(r, r.wall.width), r.wall.width,
                 r.wall.rmin, r.wall.rmax);
    std::fclose(fp);
}

/* TrackWall (bubble.cpp:543-560) */
bool track_wall(Run &r, int it) {
    const int start = wall_track_start(r);
    if (it == start) {
        if (!wall_finder(r)) return false;
        r.wall.dini = r.wall.width;
        std::cout << "initial wall width: " << r.wall.dini << std::endl;
        out_gamma(r);
    } else if (it > start && it % kWallTrackEvery == 0 && r.line.t < r.o.L / 2) {
        if (!wall_finder(r)) return false;
        out_gamma(r);
        std::cout << "gamma factor: " << gamma_factor(r, r.wall.width) << std::endl;
    }
    return true;
}

/* UpdateWall (bubble.cpp:569-573): the wall at a snapshot step */
bool update_wall(Run &r, int it) {
    if (it > wall_track_start(r) && r.line.t < r.o.L / 2) return wall_finder(r);
    return true;
}

}  // namespace

int main(int argc, char **argv) {
    const auto start = std::chrono::high_resolution_clock::now();
    Run r;
    Options &o = r.o;
    if (!parse(argc, argv, o)) return 1;
    const std::string name = "Sim" + std::to_string(o.D) + "_D_" + "nt_" + std::to_string(o.nt) + "_dt_" +
                             precistr(o.dt, 5) + "_nGrids_" + std::to_string(o.nGrids) + "_L_" + precistr(o.L, 1) +
                             "_Mode_" + std::to_string(o.mode) + "_nB_" + std::to_string(o.nbubbles) + "_c_" +
                             precistr(o.c, 2) + "_FFT_" + std::to_string(1) +
                             (o.D == 1 ? "_Full1DFieldEvery_" + std::to_string(kFull1DFieldEvery) : "") + "_Mpl_" +
                             std::to_string(int(o.mpl));
    r.folder = (fs::path(o.out) / name).string();
    const double dx = double(o.L) / o.nGrids;
    const double dtmax = dx / std::sqrt(o.D);
    if (!(o.dt < dtmax)) {
        std::cout << "Stability condition dt < dx/sqrt(D) is not satisfied (dt = " << o.dt
                  << ", dx/sqrt(D) = " << dtmax << "). Stopping." << std::endl;
        return 1;
    }
    std::cout << "Stability condition dt < dx/sqrt(D) is satisfied." << std::endl;
    fs::create_directories(r.folder);
    std::cout << "Output folder: " << r.folder << std::endl;
    r.N = 1;
    for (int a = 0; a < o.D; ++a) r.N *= (size_t)o.nGrids;

    cb_params p = {o.D, o.nGrids, o.L, o.c, o.dt, o.alpha, o.expansion, o.mpl, r.DeltaV, o.precision, o.memorysave};
    cb_ic_params ic = {o.mode, o.nbubbles, o.trad, o.deltar, o.test, o.position_seed, o.thermal_seed};
    std::vector<double> phi0(r.N), pi0(r.N);
    std::string xns_in;
    if (o.mode == 0 && o.D > 1 && !o.test) {
        std::ifstream f(r.folder + "/__xns.dat");
        if (!f) {
            std::cerr << "Error: mode 0 needs the bubble positions in " << r.folder << "/__xns.dat (one \"x y z\" per line)."
                      << std::endl;
            return 1;
        }
        xns_in.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    std::vector<char> xns(64 * 8 * (size_t)std::max(1, o.nbubbles) + 64);
    size_t xlen = 0;
    int st = cb_initial_condition(&p, &ic, xns_in.empty() ? nullptr : xns_in.c_str(), phi0.data(), pi0.data(),
                                  xns.data(), xns.size(), &xlen);
    if (st != CB_OK) { std::cerr << "Error: initial condition: " << cb_last_error(nullptr) << "\n"; return 1; }
    if (o.mode == 1 && o.D > 1 && !o.test) {
        FILE *f = std::fopen((r.folder + "/__xns.dat").c_str(), "w");
        if (f) { std::fwrite(xns.data(), 1, xlen, f); std::fclose(f); }
    }
    init_energy_file(r);
    st = cb_create_from_ic(&p, phi0.data(), pi0.data(), &r.line, &r.h);
    if (st != CB_OK) { std::cerr << "Error: " << cb_last_error(nullptr) << "\n"; return 1; }
    parameters_file(r);
    energy_line(r, r.line);
    if (!snapshot(r, 0)) return 1;
    if (o.D == 1 && !full_field(r)) return 1;

    const std::vector<int> snaps = schedule(o);
    size_t next_snap = 0;
    const bool track = o.walltracking == 1 && can_track_wall(o);
    if (o.walltracking == 1 && !track)
        std::cout << "Note: wall tracking only works in 1D or with --mode -1 or -2; skipping it." << std::endl;
    init_wall(r);
    const int wall_start = wall_track_start(r);
    const int progress = std::max(1, o.nt / 20);
    int it = 1;
    while (it <= o.nt) {
        /* the next step at which something is written */
        int next = o.nt;
        next = std::min(next, ((it + kOutEnergyEvery - 1) / kOutEnergyEvery) * kOutEnergyEvery);
        if (next_snap < snaps.size()) next = std::min(next, snaps[next_snap]);
        if (o.D == 1) next = std::min(next, ((it + kFull1DFieldEvery - 1) / kFull1DFieldEvery) * kFull1DFieldEvery);
        next = std::min(next, ((it + progress - 1) / progress) * progress);
        if (track) {
            if (it <= wall_start) next = std::min(next, wall_start);
            else next = std::min(next, ((it + kWallTrackEvery - 1) / kWallTrackEvery) * kWallTrackEvery);
        }
        const bool snap = next_snap < snaps.size() && next == snaps[next_snap];
        st = cb_step(r.h, next - it + 1, CB_STEP_SUMS | (snap && o.memorysave == 0 ? CB_STEP_LOCAL : 0), &r.line);
        if (st != CB_OK) return r.fail(st, "stepping") ? 0 : 1;
        it = next + 1;
        /* the reference's order within a step (main.cpp:276-285) */
        if (track && !track_wall(r, next)) return 1;
        if (o.D == 1 && next % kFull1DFieldEvery == 0 && !full_field(r)) return 1;
        if (next % kOutEnergyEvery == 0) energy_line(r, r.line);
        if (snap) {
            if (track && !update_wall(r, next)) return 1;
            if (!snapshot(r, (int)++next_snap)) return 1;
        }
        if (next % progress == 0)
            std::cout << "step " << next << " / " << o.nt << " (" << 100 * next / o.nt << "%)" << std::endl;
    }
    if (!collect_snapshot(r)) return 1;
    cb_destroy(r.h);
    const auto end = std::chrono::high_resolution_clock::now();
    const double el = std::chrono::duration<double>(end - start).count();
    std::cout << "Elapsed time: " << el << " seconds\n";
    FILE *fp = std::fopen((r.folder + "/parameters.dat").c_str(), "a");
    if (fp) {
        std::fprintf(fp, "Elapsed time %f seconds\n", el);
        std::fclose(fp);
    }
    return 0;
}
