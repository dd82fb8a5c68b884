/* cb_main_loop.hpp -- the time loop of CoolBubble's main.cpp on the GPU.
 *
 * A CoolBubble build (reference: Henda-M/CoolBubble) that links
 * libcoolbubble_b200 includes this file in src/main.cpp just before main()
 * -- after main.cpp's own helpers PlotFieldAndPS and SnapshotFile, which it
 * calls -- and replaces the time-evolution loop of main.cpp:274-288 with
 *
 *     if (cb_main_loop(s, folder, snapshotSteps, trackWall, progressEvery) != 0) return 1;
 *
 * Everything else of main() stays: the command line, the run folder, the
 * Bubble constructor (the initial condition drawn on the host from the seed,
 * bubble.cpp:156-316), OutParameters, the t = 0 line and snapshot, the summary
 * plots. The loop hands the constructor's state to the library (cb_create),
 * then advances it on the GPU from one output step to the next (cb_step): the
 * steps main.cpp writes an energy line at (it % OutEnergyEvery == 0), its
 * snapshot steps, the wall-tracking steps (TrackWall acts only at
 * WallTrackStart() and every WallTrackEvery steps after it), the 1-D
 * FullField steps and the progress lines. At each of them the line's scalars
 * are copied into the Bubble (and the spread sums into bubble.cpp's
 * file-static variables, through cb_ref_set_spreads), so the reference's own
 * writers produce the files: outEP (EnergyDensities.dat), TrackWall /
 * UpdateWall / outGamma (gamma.dat, from the wall line read off the device),
 * outFullField (1-D), OutField (the snapshot, from fields read off the
 * device). The power spectrum of a snapshot comes from the GPU
 * (cb_power_spectrum) and is written in FourierTransform's format
 * (bubble.cpp:642-709).
 *
 * CB_PRECISION=fp32c in the environment runs the float path; the default is
 * the FP64 parity path.
 */
#ifndef CB_MAIN_LOOP_HPP
#define CB_MAIN_LOOP_HPP

#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "coolbubble_b200.h"

/* Sets bubble.cpp's file-static spread sums (bubble.cpp:44), which outEP
 * prints; defined next to bubble.cpp in the build (cb_ref_spreads.cpp). */
void cb_ref_set_spreads(double etot_var, double ekin_var, double egrad_var, double epot_var, double avphi_var,
                        double avphip_var);

namespace cb_binding {

inline int fail(cb_handle *h, int status, const char *what) {
    std::cerr << "Error: " << what << ": " << cb_last_error(h) << " (" << cb_status_string(status) << ")"
              << std::endl;
    return 1;
}

/* The scalars oneStep leaves in the Bubble (bubble.cpp:838-875). */
inline void copy_line(Bubble &s, const cb_sums &o) {
    s.t = o.t;
    s.a = o.a;
    s.ap = o.ap;
    s.H = o.H;
    s.C = o.C;
    s.Etot = o.etot;
    s.Ekintot = o.ekin;
    s.Egradtot = o.egrad;
    s.Epottot = o.epot;
    s.avphi = o.avphi;
    s.avphiP = o.avphip;
    s.EkinHalfPrev = o.ekin_half_prev;
    cb_ref_set_spreads(o.etot_var, o.ekin_var, o.egrad_var, o.epot_var, o.avphi_var, o.avphip_var);
}

/* Site index of lattice point (i0, i1, i2) (gridfuncs.cpp:25-26, 65-70). */
inline size_t site(int i0, int i1, int i2) {
    if (D == 1) return (size_t)i0;
    if (D == 2) return (size_t)i0 * nGrids + i1;
    return ((size_t)i0 * nGrids + i1) * nGrids + i2;
}

/* The wall finder reads phi along axis 0 from the tracked bubble's centre
 * (bubble.cpp:588-592): bring exactly those values into s.phi. */
inline int fetch_wall_line(cb_handle *h, Bubble &s) {
    std::vector<double> line(nGrids);
    const int c0 = D == 1 ? 0 : s.wallCentre[0], c1 = D >= 2 ? s.wallCentre[1] : 0, c2 = D >= 3 ? s.wallCentre[2] : 0;
    const int st = cb_get_line(h, c0, c1, c2, nGrids, line.data());
    if (st != CB_OK) return fail(h, st, "reading the wall line");
    for (int m = 0; m < nGrids; ++m) s.phi[site((c0 + m) % nGrids, c1, c2)] = line[m];
    return 0;
}

/* FourierTransform(itPlot) (bubble.cpp:642-709): the shells from the GPU, the
 * file in the reference's format. */
inline int write_spectrum(cb_handle *h, Bubble &s, int itPlot) {
    if (FFT != 1) return 0;
    const int nb = cb_nbins(D, nGrids);
    std::vector<double> pw(nb), ws(nb), ks(nb);
    const int st = cb_power_spectrum(h, pw.data(), ws.data(), ks.data(), nb);
    if (st != CB_OK) return fail(h, st, "power spectrum");
    std::fstream dat((s.folder + "/_phi_k_t=" + dataName(itPlot) + ".dat").c_str(), std::ios::out);
    dat << "# t    a        (then one line per |k| bin: k_comoving  k_physical  Delta(k))" << std::endl;
    dat << s.t << " " << s.a << std::endl;
    for (int b = 0; b < nb; ++b)
        if (ws[b] > 0) {
            const double kMean = ks[b] / ws[b];
            dat << kMean << "   " << kMean / s.a << "   " << pw[b] / ws[b] << std::endl;
        }
    return 0;
}

}  // namespace cb_binding

/* main.cpp:274-288 on the GPU; returns 0, or 1 after printing the error. */
static int cb_main_loop(Bubble &s, const std::string &folder, const std::vector<int> &snapshotSteps, bool trackWall,
                        int progressEvery) {
    using namespace cb_binding;
    const char *prec = std::getenv("CB_PRECISION");
    /* positional: def.h defines `expansion` and `memorysave` as macros, so the
     * fields cannot be named here (d, n_grids, L, c, dt, alpha, expansion,
     * mpl, delta_v, precision, memorysave) */
    const cb_params p = {D, nGrids, (double)L, c, (double)TIME_STEP, ALPHAVAL, expansion, (double)Mpl, s.DeltaV,
                         (prec && std::string(prec) == "fp32c") ? CB_FP32C : CB_FP64, memorysave};
    const cb_scalars s0 = {s.t, s.a, s.ap, s.H, s.EkinHalfPrev, s.Etot};
    cb_handle *h = nullptr;
    int st = cb_create(&p, s.phi, s.pi, &s0, &h);
    if (st != CB_OK) return fail(nullptr, st, "handing the run to the GPU");

    const int wallStart = trackWall ? s.WallTrackStart() : -1;
    size_t nextSnapshot = 0;
    auto wall_step = [&](int it) { return trackWall && (it == wallStart || (it > wallStart && it % WallTrackEvery == 0)); };
    auto is_snapshot = [&](int it) { return nextSnapshot < snapshotSteps.size() && it == snapshotSteps[nextSnapshot]; };
    auto event = [&](int it) {
        return it == nt || wall_step(it) || (D == 1 && it % Full1DFieldEvery == 0) || it % OutEnergyEvery == 0 ||
               is_snapshot(it) || it % progressEvery == 0;
    };
    int it = 0;
    while (it < nt) {
        int next = it + 1;
        while (!event(next)) ++next;
        const bool snap = is_snapshot(next);
        int flags = CB_STEP_SUMS;
        if (snap && memorysave == 0) flags |= CB_STEP_LOCAL;
        cb_sums o;
        if ((st = cb_step(h, next - it, flags, &o)) != CB_OK) { fail(h, st, "stepping"); cb_destroy(h); return 1; }
        it = next;
        copy_line(s, o);
        if (wall_step(it) || (trackWall && snap))
            if (fetch_wall_line(h, s)) { cb_destroy(h); return 1; }
        if (trackWall) s.TrackWall(it);
        if (D == 1 && it % Full1DFieldEvery == 0) {
            if ((st = cb_get_fields(h, s.phi, nullptr, nullptr, nullptr, nullptr)) != CB_OK) {
                fail(h, st, "reading the field");
                cb_destroy(h);
                return 1;
            }
            s.outFullField();
        }
        if (it % OutEnergyEvery == 0) s.outEP();
        if (snap) {
            if (trackWall) s.UpdateWall(it);
            /* SaveSnapshot (main.cpp:192-198): the fields from the device, the spectrum from the GPU */
            const bool loc = memorysave == 0;
            st = cb_get_fields(h, s.phi, s.pi, loc ? s.Ekin : nullptr, loc ? s.gradphi : nullptr,
                               loc ? s.potEnergy : nullptr);
            if (st != CB_OK) { fail(h, st, "reading the fields"); cb_destroy(h); return 1; }
            const int n = (int)++nextSnapshot;
            std::cout << "snapshot " << n << " at t = " << s.t << std::endl;
            s.OutField(n);
            if (write_spectrum(h, s, n)) { cb_destroy(h); return 1; }
            PlotFieldAndPS(folder, SnapshotFile(n), s, WallTracking == 1 ? s.GammaFactor(s.WallWidth) : 0.0);
        }
        if (it % progressEvery == 0)
            std::cout << "step " << it << " / " << nt << " (" << 100 * it / nt << "%)" << std::endl;
    }
    /* leave the Bubble holding the final fields, as the reference's loop does */
    st = cb_get_fields(h, s.phi, s.pi, nullptr, nullptr, nullptr);
    if (st != CB_OK) fail(h, st, "reading the final fields");
    cb_destroy(h);
    return st == CB_OK ? 0 : 1;
}

#endif
