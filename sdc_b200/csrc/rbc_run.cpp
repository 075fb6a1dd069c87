// rbc_run.cpp -- command-line driver over the C ABI, mirroring the reference's main.cu.
//
// Options follow gpu_flow/code/main.cu:61-232 and code/README.txt (only the ones of the
// solver path):
//   -nmodes M N L        physical points in x, y and vertical modes (mandatory)
//   -clength Lx Ly       box lengths (mandatory)
//   -ra Ra  -pr Pr       Rayleigh and Prandtl numbers (mandatory)
//   -dt dt  -t T         time step and final time (mandatory); iterations = ceil(T/dt)
//   -nfiles n            state dumps during the run (theta_%08d.bin ... every iters/n)
//   -files th f g F G    restart from reference dump files (FP32 or FP64)
//   -history file        also restore the AB2 history (exact restart; the reference has none)
//   -device d  -dir path -seed s  -particles n
//   -init_amp a -init_kmax k   seeded initial condition (replaces init_random)
//   -init_isr | -init_dislocation | -init_rectangle | -init_sv | -init_cr |
//   -init_giantspiral | -init_test   pattern initial conditions (main.cu:88-98, 326-352)
//   -init_mode m  -init_noise a      their mode (default Lx/2) and the noise of the other
//                                    modes (default 1e-6, init_random's amplitude)
//   -form fp64|mixed|colloc   precision form (-colloc_nq Q: collocation levels of colloc)
//   -diag n              print Nu_wall, Nu_vol, KE every n steps
//   -real_bytes 4|8      element size of the written dumps (4 = the reference's default)
//   -freeze_circle N     from iteration N on, hold the field inside the circle of radius 0.8
//                        (freeze_operator, main.cu:222-223, 569-577)
//   -temp_circle N       from iteration N + 1 on, heat theta inside the frame of width 0.1 by
//                        1.5/100 per iteration (masktemp, main.cu:228-229, 580-589)
//   -penalized rectangle|circle|diskarray|everywhere   the penalized operator with that mask
//                        (the reference's PENALIZED build targets)
//   -eta e               its eta (main.cu:117-123; default 0.01)
//   -mean_F F            force the mean flow F of the lowest mode to F before every step
//                        (main.cu:139-140, 566-568)
// Tracers the reference's way (main.cu:150-199, 490-532, 620-660, 719-726):
//   -npart n -le_count k -le D1 .. Dk   k tracer sets of n tracers, set s with diffusivity
//                        Ds; as in the reference, no tracers without -le
//   -multitracer         without -le: the ten diffusivities of the reference's MULTITRACER
//                        builds (1e1, 3, 1, 0.3, 0.1, 0.03, 0.01, 1e-3, 1e-4, 1e-5; main.cu:201-207)
//   -part_center | -part_center_sigma | -part_diagonal | -part_pairs |
//   -part_coord_sigma x y  start patterns (sigma 0.125), -part_sigma s overrides sigma
//   -write_tracks_every p  record every p-th step; at each state dump the recorded frames
//                        of set s go to particles_le<Ds>_<step>.trkss
//   -calc_secondmoment   second moment of each set after every step, secondmoment_<s>.dat
//   -no_step_time        advance the tracers only, on the fixed initial flow
//   -snapshot_freq n     accepted; the reference's snapshot output is disabled, so is ours
// Writes simulation.log (main.cu:402-426) and returns non-zero on any library error.
#include "rbc.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <initializer_list>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <sys/stat.h>

namespace {

struct Args {
    int argc;
    char** argv;
    int find(const char* name) const
    {
        for (int i = 1; i < argc; ++i)
            if (!std::strcmp(argv[i], name)) return i;
        return -1;
    }
    bool has(const char* name) const { return find(name) >= 0; }
    // the k-th value after option `name`; an option name ends the values (a negative number
    // such as -0.5 is a value)
    static bool is_option(const char* s) { return s[0] == '-' && std::isalpha((unsigned char)s[1]); }
    const char* str(const char* name, int k = 0) const
    {
        const int i = find(name);
        if (i < 0 || i + 1 + k >= argc) return nullptr;
        for (int j = i + 1; j <= i + 1 + k; ++j)
            if (is_option(argv[j])) return nullptr;
        return argv[i + 1 + k];
    }
    double num(const char* name, double def, int k = 0, bool mandatory = false) const
    {
        const char* s = str(name, k);
        if (!s) {
            if (mandatory) {
                std::fprintf(stderr, "missing mandatory option %s\n", name);
                std::exit(2);
            }
            return def;
        }
        return std::atof(s);
    }
};

int check(rbc_status s, rbc_handle* h, const char* what)
{
    if (s == RBC_OK) return 0;
    std::fprintf(stderr, "%s: %s (%s)\n", what, rbc_status_string(s), h ? rbc_last_error(h) : "");
    return 1;
}

} // namespace

int main(int argc, char** argv)
{
    Args a{argc, argv};
    if (argc < 2 || a.has("-h") || a.has("--help")) {
        std::printf("usage: rbc_run -nmodes M N L -clength Lx Ly -ra Ra -pr Pr -dt dt -t T [options]\n");
        return argc < 2 ? 2 : 0;
    }
    rbc_params p{};
    p.nx = (int)a.num("-nmodes", 0, 0, true);
    p.ny = (int)a.num("-nmodes", 0, 1, true);
    p.nz = (int)a.num("-nmodes", 0, 2, true);
    p.lx = a.num("-clength", 0, 0, true);
    p.ly = a.num("-clength", 0, 1, true);
    p.ra = a.num("-ra", 0, 0, true);
    p.pr = a.num("-pr", 0, 0, true);
    p.dt = a.num("-dt", 0, 0, true);
    const double tfinal = a.num("-t", 0, 0, true);
    p.device = (int)a.num("-device", 0);
    p.n_tracers = (int)a.num("-particles", 0);
    const char* form = a.str("-form");
    p.form = (form && !std::strcmp(form, "mixed"))    ? RBC_FORM_MIXED
             : (form && !std::strcmp(form, "colloc")) ? RBC_FORM_COLLOC
                                                      : RBC_FORM_FP64;
    p.colloc_nq = (int)a.num("-colloc_nq", 0);
    const int nfiles = (int)a.num("-nfiles", 1);
    const unsigned long long seed = (unsigned long long)a.num("-seed", 1);
    const int diag_every = (int)a.num("-diag", 0);
    const int real_bytes = (int)a.num("-real_bytes", 4);
    const long long freeze_at = (long long)a.num("-freeze_circle", 0);
    const long long heat_at = (long long)a.num("-temp_circle", 0);
    p.field_ops = (freeze_at > 0 ? RBC_FIELD_FREEZE : 0) | (heat_at > 0 ? RBC_FIELD_HEAT : 0);
    if (const char* pen = a.str("-penalized")) {
        static const char* kMasks[] = {"rectangle", "circle", "diskarray", "everywhere"};
        p.penalization_mask = -1;
        for (int i = 0; i < 4; ++i)
            if (!std::strcmp(pen, kMasks[i])) p.penalization_mask = i;
        if (p.penalization_mask < 0) {
            std::fprintf(stderr, "unknown -penalized mask %s\n", pen);
            return 2;
        }
        p.penalization_eta = a.num("-eta", 0.01);
    }
    p.mean_F = a.num("-mean_F", 0.0);
    // tracers as main.cu configures them
    const int npart = (int)a.num("-npart", 0);
    std::vector<double> lewis;
    if (a.has("-le") || a.has("-multitracer")) {
        if (a.has("-le")) {
            const int le_count = std::max(1, (int)a.num("-le_count", 1));
            for (int k = 0; k < le_count; ++k) lewis.push_back(a.num("-le", 0.0, k, true));
        } else {
            lewis = {1e1, 3e0, 1e0, 3e-1, 1e-1, 3e-2, 1e-2, 1e-3, 1e-4, 1e-5};
        }
        const int le_count = (int)lewis.size();
        if (npart > 0) {
            p.n_tracers = npart * le_count;
            p.tracer_sets = le_count;
            p.tracer_diffusivity = lewis[0];
        }
    }
    const int nsets = p.tracer_sets > 1 ? p.tracer_sets : 1;
    if (lewis.empty()) lewis.assign(nsets, p.tracer_diffusivity); // -particles: one set, no -le
    int part_type = RBC_TRACERS_RANDOM;
    double part_sigma = 0.0, part_cx = 0.0, part_cy = 0.0;
    if (a.has("-part_center")) part_type = RBC_TRACERS_CENTER;
    if (a.has("-part_center_sigma")) { part_type = RBC_TRACERS_CENTER_SIGMA; part_sigma = 0.125; }
    if (a.has("-part_diagonal")) part_type = RBC_TRACERS_DIAGONAL;
    if (a.has("-part_pairs")) part_type = RBC_TRACERS_PAIRS;
    if (a.has("-part_coord_sigma")) {
        part_type = RBC_TRACERS_COORD_SIGMA;
        part_cx = a.num("-part_coord_sigma", 0.0, 0, true);
        part_cy = a.num("-part_coord_sigma", 0.0, 1, true);
        part_sigma = 0.125;
    }
    if (a.has("-part_sigma")) part_sigma = a.num("-part_sigma", 0.0, 0, true);
    const bool write_tracks = a.has("-write_tracks_every") && p.n_tracers > 0;
    const int track_every = std::max(1, (int)a.num("-write_tracks_every", 1));
    if (write_tracks) {
        p.track_frames = 256;
        p.track_period = track_every;
    }
    const bool moments = a.has("-calc_secondmoment") && p.n_tracers > 0;
    const bool do_step = !a.has("-no_step_time");
    const char* dir = a.str("-dir");
    std::string out = dir ? dir : ".";
    if (dir) mkdir(dir, 0755);

    // number of iterations as main.cu:275-280 (iCeil(final_t / delta_t))
    const long long iters = (long long)std::ceil(tfinal / p.dt);
    const long long write_every = nfiles > 0 ? iters / nfiles : 0;

    rbc_handle* h = nullptr;
    if (check(rbc_create(&p, &h), nullptr, "rbc_create")) return 1;
    int rc = 0;
    if (a.has("-files")) {
        rc |= check(rbc_load_state(h, a.str("-files", 0), a.str("-files", 1), a.str("-files", 2), a.str("-files", 3),
                                   a.str("-files", 4)),
                    h, "rbc_load_state");
        if (!rc && a.has("-history")) rc |= check(rbc_load_history(h, a.str("-history")), h, "rbc_load_history");
    } else {
        static const char* kPatterns[] = {"-init_isr", "-init_dislocation", "-init_rectangle", "-init_sv",
                                          "-init_cr", "-init_giantspiral", "-init_test"};
        int pattern = 0;
        for (int i = 0; i < 7; ++i)
            if (a.has(kPatterns[i])) pattern = i + 1;
        if (pattern)
            rc |= check(rbc_init_pattern(h, pattern, a.num("-init_mode", p.lx / 2.0), a.num("-init_amp", 1e-6), seed,
                                         pattern == RBC_INIT_TEST ? 0.0 : a.num("-init_noise", 1e-6)),
                        h, "rbc_init_pattern");
        else
            rc |= check(rbc_init_fields(h, seed, a.num("-init_amp", 1e-3), a.num("-init_kmax", 4.0)), h,
                        "rbc_init_fields");
    }
    if (!rc && p.n_tracers > 0) {
        if (npart > 0) {
            // one particle_tracer per Lewis number (main.cu:494-500), each with its own draws
            for (int k = 0; k < nsets && !rc; ++k) {
                rc |= check(rbc_tracer_set_diffusivity(h, k, lewis[k]), h, "rbc_tracer_set_diffusivity");
                rc |= check(rbc_tracers_init_set(h, k, part_type, seed + (unsigned long long)k, part_cx, part_cy, 0.0,
                                                 part_sigma),
                            h, "rbc_tracers_init_set");
            }
        } else {
            rc |= check(rbc_tracers_seed(h, seed), h, "rbc_tracers_seed");
        }
    }
    if (rc) {
        rbc_destroy(h);
        return 1;
    }

    {
        FILE* log = std::fopen((out + "/simulation.log").c_str(), "w");
        if (log) {
            std::fprintf(log, "Simulation of Rayleigh-Benard convection (sm_100a)\nRayleigh-Number: %g\nPrandtl-Number: %g\n"
                              "delta t: %g\nfinal t: %g\nnumber of files: %d\nnumber of iterations: %lld\n"
                              "eta(penalization): %g\ncube length x direction: %g\ncube length y direction: %g\ncube length z direction: 1\n"
                              "number of x modes: %d\nnumber of y modes: %d\nnumber of z modes: %d\ncommand string: ",
                         p.ra, p.pr, p.dt, tfinal, nfiles, iters, p.penalization_eta, p.lx, p.ly, p.nx, p.ny, p.nz);
            for (int i = 0; i < argc; ++i) std::fprintf(log, "%s ", argv[i]);
            std::fprintf(log, "\n");
            std::fclose(log);
        }
    }

    // tracer outputs: recorded frames since the last dump, the second-moment file
    std::vector<float> frames, ring(write_tracks ? (size_t)256 * 3 * p.n_tracers : 0);
    std::vector<unsigned int> frame_steps, ring_steps(write_tracks ? 256 : 0);
    std::vector<FILE*> m2;
    if (moments) {
        // one datapoint_writer per set (main.cu:521-529, output/datapoint_writer.cu:21-45)
        for (int k = 0; k < nsets; ++k) {
            char name[64];
            std::snprintf(name, sizeof name, "/secondmoment_%d.dat", k);
            FILE* f = std::fopen((out + name).c_str(), "w");
            if (!f) {
                std::fprintf(stderr, "cannot open %s%s\n", out.c_str(), name);
                rc = 1;
                break;
            }
            std::fprintf(f, "# Data point writer\n# Le %.9f\n# Data ordering: t, val\n", lewis[k]);
            m2.push_back(f);
        }
    }

    long long done = 0;
    while (done < iters && !rc) {
        // iteration i of main.cu:556; the field operators run before its step (main.cu:569-589)
        const long long i = done + 1;
        if (freeze_at > 0) {
            rc |= check(rbc_freeze_apply(h), h, "rbc_freeze_apply");
            if (i == freeze_at) rc |= check(rbc_freeze_mask(h, RBC_MASK_CIRCLE, 0.8), h, "rbc_freeze_mask");
        }
        if (heat_at > 0) {
            rc |= check(rbc_heat_apply(h), h, "rbc_heat_apply");
            if (i == heat_at) rc |= check(rbc_heat_mask(h, RBC_MASK_RECTANGLE, 0.1, 1.5 / 100), h, "rbc_heat_mask");
        }
        if (rc) break;
        long long chunk = iters - done;
        // steps run in one call only while no operator acts at their iterations
        for (long long at : {freeze_at, heat_at})
            if (at > 0) chunk = std::min(chunk, at > i ? at - i : 1);
        if (write_every > 0) chunk = std::min(chunk, write_every - done % write_every);
        if (diag_every > 0) chunk = std::min(chunk, diag_every - done % diag_every);
        if (write_tracks) chunk = std::min(chunk, (long long)255 * track_every); // ring of 256 frames
        if (moments || !do_step) chunk = 1;
        if (do_step) rc |= check(rbc_step(h, (int)chunk), h, "rbc_step");
        else rc |= check(rbc_tracers_advance(h), h, "rbc_tracers_advance");
        done += chunk;
        if (rc) break;
        if (write_tracks) {
            int n = 0;
            rc |= check(rbc_tracks_read(h, ring.data(), ring_steps.data(), 256, &n), h, "rbc_tracks_read");
            frames.insert(frames.end(), ring.begin(), ring.begin() + (size_t)n * 3 * p.n_tracers);
            frame_steps.insert(frame_steps.end(), ring_steps.begin(), ring_steps.begin() + n);
        }
        for (int k = 0; k < (int)m2.size(); ++k) {
            double mo[4];
            rc |= check(rbc_tracer_moments_set(h, k, mo), h, "rbc_tracer_moments_set");
            std::fprintf(m2[k], "%g\t%g\n", done * p.dt, mo[2]);
        }
        if (diag_every > 0 && done % diag_every == 0) {
            rbc_diag d;
            rc |= check(rbc_diagnostics(h, &d), h, "rbc_diagnostics");
            std::printf("step %lld t %.6f Nu_wall %.12f Nu_vol %.12f KE %.6e\n", done, done * p.dt, d.nu_wall, d.nu_vol, d.ke);
        }
        if (write_every > 0 && done % write_every == 0) {
            rc |= check(rbc_save_state(h, out.c_str(), done, real_bytes), h, "rbc_save_state");
            char path[4096];
            std::snprintf(path, sizeof path, "%s/history_%08lld.bin", out.c_str(), done);
            if (do_step) rc |= check(rbc_save_history(h, path), h, "rbc_save_history"); // none without steps
            if (write_tracks && !frame_steps.empty()) {
                // one track file per set (main.cu:719-725): its columns of every frame
                const int nf = (int)frame_steps.size(), ns = p.n_tracers / nsets;
                std::vector<float> part((size_t)nf * 3 * ns);
                for (int k = 0; k < nsets; ++k) {
                    for (int fr = 0; fr < nf; ++fr)
                        for (int d = 0; d < 3; ++d)
                            std::memcpy(&part[((size_t)fr * 3 + d) * ns],
                                        &frames[((size_t)fr * 3 + d) * p.n_tracers + (size_t)k * ns], ns * sizeof(float));
                    char desc[512];
                    std::snprintf(desc, sizeof desc,
                                  "Particle tracks.  Simulation: Ra=%.1lf Pr=%.1lf Size=%.1lfx%.1lfx1.0  Technical: "
                                  "Modes=%dx%dx%d dt=%.3lf  Tracks: Le=%.0le ",
                                  p.ra, p.pr, p.lx, p.ly, p.nx, p.ny, p.nz, p.dt, lewis[k]);
                    std::snprintf(path, sizeof path, "%s/particles_le%.0le_%08lld.trkss", out.c_str(), lewis[k], done);
                    rc |= check(rbc_track_write(path, desc, part.data(), frame_steps.data(), nf, ns), nullptr,
                                "rbc_track_write");
                }
                frames.clear();
                frame_steps.clear();
            }
        }
    }
    for (FILE* f : m2) std::fclose(f);
    rbc_destroy(h);
    return rc;
}
