/* rbc.h -- C ABI of the B200-native Boussinesq Rayleigh-Benard step (libsdc_b200.so).
 *
 * Drop-in boundary for the solver path of jceyy/sdc gpu_flow/code: field init, the IMEX
 * step, the nonlinear operator, tracer advance and diagnostics. Plain pointers and sizes
 * only. Spectral fields use the reference layout of matrix_device
 * (gpu_flow/code/matrix/matrix_device.h:13-66): complex numbers as interleaved
 * (re, im) doubles, index c + (Nx/2+1) * (r + Ny * k) for kx index c, ky index r
 * (ky = r for r <= Ny/2, r - Ny above) and vertical mode k. F and G hold L complex
 * values (imaginary parts are zero after every step, as in the reference).
 *
 * Every function returns an rbc_status; none exits the process (the reference calls
 * exit() through EXIT_ERROR, gpu_flow/code/cuda_defines.h:50-51). rbc_last_error()
 * gives the message of the last failure on a handle. A handle may be used from one
 * host thread at a time; all device work runs on the handle's CUDA stream, and no
 * device memory is allocated after rbc_create().
 */
#ifndef SDC_B200_RBC_H
#define SDC_B200_RBC_H

#ifdef __cplusplus
extern "C" {
#endif

#define RBC_ABI_VERSION 1

typedef struct rbc_handle rbc_handle;

typedef enum {
    RBC_OK = 0,
    RBC_ERR_INVALID_ARG = 1,
    RBC_ERR_CUDA = 2,
    RBC_ERR_NAN = 3,          /* a non-finite value appeared in the state */
    RBC_ERR_TIMEOUT = 4,
    RBC_ERR_IO = 5,
    RBC_ERR_UNSUPPORTED = 6,
    RBC_ERR_OUT_OF_MEMORY = 7
} rbc_status;

typedef enum {
    RBC_FORM_FP64 = 0,        /* plain step: everything in FP64 */
    RBC_FORM_MIXED = 1,       /* FP32 synthesis, products, contraction and FFTs;
                                 FP64 implicit solve, mean flow and diagnostics */
    RBC_FORM_COLLOC = 2       /* as MIXED, with the nonlinear products formed on colloc_nq
                                 Gauss-Legendre levels in z: the vertical mode -> level
                                 synthesis and the level -> mode projection are tensor-core
                                 products (tcgen05, TF32 operands split in two, FP32
                                 accumulation) on TMA-staged tiles; FP64 implicit solve,
                                 mean flow and diagnostics */
} rbc_form;

/* Construction parameters. Replaces main.cu's -nmodes M N L, -clength Lx Ly, -ra,
 * -pr, -dt, -device (gpu_flow/code/main.cu:64-112) and the operator constructors
 * Coeff<double>(L), linear_implicit_operator::init_operator, inverse_B_matrix::init_operator,
 * nonlinear_operator_rayleigh_noslip::init_operator, implicit_explicit_step::init_timestepping
 * (main.cu:431-454). */
typedef struct {
    int nx;          /* physical grid points in x (Nx = 2^a 3^b, 8..1024) */
    int ny;          /* physical grid points in y (same rule) */
    int nz;          /* vertical Galerkin modes L */
    double lx, ly;   /* box lengths in units of the layer depth */
    double ra, pr;   /* Rayleigh and Prandtl numbers */
    double dt;       /* time step */
    int form;        /* rbc_form */
    int n_tracers;   /* passive tracers (0: none) */
    int device;      /* CUDA device ordinal */
    int diag_capacity; /* per-step diagnostics ring entries (0: 4096) */
    int tune;        /* 1: time the launch tilings of the FFT kernels at creation and keep
                        the fastest (project autotuner); 0: built-in heuristic */
    double tracer_diffusivity; /* D, the reference's -le value: after every RK4 advance each
                        coordinate moves by sqrt(2 D dt) N(0,1) (diffuse_particles,
                        gpu_flow/code/particle/particle_tracer.cu:194-199, 690-716); 0: none */
    unsigned long long noise_seed; /* seed of that noise (see rbc_tracers_advance) */
    int track_frames;  /* device ring of recorded tracer positions, in frames (0: no tracks) */
    int track_period;  /* steps between recorded frames (0 or 1: every step) */
    int field_ops;     /* buffers of the field operators: RBC_FIELD_FREEZE | RBC_FIELD_HEAT
                          (0: none; see rbc_freeze_mask and rbc_heat_mask) */
    double penalization_eta; /* eta > 0: the penalized nonlinear operator of the reference's
                          PENALIZED builds (-eta, main.cu:117-123; 0.01 there by default);
                          0: none */
    int penalization_mask;   /* rbc_pen_mask: the build target's mask */
    int tracer_sets;   /* the tracers form this many equal consecutive sets (0 or 1: one),
                          as the reference makes one particle_tracer per Lewis number
                          (main.cu:490-505); each set has its own diffusivity
                          (rbc_tracer_set_diffusivity), start pattern (rbc_tracers_init_set)
                          and moments (rbc_tracer_moments_set) */
    double mean_F;     /* nonzero: before every step F of the lowest vertical mode is set to
                          (mean_F, 0), the reference's -mean_F (force_mean, util.cu:74-81,
                          main.cu:139-140, 566-568); 0: no forcing */
    int colloc_nq;     /* RBC_FORM_COLLOC: Gauss-Legendre collocation levels in z, a multiple
                          of 8 from nz to 32 (0: 2 nz rounded up to a multiple of 8); the
                          level rule aliases the triple products of the top modes (4 nz
                          levels would reproduce the exact Galerkin integrals to ~1e-9 of their
                          scale); other forms: ignored */
} rbc_params;

/* Masks of the penalized operator (nonlinear_operator_rayleigh_noslip.cu:1653-1738; 1 in
 * the penalized region, integer arithmetic on the Nx x Ny grid):
 *   RECTANGLE   a frame 3 points wide (make rectangle, the default)
 *   CIRCLE      outside the centred circle of radius min(Nx, Ny)/2 - 3 (make circle)
 *   DISK_ARRAY  3 x 2 disks at the cell centres where the squared distance is below
 *               min(Nx/6, Ny/4) (make diskarray; the reference compares a squared distance
 *               with that length)
 *   EVERYWHERE  every point (the reference's unused init_mask_physical_space_everywhere) */
typedef enum {
    RBC_PEN_RECTANGLE = 0, RBC_PEN_CIRCLE = 1, RBC_PEN_DISK_ARRAY = 2, RBC_PEN_EVERYWHERE = 3
} rbc_pen_mask;

#define RBC_FIELD_FREEZE 1 /* frozen planes [3][L][Ny][Nx] and their mask */
#define RBC_FIELD_HEAT 2   /* heating mask [Ny][Nx] */
#define RBC_FIELD_SCALE 4  /* mask of rbc_masker [Ny][Nx] */

/* Diagnostics of the state after a step (no reference counterpart). */
typedef struct {
    double nu_wall;  /* 1 - d<theta>_xy/dz at z = -1/2 */
    double nu_vol;   /* 1 + <w theta>_V */
    double ke;       /* 1/2 <u^2 + v^2 + w^2>_V */
    long long step;  /* steps taken since construction */
} rbc_diag;

/* Five host buffers in the reference layout (see top of file). */
typedef struct {
    double* theta; double* f; double* g; double* F; double* G;
} rbc_state;

/* --- construction -------------------------------------------------------------- */
rbc_status rbc_create(const rbc_params* p, rbc_handle** out);
void rbc_destroy(rbc_handle* h);
const char* rbc_last_error(const rbc_handle* h);
const char* rbc_status_string(rbc_status s);
/* Sets the CUDA stream (cudaStream_t) for all later device work; NULL restores the
 * handle's own stream. */
rbc_status rbc_set_stream(rbc_handle* h, void* stream);

/* --- fields -------------------------------------------------------------------- */
/* Seeded initial condition: theta of the lowest vertical mode gets N(0, amplitude^2)
 * real and imaginary parts on all (c, r) with c^2 + ky^2 <= kmax^2 (SplitMix64 +
 * Box-Muller, visited r-major then c), then the Hermitian fix of make_real_signal
 * (gpu_flow/code/util/util.cu:213-224); f = g = F = G = 0. Replaces
 * matrix_device_init::init_random (gpu_flow/code/util/init.cu:9-20) and main.cu:300-396.
 * The next step is an Euler step. */
rbc_status rbc_init_fields(rbc_handle* h, unsigned long long seed, double amplitude, double kmax);
/* Pattern initial conditions of matrix_device_init (gpu_flow/code/util/init.cu:22-310),
 * selected in the reference by main.cu's -init_* options (main.cu:88-98, 326-352). The
 * pattern is evaluated in FP64 on the Nx x Ny grid of the unit square and its unnormalised
 * R2C transform becomes theta's lowest vertical mode; every other entry of theta gets
 * uniform noise in [-noise, noise) (the reference's init_random left its +-1e-6 noise
 * there); f = g = F = G = 0; then the Hermitian fix. `mode` is the reference's -init_mode
 * (default Lx/2), truncated to an integer as its int parameters do; `amplitude` is
 * max_amplitude (1e-6 in the reference).
 *   ISR          amp cos(2 pi (mode x) + phase), phase uniform in [0, 2 pi)
 *   DISLOCATION  amp cos(2 pi mode x - phi_1 + phi_2), defects at (1/2, 1/4), (1/2, 3/4)
 *   RECTANGLE    amp cos(2 pi x_m x) with x_m = (Lx / (Nx - 1)) (Nx - 5) / 2, and a strip
 *                x < 1/8 of uniform noise in [-amp, amp)
 *   SV           amp cos(2 pi (mode y + phase(x, y))), x_frac 0.2
 *   CR           amp cos(2 pi mode y - phi_1 + phi_2), x_frac 0.8
 *   GIANTSPIRAL  amp cos(2 pi mode r - phi_1 + phi_2), centre (1/2, 1/2), defect (0.8, 1/2)
 *   TEST         init_test: theta and f = amp sin(c) on row 0, columns c > 0, every mode;
 *                F_k = amp cos(k); no noise
 * The random draws (isr phase, rectangle strip, noise) come from the SplitMix64 stream of
 * `seed` in that order. The next step is an Euler step. */
typedef enum {
    RBC_INIT_ISR = 1, RBC_INIT_DISLOCATION = 2, RBC_INIT_RECTANGLE = 3, RBC_INIT_SV = 4,
    RBC_INIT_CR = 5, RBC_INIT_GIANTSPIRAL = 6, RBC_INIT_TEST = 7
} rbc_init_pattern_type;
rbc_status rbc_init_pattern(rbc_handle* h, int pattern, double mode, double amplitude, unsigned long long seed,
                            double noise);
/* Upload / download the state (host buffers, reference layout). rbc_set_state applies
 * the 2/3 dealiasing of the reference's first dealias_data call and resets the AB2
 * history, as a restart from dump files does (main.cu:290-385,
 * implicit_explicit_stepping.cu:43-52). */
rbc_status rbc_set_state(rbc_handle* h, const double* theta, const double* f, const double* g,
                         const double* F, const double* G);
rbc_status rbc_get_state(rbc_handle* h, double* theta, double* f, double* g, double* F, double* G);

/* --- files in the reference's dump format ------------------------------------- */
/* One matrix of a dump file (matrix_folder_writer::read_binary_file,
 * gpu_flow/code/output/matrix_folder_writer.cu:3-58): FP32 (the reference's default
 * build) or FP64 complex, told apart by the file size; values are returned as FP64
 * interleaved complex. dims receives the matrix dimensions (x fastest), *ndims their
 * count; out may be NULL to query the dimensions only. Host only, no GPU needed. */
rbc_status rbc_dump_read(const char* path, int index, int* dims, int maxdims, int* ndims,
                         double* out, long long maxvals);
/* Writes one matrix (write_binary_file, matrix_folder_writer.cu:61-101) with 4- or
 * 8-byte reals. Host only. */
rbc_status rbc_dump_write(const char* path, const int* dims, int ndims, const double* data, int real_bytes);
/* The state as the five files theta_%08d.bin, f_, g_, F_, G_ in directory dir, as
 * main.cu:697-713 names them (real_bytes 4 = the reference's FP32 files, 8 = FP64). */
rbc_status rbc_save_state(rbc_handle* h, const char* dir, long long step, int real_bytes);
/* Reads the five files of a reference run (main.cu:355-385, with the same dimension
 * checks) into the state; like rbc_set_state the next step is an Euler step. */
rbc_status rbc_load_state(rbc_handle* h, const char* theta, const char* f, const char* g,
                          const char* F, const char* G);
/* AB2 history (B^-1 N of the previous step) as one FP64 file of five matrices. The
 * reference never saves it, so its restarts take an Euler step
 * (implicit_explicit_stepping.cu:43-52); with this file a restart continues exactly. */
rbc_status rbc_save_history(rbc_handle* h, const char* path);
rbc_status rbc_load_history(rbc_handle* h, const char* path);

/* --- step ---------------------------------------------------------------------- */
/* nsteps iterations of the reference loop body (main.cu:612-637): step_time
 * (implicit_explicit_stepping.cu:32-97), make_real_signal, and the tracer advance when
 * tracers exist. Waits for completion; RBC_ERR_NAN if a non-finite value appeared. */
rbc_status rbc_step(rbc_handle* h, int nsteps);
/* Same, enqueued on the handle's stream without waiting. */
rbc_status rbc_step_async(rbc_handle* h, int nsteps);
rbc_status rbc_synchronize(rbc_handle* h);

/* --- nonlinear operator -------------------------------------------------------- */
/* The reference's nonlinear_operator_rayleigh_noslip::calculate_operator(theta, f, g, F, G)
 * (gpu_flow/code/operator/nonlinear_operator_rayleigh_noslip.cu:83-1394) on host buffers:
 * reads `in`, writes the five operator results to `out` (caller-owned; the reference
 * returned a new matrix_folder*[5]). The input is dealiased first, as step_time does
 * before calling it. Does not change the solver state. */
rbc_status rbc_nonlinear(rbc_handle* h, const rbc_state* in, rbc_state* out);

/* --- tracers ------------------------------------------------------------------- */
/* Positions as three blocks x[n], y[n], z[n] (z in (-1/2, 1/2)); replaces
 * particle_tracer::init_positions and get_particle_positions
 * (gpu_flow/code/particle/particle_tracer.h:65-87). n must equal params.n_tracers. */
rbc_status rbc_tracers_set(rbc_handle* h, const double* xyz, int n);
rbc_status rbc_tracers_get(rbc_handle* h, double* xyz, int n);
/* Uniform seeded positions in [0,Lx) x [0,Ly) x (-1/2,1/2) (SplitMix64). */
rbc_status rbc_tracers_seed(rbc_handle* h, unsigned long long seed);
/* Initial positions by pattern, as particle_tracer::init_positions
 * (particle_tracer.cu:58-137, 376-450). Uniform and normal draws come from the
 * SplitMix64 stream of `seed` (uniform ((u >> 11) + 1/2) 2^-53, normal by Box-Muller
 * cos(2 pi u2) sqrt(-2 ln u1)):
 *   RANDOM        x = Lx u, y = Ly u, z = u - 1/2 per particle (= rbc_tracers_seed)
 *   CENTER        all at (Lx/2, Ly/2, 0)
 *   CENTER_SIGMA  (Lx/2, Ly/2, 0) + sigma N(0,1) per coordinate
 *   DIAGONAL      x = Lx i / n, y = Ly i / n, z = 0
 *   PAIRS         particles 2i and 2i+1 at the same (Lx u, Ly u, 0); n even
 *   COORD_SIGMA   (cx, cy, cz) + sigma N(0,1) per coordinate
 * Like the reference, the sigma spread is not reflected at the lids. */
typedef enum {
    RBC_TRACERS_RANDOM = 0, RBC_TRACERS_CENTER = 1, RBC_TRACERS_CENTER_SIGMA = 2,
    RBC_TRACERS_DIAGONAL = 3, RBC_TRACERS_PAIRS = 4, RBC_TRACERS_COORD_SIGMA = 5
} rbc_tracer_init;
rbc_status rbc_tracers_init(rbc_handle* h, int type, unsigned long long seed, double cx, double cy,
                            double cz, double sigma);
/* One tracer step with the current velocity field (particle_tracer::step_particles,
 * particle_tracer.cu:141-212: RK4, trilinear interpolation on 128 z levels, periodic x/y,
 * then the diffusion step when tracer_diffusivity > 0, then reflection at
 * z = +-(1/2 - 1e-3)); rbc_step calls it after every fluid step. The diffusion normals
 * are counter-based: for the positions of step m, particle t and coordinate d, the
 * uniforms are elements 2j and 2j+1 (0-based) of the SplitMix64 stream of noise_seed
 * with j = 3 (m n + t) + d, and the normal is cos(2 pi u2) sqrt(-2 ln u1). */
rbc_status rbc_tracers_advance(rbc_handle* h);
/* Moments of the current positions in FP64 (particle_tracer::calc_secondmoment and
 * calc_pair_secondmoment, particle_tracer.cu:217-259, 771-870):
 *   out[0] = <x>, out[1] = <y>, out[2] = <x^2 + y^2> - <x>^2 - <y>^2,
 *   out[3] = sum over pairs (2i, 2i+1) of dx^2 + dy^2, each |d| above half the box
 *            replaced by box - |d| (PERIODIC), divided by n/2 (integer division). */
rbc_status rbc_tracer_moments(rbc_handle* h, double* out);
/* Tracer sets (rbc_params.tracer_sets): set s holds tracers [s n/sets, (s + 1) n/sets).
 * rbc_tracer_set_diffusivity sets the D of one set (params.tracer_diffusivity is every set's
 * initial value; takes effect from the next advance, captured step graphs included);
 * rbc_tracers_init_set gives one set the start pattern of rbc_tracers_init (n/sets tracers);
 * rbc_tracer_moments_set returns rbc_tracer_moments of one set. */
rbc_status rbc_tracer_set_diffusivity(rbc_handle* h, int set, double D);
rbc_status rbc_tracers_init_set(rbc_handle* h, int set, int type, unsigned long long seed, double cx, double cy,
                                double cz, double sigma);
rbc_status rbc_tracer_moments_set(rbc_handle* h, int set, double* out);
/* Recorded tracks (the reference's position buffer, get_particle_positions and
 * track_writer::append, particle_tracer.cu:273-309, output/track_writer.cu:21-70).
 * With track_frames > 0 the positions of every step m with m % track_period == 0 are
 * kept as FP32 frames (the reference's TRACK_FLOAT_REAL) in a device ring; the frame of
 * the initial positions is recorded when tracers are set on such a step. This call moves
 * the unread frames, oldest first, to xyz[frame][3][n] (x, y, z blocks) and their step
 * numbers to times; *nframes receives the count (at most max_frames; the rest stay
 * unread). rbc_step refuses (RBC_ERR_INVALID_ARG) to run steps whose frames would not
 * fit in the ring, as step_particles stops on a full buffer. */
rbc_status rbc_tracks_read(rbc_handle* h, float* xyz, unsigned int* times, int max_frames, int* nframes);
/* Writes frames as a TRKSS track file, version 'a' (track_movie::Write,
 * gpu_flow/code/output/track_movie.cpp:256-325): "TRKSS", 'a', uint32 tracks, uint32
 * frame rate 1, uint32 length + description, uint32 first and last frame time, uint32
 * frame count, then per frame uint32 time and x, y, z float32 per track. Host only. */
rbc_status rbc_track_write(const char* path, const char* description, const float* xyz,
                           const unsigned int* times, int nframes, int n);

/* --- diagnostics --------------------------------------------------------------- */
/* Diagnostics of the latest step (or of the initial state before any step). Waits for the
 * handle's stream and, like rbc_synchronize, returns RBC_ERR_NAN once a non-finite value
 * has appeared: rbc_step_async followed by rbc_diagnostics advances and reads the result
 * with one host wait. */
rbc_status rbc_diagnostics(rbc_handle* h, rbc_diag* out);
/* The last min(n, steps, capacity) per-step entries, oldest first; *count receives the
 * number written. */
rbc_status rbc_diag_history(rbc_handle* h, rbc_diag* out, int n, int* count);
/* Pipelined reads of the per-step diagnostics (no reference counterpart): ..._async
 * enqueues, on the handle's stream, a copy of the newest entry and the error word into one
 * of RBC_DIAG_SLOTS pinned host slots and returns its ticket without waiting; ..._get waits
 * for that copy only (not for work enqueued after it) and returns the entry, or
 * RBC_ERR_NAN as rbc_diagnostics does. A loop of rbc_step_async(h, 1), rbc_diagnostics_async
 * and rbc_diagnostics_get of the previous ticket keeps the next step queued while the host
 * reads the last one. Tickets older than the last RBC_DIAG_SLOTS are rejected. Before the
 * first step the entry has step 0 and NaN values. */
#define RBC_DIAG_SLOTS 8
rbc_status rbc_diagnostics_async(rbc_handle* h, long long* ticket);
rbc_status rbc_diagnostics_get(rbc_handle* h, long long ticket, rbc_diag* out);
/* Radial shell spectrum of theta(x, y, z): sum of |theta_hat|^2 over the half spectrum
 * in nbins shells of width |q_max| / nbins, as energy_spectrum_2d::reduce_spectrum
 * (gpu_flow/code/postProcessing/energy_spectrum_2d.cu:85-129). */
rbc_status rbc_spectrum(rbc_handle* h, double z, double* bins, int nbins);

/* --- ensembles ------------------------------------------------------------------ */
/* Batched form (no reference counterpart): n independent runs with their own grids,
 * mode counts, Ra, Pr and dt, advanced together. Every ensemble step is one CUDA graph
 * in which each member's step is a branch on one of `nstreams` worker streams (members
 * are spread over the streams by estimated cost, longest first), so the members' kernels
 * run concurrently. Members are ordinary handles (initialise them with
 * rbc_ensemble_member + rbc_init_fields / rbc_set_state). */
typedef struct rbc_ensemble rbc_ensemble;
rbc_status rbc_ensemble_create(const rbc_params* members, int n, int nstreams, rbc_ensemble** out);
void rbc_ensemble_destroy(rbc_ensemble* e);
rbc_handle* rbc_ensemble_member(rbc_ensemble* e, int i);
/* nsteps steps of every member; waits for completion (RBC_ERR_NAN if any member blew up). */
rbc_status rbc_ensemble_step(rbc_ensemble* e, int nsteps);
/* Text of the last error of rbc_ensemble_step ("" when none). */
const char* rbc_ensemble_last_error(const rbc_ensemble* e);
/* Device time in ms (CUDA events on the ensemble's root stream) of the graph-replayed steps
 * of the last rbc_ensemble_step call; 0 when that call replayed none (its first steps, and
 * steps of members with tracers, are enqueued eagerly and not timed here). */
rbc_status rbc_ensemble_elapsed(const rbc_ensemble* e, float* ms);
/* Column-block width W and row pairs per CTA NP chosen for a handle (after tuning). */
rbc_status rbc_launch_config(const rbc_handle* h, int* W, int* NP);

/* --- inspection (tests, tools) ------------------------------------------------- */
/* Physical fields of the current state: 8 blocks [L][Ny][Nx] in the order
 * d_x f, d_y f, q^2 f, d_y g + F, -d_x g + G, theta, d_x theta, d_y theta
 * (the synthesis of nonlinear_operator_rayleigh_noslip.cu:112-233). */
rbc_status rbc_synthesis(rbc_handle* h, double* out);
/* Galerkin table by the reference getter name ("Iac", "Ia1" L*L; "Ibbb", "Ibb1", "Ib11",
 * "I111", "Iabc", "Iac1", "Iaab", "Iaa1", "Iab2", "Ia12" L^3; "lambda" L), index order of
 * gpu_flow/code/util/coeff.cu:1151-1222. Returns the count written in *count. */
rbc_status rbc_table(rbc_handle* h, const char* name, double* out, int* count);
/* Same tables without a handle or a GPU (host computation only). */
rbc_status rbc_galerkin_table(int nz, const char* name, double* out, int* count);
/* Stage timing (CUDA events on the handle's stream around every kernel): runs nsteps
 * steps and returns the mean milliseconds per launch of each kernel kind in
 * ms[RBC_NSTAGE] and the launches per step in counts[RBC_NSTAGE], in the order
 * synth_columns, rows_c2r, tracers, contract, rows_r2c, columns_combine, update.
 * Replaces the reference's -DTIMER host Timer (gpu_flow/code/util/util.cu:230-281). */
#define RBC_NSTAGE 7
rbc_status rbc_stage_times(rbc_handle* h, int nsteps, double* ms, int* counts);
/* FP64 FMA throughput of the device in TFLOP/s (roofline denominator of the FP64
 * contraction; no reference counterpart). */
rbc_status rbc_measure_fp64_peak(int device, double* tflops);
/* --- nonlinear operator without device allocation ----------------------------- */
/* No counterpart in the reference. For callers that cannot call cudaMalloc: a plug-in
 * inside a host framework that has already reserved the device's memory for its own
 * caching allocator (a new cudaMalloc there fails or fragments that pool), or a
 * latency-critical loop that must not pay the implicit device-wide synchronisation of
 * cudaMalloc/cudaFree. The same operator as rbc_nonlinear, without a handle, on DEVICE
 * buffers in the reference layout (inputs theta, f, g [nz][ny][nx/2+1] and F, G [nz]
 * complex; the five outputs alike). It calls no cudaMalloc, cudaFree or allocating
 * library routine: all scratch and tables live in one file-scope __device__ array of
 * RBC_NOALLOC_SCRATCH_BYTES, which every GPU that loads this library holds until the
 * process exits. Limits: nx, ny <= 64 (2^a 3^b, even), 2 <= nz <= 4; larger sizes return
 * RBC_ERR_INVALID_ARG with the reason in errbuf (may be NULL). Set-up happens inside the
 * calls: the first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, with that device current), and the first call of a grid size
 * (nx, ny, nz) on a device, or the first after a call of another size, copies that size's
 * twiddle and coefficient tables into the array from host memory. Make the first call
 * before any stream capture. Every call shares the array and leaves its contents behind
 * (each call rewrites the scratch it reads): calls that overlap on the GPU -- on different
 * streams, or from several host threads -- race and must be serialised by the caller.
 * Work is enqueued on `stream` (cudaStream_t, NULL = legacy default stream) and not
 * waited for; the caller's current device is restored before the call returns. */
#define RBC_NOALLOC_MAX_NX 64
#define RBC_NOALLOC_MAX_NY 64
#define RBC_NOALLOC_MAX_NZ 4
#define RBC_NOALLOC_SCRATCH_BYTES (8u << 20)
rbc_status rbc_nonlinear_noalloc(int device, int nx, int ny, int nz, double lx, double ly, double pr,
                                 const double* theta, const double* f, const double* g,
                                 const double* F, const double* G,
                                 double* out_theta, double* out_f, double* out_g,
                                 double* out_F, double* out_G, void* stream, char* errbuf, int errlen);

/* Device kernel launches issued by the last rbc_step call (for launch accounting). */
long long rbc_kernel_launches(const rbc_handle* h);

/* Second-order structure function of a mid-plane field over nsamples displacements
 * r_i = r_min + i (r_max - r_min) / nsamples along x (direction 0) or y (1), i < nsamples:
 * out[i] = sum over the half spectrum of |FFT[a(x + r) - a(x)] / P|^2. Replaces
 * structure_function_2d::calculate_{temperature,u_1,u_2}_structure_function_{x,y}
 * (gpu_flow/code/postProcessing/structure_function_2d.h:19-54, .cu:32-405), with its field
 * definitions: field 0 theta from mode 0 only, 1 u_1, 2 u_2 from C'_1, C'_2 at z = 0 (its
 * literal lambdas) and mode 0 of g. The reference's result is complex with a zero imaginary
 * part; the real part is returned. */
typedef enum { RBC_SF_THETA = 0, RBC_SF_U1 = 1, RBC_SF_U2 = 2 } rbc_sf_field;
rbc_status rbc_structure_function(rbc_handle* h, int field, int direction, double r_min, double r_max,
                                  int nsamples, double* out);

/* --- field operators of the iteration loop ----------------------------------------- */
/* The reference's freeze and heating operators (main.cu:569-590, -freeze_circle N and
 * -temp_circle N). Both work plane by plane (each vertical mode of a field on its own) on
 * the physical Nx x Ny grid of the unnormalised C2R, where a mask [Ny][Nx] (row-major,
 * column = x index) is 1 to keep the current value; then they scale by 1/(Nx Ny) and
 * return with the unnormalised R2C, which the next step dealiases. Masks:
 *   RBC_MASK_CIRCLE     1 where (col - cx Nx)^2 + (row - cy Ny)^2 > (size/2 min(Nx, Ny))^2
 *   RBC_MASK_RECTANGLE  1 where col < size Nx, col > (1 - size) Nx, row < size Ny or
 *                       row > (1 - size) Ny (a frame of width size around the box)
 * with (cx, cy) = (0.5, 0.5) for the freeze and (0.2, 0.3) for the heating, as the
 * reference's kernels fix them. The handle needs the buffers named in
 * rbc_params.field_ops. A pending tracer advance runs on the state before an operator
 * changes it; the AB2 history is kept (the reference's stepper keeps its res_1). */
typedef enum { RBC_MASK_CIRCLE = 0, RBC_MASK_RECTANGLE = 1 } rbc_mask_shape;
/* Takes the mask and the C2R of theta, f and g (the frozen planes) of the current state.
 * Replaces freeze_operator::freeze_circle / freeze_rectangle
 * (gpu_flow/code/operator/freeze_operator.cu:34-111; main.cu calls freeze_circle(0.8)).
 * The state is left as it is; the reference's out-of-place cuFFT C2R there may overwrite
 * its input, which cuFFT leaves unspecified. */
rbc_status rbc_freeze_mask(rbc_handle* h, int shape, double size);
/* theta, f, g = R2C(mask ? C2R(field) : frozen) / (Nx Ny); F and G untouched. No-op before
 * rbc_freeze_mask. Replaces freeze_operator::calculate_operator (freeze_operator.cu:120-208). */
rbc_status rbc_freeze_apply(rbc_handle* h);
/* Sets the heating mask and increment (the reference adds 1.5/100). Replaces
 * masktemp::temp_circle / temp_rectangle (gpu_flow/code/operator/masktemp.cu:36-95; main.cu
 * calls temp_rectangle(0.1)); the reference's unused C2R copy of theta is not taken. */
rbc_status rbc_heat_mask(rbc_handle* h, int shape, double size, double increment);
/* theta = R2C(mask ? C2R(theta) : C2R(theta) + increment) / (Nx Ny), every vertical mode.
 * No-op before rbc_heat_mask. Replaces masktemp::calculate_operator (masktemp.cu:104-157). */
rbc_status rbc_heat_apply(rbc_handle* h);
/* The interactive temperature mask: theta = R2C(mask ? C2R(theta) : factor C2R(theta)) / (Nx Ny)
 * for every vertical mode, with mask 1 outside the circle of radius radius/2 min(Nx, Ny)
 * centred at column y Nx and row x Ny (the reference swaps x and y there). Replaces
 * masking::set_mask_parameters + masking::masker (gpu_flow/code/operator/masking.cu:24-29,
 * 78-118), which main.cu calls with the UDP viewer's input (main.cu:676-683; defaults
 * x = y = 0.5, radius 0.15, factor 1.1). Needs RBC_FIELD_SCALE. */
rbc_status rbc_masker(rbc_handle* h, double x, double y, double radius, double factor);
/* Drops the frozen planes and the heating mask (later applies are no-ops again). */
rbc_status rbc_field_ops_reset(rbc_handle* h);

/* --- learned surrogate ----------------------------------------------------------- */
/* No counterpart in the reference (jceyy/sdc has no learned component). A Fourier neural
 * operator over the horizontal plane advances a solver's state by one surrogate interval
 * (interval_steps plain steps) at a time. Its input and output are the collocation
 * fields theta, u, v, w at the nq Gauss-Legendre levels z_q of (-1/2, 1/2): FP32
 * [ny][nx][4 nq], channel = field * nq + q. The network predicts their normalized
 * increment; the increment is projected back onto (theta, f, g, F, G) by least squares
 * in z (exact for fields in the span of the basis) and added to the FP64 state. BF16
 * GEMMs with FP32 accumulation, FP32 loss and Adam. Layout of the parameter vector:
 * sdc_b200/csrc/fno.cu. One surrogate serves solvers of one grid (nx, ny, nz). */
typedef struct rbc_fno rbc_fno;
typedef struct {
    int nx, ny;        /* horizontal grid of the solvers it serves */
    int nz;            /* their vertical Galerkin modes */
    int nq;            /* collocation levels (nq >= nz; channels C = 4 nq <= 256) */
    int width;         /* channels of the spectral layers (8..64, a multiple of 8) */
    int modes;         /* retained Fourier modes per direction: kx < m, |ky| < m (+ ky = -m) */
    int layers;        /* spectral layers */
    int hidden;        /* hidden width of the projection (8..256) */
    int max_batch;     /* largest training batch */
    int device;
    unsigned long long seed; /* weight initialisation (SplitMix64) */
    int interval_steps;      /* plain steps one application of the network replaces */
    int physics_mean;        /* 1: after the network, the horizontal-mean modes (theta_k at
                                q = 0, F_k, G_k; they set Nu_wall) are advanced by the plain
                                step's own q = 0 recursion over interval_steps steps, forced by
                                the solver's nonlinear operator at the interval start (linear
                                in time with the previous interval's); 0: from the network */
    int gemm_path;           /* 0: products with K-contiguous rows, N <= 256 and >= 128 rows on
                                the 5th-generation tensor cores (tcgen05, TMEM accumulator),
                                the rest on mma.sync tiles; 1: mma.sync tiles for all */
} rbc_fno_params;
rbc_status rbc_fno_create(const rbc_fno_params* p, rbc_fno** out);
/* BF16 GEMM of the surrogate's kernels on device buffers (no reference counterpart; the
 * numerics check of its tensor-core paths): C[M][N] (FP32, row-major) = A[M][K] B[K][N]
 * (BF16, row-major, FP32 accumulation). path 0: the tcgen05 kernel (TMA-staged A, TMEM
 * accumulator; N <= 256, K <= 256 and a multiple of 8, A 16-byte aligned, B^T within 64 KB,
 * else RBC_ERR_INVALID_ARG), 1: mma.sync tiles. Work on `stream` (NULL: legacy default
 * stream), waited for before the call returns; RBC_ERR_CUDA if a tensor-core wait gave up. */
rbc_status rbc_gemm_bf16(int device, const void* A, const void* B, float* C, int M, int N, int K, int path,
                         void* stream);
void rbc_fno_destroy(rbc_fno* m);
const char* rbc_fno_last_error(const rbc_fno* m);
long long rbc_fno_num_params(const rbc_fno* m);
rbc_status rbc_fno_get_params(rbc_fno* m, float* out, long long n);
rbc_status rbc_fno_set_params(rbc_fno* m, const float* in, long long n); /* resets Adam */
/* Normalization [4][C]: input mean, input std, increment mean, increment std. */
rbc_status rbc_fno_get_norm(rbc_fno* m, float* out);
rbc_status rbc_fno_set_norm(rbc_fno* m, const float* in);
/* The bare network on host buffers x, y [batch][ny][nx][C] (already normalized). */
rbc_status rbc_fno_forward(rbc_fno* m, const float* x, int batch, float* y);
/* Mean-squared-error loss of the network on (x, target) and its gradient with respect to
 * the parameter vector (n = rbc_fno_num_params). */
rbc_status rbc_fno_loss_grad(rbc_fno* m, const float* x, const float* target, int batch, double* loss,
                             float* grad);
/* Collocation fields of a solver's state (out [ny][nx][4 nq]), and the increment form:
 * state += projection of delta [ny][nx][4 nq] (the next step is an Euler step). */
rbc_status rbc_fno_colloc_get(rbc_fno* m, rbc_handle* h, float* out);
rbc_status rbc_fno_colloc_add(rbc_fno* m, rbc_handle* h, const float* delta);
/* Snapshot store on the device (nslots collocation snapshots), filled from solvers. */
rbc_status rbc_fno_dataset_reserve(rbc_fno* m, int nslots);
rbc_status rbc_fno_dataset_capture(rbc_fno* m, rbc_handle* h, int slot);
/* Trains on the pairs (src[i] -> dst[i]) of the store: `epochs` passes in shuffled
 * batches (seeded), Adam with a cosine decay from lr to lr / 50; fit_norm = 1 first sets
 * the normalization from these pairs. epoch_loss[e] = mean loss of epoch e. */
rbc_status rbc_fno_train(rbc_fno* m, const int* src, const int* dst, int npairs, int epochs, int batch, double lr,
                         unsigned long long seed, int fit_norm, double* epoch_loss);
/* Options of later rbc_fno_train calls. augment: 0 none; 1 each training pair mapped by
 * a random reflection of the periodic box (x -> -x and/or y -> -y, velocities as
 * vectors); 2 also the transpose x <-> y (square boxes: nx == ny and Lx == Ly). With
 * augmentation the normalization gives the velocity channels mean 0 (and, with 2, one
 * shared std). noise_rel > 0 adds N(0, (noise_rel * increment std)^2) noise per channel
 * to each training input and trains toward the true next state from the noisy one, so
 * that the network pulls drifted states back during a rollout. pushforward = 1: on every
 * other iteration a pair's input is the network's own prediction from the previous
 * snapshot of the same run (no gradient through that first application), trained toward
 * the pair's true next state (pairs without a previous one use their own input). */
rbc_status rbc_fno_set_train_options(rbc_fno* m, int augment, double noise_rel, int pushforward);
/* n surrogate intervals of the solver's state. */
rbc_status rbc_fno_advance(rbc_fno* m, rbc_handle* h, int n);

/* Rollout with the plain step as judge: every judge_every-th interval the surrogate and
 * the plain step (interval_steps steps) each advance the same state; the rollout
 * keeps the plain result and compares Nu_wall (relative error) and the theta spectrum at
 * z = 0 (relative L2 error over spec_bins bins; 0 bins or spec_tol <= 0: not checked).
 * When an error exceeds its tolerance the plain step takes over for fallback_intervals
 * intervals (-1: the rest of the run). */
typedef struct {
    int intervals;
    int judge_every;
    double nu_tol;
    double spec_tol;
    int spec_bins;
    int fallback_intervals;
} rbc_surrogate_params;
typedef struct {
    int surrogate_intervals, plain_intervals, checks, fallbacks;
    double max_nu_err, max_spec_err, last_nu_err, last_spec_err;
    double ms;         /* device time of the rollout (CUDA events on the solver's stream) */
} rbc_surrogate_report;
/* nu_trace (may be NULL; at most 65536 intervals): Nu_wall after every interval. */
rbc_status rbc_surrogate_run(rbc_fno* m, rbc_handle* h, const rbc_surrogate_params* p, rbc_surrogate_report* rep,
                             double* nu_trace);

#ifdef __cplusplus
}
#endif
#endif /* SDC_B200_RBC_H */
