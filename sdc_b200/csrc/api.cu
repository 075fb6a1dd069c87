// api.cu -- C ABI (include/rbc.h) of the B200-native RBC step: handle, device buffers,
// launch sequence, layout conversion, spectrum. Kernels live in the *.cuh headers.
#include "rbc.h"
#include "common.cuh"
#include "contract_kernel.cuh"
#include "fft.cuh"
#include "galerkin.h"
#include "step_kernels.cuh"
#include "tracer_kernel.cuh"
#include "update_kernel.cuh"
#include "colloc_kernels.cuh"
#include "colloc_tc.cuh"
#include "mask_kernels.cuh"
#include "pen_kernels.cuh"
#include "solver_internal.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

using namespace rbck;

// ------------------------------------------------------------------ helpers
namespace {

struct CudaError {
    cudaError_t e;
    const char* what;
};

#define RBC_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) throw CudaError{e_, #call};                               \
    } while (0)

struct ArgError {
    std::string msg;
};

// Most collocation levels of RBC_FORM_COLLOC (the TMEM columns of the level products).
constexpr int kMaxCollocLevels = 32;

template <typename T> T* dalloc(size_t n, std::vector<void*>& owned)
{
    void* p = nullptr;
    if (n == 0) n = 1;
    RBC_CUDA(cudaMalloc(&p, n * sizeof(T)));
    owned.push_back(p);
    return static_cast<T*>(p);
}

bool fft_len_ok(int n)
{
    if (n < 8 || n > 1024 || (n & 1)) return false;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    return n == 1;
}

} // namespace

// ------------------------------------------------------------------ handle
struct rbc_handle {
    rbc_params prm{};
    unsigned long long uid = 0;   // unique per handle in the process (never reused)
    rbchost::GridInfo gi;
    rbchost::Tables tab;
    Geom G{};
    int W = 4, NP = 8;
    bool mixed = false;
    int colloc_nq = 0;            // collocation form: levels of its nonlinear products (0: other forms)
    float* col_bimg = nullptr;    // its basis operands (shared-memory image, hi then lo)
    float* col_proj = nullptr;    // its level -> mode table [NKIND][Q][Lp]
    int col_grid = 0;
    size_t col_smem = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    std::vector<void*> owned;
    // state (FP64, CM) and AB2 history
    double2 *th = nullptr, *f = nullptr, *g = nullptr, *FG = nullptr;
    double2 *hist = nullptr, *hFG = nullptr;
    bool have_hist = false;
    // operators
    int* cls = nullptr;
    double *optab = nullptr, *diag_tab = nullptr;
    void* coef = nullptr; // R
    double2 *twx = nullptr, *twy = nullptr;
    rbcfft::Plan px{}, py{};
    // scratch (R precision)
    void *H = nullptr, *phys = nullptr, *grp = nullptr, *gh = nullptr, *N = nullptr;
    double* NFG = nullptr;
    // diagnostics
    double *partial = nullptr, *th00 = nullptr, *ring = nullptr;
    unsigned int* ticket = nullptr;
    long long* step_counter = nullptr;
    int* err = nullptr;
    int ring_cap = 4096;
    int upd_blocks = 0;
    int upd_nlow = 0, upd_nkr = 0;  // kept rows r < upd_nlow or r >= upd_nlow + (Ny - upd_nkr)
    long long host_steps = 0;
    // staging for layout conversion
    double2* stage = nullptr;
    // tracers
    int ntr = 0;
    double* trpos = nullptr;      // [3][ntr]
    double* zbasis = nullptr;     // [128][3][L]
    void* nv = nullptr;           // [Ny*Nx][NodeRec] node records for the tracers (R)
    bool tracer_pending = false;  // a fluid step ran whose tracer advance is not done yet
    double tr_sigma = 0.0;        // sqrt(2 D dt) of the diffusion step
    int tr_sets = 1, tr_per_set = 0;  // equal consecutive tracer sets
    double* set_sig = nullptr;    // [tr_sets] sqrt(2 D dt) of each set (device)
    std::vector<double> set_sig_host;
    float* trk = nullptr;         // [trk_cap][3][ntr] recorded frames
    int trk_cap = 0, trk_period = 1;
    long long trk_next = 0;       // step of the oldest unread frame (a multiple of trk_period)
    double* trsums = nullptr;     // [4] moment sums
    long long* tr_step = nullptr; // step counter as of the tracer advance (see snapshot_step)
    // the tracer advance runs on a side stream, forked after the contraction and joined
    // after the update, so that it overlaps the analysis FFTs and the update
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool join_pending = false;
    long long launches = 0;
    int contract_grid = 0, contract_smem = 0;
    // field operators of the iteration loop (freeze, heating), when rbc_params.field_ops
    // asks for their buffers
    unsigned char *fmask = nullptr, *hmask = nullptr, *smask = nullptr; // [Ny][Nx], 1 keeps the value
    double* frozen = nullptr;                        // [3][L][Ny][Nx] C2R of theta, f, g
    bool frozen_set = false, heat_set = false;
    double heat_inc = 0.0;
    int mask_nb = 1;                                 // row pairs per k_mask_rows CTA
    // pipelined diagnostics: pinned slots of [4] doubles + the error word, one event each
    struct DiagSlot { double v[4]; int err; int pad; };
    DiagSlot* dslot = nullptr;
    cudaEvent_t dev_ev[RBC_DIAG_SLOTS] = {};
    long long dticket = 0;                           // tickets issued
    // penalized operator (rbc_params.penalization_eta > 0)
    bool penalized = false;
    double *pen_mask = nullptr, *pen_cf = nullptr, *pen_ia2 = nullptr, *pen_partial = nullptr;
    int pen_blocks = 0;
    // CUDA graphs of one steady-state (AB2) step: [0] without, [1] with the pending
    // tracer advance at its start
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // kChainSteps steady steps with pending tracer advances in one graph: each advance is
    // joined just before the next step's contraction (which rewrites the node records it
    // reads) instead of at the end of its own step, so it also overlaps the next synthesis
    cudaGraphExec_t graph_chain = nullptr;
    cudaStream_t graph_chain_stream = nullptr;
    int graph_chain_launches = 0;
    bool chain_tracers = false;   // while capturing that graph
    bool k1_dep = false;          // K1 follows the previous step's update inside such a graph
    // programmatic dependent launches off: set for ensemble members, whose steps run as
    // concurrent graph branches (CTAs waiting at griddepcontrol.wait would hold SM
    // resources the other branches can use)
    bool no_pdl = false;
    cudaStream_t graph_stream[2] = {nullptr, nullptr};
    int graph_launches[2] = {0, 0};
    bool use_graphs = true;
    // stage timing: events recorded around each launch while `profiling`
    bool profiling = false;
    struct Mark { int stage; cudaEvent_t a, b; };
    std::vector<Mark> marks;
    std::vector<cudaEvent_t> evpool;
    size_t evnext = 0;
    std::string last_error;
};

static rbc_status fail(rbc_handle* h, rbc_status s, const std::string& m)
{
    if (h) h->last_error = m;
    return s;
}

// Stage ids for rbc_stage_times.
enum { ST_SYNTH = 0, ST_C2R, ST_TRACER, ST_CONTRACT, ST_R2C, ST_COMBINE, ST_UPDATE };
static cudaEvent_t pool_event(rbc_handle* h)
{
    if (h->evnext == h->evpool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        h->evpool.push_back(e);
    }
    return h->evpool[h->evnext++];
}
struct StageScope {
    rbc_handle* h;
    int stage;
    cudaEvent_t a = nullptr;
    StageScope(rbc_handle* h_, int s) : h(h_), stage(s)
    {
        if (h->profiling) {
            a = pool_event(h);
            cudaEventRecord(a, h->stream);
        }
    }
    ~StageScope()
    {
        if (h->profiling) {
            cudaEvent_t b = pool_event(h);
            cudaEventRecord(b, h->stream);
            h->marks.push_back({stage, a, b});
        }
    }
};

// ------------------------------------------------------------------ layout kernels
// reference [L][Ny][mox] <-> CM [L][ckp][Ny]; set applies the 2/3 mask.
__global__ void k_ref_to_cm(const double2* __restrict__ src, double2* __restrict__ dst, Geom G, int nmat)
{
    const size_t n = (size_t)nmat * G.ckp * G.ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % G.ny);
        const size_t t = e / G.ny;
        const int c = (int)(t % G.ckp);
        const int k = (int)(t / G.ckp);
        double2 v = make_double2(0, 0);
        if (c < G.ckeep && row_kept(r, G.ny)) v = src[((size_t)k * G.ny + r) * G.mox + c];
        dst[e] = v;
    }
}
__global__ void k_cm_to_ref(const double2* __restrict__ src, double2* __restrict__ dst, Geom G, int nmat)
{
    const size_t n = (size_t)nmat * G.ny * G.mox;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % G.mox);
        const size_t t = e / G.mox;
        const int r = (int)(t % G.ny);
        const int k = (int)(t / G.ny);
        double2 v = make_double2(0, 0);
        if (c < G.ckp) v = src[((size_t)k * G.ckp + c) * G.ny + r];
        dst[e] = v;
    }
}

// Spectrum: one CTA per bin, deterministic block reduction over the half spectrum
// (energy_spectrum_2d.cu:85-129 bins; theta(z) = sum_i S_i(z) theta_i per wavenumber).
__global__ void k_spectrum(const double2* __restrict__ th, Geom G, double z, int nbins, double* __restrict__ bins)
{
    const int b = blockIdx.x;
    const double mmx = 2.0 * kPi * (G.mox - 1) / G.lx, mmy = 2.0 * kPi * (G.ny / 2) / G.ly;
    const double inc = sqrt(mmx * mmx + mmy * mmy) / ((double)nbins);
    const double lo = b * inc, hi = (b + 1) * inc;
    double acc = 0.0;
    for (int e = threadIdx.x; e < G.ckeep * G.ny; e += blockDim.x) {
        const int c = e / G.ny, r = e - c * G.ny;
        const double cx = 2.0 * kPi * c / G.lx;
        const double cy = r <= G.ny / 2 ? 2.0 * kPi * r / G.ly : 2.0 * kPi * (G.ny - r) / G.ly;
        const double a = sqrt(cx * cx + cy * cy);
        if (lo <= a && hi > a) {
            double2 v = make_double2(0, 0);
            for (int i = 0; i < G.L; ++i) {
                const double s = sin(kPi * (i + 1) * (z + 0.5));
                const double2 t = th[((size_t)i * G.ckp + c) * G.ny + r];
                v = make_double2(v.x + s * t.x, v.y + s * t.y);
            }
            acc += v.x * v.x + v.y * v.y;
        }
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) bins[b] = red[0];
}

// Second-order structure functions of the mid-plane fields, one CTA per displacement
// (structure_function_2d.cu:32-405). The reference forms the spectrum of the shifted
// difference D(k) = (e^{i k.r} - 1) A(k), transforms it to physical space, raises it to
// the power order/2 = 1 (its only caller uses order 2), transforms back, scales by 1/P
// and sums |.|^2 over the half spectrum. For a dealiased state with the Hermitian kx = 0
// column that round trip is the identity, so the sum is taken directly:
//   S2(r) = sum_k (2 - 2 cos(k.r)) |A(k)|^2.
// A(k) is the reference's mid-plane field, including its fixed choices
// (twiddle_by_shift_*, structure_function_2d.cu:444-656): theta: theta_0 (mode 0 only);
// u1: i kx sum_{m<2} z_m f_m + i ky g_0; u2: i ky sum_{m<2} z_m f_m - i kx g_0, with
// z_m = C'_m(0) from its literal lambdas 4.73004074 and 7.85320462. Wavenumber rows
// r <= Ny/2 count as positive (get_wave_number_by_index_real_matrix_structure_function).
__global__ void k_structure_function(const double2* __restrict__ th, const double2* __restrict__ f,
                                     const double2* __restrict__ g, Geom G, int field, int dir, double r_min,
                                     double r_inc, double* __restrict__ out)
{
    const int b = blockIdx.x;
    const double rd = r_min + b * r_inc;
    const double r1 = dir == 0 ? rd : 0.0, r2 = dir == 1 ? rd : 0.0;
    const double la = 4.73004074, lb = 7.85320462;
    const double z0 = la * sinh(la * 0.0) / cosh(la * 0.5) + la * sin(la * 0.0) / cos(la * 0.5);
    const double z1 = lb * cosh(lb * 0.0) / sinh(lb * 0.5) - lb * cos(lb * 0.0) / sin(lb * 0.5);
    const size_t plane = (size_t)G.ckp * G.ny;
    double acc = 0.0;
    for (int e = threadIdx.x; e < G.ckeep * G.ny; e += blockDim.x) {
        const int c = e / G.ny, r = e - c * G.ny;
        const double kx = c * 2 * kPi / G.lx;
        const double ky = (r < G.ny / 2 + 1 ? r : r - G.ny) * 2 * kPi / G.ly;
        const size_t o = (size_t)c * G.ny + r;
        double2 a;
        if (field == 0) {
            a = th[o];
        } else {
            double2 fz = f[o] * z0;
            if (G.L > 1) fz = fz + f[plane + o] * z1;
            const double2 g0 = g[o];
            // u1 = i kx fz + i ky g0, u2 = i ky fz - i kx g0
            a = field == 1 ? make_double2(-(kx * fz.y + ky * g0.y), kx * fz.x + ky * g0.x)
                           : make_double2(-(ky * fz.y - kx * g0.y), ky * fz.x - kx * g0.x);
        }
        acc += (2.0 - 2.0 * cos(kx * r1 + ky * r2)) * (a.x * a.x + a.y * a.y);
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) red[threadIdx.x] += red[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = red[0];
}

// ------------------------------------------------------------------ dispatch
// Launch of a step kernel that follows another kernel of the step on the same stream: with
// programmatic stream serialization, so that its CTAs start and load their constant tables
// while the predecessor drains (the kernel fences with pdl_wait before it touches step data).
// Every CTA of every kernel launched this way executes pdl_wait before it can exit, so the
// waits chain: a kernel's wait returns after all earlier kernels of the step completed.
// Step data is read through L2 only (ld_cg / copy_cg, common.cuh): with L1-cached reads the
// penalized operator read stale group values after its read-modify-write kernel. Plain
// launches while stage timing brackets every kernel with events.
template <typename... KArgs, typename... Args>
static void launch_dep(rbc_handle* h, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = (h->profiling || h->no_pdl) ? 0 : 1;
    RBC_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
}

template <typename R, int L> static void setup_contract(rbc_handle* h)
{
    const int smem = (int)(rbcprog::NUNIT * L * L * rbcprog::half_len(L) * sizeof(R));
    RBC_CUDA(cudaFuncSetAttribute(k_contract<R, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int dev = 0, nsm = 148, per = 0;
    RBC_CUDA(cudaGetDevice(&dev));
    RBC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    RBC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_contract<R, L>, 128, smem));
    if (per < 1) per = 1;
    const int need = (h->G.P + 127) / 128;
    h->contract_grid = need < nsm * per ? need : nsm * per;
    h->contract_smem = smem;
}

// The collocation form's contraction (colloc_tc.cuh): the basis operands in the tensor
// cores' shared-memory image (hi and lo TF32 parts), the weighted level -> mode table, the
// launch shape.
template <typename R, int L> static void setup_colloc(rbc_handle* h)
{
    const int Q = h->colloc_nq;
    const CollocGeom cg = colloc_geom(L, Q);
    int dev = 0, optin = 0, nsm = 148, per = 0;
    RBC_CUDA(cudaGetDevice(&dev));
    RBC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    RBC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    h->col_smem = (size_t)cg.smem + 1024;
    if (cg.tcols > 512 || h->col_smem > (size_t)optin) throw ArgError{"collocation levels exceed the tensor-core tile"};
    rbchost::CollocContract t;
    rbchost::colloc_contract_tables(L, Q, t);
    std::vector<float> img(cg.b_bytes / sizeof(float), 0.0f);
    for (int f = 0; f < 8; ++f) {
        const int p0 = rbccol::field_first_pair(f), np = rbccol::field_pairs(f);
        for (int j = 0; j < np; ++j) {
            const int kind = rbccol::spair_at(p0 + j).kind;
            for (int q = 0; q < Q; ++q)
                for (int i = 0; i < L; ++i) {
                    const double v = t.basis[((size_t)kind * L + i) * Q + q];
                    uint32_t bits;
                    const float vf = (float)v;
                    std::memcpy(&bits, &vf, 4);
                    bits &= 0xFFFFE000u; // TF32 part
                    float hi;
                    std::memcpy(&hi, &bits, 4);
                    const float lo = (float)(v - (double)hi);
                    const unsigned o = cg.b_off[f] + colloc_kmajor_off(j * Q + q, i, cg.Kp);
                    img[o / 4] = hi;
                    img[(cg.b_half + o) / 4] = lo;
                }
        }
    }
    std::vector<float> proj((size_t)rbccol::NKIND * Q * cg.Lp, 0.0f);
    for (int c = 0; c < rbccol::NKIND; ++c)
        for (int q = 0; q < Q; ++q)
            for (int k = 0; k < L; ++k) proj[((size_t)c * Q + q) * cg.Lp + k] = (float)t.proj[((size_t)c * Q + q) * L + k];
    h->col_bimg = dalloc<float>(img.size(), h->owned);
    h->col_proj = dalloc<float>(proj.size(), h->owned);
    RBC_CUDA(cudaMemcpy(h->col_bimg, img.data(), img.size() * sizeof(float), cudaMemcpyHostToDevice));
    RBC_CUDA(cudaMemcpy(h->col_proj, proj.data(), proj.size() * sizeof(float), cudaMemcpyHostToDevice));
    RBC_CUDA(cudaFuncSetAttribute(k_colloc_contract<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->col_smem));
    RBC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_colloc_contract<L>, kColThreads, h->col_smem));
    if (per < 1) throw ArgError{"collocation contraction does not fit an SM"};
    // one CTA per SM at most holds the TMEM columns without waiting for another CTA's
    if (cg.tcols * per > 512) per = 512 / cg.tcols;
    const int ntiles = (h->G.P + kColM - 1) / kColM;
    h->col_grid = std::min(ntiles, nsm * per);
}

template <typename R, int L> static void launch_contract(rbc_handle* h)
{
    StageScope sc(h, ST_CONTRACT);
    if constexpr (std::is_same<R, float>::value) {
        if (h->colloc_nq > 0) {
            CollocArgs A;
            A.phys = (const float*)h->phys;
            A.grp = (float*)h->grp;
            A.nv = h->tracer_pending ? (float*)h->nv : nullptr;
            A.step_counter = h->step_counter;
            A.step_copy = h->tr_step;
            A.bimg = h->col_bimg;
            A.proj = h->col_proj;
            A.P = h->G.P;
            A.ntiles = (h->G.P + kColM - 1) / kColM;
            A.err = h->err;
            launch_dep(h, k_colloc_contract<L>, dim3(h->col_grid), dim3(kColThreads), h->col_smem, A, h->colloc_nq);
            RBC_CUDA(cudaGetLastError());
            ++h->launches;
            return;
        }
    }
    R* nv = h->tracer_pending ? (R*)h->nv : nullptr; // node records for the tracer advance
    launch_dep(h, k_contract<R, L>, dim3(h->contract_grid), dim3(128), (size_t)h->contract_smem, (const R*)h->phys,
               (R*)h->grp, (const R*)h->coef, h->G.P, nv, (const long long*)h->step_counter, h->tr_step);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

template <typename R, int L> static void launch_node_records(rbc_handle* h)
{
    const int grid = std::min((h->G.P + 255) / 256, 148 * 8);
    k_node_records<R, L><<<grid, 256, 0, h->stream>>>((const R*)h->phys, h->G.P, (R*)h->nv);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

template <typename R, int L> static void launch_update(rbc_handle* h)
{
    UpdateArgs A;
    A.G = h->G;
    A.cls = h->cls;
    A.optab = h->optab;
    A.diag_tab = h->diag_tab;
    A.N = h->N;
    A.NFG = h->NFG;
    A.th = h->th;
    A.f = h->f;
    A.g = h->g;
    A.FG = h->FG;
    A.hist = h->hist;
    A.hFG = h->hFG;
    A.first = h->have_hist ? 0 : 1;
    A.partial = h->partial;
    A.ticket = h->ticket;
    A.th00 = h->th00;
    A.ring = h->ring;
    A.ring_cap = h->ring_cap;
    A.step_counter = h->step_counter;
    A.err = h->err;
    A.nlow = h->upd_nlow;
    A.nkr = h->upd_nkr;
    StageScope sc(h, ST_UPDATE);
    launch_dep(h, k_update<R, L>, dim3(h->upd_blocks), dim3(kThreads), 0, A);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

#define RBC_DISPATCH_L(FN, R, Lv, h)                                                    \
    switch (Lv) {                                                                         \
    case 2: FN<R, 2>(h); break;                                                           \
    case 3: FN<R, 3>(h); break;                                                           \
    case 4: FN<R, 4>(h); break;                                                           \
    case 5: FN<R, 5>(h); break;                                                           \
    case 6: FN<R, 6>(h); break;                                                           \
    case 8: FN<R, 8>(h); break;                                                           \
    case 12: FN<R, 12>(h); break;                                                         \
    default: throw ArgError{"unsupported number of vertical modes"};                      \
    }

static bool L_supported(int L, bool mixed)
{
    (void)mixed;
    return L == 2 || L == 3 || L == 4 || L == 5 || L == 6 || L == 8 || L == 12;
}

// Lanes per transform of the register FFT for the x and y lengths (0: Stockham passes),
// and the length that selects the register-FFT kernels (0: the Stockham kernels).
static int rx_x(const rbc_handle* h) { return rbcfft::reg_fft_lanes(h->G.nx); }
static int rx_y(const rbc_handle* h) { return rbcfft::reg_fft_lanes(h->G.ny); }
static int reg_nx(const rbc_handle* h) { return rx_x(h) ? h->G.nx : 0; }
static int reg_ny(const rbc_handle* h) { return rx_y(h) ? h->G.ny : 0; }
// Row pairs (transforms) a row-kernel CTA can hold: one per TL lanes of kThreads threads,
// or one Stockham chunk.
static int max_row_pairs(const rbc_handle* h) { return rx_x(h) ? kThreads / rx_x(h) : h->px.chunk; }

template <typename R> static size_t smem_cols(const rbc_handle* h, int nfield)
{
    const size_t c = sizeof(typename cplx_t<R>::type);
    if (const int rx = rx_y(h))
        return c * ((size_t)h->G.ny + (size_t)nfield * h->W * tp_stride(h->G.ny)) +
               sizeof(double2) * 3 * (size_t)h->W * h->G.ny;
    return c * ((size_t)h->G.ny + (size_t)nfield * h->W * h->py.stride);
}
template <typename R> static size_t smem_combine(const rbc_handle* h)
{
    const int rx = rx_y(h);
    return sizeof(typename cplx_t<R>::type) * ((size_t)h->G.ny + 13 * (size_t)(rx ? tp_stride(h->G.ny) : h->py.stride));
}
template <typename R> static size_t smem_rows(const rbc_handle* h)
{
    const int rx = rx_x(h);
    return sizeof(typename cplx_t<R>::type) * ((size_t)h->G.nx + (size_t)h->NP * (rx ? tp_stride(h->G.nx) : h->px.stride));
}

// Grid of the analysis row kernel: at most the CTAs that are resident at once (each CTA
// then loops over its items and prefetches the next one), never more than the items.
template <typename K> static int resident_grid(const rbc_handle* h, K kernel, int threads, size_t smem, int items)
{
    (void)h;
    int dev = 0, nsm = 148, per = 0;
    RBC_CUDA(cudaGetDevice(&dev));
    RBC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    RBC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
    const long long res = (long long)nsm * (per > 0 ? per : 1);
    return (int)std::min<long long>(items, res);
}

template <typename R> static void launch_tracer_from_synthesis(rbc_handle* h);

// Synthesis: K1 (columns) + K2 (rows) into h->phys from the state in (th, f, g, FG).
template <typename R>
static void run_synthesis(rbc_handle* h, const double2* th, const double2* f, const double2* g, const double2* FG)
{
    typedef typename cplx_t<R>::type C;
    const Geom& G = h->G;
    dim3 g1(G.ckw / h->W, G.L);
    {
    StageScope sc(h, ST_SYNTH);
    const size_t sm = smem_cols<R>(h, 8);
    switch (reg_ny(h)) {
#define RBC_SYNTH_TP(NN)                                                                                                          \
    case NN:                                                                                                                      \
        if (h->k1_dep) launch_dep(h, k_synth_columns_tp<R, NN>, g1, dim3(8 * h->W * rx_y(h)), sm, G, h->W, (const double2*)h->twy, th, f, g, FG, (C*)h->H); \
        else k_synth_columns_tp<R, NN><<<g1, 8 * h->W * rx_y(h), sm, h->stream>>>(G, h->W, h->twy, th, f, g, FG, (C*)h->H); \
        break;
    RBC_SYNTH_TP(512)
    RBC_SYNTH_TP(256)
    RBC_SYNTH_TP(192)
    RBC_SYNTH_TP(128)
    RBC_SYNTH_TP(64)
#undef RBC_SYNTH_TP
    default:
        if (h->k1_dep) launch_dep(h, k_synth_columns<R>, g1, dim3(kThreads), sm, G, h->W, h->py, (const double2*)h->twy, th, f, g, FG, (C*)h->H);
        else k_synth_columns<R><<<g1, kThreads, sm, h->stream>>>(G, h->W, h->py, h->twy, th, f, g, FG, (C*)h->H);
    }
    RBC_CUDA(cudaGetLastError());
    }
    const int rows = 8 * G.L * G.ny;
    StageScope sc(h, ST_C2R);
    const int nb = rows / (2 * h->NP);
    const size_t sm = smem_rows<R>(h);
    const dim3 tb(h->NP * rx_x(h));
    switch (reg_nx(h)) {
    case 512: launch_dep(h, k_rows_c2r_tp<R, 512>, dim3(nb), tb, sm, G, h->NP, (const double2*)h->twx, (const C*)h->H, (R*)h->phys); break;
    case 256: launch_dep(h, k_rows_c2r_tp<R, 256>, dim3(nb), tb, sm, G, h->NP, (const double2*)h->twx, (const C*)h->H, (R*)h->phys); break;
    case 192: launch_dep(h, k_rows_c2r_tp<R, 192>, dim3(nb), tb, sm, G, h->NP, (const double2*)h->twx, (const C*)h->H, (R*)h->phys); break;
    case 128: launch_dep(h, k_rows_c2r_tp<R, 128>, dim3(nb), tb, sm, G, h->NP, (const double2*)h->twx, (const C*)h->H, (R*)h->phys); break;
    case 64: launch_dep(h, k_rows_c2r_tp<R, 64>, dim3(nb), tb, sm, G, h->NP, (const double2*)h->twx, (const C*)h->H, (R*)h->phys); break;
    default: launch_dep(h, k_rows_c2r<R>, dim3(nb), dim3(kThreads), sm, G, h->NP, h->px, (const double2*)h->twx, (const C*)h->H, (R*)h->phys);
    }
    RBC_CUDA(cudaGetLastError());
    h->launches += 2;
}

// Nonlinear operator from phys into N / NFG: K3 + K4 + K5 over the columns of G.
static void join_tracer(rbc_handle* h)
{
    if (!h->join_pending) return;
    RBC_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    h->join_pending = false;
}

// The tracer advance of step m reads m (diffusion noise, track frame) while, on the side
// stream, the update kernel of the step it overlaps increments the step counter: the
// advance reads a copy taken on the main stream before the fork (inside the step, by the
// contraction kernel that writes the node records; here, for an advance from a synthesis
// that no step starts from).
static void snapshot_step(rbc_handle* h)
{
    RBC_CUDA(cudaMemcpyAsync(h->tr_step, h->step_counter, sizeof(long long), cudaMemcpyDeviceToDevice, h->stream));
}

// Forward x and y transforms of the contracted groups (after the contraction). With a
// pending tracer advance the tracer kernel is forked onto the side stream right after
// the contraction that wrote its node records; defer_join leaves the join to the caller
// (run_step joins after the update), otherwise it is joined here.
template <typename R, int L> static void launch_penalize(rbc_handle* h);
template <typename R, int L> static void launch_penalize_fg(rbc_handle* h);

template <typename R> static void run_analysis(rbc_handle* h, const Geom& G, bool defer_join = false)
{
    typedef typename cplx_t<R>::type C;
    join_tracer(h); // an advance still reading the node records ends before they are rewritten
    RBC_DISPATCH_L(launch_contract, R, G.L, h); // with a pending advance it also copies the step counter
    if (h->tracer_pending) {
        if (h->side && !h->profiling) {
            RBC_CUDA(cudaEventRecord(h->ev_fork, h->stream));
            RBC_CUDA(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
            cudaStream_t main_stream = h->stream;
            h->stream = h->side;
            launch_tracer_from_synthesis<R>(h);
            h->stream = main_stream;
            RBC_CUDA(cudaEventRecord(h->ev_join, h->side));
            h->join_pending = true;
        } else {
            launch_tracer_from_synthesis<R>(h);
        }
    }
    if (h->penalized) RBC_DISPATCH_L(launch_penalize, R, G.L, h);
    const int rows = 13 * G.L * G.ny;
    {
    StageScope sc(h, ST_R2C);
    const int nb = rows / (2 * h->NP);
    const size_t sm = smem_rows<R>(h);
    const dim3 tb(h->NP * rx_x(h));
    switch (reg_nx(h)) {
    case 512: launch_dep(h, k_rows_r2c_tp<R, 512>, dim3(resident_grid(h, k_rows_r2c_tp<R, 512>, tb.x, sm, nb)), tb, sm, G, h->NP, nb, (const double2*)h->twx, (const R*)h->grp, (C*)h->gh); break;
    case 256: launch_dep(h, k_rows_r2c_tp<R, 256>, dim3(resident_grid(h, k_rows_r2c_tp<R, 256>, tb.x, sm, nb)), tb, sm, G, h->NP, nb, (const double2*)h->twx, (const R*)h->grp, (C*)h->gh); break;
    case 192: launch_dep(h, k_rows_r2c_tp<R, 192>, dim3(resident_grid(h, k_rows_r2c_tp<R, 192>, tb.x, sm, nb)), tb, sm, G, h->NP, nb, (const double2*)h->twx, (const R*)h->grp, (C*)h->gh); break;
    case 128: launch_dep(h, k_rows_r2c_tp<R, 128>, dim3(resident_grid(h, k_rows_r2c_tp<R, 128>, tb.x, sm, nb)), tb, sm, G, h->NP, nb, (const double2*)h->twx, (const R*)h->grp, (C*)h->gh); break;
    case 64: launch_dep(h, k_rows_r2c_tp<R, 64>, dim3(resident_grid(h, k_rows_r2c_tp<R, 64>, tb.x, sm, nb)), tb, sm, G, h->NP, nb, (const double2*)h->twx, (const R*)h->grp, (C*)h->gh); break;
    default: launch_dep(h, k_rows_r2c<R>, dim3(nb), dim3(kThreads), sm, G, h->NP, h->px, (const double2*)h->twx, (const R*)h->grp, (C*)h->gh);
    }
    RBC_CUDA(cudaGetLastError());
    }
    dim3 g5(G.ckw, G.L);
    {
    StageScope sc(h, ST_COMBINE);
    const size_t sm = smem_combine<R>(h);
    const dim3 tb(std::min(13 * rx_y(h), kThreads));
    switch (reg_ny(h)) {
    case 512: launch_dep(h, k_columns_combine_tp<R, 512>, g5, tb, sm, G, (const double2*)h->twy, (const C*)h->gh, (C*)h->N, h->NFG); break;
    case 256: launch_dep(h, k_columns_combine_tp<R, 256>, g5, tb, sm, G, (const double2*)h->twy, (const C*)h->gh, (C*)h->N, h->NFG); break;
    case 192: launch_dep(h, k_columns_combine_tp<R, 192>, g5, tb, sm, G, (const double2*)h->twy, (const C*)h->gh, (C*)h->N, h->NFG); break;
    case 128: launch_dep(h, k_columns_combine_tp<R, 128>, g5, tb, sm, G, (const double2*)h->twy, (const C*)h->gh, (C*)h->N, h->NFG); break;
    case 64: launch_dep(h, k_columns_combine_tp<R, 64>, g5, tb, sm, G, (const double2*)h->twy, (const C*)h->gh, (C*)h->N, h->NFG); break;
    default: launch_dep(h, k_columns_combine<R>, g5, dim3(kThreads), sm, G, h->py, (const double2*)h->twy, (const C*)h->gh, (C*)h->N, h->NFG);
    }
    RBC_CUDA(cudaGetLastError());
    }
    h->launches += 2;
    if (h->penalized) RBC_DISPATCH_L(launch_penalize_fg, R, G.L, h);
    if (!defer_join) join_tracer(h);
}


// ------------------------------------------------------------------ tracers
// 128 z levels of particle_tracer.cu:151-154 and the basis values of
// calculate_velocity_operator.cu:458-488 (get_z_coeff_at), host FP64.
static void tracer_setup(rbc_handle* h)
{
    h->ntr = h->prm.n_tracers;
    if (h->ntr == 0) return;
    const int L = h->G.L;
    const double zmax = 0.5f - 1e-3;
    std::vector<double> zb((size_t)kZNum * 3 * L);
    for (int l = 0; l < kZNum; ++l) {
        double z = -zmax + l * (zmax - -zmax) / (kZNum - 1);
        if (z < -0.5) z = -0.5;
        else if (z > 0.5) z = 0.5;
        for (int i = 0; i < L; ++i) {
            const int m = i + 1;
            const double lam = h->tab.lambda[i], lz = lam * z;
            double C, D;
            if (m % 2 == 1) {
                const double ich = 1.0 / std::cosh(lam * 0.5), ic = 1.0 / std::cos(lam * 0.5);
                C = std::cosh(lz) * ich - std::cos(lz) * ic;
                D = lam * (std::sinh(lz) * ich + std::sin(lz) * ic);
            } else {
                const double ish = 1.0 / std::sinh(lam * 0.5), is = 1.0 / std::sin(lam * 0.5);
                C = std::sinh(lz) * ish - std::sin(lz) * is;
                D = lam * (std::cosh(lz) * ish - std::cos(lz) * is);
            }
            zb[((size_t)l * 3 + 0) * L + i] = C;
            zb[((size_t)l * 3 + 1) * L + i] = std::sin(kPi * m * (z + 0.5));
            zb[((size_t)l * 3 + 2) * L + i] = D;
        }
    }
    h->zbasis = dalloc<double>(zb.size(), h->owned);
    RBC_CUDA(cudaMemcpy(h->zbasis, zb.data(), zb.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->trpos = dalloc<double>(3 * (size_t)h->ntr, h->owned);
    const size_t rsz = h->mixed ? sizeof(float) : sizeof(double);
    h->nv = dalloc<unsigned char>((size_t)h->G.P * node_rec_len(L) * rsz, h->owned);
    RBC_CUDA(cudaMemset(h->trpos, 0, 3 * (size_t)h->ntr * sizeof(double)));
    h->trsums = dalloc<double>(4, h->owned);
    h->tr_step = dalloc<long long>(1, h->owned);
    RBC_CUDA(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    RBC_CUDA(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    RBC_CUDA(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    const double D = h->prm.tracer_diffusivity;
    h->tr_sigma = D > 0 ? std::sqrt(2.0 * D * h->G.dt) : 0.0;
    h->tr_sets = h->prm.tracer_sets > 1 ? h->prm.tracer_sets : 1;
    h->tr_per_set = h->ntr / h->tr_sets;
    h->set_sig_host.assign(h->tr_sets, h->tr_sigma);
    h->set_sig = dalloc<double>(h->tr_sets, h->owned);
    RBC_CUDA(cudaMemcpy(h->set_sig, h->set_sig_host.data(), h->tr_sets * sizeof(double), cudaMemcpyHostToDevice));
    h->trk_period = h->prm.track_period > 1 ? h->prm.track_period : 1;
    h->trk_cap = h->prm.track_frames;
    if (h->trk_cap > 0) {
        h->trk = dalloc<float>((size_t)h->trk_cap * 3 * h->ntr, h->owned);
        RBC_CUDA(cudaMemset(h->trk, 0, (size_t)h->trk_cap * 3 * h->ntr * sizeof(float)));
    }
}

// Step of the newest tracer positions: the fluid steps taken, minus a pending advance.
static long long tracer_time(const rbc_handle* h) { return h->host_steps - (h->tracer_pending ? 1 : 0); }

// Unread track frames if the tracer positions were at step `upto`.
static long long track_frames_until(const rbc_handle* h, long long upto)
{
    if (upto < h->trk_next) return 0;
    return upto / h->trk_period - h->trk_next / h->trk_period + 1;
}

// New positions were set at the current step: the track restarts there.
static void track_reset(rbc_handle* h)
{
    if (!h->trk) return;
    const long long m = h->host_steps, P = h->trk_period;
    h->trk_next = ((m + P - 1) / P) * P;
    if (m % P == 0) {
        float* fr = h->trk + (size_t)((m / P) % h->trk_cap) * 3 * h->ntr;
        k_track_frame<<<(3 * h->ntr + 255) / 256, 256, 0, h->stream>>>(h->trpos, fr, h->ntr);
        RBC_CUDA(cudaGetLastError());
    }
}

// Steps whose frames would overrun the ring are refused (particle_tracer.cu:145-147).
static bool track_room(const rbc_handle* h, long long nsteps)
{
    return !h->trk || track_frames_until(h, h->host_steps + nsteps) <= h->trk_cap;
}
static const char* kTrackFull = "track ring full: read the recorded frames (rbc_tracks_read) before stepping on";

template <typename R, int L> static void launch_tracer_L(rbc_handle* h)
{
    TracerArgs A;
    A.nv = h->nv;
    A.zbasis = h->zbasis;
    A.pos = h->trpos;
    A.n = h->ntr;
    A.nx = h->G.nx;
    A.ny = h->G.ny;
    A.L = L;
    A.lx = h->G.lx;
    A.ly = h->G.ly;
    A.dt = h->G.dt;
    A.zmax = 0.5f - 1e-3;
    A.sx = h->G.nx / h->G.lx;
    A.sy = h->G.ny / h->G.ly;
    A.sz = (kZNum - 1) / (2 * A.zmax);
    A.inx = 1.0 / h->G.nx;
    A.iny = 1.0 / h->G.ny;
    A.set_sigma = h->set_sig;
    A.per_set = h->tr_per_set;
    A.noise_seed = h->prm.noise_seed;
    A.step_counter = h->tr_step;
    A.track = h->trk;
    A.track_cap = h->trk_cap;
    A.track_period = h->trk_period;
    StageScope sc(h, ST_TRACER);
    // 8 lanes per tracer; each team's 4 corner records in shared memory
    k_tracers<R, L><<<(8 * h->ntr + kTracerThreads - 1) / kTracerThreads, kTracerThreads, tracer_smem<R, L>(),
                      h->stream>>>(A);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

// Tracer advance with the velocity of the synthesis currently in h->phys.
template <typename R> static void launch_tracer_from_synthesis(rbc_handle* h)
{
    if (h->ntr == 0) return;
    RBC_DISPATCH_L(launch_tracer_L, R, h->G.L, h);
}

// One iteration of the reference loop (main.cu:612-637). The tracer advance of a step
// needs the velocity of the state after it, which is exactly the synthesis the next
// step starts with; it is therefore run there (or by flush_tracers).
__global__ void k_force_mean(double2* __restrict__ FG, double v) { FG[0] = make_double2(v, 0.0); }

template <typename R> static void flush_tracers_t(rbc_handle* h, bool overlap);

template <typename R> static void run_step(rbc_handle* h)
{
    if (h->prm.mean_F != 0.0) {
        // force_mean comes before the step, after the previous step's tracer advance, which
        // must see the unforced mean flow: a pending advance runs on its own synthesis first
        flush_tracers_t<R>(h, false);
        k_force_mean<<<1, 1, 0, h->stream>>>(h->FG, h->prm.mean_F);
        RBC_CUDA(cudaGetLastError());
        ++h->launches;
    }
    run_synthesis<R>(h, h->th, h->f, h->g, h->FG);
    run_analysis<R>(h, h->G, true); // the contraction also writes the tracers' node records
    h->tracer_pending = false;
    RBC_DISPATCH_L(launch_update, R, h->G.L, h);
    if (!h->chain_tracers) join_tracer(h); // in a chain the next step's analysis joins it
    h->have_hist = true;
    h->tracer_pending = h->ntr > 0;
    ++h->host_steps;
}

// overlap: the advance goes to the side stream and the caller calls join_tracer(h) once
// the work it overlaps (which must leave the tracer data and node records alone) is enqueued.
template <typename R> static void flush_tracers_t(rbc_handle* h, bool overlap)
{
    if (!h->tracer_pending) return;
    run_synthesis<R>(h, h->th, h->f, h->g, h->FG);
    RBC_DISPATCH_L(launch_node_records, R, h->G.L, h); // no step starts from this synthesis
    snapshot_step(h);
    if (overlap && h->side && !h->profiling) {
        RBC_CUDA(cudaEventRecord(h->ev_fork, h->stream));
        RBC_CUDA(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
        cudaStream_t main_stream = h->stream;
        h->stream = h->side;
        launch_tracer_from_synthesis<R>(h);
        h->stream = main_stream;
        RBC_CUDA(cudaEventRecord(h->ev_join, h->side));
        h->join_pending = true;
    } else {
        launch_tracer_from_synthesis<R>(h);
    }
    h->tracer_pending = false;
}
static void flush_tracers(rbc_handle* h, bool overlap = false)
{
    if (h->mixed) flush_tracers_t<float>(h, overlap);
    else flush_tracers_t<double>(h, overlap);
}

template <typename R, int L> static void set_tracer_attribute(rbc_handle*)
{
    RBC_CUDA(cudaFuncSetAttribute(k_tracers<R, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tracer_smem<R, L>()));
}

// The dynamic shared-memory limit is an attribute of the kernel, shared by every handle
// in the process; it is set to the device's opt-in maximum (a cap only: occupancy follows
// the size each launch asks for), so handles of different shapes can run side by side.
template <typename R> static void set_attributes(rbc_handle* h)
{
    int dev = 0, optin = 0;
    RBC_CUDA(cudaGetDevice(&dev));
    RBC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t need = std::max({smem_cols<R>(h, 8), smem_combine<R>(h), smem_rows<R>(h)});
    if (need > (size_t)optin) throw ArgError{"grid too large for the FFT kernels' shared memory"};
    RBC_CUDA(cudaFuncSetAttribute(k_synth_columns<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_columns_combine<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_c2r<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_r2c<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_synth_columns_tp<R, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_synth_columns_tp<R, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_synth_columns_tp<R, 192>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_synth_columns_tp<R, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_synth_columns_tp<R, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_c2r_tp<R, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_c2r_tp<R, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_c2r_tp<R, 192>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_c2r_tp<R, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_c2r_tp<R, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_r2c_tp<R, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_r2c_tp<R, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_r2c_tp<R, 192>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_r2c_tp<R, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_rows_r2c_tp<R, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_columns_combine_tp<R, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_columns_combine_tp<R, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_columns_combine_tp<R, 192>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_columns_combine_tp<R, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_columns_combine_tp<R, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    if (h->prm.n_tracers > 0) RBC_DISPATCH_L(set_tracer_attribute, R, h->G.L, h);
}

// ------------------------------------------------------------------ autotuner
// Times the four FFT kernels (synthesis columns and rows, analysis rows and columns)
// for every admissible column block W in {1, 2, 4} and row-pair count NP (divisors of
// Ny/2 up to the FFT chunk) on the handle's own scratch, and keeps the fastest pair.
static void autotune(rbc_handle* h)
{
    Geom& G = h->G;
    const bool mixed = h->mixed;
    const size_t csz = mixed ? sizeof(float2) : sizeof(double2);
    int best_W = h->W, best_NP = h->NP;
    float best = 1e30f;
    cudaEvent_t a, b;
    RBC_CUDA(cudaEventCreate(&a));
    RBC_CUDA(cudaEventCreate(&b));
    int dev = 0, optin = 0;
    RBC_CUDA(cudaGetDevice(&dev));
    RBC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    (void)csz;
    for (int W = 1; W <= 4; W *= 2) {
        if (8 * W > h->py.chunk && W > 1) continue;
        if (rx_y(h) && 8 * W * rx_y(h) > kThreads) continue;
        for (int NP = 1; NP <= 32 && NP <= max_row_pairs(h); ++NP) {
            if ((G.ny / 2) % NP) continue;
            if (rx_x(h) && NP * rx_x(h) > kThreads) continue;
            const int W0 = h->W, NP0 = h->NP;
            h->W = W;
            h->NP = NP;
            const size_t need = mixed ? std::max({smem_cols<float>(h, 8), smem_combine<float>(h), smem_rows<float>(h)})
                                      : std::max({smem_cols<double>(h, 8), smem_combine<double>(h), smem_rows<double>(h)});
            if (need > (size_t)optin) {
                h->W = W0;
                h->NP = NP0;
                continue;
            }
            G.ckw = ((G.ckeep + W - 1) / W) * W;
            if (mixed) set_attributes<float>(h);
            else set_attributes<double>(h);
            float t = 0;
            for (int rep = 0; rep < 4; ++rep) {
                RBC_CUDA(cudaEventRecord(a, h->stream));
                if (mixed) { run_synthesis<float>(h, h->th, h->f, h->g, h->FG); run_analysis<float>(h, G); }
                else { run_synthesis<double>(h, h->th, h->f, h->g, h->FG); run_analysis<double>(h, G); }
                RBC_CUDA(cudaEventRecord(b, h->stream));
                RBC_CUDA(cudaEventSynchronize(b));
                float ms = 0;
                RBC_CUDA(cudaEventElapsedTime(&ms, a, b));
                if (rep > 0) t += ms; // first repetition warms up
            }
            if (t < best) { best = t; best_W = W; best_NP = NP; }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->W = best_W;
    h->NP = best_NP;
    G.ckw = ((G.ckeep + best_W - 1) / best_W) * best_W;
    if (mixed) set_attributes<float>(h);
    else set_attributes<double>(h);
    h->launches = 0;
}

// ------------------------------------------------------------------ penalization
// Mask of the reference's PENALIZED builds (see rbc_pen_mask), [Ny][Nx], col = index % Nx.
static void pen_mask_host(int nx, int ny, int kind, std::vector<double>& m)
{
    m.assign((size_t)nx * ny, 0.0);
    for (int row = 0; row < ny; ++row)
        for (int col = 0; col < nx; ++col) {
            bool in = false;
            if (kind == RBC_PEN_RECTANGLE) {
                in = col < 3 || col > nx - 4 || row < 3 || row > ny - 4;
            } else if (kind == RBC_PEN_CIRCLE) {
                const int mn = std::min(nx, ny);
                in = (col - nx / 2) * (col - nx / 2) + (row - ny / 2) * (row - ny / 2) > (mn / 2 - 3) * (mn / 2 - 3);
            } else if (kind == RBC_PEN_DISK_ARRAY) {
                const int r = std::min(nx / 6, ny / 4);
                for (int a = 0; a < 3 && !in; ++a)
                    for (int b = 0; b < 2 && !in; ++b) {
                        const int cx = a * nx / 3 + nx / 6, cy = b * ny / 2 + ny / 4;
                        in = (cx - col) * (cx - col) + (cy - row) * (cy - row) < r;
                    }
            } else {
                in = true;
            }
            m[(size_t)row * nx + col] = in ? 1.0 : 0.0;
        }
}

// Mask, group coefficients (layout of k_penalize) and the partial-sum buffer.
static void penalization_setup(rbc_handle* h)
{
    const rbc_params& p = h->prm;
    if (!(p.penalization_eta > 0)) return;
    const Geom& G = h->G;
    const int L = G.L;
    std::vector<double> m;
    pen_mask_host(G.nx, G.ny, p.penalization_mask, m);
    const double pe = p.pr / p.penalization_eta;
    const auto& T = h->tab;
    auto Iac = [&](int a, int c) { return T.Iac[a + c * L]; };
    auto Ia2 = [&](int a, int c) { return T.Ia2[a + c * L]; };
    std::vector<double> cf((size_t)2 * L * 4 * L, 0.0);
    auto at = [&](int g, int k, int f, int j) -> double& { return cf[((size_t)g * L + k) * 4 * L + f * L + j]; };
    for (int k = 0; k < L; ++k)
        for (int j = 0; j < L; ++j) {
            const double d = j == k ? 0.5 * pe : 0.0;
            at(0, k, 0, j) = pe * Iac(j, k);  // d_x: u11
            at(0, k, 1, j) = pe * Ia2(j, k);  //      u21 (the reference's third "g" summand)
            at(0, k, 2, j) = pe * Ia2(k, j);  //      u12
            at(1, k, 0, j) = -pe * Ia2(j, k); // d_y: u11 (first "g" summand)
            at(1, k, 1, j) = pe * Iac(j, k);  //      u21
            at(1, k, 2, j) = d;               //      u12 (second "g" summand)
            at(1, k, 3, j) = pe * Ia2(k, j) - d; //   u22 (and the fourth "g" summand)
        }
    h->pen_mask = dalloc<double>(m.size(), h->owned);
    RBC_CUDA(cudaMemcpy(h->pen_mask, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->pen_cf = dalloc<double>(cf.size(), h->owned);
    RBC_CUDA(cudaMemcpy(h->pen_cf, cf.data(), cf.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->pen_ia2 = dalloc<double>(T.Ia2.size(), h->owned);
    RBC_CUDA(cudaMemcpy(h->pen_ia2, T.Ia2.data(), T.Ia2.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->pen_blocks = (G.P + kPenThreads - 1) / kPenThreads;
    h->pen_partial = dalloc<double>((size_t)h->pen_blocks * 4 * L, h->owned);
    h->penalized = true;
}

template <typename R, int L> static void launch_penalize(rbc_handle* h)
{
    const rbc_params& p = h->prm;
    launch_dep(h, k_penalize<R, L>, dim3(h->pen_blocks), dim3(kPenThreads), 0, (const R*)h->phys, (R*)h->grp,
               (const double*)h->pen_mask, (const double*)h->pen_cf, h->G.P, p.pr / p.penalization_eta,
               0.5 / p.penalization_eta, h->pen_partial);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

template <typename R, int L> static void launch_penalize_fg(rbc_handle* h)
{
    launch_dep(h, k_penalize_fg<L>, dim3(1), dim3(kPenFgThreads), 0, (const double*)h->pen_partial, h->pen_blocks,
               (const double*)h->pen_ia2, 1.0 / (h->prm.penalization_eta * h->G.P), h->NFG);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* rbc_status_string(rbc_status s)
{
    switch (s) {
    case RBC_OK: return "ok";
    case RBC_ERR_INVALID_ARG: return "invalid argument";
    case RBC_ERR_CUDA: return "CUDA error";
    case RBC_ERR_NAN: return "non-finite value in the state";
    case RBC_ERR_TIMEOUT: return "timeout";
    case RBC_ERR_IO: return "I/O error";
    case RBC_ERR_UNSUPPORTED: return "unsupported";
    case RBC_ERR_OUT_OF_MEMORY: return "out of device memory";
    }
    return "unknown status";
}

const char* rbc_last_error(const rbc_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

static void free_all(rbc_handle* h)
{
    for (int v = 0; v < 2; ++v)
        if (h->graph[v]) cudaGraphExecDestroy(h->graph[v]);
    if (h->graph_chain) cudaGraphExecDestroy(h->graph_chain);
    h->graph_chain = nullptr;
    for (cudaEvent_t e : h->evpool) cudaEventDestroy(e);
    h->evpool.clear();
    for (void* p : h->owned) cudaFree(p);
    h->owned.clear();
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    h->own_stream = nullptr;
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    h->side = nullptr;
    h->ev_fork = h->ev_join = nullptr;
    for (auto& e : h->dev_ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    if (h->dslot) cudaFreeHost(h->dslot);
    h->dslot = nullptr;
}

void rbc_destroy(rbc_handle* h)
{
    if (!h) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(h->prm.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->side) cudaStreamSynchronize(h->side);
    free_all(h);
    cudaSetDevice(cur);
    delete h;
}

static void twiddles(int n, std::vector<double2>& tw)
{
    tw.resize(n);
    for (int t = 0; t < n; ++t) {
        const long double a = -2.0L * 3.14159265358979323846264338327950288L * t / n;
        tw[t] = make_double2((double)cosl(a), (double)sinl(a));
    }
}

// ------------------------------------------------------------------ field operators
static size_t smem_mask_cols(const rbc_handle* h, int W)
{
    return (size_t)(h->G.ny + W * h->py.stride) * sizeof(double2);
}
static size_t smem_mask_rows(const rbc_handle* h, int nb)
{
    return (size_t)(h->G.nx + nb * h->px.stride + 2 * nb * h->G.ckeep) * sizeof(double2);
}

// Buffers of the freeze and heating operators. Their column and row passes use the
// synthesis scratch H (8 L planes of R complex values; 3 L FP64 planes fit in both forms).
static void field_ops_setup(rbc_handle* h)
{
    const int ops = h->prm.field_ops;
    if (!ops) return;
    const Geom& G = h->G;
    if (ops & RBC_FIELD_FREEZE) {
        h->fmask = dalloc<unsigned char>((size_t)G.P, h->owned);
        h->frozen = dalloc<double>((size_t)3 * G.L * G.P, h->owned);
    }
    if (ops & RBC_FIELD_HEAT) h->hmask = dalloc<unsigned char>((size_t)G.P, h->owned);
    if (ops & RBC_FIELD_SCALE) h->smask = dalloc<unsigned char>((size_t)G.P, h->owned);
    int dev = 0, optin = 0;
    RBC_CUDA(cudaGetDevice(&dev));
    RBC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    // row pairs per CTA: the most that leave room for two CTAs per SM
    int nb = h->px.chunk;
    while (nb > 1 && smem_mask_rows(h, nb) > (size_t)optin / 2) nb /= 2;
    if (smem_mask_rows(h, nb) > (size_t)optin || smem_mask_cols(h, h->py.chunk) > (size_t)optin)
        throw ArgError{"grid too large for the field operators' shared memory"};
    h->mask_nb = nb;
    RBC_CUDA(cudaFuncSetAttribute(k_mask_cols<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_mask_cols<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    RBC_CUDA(cudaFuncSetAttribute(k_mask_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
}

// One operator over the first nfields of (theta, f, g): KM1, KM2 and (unless the pass
// only takes the frozen planes) KM3.
static void mask_pass(rbc_handle* h, int nfields, int op, const unsigned char* mask, double increment)
{
    const Geom& G = h->G;
    MaskFields fl{{h->th, h->f, h->g}};
    const int planes = nfields * G.L;
    double2* S = static_cast<double2*>(h->H);
    // column CTAs: about four per SM over all planes, each with a thread per butterfly
    int rmin = 1 << 30;
    for (int i = 0; i < h->py.npass; ++i) rmin = std::min(rmin, h->py.radix[i]);
    const int W = std::max(1, std::min(h->py.chunk, (G.ckeep * planes + 4 * 148 - 1) / (4 * 148)));
    const int tc = std::min(kThreads, std::max(32, (W * G.ny / rmin + 31) / 32 * 32));
    const dim3 gc((G.ckeep + W - 1) / W, planes);
    const size_t smc = smem_mask_cols(h, W);
    k_mask_cols<1><<<gc, tc, smc, h->stream>>>(G, W, h->py, h->twy, fl, S);
    RBC_CUDA(cudaGetLastError());
    const int nb = h->mask_nb;
    k_mask_rows<<<dim3((G.ny + 2 * nb - 1) / (2 * nb), planes), kThreads, smem_mask_rows(h, nb), h->stream>>>(
        G, nb, h->px, h->twx, S, op, mask, h->frozen, increment);
    RBC_CUDA(cudaGetLastError());
    h->launches += 2;
    if (op == MASK_SNAPSHOT) return;
    k_mask_cols<-1><<<gc, tc, smc, h->stream>>>(G, W, h->py, h->twy, fl, S);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

static void make_mask(rbc_handle* h, unsigned char* mask, int shape, double cx, double cy, double size)
{
    const int P = h->G.P;
    k_field_mask<<<(P + 255) / 256, 256, 0, h->stream>>>(mask, h->G.nx, h->G.ny, shape, cx, cy, size);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}

rbc_status rbc_create(const rbc_params* p, rbc_handle** out)
{
    if (!p || !out) return RBC_ERR_INVALID_ARG;
    *out = nullptr;
    if (!fft_len_ok(p->nx) || !fft_len_ok(p->ny)) return RBC_ERR_INVALID_ARG;
    if (!(p->lx > 0 && p->ly > 0 && p->pr > 0 && p->dt > 0) || p->n_tracers < 0) return RBC_ERR_INVALID_ARG;
    if (p->tracer_sets < 0 || (p->tracer_sets > 1 && (p->n_tracers == 0 || p->n_tracers % p->tracer_sets)))
        return RBC_ERR_INVALID_ARG;
    if (!(p->tracer_diffusivity >= 0 && std::isfinite(p->tracer_diffusivity)) || p->track_frames < 0 ||
        p->track_period < 0 || (p->track_frames > 0 && p->n_tracers == 0))
        return RBC_ERR_INVALID_ARG;
    if (p->form != RBC_FORM_FP64 && p->form != RBC_FORM_MIXED && p->form != RBC_FORM_COLLOC)
        return RBC_ERR_INVALID_ARG;
    if (p->form == RBC_FORM_COLLOC && (p->colloc_nq < 0 || p->colloc_nq % 8 ||
                                       (p->colloc_nq > 0 && p->colloc_nq < p->nz) || p->colloc_nq > kMaxCollocLevels))
        return RBC_ERR_INVALID_ARG;
    if (p->field_ops & ~(RBC_FIELD_FREEZE | RBC_FIELD_HEAT | RBC_FIELD_SCALE)) return RBC_ERR_INVALID_ARG;
    if (!std::isfinite(p->mean_F)) return RBC_ERR_INVALID_ARG;
    if (!(p->penalization_eta >= 0 && std::isfinite(p->penalization_eta)) || p->penalization_mask < 0 ||
        p->penalization_mask > RBC_PEN_EVERYWHERE)
        return RBC_ERR_INVALID_ARG;
    if (!L_supported(p->nz, p->form != RBC_FORM_FP64)) return RBC_ERR_UNSUPPORTED;
    rbc_handle* h = new rbc_handle;
    h->prm = *p;
    {
        static std::atomic<unsigned long long> next_uid{1};
        h->uid = next_uid++;
    }
    h->mixed = p->form != RBC_FORM_FP64;
    // default: 2 nz levels, rounded up to the tensor-core K granularity of 8
    h->colloc_nq = p->form == RBC_FORM_COLLOC ? (p->colloc_nq > 0 ? p->colloc_nq : std::max(8, (2 * p->nz + 7) / 8 * 8)) : 0;
    if (p->diag_capacity > 0) h->ring_cap = p->diag_capacity;
    try {
        RBC_CUDA(cudaSetDevice(p->device));
        rbchost::grid_info(p->nx, p->ny, p->nz, p->lx, p->ly, p->ra, p->pr, p->dt, h->gi);
        // the collocation form's nonlinear tensors are its level rule's sums
        rbchost::build_tables(p->nz, h->tab, h->colloc_nq);
        const size_t csz = h->mixed ? sizeof(float2) : sizeof(double2);
        h->px = rbcfft::make_plan(p->nx);
        h->py = rbcfft::make_plan(p->ny);
        // synthesis CTAs take W columns (8 W transforms) to fill one FFT chunk
        int W = 1;
        while (W < 4 && 8 * (2 * W) <= h->py.chunk) W *= 2;
        h->W = W;
        // row kernels: NP row pairs per CTA, a divisor of Ny/2 that fits one CTA's transforms
        int NP = 1;
        const int tlx = rbcfft::reg_fft_lanes(p->nx);
        for (int c = 1; c <= 32 && c <= (tlx ? kThreads / tlx : h->px.chunk); ++c)
            if ((p->ny / 2) % c == 0) NP = c;
        h->NP = NP;
        Geom& G = h->G;
        G.nx = p->nx;
        G.ny = p->ny;
        G.mox = p->nx / 2 + 1;
        G.L = p->nz;
        G.ckeep = h->gi.ckeep;
        G.ckw = ((G.ckeep + W - 1) / W) * W;
        G.ckp = ((G.mox + 3) / 4) * 4; // stride padded for any column block W <= 4
        G.P = p->nx * p->ny;
        G.lx = p->lx;
        G.ly = p->ly;
        G.pr = p->pr;
        G.dt = p->dt;
        RBC_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
        h->stream = h->own_stream;
        const int L = G.L;
        const size_t plane = (size_t)G.ckp * G.ny;
        h->th = dalloc<double2>(plane * L, h->owned);
        h->f = dalloc<double2>(plane * L, h->owned);
        h->g = dalloc<double2>(plane * L, h->owned);
        h->FG = dalloc<double2>(2 * L, h->owned);
        h->hist = dalloc<double2>(3 * plane * L, h->owned);
        h->hFG = dalloc<double2>(2 * L, h->owned);
        // operators
        rbchost::OperatorTables op;
        rbchost::build_operator_tables(h->gi, h->tab, op);
        std::vector<int> cls_cm(plane, -1);
        for (int c = 0; c < G.ckeep; ++c)
            for (int r = 0; r < G.ny; ++r) cls_cm[(size_t)c * G.ny + r] = op.cls[(size_t)r * G.mox + c];
        h->cls = dalloc<int>(plane, h->owned);
        RBC_CUDA(cudaMemcpy(h->cls, cls_cm.data(), plane * sizeof(int), cudaMemcpyHostToDevice));
        // parity-packed rows of B_ff^-1 and the implicit blocks (update_kernel.cuh)
        {
            const int H = op_half(L), RW = op_row(L);
            std::vector<double> pk((size_t)op.nclass * L * RW, 0.0);
            for (int c = 0; c < op.nclass; ++c)
                for (int b = 0; b < 5; ++b) {
                    const double* m = b == 0 ? &op.binv[(size_t)c * L * L] : &op.imp[((size_t)c * 4 + b - 1) * L * L];
                    for (int k = 0; k < L; ++k)
                        for (int j = 0; j < L; ++j) {
                            const double v = m[(size_t)k * L + j];
                            if ((j - k) & 1) {
                                if (v != 0.0) throw ArgError{"operator tables couple modes of opposite parity"};
                            } else {
                                pk[((size_t)c * L + k) * RW + (size_t)b * H + j / 2] = v;
                            }
                        }
                }
            h->optab = dalloc<double>(pk.size(), h->owned);
            RBC_CUDA(cudaMemcpy(h->optab, pk.data(), pk.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
        std::vector<double> dtab;
        dtab.insert(dtab.end(), h->tab.CpCp.begin(), h->tab.CpCp.end());
        dtab.insert(dtab.end(), h->tab.CC.begin(), h->tab.CC.end());
        dtab.insert(dtab.end(), h->tab.CS.begin(), h->tab.CS.end());
        for (int t = 0; t < 3; ++t) // the diagnostics skip the opposite-parity entries too
            for (int k = 0; k < L; ++k)
                for (int j = 0; j < L; ++j)
                    if (((j - k) & 1) && dtab[(size_t)t * L * L + k + (size_t)j * L] != 0.0)
                        throw ArgError{"diagnostic integrals couple modes of opposite parity"};
        h->diag_tab = dalloc<double>(dtab.size(), h->owned);
        RBC_CUDA(cudaMemcpy(h->diag_tab, dtab.data(), dtab.size() * sizeof(double), cudaMemcpyHostToDevice));
        std::vector<double> coef;
        rbchost::pack_contraction(h->tab, coef);
        if (h->mixed) {
            std::vector<float> cf(coef.begin(), coef.end());
            h->coef = dalloc<float>(cf.size(), h->owned);
            RBC_CUDA(cudaMemcpy(h->coef, cf.data(), cf.size() * sizeof(float), cudaMemcpyHostToDevice));
        } else {
            h->coef = dalloc<double>(coef.size(), h->owned);
            RBC_CUDA(cudaMemcpy(h->coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
        std::vector<double2> tw;
        twiddles(G.nx, tw);
        h->twx = dalloc<double2>(G.nx, h->owned);
        RBC_CUDA(cudaMemcpy(h->twx, tw.data(), G.nx * sizeof(double2), cudaMemcpyHostToDevice));
        twiddles(G.ny, tw);
        h->twy = dalloc<double2>(G.ny, h->owned);
        RBC_CUDA(cudaMemcpy(h->twy, tw.data(), G.ny * sizeof(double2), cudaMemcpyHostToDevice));
        // scratch
        const size_t rsz = h->mixed ? sizeof(float) : sizeof(double);
        h->H = dalloc<unsigned char>(8 * plane * L * csz, h->owned);
        h->phys = dalloc<unsigned char>((size_t)8 * L * G.P * rsz, h->owned);
        h->grp = dalloc<unsigned char>((size_t)13 * L * G.P * rsz, h->owned);
        h->gh = dalloc<unsigned char>(13 * plane * L * csz, h->owned);
        h->N = dalloc<unsigned char>(3 * plane * L * csz, h->owned);
        h->NFG = dalloc<double>(2 * L, h->owned);
        // the 2/3 rule keeps a prefix and a suffix of the rows
        h->upd_nlow = 0;
        while (h->upd_nlow < G.ny && row_kept(h->upd_nlow, G.ny)) ++h->upd_nlow;
        h->upd_nkr = 0;
        for (int r = 0; r < G.ny; ++r)
            if (row_kept(r, G.ny)) ++h->upd_nkr;
        for (int r = 0; r < G.ny; ++r) {
            const bool want = r < h->upd_nlow || r >= h->upd_nlow + (G.ny - h->upd_nkr);
            if (want != row_kept(r, G.ny)) throw ArgError{"kept rows are not a prefix and a suffix"};
        }
        switch (L) {
        case 2: h->upd_blocks = update_blocks<2>(G.ckeep, h->upd_nkr); break;
        case 3: h->upd_blocks = update_blocks<3>(G.ckeep, h->upd_nkr); break;
        case 4: h->upd_blocks = update_blocks<4>(G.ckeep, h->upd_nkr); break;
        case 5: h->upd_blocks = update_blocks<5>(G.ckeep, h->upd_nkr); break;
        case 6: h->upd_blocks = update_blocks<6>(G.ckeep, h->upd_nkr); break;
        case 8: h->upd_blocks = update_blocks<8>(G.ckeep, h->upd_nkr); break;
        default: h->upd_blocks = update_blocks<12>(G.ckeep, h->upd_nkr); break;
        }
        h->partial = dalloc<double>(2 * (size_t)h->upd_blocks, h->owned);
        h->th00 = dalloc<double>(L, h->owned);
        h->ring = dalloc<double>(4 * ((size_t)h->ring_cap + 1), h->owned); // + the newest entry
        h->ticket = dalloc<unsigned int>(1, h->owned);
        h->step_counter = dalloc<long long>(1, h->owned);
        h->err = dalloc<int>(1, h->owned);
        h->stage = dalloc<double2>((size_t)G.ny * G.mox * L, h->owned);
        RBC_CUDA(cudaMemset(h->ticket, 0, sizeof(unsigned int)));
        RBC_CUDA(cudaMemset(h->step_counter, 0, sizeof(long long)));
        RBC_CUDA(cudaMemset(h->err, 0, sizeof(int)));
        RBC_CUDA(cudaMemset(h->ring, 0, 4 * ((size_t)h->ring_cap + 1) * sizeof(double)));
        RBC_CUDA(cudaMemset(h->th, 0, plane * L * sizeof(double2)));
        RBC_CUDA(cudaMemset(h->f, 0, plane * L * sizeof(double2)));
        RBC_CUDA(cudaMemset(h->g, 0, plane * L * sizeof(double2)));
        RBC_CUDA(cudaMemset(h->FG, 0, 2 * L * sizeof(double2)));
        RBC_CUDA(cudaMemset(h->hist, 0, 3 * plane * L * sizeof(double2)));
        RBC_CUDA(cudaMemset(h->hFG, 0, 2 * L * sizeof(double2)));
        RBC_CUDA(cudaMemset(h->H, 0, 8 * plane * L * csz));
        RBC_CUDA(cudaMemset(h->gh, 0, 13 * plane * L * csz));
        RBC_CUDA(cudaMemset(h->N, 0, 3 * plane * L * csz));
        if (h->mixed) {
            set_attributes<float>(h);
            RBC_DISPATCH_L(setup_contract, float, G.L, h);
            if (h->colloc_nq > 0) RBC_DISPATCH_L(setup_colloc, float, G.L, h);
        } else {
            set_attributes<double>(h);
            RBC_DISPATCH_L(setup_contract, double, G.L, h);
        }
        tracer_setup(h);
        RBC_CUDA(cudaHostAlloc((void**)&h->dslot, RBC_DIAG_SLOTS * sizeof(rbc_handle::DiagSlot), cudaHostAllocDefault));
        for (auto& e : h->dev_ev) RBC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        field_ops_setup(h);
        penalization_setup(h);
        RBC_CUDA(cudaDeviceSynchronize());
        if (p->tune) autotune(h);
    } catch (const CudaError& e) {
        std::string m = std::string("rbc_create: ") + e.what + ": " + cudaGetErrorString(e.e);
        std::fprintf(stderr, "%s\n", m.c_str());
        const bool oom = e.e == cudaErrorMemoryAllocation;
        free_all(h);
        delete h;
        return oom ? RBC_ERR_OUT_OF_MEMORY : RBC_ERR_CUDA;
    } catch (const ArgError& e) {
        free_all(h);
        delete h;
        return RBC_ERR_UNSUPPORTED;
    }
    *out = h;
    return RBC_OK;
}

rbc_status rbc_set_stream(rbc_handle* h, void* stream)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return RBC_OK;
}

#define RBC_GUARD(h)                                                                        \
    if (!h) return RBC_ERR_INVALID_ARG;                                                     \
    try {                                                                                   \
        RBC_CUDA(cudaSetDevice(h->prm.device));
#define RBC_GUARD_END(h)                                                                    \
    }                                                                                       \
    catch (const CudaError& e) {                                                            \
        return fail(h, e.e == cudaErrorMemoryAllocation ? RBC_ERR_OUT_OF_MEMORY : RBC_ERR_CUDA, \
                    std::string(e.what) + ": " + cudaGetErrorString(e.e));                   \
    }                                                                                       \
    catch (const ArgError& e) {                                                             \
        return fail(h, RBC_ERR_UNSUPPORTED, e.msg);                                         \
    }

static void upload_field(rbc_handle* h, const double* src, double2* dst, int nmat)
{
    // only the kept band crosses to the device: the kept prefix and suffix of rows of every
    // matrix, columns c < ckeep (k_ref_to_cm reads nothing else of the staging copy), as two
    // strided copies
    const Geom& G = h->G;
    const size_t rowb = (size_t)G.mox * sizeof(double2);
    const int nlow = h->upd_nlow, nkr = h->upd_nkr;
    for (int part = 0; part < 2; ++part) {
        const int r0 = part == 0 ? 0 : nlow + (G.ny - nkr), nr = part == 0 ? nlow : nkr - nlow;
        if (nr <= 0) continue;
        cudaMemcpy3DParms cp = {};
        cp.srcPtr = make_cudaPitchedPtr(const_cast<double*>(src), rowb, rowb, G.ny);
        cp.dstPtr = make_cudaPitchedPtr(h->stage, rowb, rowb, G.ny);
        cp.srcPos = make_cudaPos(0, r0, 0);
        cp.dstPos = make_cudaPos(0, r0, 0);
        cp.extent = make_cudaExtent((size_t)G.ckeep * sizeof(double2), nr, nmat);
        cp.kind = cudaMemcpyHostToDevice;
        RBC_CUDA(cudaMemcpy3DAsync(&cp, h->stream));
    }
    k_ref_to_cm<<<512, 256, 0, h->stream>>>(h->stage, dst, h->G, nmat);
    RBC_CUDA(cudaGetLastError());
}
static void download_field(rbc_handle* h, const double2* src, double* dst, int nmat)
{
    const size_t n = (size_t)h->G.ny * h->G.mox * nmat;
    k_cm_to_ref<<<512, 256, 0, h->stream>>>(src, h->stage, h->G, nmat);
    RBC_CUDA(cudaGetLastError());
    RBC_CUDA(cudaMemcpyAsync(dst, h->stage, n * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
}

rbc_status rbc_set_state(rbc_handle* h, const double* th, const double* f, const double* g, const double* F, const double* G)
{
    if (!th || !f || !g || !F || !G) return fail(h, RBC_ERR_INVALID_ARG, "null state buffer");
    RBC_GUARD(h)
    flush_tracers(h);
    const int L = h->G.L;
    upload_field(h, th, h->th, L);
    upload_field(h, f, h->f, L);
    upload_field(h, g, h->g, L);
    std::vector<double2> fg(2 * L);
    std::memcpy(fg.data(), F, L * sizeof(double2));
    std::memcpy(fg.data() + L, G, L * sizeof(double2));
    RBC_CUDA(cudaMemcpyAsync(h->FG, fg.data(), 2 * L * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    h->have_hist = false;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_get_state(rbc_handle* h, double* th, double* f, double* g, double* F, double* G)
{
    if (!th || !f || !g || !F || !G) return fail(h, RBC_ERR_INVALID_ARG, "null state buffer");
    RBC_GUARD(h)
    const int L = h->G.L;
    download_field(h, h->th, th, L);
    download_field(h, h->f, f, L);
    download_field(h, h->g, g, L);
    std::vector<double2> fg(2 * L);
    RBC_CUDA(cudaMemcpyAsync(fg.data(), h->FG, 2 * L * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    std::memcpy(F, fg.data(), L * sizeof(double2));
    std::memcpy(G, fg.data() + L, L * sizeof(double2));
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_init_fields(rbc_handle* h, unsigned long long seed, double amplitude, double kmax)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    const int L = h->G.L;
    const size_t n = (size_t)h->G.ny * h->G.mox * L;
    std::vector<double> th(2 * n), zero(2 * n, 0.0), fg(2 * L, 0.0);
    rbchost::seeded_theta(h->gi, seed, amplitude, kmax, th.data());
    return rbc_set_state(h, th.data(), zero.data(), zero.data(), fg.data(), fg.data());
}

rbc_status rbc_init_pattern(rbc_handle* h, int pattern, double mode, double amplitude, unsigned long long seed,
                            double noise)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (pattern < RBC_INIT_ISR || pattern > RBC_INIT_TEST || !std::isfinite(mode) || !std::isfinite(amplitude) ||
        !(noise >= 0))
        return fail(h, RBC_ERR_INVALID_ARG, "unknown pattern or bad amplitude");
    const int L = h->G.L;
    const size_t n = (size_t)h->G.ny * h->G.mox * L;
    std::vector<double> th(2 * n), f(2 * n, 0.0), g(2 * n, 0.0), F(2 * L, 0.0), G(2 * L, 0.0);
    rbchost::pattern_theta(h->gi, pattern, mode, amplitude, seed, noise, th.data(), f.data(), F.data());
    return rbc_set_state(h, th.data(), f.data(), g.data(), F.data(), G.data());
}

static rbc_status check_err(rbc_handle* h)
{
    int e = 0;
    RBC_CUDA(cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    if (e & RBC_DEVERR_NAN) return fail(h, RBC_ERR_NAN, "non-finite value in the state");
    if (e) return fail(h, RBC_ERR_CUDA, "device error word set");
    return RBC_OK;
}

// Captures one steady-state step (history present; tracer advance pending or not) on
// the current stream into an executable graph.
static void capture_step(rbc_handle* h, int variant)
{
    if (h->graph[variant]) {
        cudaGraphExecDestroy(h->graph[variant]);
        h->graph[variant] = nullptr;
    }
    const bool hist = h->have_hist, pend = h->tracer_pending;
    const long long launches = h->launches, hs = h->host_steps;
    h->have_hist = true;
    h->tracer_pending = variant == 1;
    cudaGraph_t g = nullptr;
    RBC_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->launches = 0;
    try {
        if (h->mixed) run_step<float>(h);
        else run_step<double>(h);
    } catch (...) {
        cudaStreamEndCapture(h->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    RBC_CUDA(cudaStreamEndCapture(h->stream, &g));
    h->graph_launches[variant] = (int)h->launches;
    cudaError_t e = cudaGraphInstantiate(&h->graph[variant], g, 0);
    cudaGraphDestroy(g);
    RBC_CUDA(e);
    h->graph_stream[variant] = h->stream;
    h->have_hist = hist;
    h->tracer_pending = pend;
    h->launches = launches;
    h->host_steps = hs;
}

constexpr int kChainSteps = 8;

// Captures kChainSteps steady steps, each with a pending tracer advance, into one graph.
static void capture_chain(rbc_handle* h)
{
    if (h->graph_chain) {
        cudaGraphExecDestroy(h->graph_chain);
        h->graph_chain = nullptr;
    }
    const bool hist = h->have_hist, pend = h->tracer_pending;
    const long long launches = h->launches, hs = h->host_steps;
    cudaGraph_t g = nullptr;
    RBC_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->launches = 0;
    h->chain_tracers = true;
    try {
        for (int i = 0; i < kChainSteps; ++i) {
            h->have_hist = true;
            h->tracer_pending = true;
            h->k1_dep = i > 0; // after the previous step's update, which wrote the state
            if (h->mixed) run_step<float>(h);
            else run_step<double>(h);
        }
        h->k1_dep = false;
        join_tracer(h); // the last advance
    } catch (...) {
        h->chain_tracers = false;
        h->k1_dep = false;
        h->join_pending = false;
        cudaStreamEndCapture(h->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    h->chain_tracers = false;
    RBC_CUDA(cudaStreamEndCapture(h->stream, &g));
    h->graph_chain_launches = (int)h->launches;
    cudaError_t e = cudaGraphInstantiate(&h->graph_chain, g, 0);
    cudaGraphDestroy(g);
    RBC_CUDA(e);
    h->graph_chain_stream = h->stream;
    h->have_hist = hist;
    h->tracer_pending = pend;
    h->launches = launches;
    h->host_steps = hs;
}

// Instantiates every steady-step graph a run on the current stream can replay (the
// single step with and without a pending tracer advance, and the kChainSteps chain when
// tracers are on) the first time any of them is needed, so that a later call replays
// graphs only and never captures and instantiates in the middle of a run of steps.
static void prepare_graphs(rbc_handle* h)
{
    if (h->ntr > 0) {
        if (!h->graph[1] || h->graph_stream[1] != h->stream) capture_step(h, 1);
        if (!h->graph_chain || h->graph_chain_stream != h->stream) capture_chain(h);
    }
    if (!h->graph[0] || h->graph_stream[0] != h->stream) capture_step(h, 0);
}

rbc_status rbc_step_async(rbc_handle* h, int nsteps)
{
    if (nsteps < 0) return fail(h, RBC_ERR_INVALID_ARG, "negative step count");
    if (h && !track_room(h, nsteps)) return fail(h, RBC_ERR_INVALID_ARG, kTrackFull);
    RBC_GUARD(h)
    h->launches = 0;
    for (int s = 0; s < nsteps; ++s) {
        // graphs need a real stream (the legacy default stream cannot be captured)
        if (h->use_graphs && h->have_hist && !h->profiling && h->stream != nullptr) {
            prepare_graphs(h);
            if (h->tracer_pending && h->ntr > 0 && nsteps - s >= kChainSteps) {
                if (!h->graph_chain || h->graph_chain_stream != h->stream) capture_chain(h);
                RBC_CUDA(cudaGraphLaunch(h->graph_chain, h->stream));
                h->launches += h->graph_chain_launches;
                h->tracer_pending = true;
                h->host_steps += kChainSteps;
                s += kChainSteps - 1;
                continue;
            }
            const int v = h->tracer_pending ? 1 : 0;
            if (!h->graph[v] || h->graph_stream[v] != h->stream) capture_step(h, v);
            RBC_CUDA(cudaGraphLaunch(h->graph[v], h->stream));
            h->launches += h->graph_launches[v];
            h->tracer_pending = h->ntr > 0;
            ++h->host_steps;
        } else {
            if (h->mixed) run_step<float>(h);
            else run_step<double>(h);
        }
    }
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_synchronize(rbc_handle* h)
{
    RBC_GUARD(h)
    return check_err(h); // its read of the error word waits for all work on the stream
    RBC_GUARD_END(h)
}

rbc_status rbc_step(rbc_handle* h, int nsteps)
{
    rbc_status s = rbc_step_async(h, nsteps);
    if (s != RBC_OK) return s;
    return rbc_synchronize(h);
}

long long rbc_kernel_launches(const rbc_handle* h) { return h ? h->launches : 0; }

rbc_status rbc_stage_times(rbc_handle* h, int nsteps, double* ms, int* counts)
{
    if (!ms || !counts || nsteps <= 0) return fail(h, RBC_ERR_INVALID_ARG, "bad arguments");
    RBC_GUARD(h)
    h->marks.clear();
    // events for all launches exist before anything is queued
    h->evnext = 0;
    for (int i = 0; i < 2 * RBC_NSTAGE * (nsteps + 1); ++i) pool_event(h);
    h->evnext = 0;
    // head start: queue unprofiled steps first so that the profiled launches are
    // enqueued while the GPU is still busy (no host gaps inside the event pairs)
    for (int s = 0; s < nsteps; ++s) {
        if (h->mixed) run_step<float>(h);
        else run_step<double>(h);
    }
    h->profiling = true;
    for (int s = 0; s < nsteps; ++s) {
        if (h->mixed) run_step<float>(h);
        else run_step<double>(h);
    }
    flush_tracers(h);
    h->profiling = false;
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    double tot[RBC_NSTAGE] = {0};
    int cnt[RBC_NSTAGE] = {0};
    for (auto& m : h->marks) {
        float t = 0;
        cudaEventElapsedTime(&t, m.a, m.b);
        tot[m.stage] += t;
        cnt[m.stage] += 1;
    }
    h->marks.clear();
    for (int i = 0; i < RBC_NSTAGE; ++i) {
        ms[i] = cnt[i] ? tot[i] / cnt[i] : 0.0;
        counts[i] = cnt[i] / nsteps;
    }
    return check_err(h);
    RBC_GUARD_END(h)
}

rbc_status rbc_save_state(rbc_handle* h, const char* dir, long long step, int real_bytes)
{
    if (!h || !dir || (real_bytes != 4 && real_bytes != 8)) return fail(h, RBC_ERR_INVALID_ARG, "bad arguments");
    const Geom& G = h->G;
    const int L = G.L;
    const size_t n = (size_t)L * G.ny * G.mox;
    std::vector<double> th(2 * n), f(2 * n), g(2 * n), F(2 * L), Gm(2 * L);
    rbc_status s = rbc_get_state(h, th.data(), f.data(), g.data(), F.data(), Gm.data());
    if (s != RBC_OK) return s;
    const int d3[3] = {G.mox, G.ny, L}, d1[3] = {1, 1, L};
    const char* names[5] = {"theta", "f", "g", "F", "G"};
    const double* data[5] = {th.data(), f.data(), g.data(), F.data(), Gm.data()};
    for (int i = 0; i < 5; ++i) {
        char path[4096];
        std::snprintf(path, sizeof path, "%s/%s_%08lld.bin", dir, names[i], step);
        s = rbc_dump_write(path, i < 3 ? d3 : d1, 3, data[i], real_bytes);
        if (s != RBC_OK) return fail(h, s, std::string("cannot write ") + path);
    }
    return RBC_OK;
}

rbc_status rbc_load_state(rbc_handle* h, const char* tp, const char* fp, const char* gp, const char* Fp, const char* Gp)
{
    if (!h || !tp || !fp || !gp || !Fp || !Gp) return fail(h, RBC_ERR_INVALID_ARG, "null path");
    const Geom& G = h->G;
    const int L = G.L;
    const size_t n = (size_t)L * G.ny * G.mox;
    std::vector<double> buf[5];
    const char* paths[5] = {tp, fp, gp, Fp, Gp};
    for (int i = 0; i < 5; ++i) {
        int dims[8], nd = 0;
        const size_t want = i < 3 ? n : (size_t)L;
        buf[i].assign(2 * want, 0.0);
        rbc_status s = rbc_dump_read(paths[i], 0, dims, 8, &nd, nullptr, 0);
        if (s != RBC_OK) return fail(h, s, std::string("cannot read ") + paths[i]);
        // matrix_has_size (gpu_flow/code/util/util.cu:32-43)
        const bool ok = nd == 3 && (i < 3 ? (dims[0] == G.mox && dims[1] == G.ny && dims[2] == L)
                                          : (dims[0] == 1 && dims[1] == 1 && dims[2] == L));
        if (!ok) return fail(h, RBC_ERR_INVALID_ARG, std::string("wrong dimensions in ") + paths[i]);
        s = rbc_dump_read(paths[i], 0, dims, 8, &nd, buf[i].data(), (long long)want);
        if (s != RBC_OK) return fail(h, s, std::string("cannot read ") + paths[i]);
    }
    return rbc_set_state(h, buf[0].data(), buf[1].data(), buf[2].data(), buf[3].data(), buf[4].data());
}

rbc_status rbc_save_history(rbc_handle* h, const char* path)
{
    if (!path) return fail(h, RBC_ERR_INVALID_ARG, "null path");
    RBC_GUARD(h)
    if (!h->have_hist) return fail(h, RBC_ERR_INVALID_ARG, "no AB2 history yet (no step since the state was set)");
    const Geom& G = h->G;
    const int L = G.L;
    const size_t n = (size_t)L * G.ny * G.mox, plane = (size_t)G.ckp * G.ny;
    std::vector<double> hv[3];
    for (int a = 0; a < 3; ++a) {
        hv[a].resize(2 * n);
        download_field(h, h->hist + a * plane * L, hv[a].data(), L);
    }
    std::vector<double2> fg(2 * L);
    RBC_CUDA(cudaMemcpyAsync(fg.data(), h->hFG, 2 * L * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    FILE* fpo = std::fopen(path, "wb");
    if (!fpo) return fail(h, RBC_ERR_IO, std::string("cannot write ") + path);
    bool ok = true;
    const int nmat = 5, nd = 3;
    ok &= std::fwrite(&nmat, 4, 1, fpo) == 1;
    for (int a = 0; a < 5; ++a) {
        const int d3[3] = {G.mox, G.ny, L}, d1[3] = {1, 1, L};
        ok &= std::fwrite(&nd, 4, 1, fpo) == 1;
        ok &= std::fwrite(a < 3 ? d3 : d1, 4, 3, fpo) == 3;
        if (a < 3) ok &= std::fwrite(hv[a].data(), 8, hv[a].size(), fpo) == hv[a].size();
        else ok &= std::fwrite(fg.data() + (a - 3) * L, 16, L, fpo) == (size_t)L;
    }
    ok &= std::fclose(fpo) == 0;
    return ok ? RBC_OK : fail(h, RBC_ERR_IO, std::string("cannot write ") + path);
    RBC_GUARD_END(h)
}

rbc_status rbc_load_history(rbc_handle* h, const char* path)
{
    if (!path) return fail(h, RBC_ERR_INVALID_ARG, "null path");
    RBC_GUARD(h)
    const Geom& G = h->G;
    const int L = G.L;
    const size_t n = (size_t)L * G.ny * G.mox, plane = (size_t)G.ckp * G.ny;
    std::vector<double> hv[5];
    for (int a = 0; a < 5; ++a) {
        int dims[8], nd = 0;
        const size_t want = a < 3 ? n : (size_t)L;
        hv[a].assign(2 * want, 0.0);
        rbc_status s = rbc_dump_read(path, a, dims, 8, &nd, hv[a].data(), (long long)want);
        if (s != RBC_OK) return fail(h, s, std::string("cannot read history ") + path);
        const bool ok = nd == 3 && (a < 3 ? (dims[0] == G.mox && dims[1] == G.ny && dims[2] == L)
                                          : (dims[0] == 1 && dims[1] == 1 && dims[2] == L));
        if (!ok) return fail(h, RBC_ERR_INVALID_ARG, std::string("wrong dimensions in ") + path);
    }
    flush_tracers(h);
    for (int a = 0; a < 3; ++a) upload_field(h, hv[a].data(), h->hist + a * plane * L, L);
    std::vector<double2> fg(2 * L);
    std::memcpy(fg.data(), hv[3].data(), L * sizeof(double2));
    std::memcpy(fg.data() + L, hv[4].data(), L * sizeof(double2));
    RBC_CUDA(cudaMemcpyAsync(h->hFG, fg.data(), 2 * L * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    h->have_hist = true;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_nonlinear(rbc_handle* h, const rbc_state* in, rbc_state* out)
{
    if (!in || !out || !in->theta || !in->f || !in->g || !in->F || !in->G || !out->theta || !out->f ||
        !out->g || !out->F || !out->G)
        return fail(h, RBC_ERR_INVALID_ARG, "null state buffer");
    RBC_GUARD(h)
    const Geom& G = h->G;
    const int L = G.L;
    const size_t plane = (size_t)G.ckp * G.ny;
    // the operator input goes into the history buffer's planes? No: use dedicated scratch
    // carved from gh (13 L planes of complex R >= 3 L planes of double2 + 2 L).
    static_assert(sizeof(double2) >= 8, "");
    double2* tmp = reinterpret_cast<double2*>(h->gh);
    const size_t need = (3 * plane * L + 2 * L) * sizeof(double2);
    const size_t have = 13 * plane * L * (h->mixed ? sizeof(float2) : sizeof(double2));
    if (need > have) throw ArgError{"scratch too small for rbc_nonlinear"};
    double2* ti = tmp;
    double2* fi = tmp + plane * L;
    double2* gi = tmp + 2 * plane * L;
    double2* FGi = tmp + 3 * plane * L;
    upload_field(h, in->theta, ti, L);
    upload_field(h, in->f, fi, L);
    upload_field(h, in->g, gi, L);
    std::vector<double2> fg(2 * L);
    std::memcpy(fg.data(), in->F, L * sizeof(double2));
    std::memcpy(fg.data() + L, in->G, L * sizeof(double2));
    RBC_CUDA(cudaMemcpyAsync(FGi, fg.data(), 2 * L * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    if (h->mixed) run_synthesis<float>(h, ti, fi, gi, FGi);
    else run_synthesis<double>(h, ti, fi, gi, FGi);
    Geom Gf = G; // every column: the reference operator returns all modes
    Gf.ckeep = G.mox;
    Gf.ckw = G.ckp;
    if (h->mixed) run_analysis<float>(h, Gf);
    else run_analysis<double>(h, Gf);
    // N (R precision, CM) -> double2 CM in the stage-adjacent scratch, then reference layout
    std::vector<double> nfg(2 * L);
    RBC_CUDA(cudaMemcpyAsync(nfg.data(), h->NFG, 2 * L * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    std::vector<double2> nh(3 * plane * L);
    if (h->mixed) {
        std::vector<float2> nf(3 * plane * L);
        RBC_CUDA(cudaMemcpyAsync(nf.data(), h->N, nf.size() * sizeof(float2), cudaMemcpyDeviceToHost, h->stream));
        RBC_CUDA(cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < nf.size(); ++i) nh[i] = make_double2(nf[i].x, nf[i].y);
    } else {
        RBC_CUDA(cudaMemcpyAsync(nh.data(), h->N, nh.size() * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
        RBC_CUDA(cudaStreamSynchronize(h->stream));
    }
    double* outs[3] = {out->theta, out->f, out->g};
    for (int a = 0; a < 3; ++a) {
        double2* o = reinterpret_cast<double2*>(outs[a]);
        std::memset(o, 0, (size_t)L * G.ny * G.mox * sizeof(double2));
        for (int k = 0; k < L; ++k)
            for (int c = 0; c < G.mox; ++c)
                for (int r = 0; r < G.ny; ++r)
                    o[((size_t)k * G.ny + r) * G.mox + c] = nh[((size_t)(a * L + k) * G.ckp + c) * G.ny + r];
    }
    for (int k = 0; k < L; ++k) {
        out->F[2 * k] = nfg[k];
        out->F[2 * k + 1] = 0.0;
        out->G[2 * k] = nfg[L + k];
        out->G[2 * k + 1] = 0.0;
    }
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_synthesis(rbc_handle* h, double* out)
{
    if (!out) return fail(h, RBC_ERR_INVALID_ARG, "null output");
    RBC_GUARD(h)
    const Geom& G = h->G;
    if (h->mixed) run_synthesis<float>(h, h->th, h->f, h->g, h->FG);
    else run_synthesis<double>(h, h->th, h->f, h->g, h->FG);
    const size_t n = (size_t)8 * G.L * G.P;
    if (h->mixed) {
        std::vector<float> v(n);
        RBC_CUDA(cudaMemcpyAsync(v.data(), h->phys, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        RBC_CUDA(cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < n; ++i) out[i] = v[i];
    } else {
        RBC_CUDA(cudaMemcpyAsync(out, h->phys, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        RBC_CUDA(cudaStreamSynchronize(h->stream));
    }
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_diagnostics(rbc_handle* h, rbc_diag* out)
{
    if (!out) return fail(h, RBC_ERR_INVALID_ARG, "null output");
    RBC_GUARD(h)
    // the update kernel keeps the newest entry after the ring; it and the error word are
    // read with one wait for the stream
    double last[4];
    int e = 0;
    RBC_CUDA(cudaMemcpyAsync(last, h->ring + 4 * (size_t)h->ring_cap, sizeof(last), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    if (e & RBC_DEVERR_NAN) return fail(h, RBC_ERR_NAN, "non-finite value in the state");
    if (e) return fail(h, RBC_ERR_CUDA, "device error word set");
    if (last[3] > 0) {
        out->nu_wall = last[0];
        out->nu_vol = last[1];
        out->ke = last[2];
        out->step = (long long)last[3];
        return RBC_OK;
    }
    // no step yet: Nu_wall of the current state only
    std::vector<double2> t((size_t)h->G.L * h->G.ckp * h->G.ny);
    RBC_CUDA(cudaMemcpyAsync(t.data(), h->th, t.size() * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    double nu = 1.0;
    for (int k = 0; k < h->G.L; ++k) nu -= (k + 1) * kPi * t[(size_t)k * h->G.ckp * h->G.ny].x;
    out->nu_wall = nu;
    out->nu_vol = NAN;
    out->ke = NAN;
    out->step = 0;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_diagnostics_async(rbc_handle* h, long long* ticket)
{
    if (!ticket) return fail(h, RBC_ERR_INVALID_ARG, "null ticket");
    RBC_GUARD(h)
    const long long t = h->dticket;
    const int sl = (int)(t % RBC_DIAG_SLOTS);
    rbc_handle::DiagSlot* d = h->dslot + sl;
    // the slot's previous copy must be done before it is overwritten
    RBC_CUDA(cudaEventSynchronize(h->dev_ev[sl]));
    RBC_CUDA(cudaMemcpyAsync(d->v, h->ring + 4 * (size_t)h->ring_cap, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                             h->stream));
    RBC_CUDA(cudaMemcpyAsync(&d->err, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaEventRecord(h->dev_ev[sl], h->stream));
    h->dticket = t + 1;
    *ticket = t;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_diagnostics_get(rbc_handle* h, long long ticket, rbc_diag* out)
{
    if (!out) return fail(h, RBC_ERR_INVALID_ARG, "null output");
    if (!h) return RBC_ERR_INVALID_ARG;
    if (ticket < 0 || ticket >= h->dticket || ticket < h->dticket - RBC_DIAG_SLOTS)
        return fail(h, RBC_ERR_INVALID_ARG, "ticket not among the last RBC_DIAG_SLOTS issued");
    RBC_GUARD(h)
    const int sl = (int)(ticket % RBC_DIAG_SLOTS);
    RBC_CUDA(cudaEventSynchronize(h->dev_ev[sl]));
    const rbc_handle::DiagSlot& d = h->dslot[sl];
    if (d.err & RBC_DEVERR_NAN) return fail(h, RBC_ERR_NAN, "non-finite value in the state");
    if (d.err) return fail(h, RBC_ERR_CUDA, "device error word set");
    if (d.v[3] > 0) {
        out->nu_wall = d.v[0];
        out->nu_vol = d.v[1];
        out->ke = d.v[2];
        out->step = (long long)d.v[3];
    } else {
        out->nu_wall = out->nu_vol = out->ke = NAN;
        out->step = 0;
    }
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_diag_history(rbc_handle* h, rbc_diag* out, int n, int* count)
{
    if (!out || !count || n < 0) return fail(h, RBC_ERR_INVALID_ARG, "bad arguments");
    RBC_GUARD(h)
    long long steps = 0;
    RBC_CUDA(cudaMemcpyAsync(&steps, h->step_counter, sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    long long avail = steps < h->ring_cap ? steps : h->ring_cap;
    if (avail > n) avail = n;
    // the newest `avail` entries are ring slots (steps - avail) .. (steps - 1) mod cap: at
    // most two contiguous pieces
    std::vector<double> buf(4 * (size_t)avail);
    const long long first = (steps - avail) % h->ring_cap;
    const long long n1 = std::min<long long>(avail, h->ring_cap - first);
    if (n1 > 0)
        RBC_CUDA(cudaMemcpyAsync(buf.data(), h->ring + 4 * (size_t)first, 4 * n1 * sizeof(double),
                                 cudaMemcpyDeviceToHost, h->stream));
    if (avail > n1)
        RBC_CUDA(cudaMemcpyAsync(buf.data() + 4 * n1, h->ring, 4 * (avail - n1) * sizeof(double),
                                 cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    for (long long i = 0; i < avail; ++i) {
        out[i].nu_wall = buf[4 * i];
        out[i].nu_vol = buf[4 * i + 1];
        out[i].ke = buf[4 * i + 2];
        out[i].step = (long long)buf[4 * i + 3];
    }
    *count = (int)avail;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_spectrum(rbc_handle* h, double z, double* bins, int nbins)
{
    if (!bins || nbins <= 0) return fail(h, RBC_ERR_INVALID_ARG, "bad spectrum arguments");
    RBC_GUARD(h)
    double* d = reinterpret_cast<double*>(h->N); // scratch: nbins doubles
    const size_t cap = 3 * (size_t)h->G.ckp * h->G.ny * h->G.L * (h->mixed ? sizeof(float2) : sizeof(double2));
    if ((size_t)nbins * sizeof(double) > cap) throw ArgError{"too many spectrum bins"};
    k_spectrum<<<nbins, 256, 0, h->stream>>>(h->th, h->G, z, nbins, d);
    RBC_CUDA(cudaGetLastError());
    RBC_CUDA(cudaMemcpyAsync(bins, d, nbins * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_structure_function(rbc_handle* h, int field, int direction, double r_min, double r_max,
                                  int nsamples, double* out)
{
    if (!out || nsamples <= 0 || field < 0 || field > 2 || direction < 0 || direction > 1 ||
        !std::isfinite(r_min) || !std::isfinite(r_max))
        return fail(h, RBC_ERR_INVALID_ARG, "bad structure-function arguments");
    RBC_GUARD(h)
    double* d = reinterpret_cast<double*>(h->N); // scratch: nsamples doubles
    const size_t cap = 3 * (size_t)h->G.ckp * h->G.ny * h->G.L * (h->mixed ? sizeof(float2) : sizeof(double2));
    if ((size_t)nsamples * sizeof(double) > cap) throw ArgError{"too many structure-function samples"};
    const double inc = (r_max - r_min) / nsamples; // the reference's sample spacing
    k_structure_function<<<nsamples, 256, 0, h->stream>>>(h->th, h->f, h->g, h->G, field, direction, r_min, inc, d);
    RBC_CUDA(cudaGetLastError());
    RBC_CUDA(cudaMemcpyAsync(out, d, nsamples * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    return RBC_OK;
    RBC_GUARD_END(h)
}

static rbc_status table_by_name(const rbchost::Tables& T, const char* name, double* out, int* count)
{
    const int L = T.L;
    const std::vector<double>* v = nullptr;
    if (!std::strcmp(name, "Iac")) v = &T.Iac;
    else if (!std::strcmp(name, "Ia1")) v = &T.Ia1;
    else if (!std::strcmp(name, "Ia2")) v = &T.Ia2;
    else if (!std::strcmp(name, "Ibb1")) v = &T.Ibb1;
    else if (!std::strcmp(name, "Ib11")) v = &T.Ib11;
    else if (!std::strcmp(name, "I111")) v = &T.I111;
    else if (!std::strcmp(name, "Iabc")) v = &T.Iabc;
    else if (!std::strcmp(name, "Iac1")) v = &T.Iac1;
    else if (!std::strcmp(name, "Iaab")) v = &T.Iaab;
    else if (!std::strcmp(name, "Iaa1")) v = &T.Iaa1;
    else if (!std::strcmp(name, "Iab2")) v = &T.Iab2;
    else if (!std::strcmp(name, "Ia12")) v = &T.Ia12;
    else if (!std::strcmp(name, "lambda")) v = &T.lambda;
    else if (!std::strcmp(name, "Ibbb")) {
        for (int k = 0; k < L; ++k)
            for (int j = 0; j < L; ++j)
                for (int i = 0; i < L; ++i) out[i + j * L + k * L * L] = T.ibbb(i, j, k);
        *count = L * L * L;
        return RBC_OK;
    }
    if (!v) return RBC_ERR_INVALID_ARG;
    std::memcpy(out, v->data(), v->size() * sizeof(double));
    *count = (int)v->size();
    return RBC_OK;
}

rbc_status rbc_table(rbc_handle* h, const char* name, double* out, int* count)
{
    if (!h || !name || !out || !count) return RBC_ERR_INVALID_ARG;
    const rbc_status s = table_by_name(h->tab, name, out, count);
    if (s != RBC_OK) return fail(h, s, std::string("unknown table ") + name);
    return RBC_OK;
}

rbc_status rbc_galerkin_table(int nz, const char* name, double* out, int* count)
{
    if (nz < 1 || nz > 16 || !name || !out || !count) return RBC_ERR_INVALID_ARG;
    rbchost::Tables T;
    rbchost::build_tables(nz, T);
    return table_by_name(T, name, out, count);
}

rbc_status rbc_tracers_set(rbc_handle* h, const double* xyz, int n)
{
    if (!xyz) return fail(h, RBC_ERR_INVALID_ARG, "null positions");
    if (!h || n != h->ntr) return fail(h, RBC_ERR_INVALID_ARG, "tracer count differs from params.n_tracers");
    RBC_GUARD(h)
    h->tracer_pending = false;
    RBC_CUDA(cudaMemcpyAsync(h->trpos, xyz, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    track_reset(h);
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_tracers_get(rbc_handle* h, double* xyz, int n)
{
    if (!xyz) return fail(h, RBC_ERR_INVALID_ARG, "null positions");
    if (!h || n != h->ntr) return fail(h, RBC_ERR_INVALID_ARG, "tracer count differs from params.n_tracers");
    RBC_GUARD(h)
    flush_tracers(h);
    RBC_CUDA(cudaMemcpyAsync(xyz, h->trpos, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_tracers_seed(rbc_handle* h, unsigned long long seed)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    std::vector<double> xyz(3 * (size_t)h->ntr);
    rbchost::seeded_positions(seed, h->ntr, h->prm.lx, h->prm.ly, xyz.data());
    return rbc_tracers_set(h, xyz.data(), h->ntr);
}

rbc_status rbc_tracers_init(rbc_handle* h, int type, unsigned long long seed, double cx, double cy, double cz,
                            double sigma)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (type < RBC_TRACERS_RANDOM || type > RBC_TRACERS_COORD_SIGMA || !(sigma >= 0))
        return fail(h, RBC_ERR_INVALID_ARG, "unknown tracer pattern or negative sigma");
    if (type == RBC_TRACERS_PAIRS && (h->ntr & 1))
        return fail(h, RBC_ERR_INVALID_ARG, "position pairs need an even number of tracers");
    std::vector<double> xyz(3 * (size_t)h->ntr);
    rbchost::tracer_pattern(type, seed, h->ntr, h->prm.lx, h->prm.ly, cx, cy, cz, sigma, xyz.data());
    return rbc_tracers_set(h, xyz.data(), h->ntr);
}

rbc_status rbc_tracer_moments(rbc_handle* h, double* out)
{
    if (!out) return fail(h, RBC_ERR_INVALID_ARG, "null output");
    RBC_GUARD(h)
    if (h->ntr == 0) return fail(h, RBC_ERR_INVALID_ARG, "no tracers");
    flush_tracers(h);
    k_tracer_sums<<<1, 1024, 0, h->stream>>>(h->trpos, h->ntr, h->ntr, h->prm.lx, h->prm.ly, h->trsums);
    RBC_CUDA(cudaGetLastError());
    double s[4];
    RBC_CUDA(cudaMemcpyAsync(s, h->trsums, sizeof s, cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    const double n = h->ntr;
    out[0] = s[0] / n;
    out[1] = s[1] / n;
    out[2] = s[2] / n - out[0] * out[0] - out[1] * out[1];
    out[3] = s[3] / (double)(h->ntr / 2);
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_tracer_set_diffusivity(rbc_handle* h, int set, double D)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (h->ntr == 0 || set < 0 || set >= h->tr_sets || !(D >= 0 && std::isfinite(D)))
        return fail(h, RBC_ERR_INVALID_ARG, "bad tracer set or diffusivity");
    RBC_GUARD(h)
    h->set_sig_host[set] = D > 0 ? std::sqrt(2.0 * D * h->G.dt) : 0.0;
    RBC_CUDA(cudaMemcpyAsync(h->set_sig + set, &h->set_sig_host[set], sizeof(double), cudaMemcpyHostToDevice,
                             h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream)); // the host value may change again right after
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_tracers_init_set(rbc_handle* h, int set, int type, unsigned long long seed, double cx, double cy,
                                double cz, double sigma)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (h->ntr == 0 || set < 0 || set >= h->tr_sets) return fail(h, RBC_ERR_INVALID_ARG, "bad tracer set");
    if (type < RBC_TRACERS_RANDOM || type > RBC_TRACERS_COORD_SIGMA || !(sigma >= 0))
        return fail(h, RBC_ERR_INVALID_ARG, "unknown tracer pattern or negative sigma");
    const int ns = h->tr_per_set, n = h->ntr;
    if (type == RBC_TRACERS_PAIRS && (ns & 1))
        return fail(h, RBC_ERR_INVALID_ARG, "position pairs need an even number of tracers per set");
    std::vector<double> all(3 * (size_t)n), part(3 * (size_t)ns);
    rbc_status st = rbc_tracers_get(h, all.data(), n);
    if (st != RBC_OK) return st;
    rbchost::tracer_pattern(type, seed, ns, h->prm.lx, h->prm.ly, cx, cy, cz, sigma, part.data());
    for (int d = 0; d < 3; ++d)
        std::memcpy(&all[(size_t)d * n + (size_t)set * ns], &part[(size_t)d * ns], ns * sizeof(double));
    return rbc_tracers_set(h, all.data(), n);
}

rbc_status rbc_tracer_moments_set(rbc_handle* h, int set, double* out)
{
    if (!out) return fail(h, RBC_ERR_INVALID_ARG, "null output");
    RBC_GUARD(h)
    if (h->ntr == 0 || set < 0 || set >= h->tr_sets) return fail(h, RBC_ERR_INVALID_ARG, "bad tracer set");
    flush_tracers(h);
    const int ns = h->tr_per_set;
    k_tracer_sums<<<1, 1024, 0, h->stream>>>(h->trpos + (size_t)set * ns, ns, h->ntr, h->prm.lx, h->prm.ly,
                                             h->trsums);
    RBC_CUDA(cudaGetLastError());
    double s[4];
    RBC_CUDA(cudaMemcpyAsync(s, h->trsums, sizeof s, cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    out[0] = s[0] / ns;
    out[1] = s[1] / ns;
    out[2] = s[2] / ns - out[0] * out[0] - out[1] * out[1];
    out[3] = s[3] / (double)(ns / 2);
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_tracks_read(rbc_handle* h, float* xyz, unsigned int* times, int max_frames, int* nframes)
{
    if (!nframes || max_frames < 0 || (max_frames > 0 && (!xyz || !times)))
        return fail(h, RBC_ERR_INVALID_ARG, "bad output buffers");
    RBC_GUARD(h)
    *nframes = 0;
    if (!h->trk) return fail(h, RBC_ERR_INVALID_ARG, "no track ring (params.track_frames = 0)");
    flush_tracers(h);
    const long long avail = track_frames_until(h, tracer_time(h));
    const int k = (int)std::min<long long>(avail, max_frames);
    const size_t fsz = 3 * (size_t)h->ntr;
    for (int i = 0; i < k; ++i) {
        const long long t = h->trk_next + (long long)i * h->trk_period;
        const float* fr = h->trk + (size_t)((t / h->trk_period) % h->trk_cap) * fsz;
        RBC_CUDA(cudaMemcpyAsync(xyz + (size_t)i * fsz, fr, fsz * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        times[i] = (unsigned int)t;
    }
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    h->trk_next += (long long)k * h->trk_period;
    *nframes = k;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_tracers_advance(rbc_handle* h)
{
    RBC_GUARD(h)
    if (h->ntr == 0) return RBC_OK;
    flush_tracers(h);
    h->tracer_pending = true; // one more advance with the current field
    flush_tracers(h);
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_launch_config(const rbc_handle* h, int* W, int* NP)
{
    if (!h || !W || !NP) return RBC_ERR_INVALID_ARG;
    *W = h->W;
    *NP = h->NP;
    return RBC_OK;
}

} // extern "C"

// ------------------------------------------------------------------ ensembles
struct rbc_ensemble {
    std::vector<rbc_handle*> members;
    std::vector<int> stream_of;             // worker stream of each member
    std::vector<cudaStream_t> streams;      // worker streams
    cudaStream_t root = nullptr;
    std::vector<cudaEvent_t> ev;            // fork + one join event per worker
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr; // around the graph-replayed steps of a call
    float last_ms = 0.0f;
    int device = 0;
    std::string last_error;
};

static double member_cost(const rbc_params& p)
{
    // algorithmic bytes of one plain step (S = (Nx/2+1) Ny, P = Nx Ny)
    const double S = (p.nx / 2 + 1.0) * p.ny, P = (double)p.nx * p.ny, L = p.nz;
    return L * (12 * S * 16 + 44 * P * 8) + 40 * L * L * S;
}

extern "C" {

rbc_status rbc_ensemble_create(const rbc_params* members, int n, int nstreams, rbc_ensemble** out)
{
    if (!members || n <= 0 || !out) return RBC_ERR_INVALID_ARG;
    *out = nullptr;
    if (nstreams <= 0) nstreams = 16;
    if (nstreams > n) nstreams = n;
    for (int i = 0; i < n; ++i)
        if (members[i].device != members[0].device) return RBC_ERR_INVALID_ARG;
    rbc_ensemble* e = new rbc_ensemble;
    e->device = members[0].device;
    for (int i = 0; i < n; ++i) {
        rbc_handle* h = nullptr;
        rbc_status s = rbc_create(&members[i], &h);
        if (s != RBC_OK) {
            rbc_ensemble_destroy(e);
            return s;
        }
        h->no_pdl = true;
        e->members.push_back(h);
    }
    // longest-processing-time-first assignment of members to worker streams
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return member_cost(members[a]) > member_cost(members[b]); });
    std::vector<double> load(nstreams, 0.0);
    e->stream_of.assign(n, 0);
    for (int i : order) {
        const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        e->stream_of[i] = s;
        load[s] += member_cost(members[i]);
    }
    cudaSetDevice(e->device);
    e->streams.resize(nstreams);
    bool ok = cudaStreamCreateWithFlags(&e->root, cudaStreamNonBlocking) == cudaSuccess;
    for (int s = 0; s < nstreams && ok; ++s) ok = cudaStreamCreateWithFlags(&e->streams[s], cudaStreamNonBlocking) == cudaSuccess;
    e->ev.resize(nstreams + 1);
    for (auto& x : e->ev) ok = ok && cudaEventCreateWithFlags(&x, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreate(&e->t0) == cudaSuccess && cudaEventCreate(&e->t1) == cudaSuccess;
    if (!ok) {
        rbc_ensemble_destroy(e);
        return RBC_ERR_CUDA;
    }
    *out = e;
    return RBC_OK;
}

void rbc_ensemble_destroy(rbc_ensemble* e)
{
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    for (auto* h : e->members) rbc_destroy(h);
    for (auto s : e->streams) if (s) cudaStreamDestroy(s);
    if (e->root) cudaStreamDestroy(e->root);
    for (auto x : e->ev) if (x) cudaEventDestroy(x);
    if (e->t0) cudaEventDestroy(e->t0);
    if (e->t1) cudaEventDestroy(e->t1);
    delete e;
}

rbc_status rbc_ensemble_elapsed(const rbc_ensemble* e, float* ms)
{
    if (!e || !ms) return RBC_ERR_INVALID_ARG;
    *ms = e->last_ms;
    return RBC_OK;
}

const char* rbc_ensemble_last_error(const rbc_ensemble* e)
{
    return e ? e->last_error.c_str() : "null ensemble";
}

rbc_handle* rbc_ensemble_member(rbc_ensemble* e, int i)
{
    if (!e || i < 0 || i >= (int)e->members.size()) return nullptr;
    return e->members[i];
}

rbc_status rbc_ensemble_step(rbc_ensemble* e, int nsteps)
{
    if (!e || nsteps < 0) return RBC_ERR_INVALID_ARG;
    if (cudaSetDevice(e->device) != cudaSuccess) return RBC_ERR_CUDA;
    e->last_error.clear();
    for (auto* h : e->members)
        if (!track_room(h, nsteps)) {
            e->last_error = kTrackFull;
            return RBC_ERR_INVALID_ARG;
        }
    try {
        const int n = (int)e->members.size();
        int s = 0;
        // work a member queued on another stream completes before its worker stream takes over
        for (int i = 0; i < n; ++i) {
            rbc_handle* h = e->members[i];
            if (h->stream != e->streams[e->stream_of[i]]) {
                if (h->stream) RBC_CUDA(cudaStreamSynchronize(h->stream));
                h->stream = e->streams[e->stream_of[i]];
            }
        }
        // members still waiting for their first (Euler) step, or with tracers, step eagerly
        bool graphable = true;
        for (auto* h : e->members) graphable = graphable && h->have_hist && h->ntr == 0;
        for (; s < nsteps && !graphable; ++s) {
            for (int i = 0; i < n; ++i) {
                rbc_handle* h = e->members[i];
                h->stream = e->streams[e->stream_of[i]];
                if (h->mixed) run_step<float>(h);
                else run_step<double>(h);
            }
            graphable = true;
            for (auto* h : e->members) graphable = graphable && h->have_hist && h->ntr == 0;
        }
        if (s < nsteps && !e->graph) {
            // one graph: fork from root to the worker streams, every member's step on its
            // stream, join back to root
            cudaGraph_t g = nullptr;
            RBC_CUDA(cudaStreamBeginCapture(e->root, cudaStreamCaptureModeThreadLocal));
            RBC_CUDA(cudaEventRecord(e->ev[0], e->root));
            for (auto st : e->streams) RBC_CUDA(cudaStreamWaitEvent(st, e->ev[0], 0));
            for (int i = 0; i < n; ++i) {
                rbc_handle* h = e->members[i];
                h->stream = e->streams[e->stream_of[i]];
                const long long hs = h->host_steps;
                if (h->mixed) run_step<float>(h);
                else run_step<double>(h);
                h->host_steps = hs;
            }
            for (size_t w = 0; w < e->streams.size(); ++w) {
                RBC_CUDA(cudaEventRecord(e->ev[w + 1], e->streams[w]));
                RBC_CUDA(cudaStreamWaitEvent(e->root, e->ev[w + 1], 0));
            }
            RBC_CUDA(cudaStreamEndCapture(e->root, &g));
            cudaError_t ce = cudaGraphInstantiate(&e->graph, g, 0);
            cudaGraphDestroy(g);
            RBC_CUDA(ce);
        }
        const int replayed = nsteps - s;
        if (replayed > 0) RBC_CUDA(cudaEventRecord(e->t0, e->root));
        for (; s < nsteps; ++s) {
            RBC_CUDA(cudaGraphLaunch(e->graph, e->root));
            for (auto* h : e->members) ++h->host_steps;
        }
        if (replayed > 0) RBC_CUDA(cudaEventRecord(e->t1, e->root));
        RBC_CUDA(cudaStreamSynchronize(e->root));
        e->last_ms = 0.0f;
        if (replayed > 0) RBC_CUDA(cudaEventElapsedTime(&e->last_ms, e->t0, e->t1));
        for (auto st : e->streams) RBC_CUDA(cudaStreamSynchronize(st));
        for (auto* h : e->members) {
            rbc_status st = check_err(h);
            if (st != RBC_OK) {
                e->last_error = rbc_last_error(h);
                return st;
            }
        }
    } catch (const CudaError& x) {
        e->last_error = std::string(x.what) + ": " + cudaGetErrorString(x.e);
        return RBC_ERR_CUDA;
    } catch (const ArgError& x) {
        e->last_error = x.msg;
        return RBC_ERR_UNSUPPORTED;
    }
    return RBC_OK;
}

} // extern "C"

// ------------------------------------------------------------------ surrogate access
// Library-internal functions of solver_internal.h (used by fno.cu).
namespace rbcint {

GridDesc grid(const rbc_handle* h)
{
    GridDesc d;
    d.nx = h->G.nx;
    d.ny = h->G.ny;
    d.L = h->G.L;
    d.ckeep = h->G.ckeep;
    d.device = h->prm.device;
    d.lx = h->G.lx;
    d.ly = h->G.ly;
    d.dt = h->G.dt;
    d.ra = h->prm.ra;
    d.pr = h->prm.pr;
    d.mixed = h->mixed;
    return d;
}

cudaStream_t stream(const rbc_handle* h) { return h->stream; }
unsigned long long uid(const rbc_handle* h) { return h->uid; }
bool has_tracers(const rbc_handle* h) { return h->ntr > 0; }
void state_changed(rbc_handle* h) { h->have_hist = false; }

void set_error(rbc_handle* h, const char* msg)
{
    if (h) h->last_error = msg;
}

template <typename R, int L> static void encode_L(rbc_handle* h, int nq, const double* basis, float* out)
{
    const int P = h->G.P;
    // 64-point blocks: a 128 x 128 plane gives 256 CTAs
    const size_t sm = (size_t)64 * (4 * nq + 1) * sizeof(float);
    k_colloc_encode<R, L><<<(P + 63) / 64, 64, sm, h->stream>>>((const R*)h->phys, P, nq, basis, out);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
}
template <typename R> static void encode_t(rbc_handle* h, int nq, const double* basis, float* out)
{
    run_synthesis<R>(h, h->th, h->f, h->g, h->FG);
    switch (h->G.L) {
    case 2: encode_L<R, 2>(h, nq, basis, out); break;
    case 3: encode_L<R, 3>(h, nq, basis, out); break;
    case 4: encode_L<R, 4>(h, nq, basis, out); break;
    case 5: encode_L<R, 5>(h, nq, basis, out); break;
    case 6: encode_L<R, 6>(h, nq, basis, out); break;
    case 8: encode_L<R, 8>(h, nq, basis, out); break;
    case 12: encode_L<R, 12>(h, nq, basis, out); break;
    default: throw ArgError{"unsupported number of vertical modes"};
    }
}

rbc_status colloc_encode(rbc_handle* h, int nq, const double* d_basis, float* d_out)
{
    if (!d_basis || !d_out || !h || nq < h->G.L) return fail(h, RBC_ERR_INVALID_ARG, "bad collocation arguments");
    RBC_GUARD(h)
    if (h->mixed) encode_t<float>(h, nq, d_basis, d_out);
    else encode_t<double>(h, nq, d_basis, d_out);
    return RBC_OK;
    RBC_GUARD_END(h)
}

// Mean-mode forcing of the current state: g = (2 Re N_theta_k(q=0), 2 Pr NF_k, 2 Pr NG_k),
// the q = 0 terms that the update kernel adds (inverse B of the nonlinear term), and the
// current mean modes y0 = (Re theta_k(q=0), F_k, G_k).
template <typename C>
__global__ void k_mean_forcing(const C* __restrict__ N, const double* __restrict__ NFG,
                               const double2* __restrict__ th, const double2* __restrict__ FG, size_t plane, int L,
                               double pr, double* __restrict__ g, double* __restrict__ y0)
{
    const int k = threadIdx.x;
    if (k >= L) return;
    g[k] = 2.0 * (double)N[(size_t)k * plane].x;
    g[L + k] = 2.0 * pr * NFG[k];
    g[2 * L + k] = 2.0 * pr * NFG[L + k];
    y0[k] = th[(size_t)k * plane].x;
    y0[L + k] = FG[k].x;
    y0[2 * L + k] = FG[L + k].x;
}

// nsub steps of the plain step's recursion for the mean modes (q = 0: theta_k, F_k, G_k
// decouple from everything else): y <- (y + dt (1.5 g_s - 0.5 g_{s-1})) / (1 + dt a),
// a = ((k+1) pi)^2 for theta and Pr ((k+1) pi)^2 for F, G, with the forcing g_s taken
// linear in time through g0 (interval start) and gp (start of the previous interval,
// nsub steps earlier); without gp the forcing is constant and the first step is Euler.
__global__ void k_mean_advance(double2* __restrict__ th, double2* __restrict__ FG, size_t plane, int L,
                               const double* __restrict__ y0, const double* __restrict__ g0,
                               const double* __restrict__ gp, int nsub, double dt, double pr)
{
    const int i = threadIdx.x;
    if (i >= 3 * L) return;
    const int kind = i / L, k = i - kind * L;
    const double mpi = (k + 1) * kPi;
    const double a = (kind ? pr : 1.0) * mpi * mpi;
    const double fac = 1.0 / (1.0 + dt * a);
    const double slope = gp ? (g0[i] - gp[i]) / nsub : 0.0;
    double y = y0[i], gprev = g0[i] - slope;
    for (int s = 0; s < nsub; ++s) {
        const double gs = g0[i] + slope * s;
        const double incr = (gp || s > 0) ? 1.5 * gs - 0.5 * gprev : gs;
        y = (y + dt * incr) * fac;
        gprev = gs;
    }
    if (kind == 0) th[(size_t)k * plane] = make_double2(y, 0.0);
    else FG[(kind - 1) * L + k] = make_double2(y, 0.0);
}

template <typename R> static void encode_forcing_t(rbc_handle* h, int nq, const double* basis, float* out, double* g,
                                                   double* y0)
{
    typedef typename cplx_t<R>::type C;
    encode_t<R>(h, nq, basis, out);
    run_analysis<R>(h, h->G);
    k_mean_forcing<C><<<1, 32, 0, h->stream>>>((const C*)h->N, h->NFG, h->th, h->FG, (size_t)h->G.ckp * h->G.ny,
                                                h->G.L, h->G.pr, g, y0);
    RBC_CUDA(cudaGetLastError());
    h->launches += 1;
}

rbc_status colloc_encode_forcing(rbc_handle* h, int nq, const double* d_basis, float* d_out, double* d_g,
                                 double* d_y0)
{
    if (!d_basis || !d_out || !d_g || !d_y0 || !h || nq < h->G.L)
        return fail(h, RBC_ERR_INVALID_ARG, "bad collocation arguments");
    RBC_GUARD(h)
    flush_tracers(h); // a pending tracer advance runs on the current state first
    if (h->mixed) encode_forcing_t<float>(h, nq, d_basis, d_out, d_g, d_y0);
    else encode_forcing_t<double>(h, nq, d_basis, d_out, d_g, d_y0);
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status mean_advance(rbc_handle* h, const double* d_y0, const double* d_g0, const double* d_gp, int nsub)
{
    if (!h || !d_y0 || !d_g0 || nsub < 1 || 3 * h->G.L > 64) return fail(h, RBC_ERR_INVALID_ARG, "bad mean-mode arguments");
    RBC_GUARD(h)
    k_mean_advance<<<1, 64, 0, h->stream>>>(h->th, h->FG, (size_t)h->G.ckp * h->G.ny, h->G.L, d_y0, d_g0, d_gp, nsub,
                                            h->G.dt, h->G.pr);
    RBC_CUDA(cudaGetLastError());
    ++h->launches;
    h->have_hist = false;
    return RBC_OK;
    RBC_GUARD_END(h)
}

size_t colloc_scratch_bytes(const rbc_handle* h)
{
    const Geom& G = h->G;
    return (size_t)4 * G.L * G.P * sizeof(double) + (size_t)4 * G.L * G.ckeep * G.ny * sizeof(double2);
}

template <int L> static void add_L(rbc_handle* h, int nq, const double* proj, const float* delta, void* scratch)
{
    const Geom& G = h->G;
    double* planes = static_cast<double*>(scratch);
    double2* rows = reinterpret_cast<double2*>(planes + (size_t)4 * L * G.P);
    const size_t sm_pr = (size_t)64 * (4 * nq + 1) * sizeof(float);
    k_colloc_project<L><<<(G.P + 63) / 64, 64, sm_pr, h->stream>>>(delta, G.P, nq, proj, planes);
    RBC_CUDA(cudaGetLastError());
    const size_t sm_row = (size_t)G.nx * (sizeof(double2) + sizeof(double));
    k_colloc_row_dft<<<4 * L * G.ny, 128, sm_row, h->stream>>>(planes, G.nx, G.ny, G.ckeep, h->twx, rows);
    RBC_CUDA(cudaGetLastError());
    const size_t sm_col = (size_t)5 * G.ny * sizeof(double2);
    if (sm_col > 48 * 1024)
        RBC_CUDA(cudaFuncSetAttribute(k_colloc_assemble<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_col));
    k_colloc_assemble<L><<<dim3(G.ckeep, L), 256, sm_col, h->stream>>>(rows, G, h->twy, h->th, h->f, h->g, h->FG);
    RBC_CUDA(cudaGetLastError());
    h->launches += 3;
}

rbc_status colloc_add(rbc_handle* h, int nq, const double* d_proj, const float* d_delta, void* d_scratch)
{
    if (!h || !d_proj || !d_delta || !d_scratch || nq < h->G.L)
        return fail(h, RBC_ERR_INVALID_ARG, "bad collocation arguments");
    RBC_GUARD(h)
    flush_tracers(h); // a pending tracer advance uses the velocity of the state before the change
    switch (h->G.L) {
    case 2: add_L<2>(h, nq, d_proj, d_delta, d_scratch); break;
    case 3: add_L<3>(h, nq, d_proj, d_delta, d_scratch); break;
    case 4: add_L<4>(h, nq, d_proj, d_delta, d_scratch); break;
    case 5: add_L<5>(h, nq, d_proj, d_delta, d_scratch); break;
    case 6: add_L<6>(h, nq, d_proj, d_delta, d_scratch); break;
    case 8: add_L<8>(h, nq, d_proj, d_delta, d_scratch); break;
    case 12: add_L<12>(h, nq, d_proj, d_delta, d_scratch); break;
    default: throw ArgError{"unsupported number of vertical modes"};
    }
    h->have_hist = false;
    return RBC_OK;
    RBC_GUARD_END(h)
}

size_t state_bytes(const rbc_handle* h)
{
    return ((size_t)3 * h->G.L * h->G.ckp * h->G.ny + 2 * (size_t)h->G.L) * sizeof(double2);
}

rbc_status state_save(rbc_handle* h, void* d_dst)
{
    if (!h || !d_dst) return fail(h, RBC_ERR_INVALID_ARG, "null buffer");
    RBC_GUARD(h)
    const size_t pl = (size_t)h->G.L * h->G.ckp * h->G.ny;
    double2* d = static_cast<double2*>(d_dst);
    RBC_CUDA(cudaMemcpyAsync(d, h->th, pl * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    RBC_CUDA(cudaMemcpyAsync(d + pl, h->f, pl * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    RBC_CUDA(cudaMemcpyAsync(d + 2 * pl, h->g, pl * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    RBC_CUDA(cudaMemcpyAsync(d + 3 * pl, h->FG, 2 * h->G.L * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status state_load(rbc_handle* h, const void* d_src)
{
    if (!h || !d_src) return fail(h, RBC_ERR_INVALID_ARG, "null buffer");
    RBC_GUARD(h)
    flush_tracers(h);
    const size_t pl = (size_t)h->G.L * h->G.ckp * h->G.ny;
    const double2* s = static_cast<const double2*>(d_src);
    RBC_CUDA(cudaMemcpyAsync(h->th, s, pl * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    RBC_CUDA(cudaMemcpyAsync(h->f, s + pl, pl * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    RBC_CUDA(cudaMemcpyAsync(h->g, s + 2 * pl, pl * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    RBC_CUDA(cudaMemcpyAsync(h->FG, s + 3 * pl, 2 * h->G.L * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    h->have_hist = false;
    return RBC_OK;
    RBC_GUARD_END(h)
}

__global__ void k_nu_wall_record(const double2* __restrict__ th, size_t plane, int L, double* __restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double v = 1.0;
        for (int k = 0; k < L; ++k) v -= (k + 1) * kPi * th[(size_t)k * plane].x;
        *out = v;
    }
}

rbc_status nu_wall_record(rbc_handle* h, double* d_out)
{
    if (!h || !d_out) return fail(h, RBC_ERR_INVALID_ARG, "null output");
    RBC_GUARD(h)
    k_nu_wall_record<<<1, 32, 0, h->stream>>>(h->th, (size_t)h->G.ckp * h->G.ny, h->G.L, d_out);
    RBC_CUDA(cudaGetLastError());
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status nu_wall(rbc_handle* h, double* nu)
{
    if (!h || !nu) return fail(h, RBC_ERR_INVALID_ARG, "null output");
    RBC_GUARD(h)
    const int L = h->G.L;
    std::vector<double2> t(L);
    RBC_CUDA(cudaMemcpy2DAsync(t.data(), sizeof(double2), h->th, (size_t)h->G.ckp * h->G.ny * sizeof(double2),
                               sizeof(double2), L, cudaMemcpyDeviceToHost, h->stream));
    RBC_CUDA(cudaStreamSynchronize(h->stream));
    double v = 1.0;
    for (int k = 0; k < L; ++k) v -= (k + 1) * kPi * t[k].x;
    *nu = v;
    return RBC_OK;
    RBC_GUARD_END(h)
}

} // namespace rbcint

// ------------------------------------------------------------------ field operators
rbc_status rbc_freeze_mask(rbc_handle* h, int shape, double size)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (!h->frozen) return fail(h, RBC_ERR_INVALID_ARG, "handle created without RBC_FIELD_FREEZE");
    if ((shape != RBC_MASK_CIRCLE && shape != RBC_MASK_RECTANGLE) || !std::isfinite(size))
        return fail(h, RBC_ERR_INVALID_ARG, "bad mask shape or size");
    RBC_GUARD(h)
    make_mask(h, h->fmask, shape, 0.5, 0.5, size);
    mask_pass(h, 3, MASK_SNAPSHOT, h->fmask, 0.0);
    h->frozen_set = true;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_freeze_apply(rbc_handle* h)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (!h->frozen_set) return RBC_OK; // freeze_operator::calculate_operator before a freeze
    RBC_GUARD(h)
    // a pending tracer advance uses the velocity of the state before the change; it runs
    // beside the operator, which leaves the tracer data alone
    flush_tracers(h, true);
    mask_pass(h, 3, MASK_FREEZE, h->fmask, 0.0);
    join_tracer(h);
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_heat_mask(rbc_handle* h, int shape, double size, double increment)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (!h->hmask) return fail(h, RBC_ERR_INVALID_ARG, "handle created without RBC_FIELD_HEAT");
    if ((shape != RBC_MASK_CIRCLE && shape != RBC_MASK_RECTANGLE) || !std::isfinite(size) || !std::isfinite(increment))
        return fail(h, RBC_ERR_INVALID_ARG, "bad mask shape, size or increment");
    RBC_GUARD(h)
    make_mask(h, h->hmask, shape, 0.2, 0.3, size);
    h->heat_set = true;
    h->heat_inc = increment;
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_heat_apply(rbc_handle* h)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (!h->heat_set) return RBC_OK; // masktemp::calculate_operator before the mask is set
    RBC_GUARD(h)
    flush_tracers(h, true);
    mask_pass(h, 1, MASK_HEAT, h->hmask, h->heat_inc);
    join_tracer(h);
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_masker(rbc_handle* h, double x, double y, double radius, double factor)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    if (!h->smask) return fail(h, RBC_ERR_INVALID_ARG, "handle created without RBC_FIELD_SCALE");
    if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(radius) || !std::isfinite(factor))
        return fail(h, RBC_ERR_INVALID_ARG, "bad mask position, radius or factor");
    RBC_GUARD(h)
    flush_tracers(h, true); // beside the operator, as in rbc_freeze_apply
    make_mask(h, h->smask, RBC_MASK_CIRCLE, y, x, radius); // column centre y Nx, row centre x Ny
    mask_pass(h, 1, MASK_SCALE, h->smask, factor);
    join_tracer(h);
    return RBC_OK;
    RBC_GUARD_END(h)
}

rbc_status rbc_field_ops_reset(rbc_handle* h)
{
    if (!h) return RBC_ERR_INVALID_ARG;
    h->frozen_set = h->heat_set = false;
    return RBC_OK;
}
