// nonlinear_static.cu -- the nonlinear operator for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: a plug-in running inside a host framework that has
// already reserved the device's memory for its own caching allocator (a new cudaMalloc
// there fails or fragments that pool), or a latency-critical loop that must not pay the
// implicit device-wide synchronisation of cudaMalloc and cudaFree. rbc_nonlinear_noalloc
// gives them the nonlinear operator without a handle and without any device allocation:
// the caller passes device buffers for the input state and the five results, and every
// scratch plane and table the kernels need lives in one file-scope __device__ array of
// fixed size (RBC_NOALLOC_SCRATCH_BYTES), which every GPU that loads this library keeps
// until the process exits.
//
// The kernels are the same as those of rbc_nonlinear (step_kernels.cuh,
// contract_kernel.cuh); only the placement of their scratch differs.
#include "rbc.h"
#include "common.cuh"
#include "contract_kernel.cuh"
#include "fft.cuh"
#include "galerkin.h"
#include "step_kernels.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

using namespace rbck;

namespace {

// The scratch array. In host code its name is only a host-side stand-in: its device
// address is obtained with cudaGetSymbolAddress (per device, see scratch_address).
__device__ __align__(256) unsigned char g_noalloc_scratch[RBC_NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
void* g_addr[64] = {nullptr}; // device address of g_noalloc_scratch, per device ordinal

// The size whose tables (twiddles, contraction coefficients) sit at the start of the
// array on each device: a call of the same size finds them there and enqueues kernels
// only; a call of another size rewrites them (its scratch planes may overlap the old
// tables' place). The host copies are kept for the life of the process.
struct TableKey {
    int nx = 0, ny = 0, nz = 0;
};
TableKey g_tables[64];
std::vector<double> g_coef[64];
std::vector<double2> g_twx[64], g_twy[64];

// Device address of the scratch array on `device` (which must be current). Looked up
// once per device and cached.
cudaError_t scratch_address(int device, void** out)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (!g_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[device] = p;
    }
    *out = g_addr[device];
    return cudaSuccess;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct Layout {
    size_t twx, twy, coef, st, FG, H, phys, grp, gh, N, NFG, total;
};

Layout layout(const Geom& G, int L)
{
    Layout l;
    size_t o = 0;
    const size_t plane = (size_t)G.ckp * G.ny;
    auto take = [&](size_t bytes) { size_t at = o; o += align256(bytes); return at; };
    l.twx = take(sizeof(double2) * G.nx);
    l.twy = take(sizeof(double2) * G.ny);
    l.coef = take(sizeof(double) * rbcprog::NUNIT * L * L * rbcprog::half_len(L));
    l.st = take(sizeof(double2) * 3 * plane * L);
    l.FG = take(sizeof(double2) * 2 * L);
    l.H = take(sizeof(double2) * 8 * plane * L);
    l.phys = take(sizeof(double) * 8 * (size_t)L * G.P);
    l.grp = take(sizeof(double) * 13 * (size_t)L * G.P);
    l.gh = take(sizeof(double2) * 13 * plane * L);
    l.N = take(sizeof(double2) * 3 * plane * L);
    l.NFG = take(sizeof(double) * 2 * L);
    l.total = o;
    return l;
}

__global__ void k_na_ref_to_cm(const double2* __restrict__ src, double2* __restrict__ dst, Geom G, int nmat)
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

__global__ void k_na_cm_to_ref(const double2* __restrict__ src, double2* __restrict__ dst, Geom G, int nmat)
{
    const size_t n = (size_t)nmat * G.ny * G.mox;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % G.mox);
        const size_t t = e / G.mox;
        const int r = (int)(t % G.ny);
        const int k = (int)(t / G.ny);
        dst[e] = src[((size_t)k * G.ckp + c) * G.ny + r];
    }
}

__global__ void k_na_fg(const double* __restrict__ nfg, double2* __restrict__ F, double2* __restrict__ Gout, int L)
{
    const int k = threadIdx.x;
    if (k < L) {
        F[k] = make_double2(nfg[k], 0.0);
        Gout[k] = make_double2(nfg[L + k], 0.0);
    }
}

struct DeviceRestore {
    int dev = -1;
    ~DeviceRestore()
    {
        if (dev >= 0) cudaSetDevice(dev);
    }
};

void say(char* buf, int len, const char* msg)
{
    if (buf && len > 0) {
        std::strncpy(buf, msg, (size_t)len - 1);
        buf[len - 1] = 0;
    }
}

template <int L> void launch_contract_na(const Geom& G, double* phys, double* grp, const double* coef, cudaStream_t s)
{
    const int smem = (int)(rbcprog::NUNIT * L * L * rbcprog::half_len(L) * sizeof(double));
    k_contract<double, L><<<(G.P + 127) / 128, 128, smem, s>>>(phys, grp, coef, G.P, nullptr, nullptr, nullptr);
}

} // namespace

extern "C" rbc_status rbc_nonlinear_noalloc(int device, int nx, int ny, int nz, double lx, double ly, double pr,
                                            const double* theta, const double* f, const double* g, const double* F,
                                            const double* Gm, double* out_theta, double* out_f, double* out_g,
                                            double* out_F, double* out_G, void* stream, char* errbuf, int errlen)
{
    say(errbuf, errlen, "");
    if (!theta || !f || !g || !F || !Gm || !out_theta || !out_f || !out_g || !out_F || !out_G) {
        say(errbuf, errlen, "rbc_nonlinear_noalloc: null buffer");
        return RBC_ERR_INVALID_ARG;
    }
    if (nx > RBC_NOALLOC_MAX_NX || ny > RBC_NOALLOC_MAX_NY || nz > RBC_NOALLOC_MAX_NZ || nz < 2) {
        char m[200];
        std::snprintf(m, sizeof m, "rbc_nonlinear_noalloc: %dx%dx%d exceeds the static scratch limit %dx%dx%d (2 <= nz)",
                      nx, ny, nz, RBC_NOALLOC_MAX_NX, RBC_NOALLOC_MAX_NY, RBC_NOALLOC_MAX_NZ);
        say(errbuf, errlen, m);
        return RBC_ERR_INVALID_ARG;
    }
    const rbcfft::Plan px = rbcfft::make_plan(nx), py = rbcfft::make_plan(ny);
    if (px.npass <= 0 || py.npass <= 0 || (nx & 1) || (ny & 1) || !(lx > 0) || !(ly > 0) || !(pr > 0)) {
        say(errbuf, errlen, "rbc_nonlinear_noalloc: invalid grid or parameters");
        return RBC_ERR_INVALID_ARG;
    }
    if (device < 0 || device >= 64) {
        say(errbuf, errlen, "rbc_nonlinear_noalloc: device ordinal out of range");
        return RBC_ERR_INVALID_ARG;
    }
    // the caller's current device is restored on every return path
    DeviceRestore restore;
    if (cudaGetDevice(&restore.dev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        say(errbuf, errlen, "rbc_nonlinear_noalloc: cudaSetDevice failed");
        return RBC_ERR_CUDA;
    }
    // an error left pending by earlier, unrelated work is not this call's failure
    (void)cudaGetLastError();
    void* base = nullptr;
    cudaError_t e = scratch_address(device, &base);
    if (e != cudaSuccess) {
        say(errbuf, errlen, cudaGetErrorString(e));
        return RBC_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // geometry exactly as rbc_create builds it
    rbchost::GridInfo gi;
    rbchost::grid_info(nx, ny, nz, lx, ly, 0.0, pr, 1.0, gi);
    int W = 1;
    while (W < 4 && 8 * (2 * W) <= py.chunk) W *= 2;
    int NP = 1;
    for (int c = 1; c <= 32 && c <= px.chunk; ++c)
        if ((ny / 2) % c == 0) NP = c;
    Geom G{};
    G.nx = nx; G.ny = ny; G.mox = nx / 2 + 1; G.L = nz;
    G.ckeep = gi.ckeep;
    G.ckw = ((G.ckeep + W - 1) / W) * W;
    G.ckp = ((G.mox + W - 1) / W) * W;
    G.P = nx * ny;
    G.lx = lx; G.ly = ly; G.pr = pr; G.dt = 1.0;
    const Layout l = layout(G, nz);
    if (l.total > RBC_NOALLOC_SCRATCH_BYTES) {
        say(errbuf, errlen, "rbc_nonlinear_noalloc: problem does not fit the static scratch");
        return RBC_ERR_INVALID_ARG;
    }
    unsigned char* b = static_cast<unsigned char*>(base);
    {
        // tables: uploaded when this device's array holds another size's (host computation
        // into process-lifetime buffers)
        std::lock_guard<std::mutex> lock(g_mu);
        TableKey& key = g_tables[device];
        if (key.nx != nx || key.ny != ny || key.nz != nz) {
            rbchost::Tables T;
            rbchost::build_tables(nz, T);
            std::vector<double>& coef = g_coef[device];
            rbchost::pack_contraction(T, coef);
            std::vector<double2>& twx = g_twx[device];
            std::vector<double2>& twy = g_twy[device];
            twx.resize(nx);
            twy.resize(ny);
            for (int t = 0; t < nx; ++t) {
                const long double a = -2.0L * 3.14159265358979323846264338327950288L * t / nx;
                twx[t] = make_double2((double)cosl(a), (double)sinl(a));
            }
            for (int t = 0; t < ny; ++t) {
                const long double a = -2.0L * 3.14159265358979323846264338327950288L * t / ny;
                twy[t] = make_double2((double)cosl(a), (double)sinl(a));
            }
            e = cudaMemcpyAsync(b + l.twx, twx.data(), sizeof(double2) * nx, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(b + l.twy, twy.data(), sizeof(double2) * ny, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(b + l.coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) {
                key = TableKey{};
                say(errbuf, errlen, cudaGetErrorString(e));
                return RBC_ERR_CUDA;
            }
            key.nx = nx;
            key.ny = ny;
            key.nz = nz;
        }
    }
    double2* st = reinterpret_cast<double2*>(b + l.st);
    const size_t plane = (size_t)G.ckp * ny;
    double2* FG = reinterpret_cast<double2*>(b + l.FG);
    // input (dealiased on the way in, as step_time does before the operator)
    k_na_ref_to_cm<<<256, 256, 0, s>>>(reinterpret_cast<const double2*>(theta), st, G, nz);
    k_na_ref_to_cm<<<256, 256, 0, s>>>(reinterpret_cast<const double2*>(f), st + plane * nz, G, nz);
    k_na_ref_to_cm<<<256, 256, 0, s>>>(reinterpret_cast<const double2*>(g), st + 2 * plane * nz, G, nz);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        say(errbuf, errlen, cudaGetErrorString(e));
        return RBC_ERR_CUDA;
    }
    e = cudaMemcpyAsync(FG, F, sizeof(double2) * nz, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(FG + nz, Gm, sizeof(double2) * nz, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) {
        say(errbuf, errlen, cudaGetErrorString(e));
        return RBC_ERR_CUDA;
    }
    typedef double2 C;
    const double2* tx = reinterpret_cast<const double2*>(b + l.twx);
    const double2* ty = reinterpret_cast<const double2*>(b + l.twy);
    C* H = reinterpret_cast<C*>(b + l.H);
    double* phys = reinterpret_cast<double*>(b + l.phys);
    double* grp = reinterpret_cast<double*>(b + l.grp);
    C* gh = reinterpret_cast<C*>(b + l.gh);
    C* N = reinterpret_cast<C*>(b + l.N);
    double* NFG = reinterpret_cast<double*>(b + l.NFG);
    const size_t smc = sizeof(C) * ((size_t)ny + 8 * (size_t)W * py.stride);
    const size_t smr = sizeof(C) * ((size_t)nx + (size_t)NP * px.stride);
    const size_t smk = sizeof(C) * ((size_t)ny + 13 * (size_t)py.stride);
    k_synth_columns<double><<<dim3(G.ckw / W, nz), kThreads, smc, s>>>(G, W, py, ty, st, st + plane * nz,
                                                                       st + 2 * plane * nz, FG, H);
    k_rows_c2r<double><<<8 * nz * ny / (2 * NP), kThreads, smr, s>>>(G, NP, px, tx, H, phys);
    const double* cf = reinterpret_cast<const double*>(b + l.coef);
    switch (nz) {
    case 2: launch_contract_na<2>(G, phys, grp, cf, s); break;
    case 3: launch_contract_na<3>(G, phys, grp, cf, s); break;
    default: launch_contract_na<4>(G, phys, grp, cf, s); break;
    }
    Geom Gf = G; // every column: the operator returns all modes
    Gf.ckeep = G.mox;
    Gf.ckw = G.ckp;
    k_rows_r2c<double><<<13 * nz * ny / (2 * NP), kThreads, smr, s>>>(Gf, NP, px, tx, grp, gh);
    k_columns_combine<double><<<dim3(Gf.ckw, nz), kThreads, smk, s>>>(Gf, py, ty, gh, N, NFG);
    k_na_cm_to_ref<<<256, 256, 0, s>>>(N, reinterpret_cast<double2*>(out_theta), Gf, nz);
    k_na_cm_to_ref<<<256, 256, 0, s>>>(N + plane * nz, reinterpret_cast<double2*>(out_f), Gf, nz);
    k_na_cm_to_ref<<<256, 256, 0, s>>>(N + 2 * plane * nz, reinterpret_cast<double2*>(out_g), Gf, nz);
    k_na_fg<<<1, 32, 0, s>>>(NFG, reinterpret_cast<double2*>(out_F), reinterpret_cast<double2*>(out_G), nz);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        say(errbuf, errlen, cudaGetErrorString(e));
        return RBC_ERR_CUDA;
    }
    return RBC_OK;
}
