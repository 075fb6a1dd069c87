// fno.cu -- learned surrogate of the RBC step: a Fourier neural operator (FNO) that
// advances the solver state by one surrogate interval (many plain steps) at a time, its
// training on snapshot pairs the solver generates, and a rollout in which the plain IMEX
// step checks the surrogate's Nusselt number and spectrum and takes over when they drift.
// No reference counterpart (jceyy/sdc has no learned component).
//
// Network (FNO-2d over the horizontal plane; the nq collocation levels of the four
// fields theta, u, v, w are its C = 4 nq channels, channel = field * nq + level):
//   h0 = x P^T + p                                   lift C -> W
//   h_{l+1} = act(h_l W_l^T + b_l + K_l(h_l))         l = 0 .. nl-1, act = GELU except last
//   K_l(h) = irfft2(R_l * rfft2(h) on kx < m, ky in [0, m) U [-m, 0))
//   y = GELU(h_nl Q1^T + q1) Q2^T + q2                project W -> H -> C
// y is the normalized increment of the collocation fields over one interval. The
// truncated transforms are products with fixed DFT matrices (Fx, Fy forward, Gy, Gx
// inverse), so every contraction runs as a BF16 GEMM with FP32 accumulation; activations
// are stored in BF16, pre-activations, the loss and the optimizer in FP32.
//
// Parameter vector (FP32, this order): P [W][C], p [W]; per layer W_l [W][W], b_l [W],
// R_l [2m][m][2][W][W] (ky index, kx, re/im, in, out); Q1 [H][W], q1 [H]; Q2 [C][H], q2 [C].
#include "rbc.h"
#include "fno_kernels.cuh"
#include "gemm_tc.cuh"

#include <cudaTypedefs.h>
#include "galerkin.h"
#include "solver_internal.h"
#include "splitmix.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

using namespace rbcfno;

namespace {

struct CudaErr {
    cudaError_t e;
    const char* what;
};
struct ArgErr {
    std::string msg;
};
#define FNO_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) throw CudaErr{e_, #call};                                 \
    } while (0)

// float -> BF16 bits, round to nearest even (the conversion the kernels use).
uint16_t bf16_bits(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

constexpr double kTwoPi = 6.283185307179586476925286766559;

} // namespace

struct rbc_fno {
    rbc_fno_params p{};
    int C = 0, W = 0, m = 0, my = 0, H = 0, nl = 0, nx = 0, ny = 0, P = 0, B = 0;
    std::string last_error;
    cudaStream_t stream = nullptr;
    std::vector<void*> owned;
    long long nparam = 0, oPw = 0, oPb = 0, oQ1w = 0, oQ1b = 0, oQ2w = 0, oQ2b = 0;
    std::vector<long long> oW, ob, oR;
    float *param = nullptr, *grad = nullptr, *am = nullptr, *av = nullptr;
    bf16* pbf = nullptr;
    long long adam_t = 0;
    bf16 *FxT = nullptr, *FyB = nullptr, *GyB = nullptr, *GxT = nullptr;
    float* norm = nullptr; // [5][C]: x mean, 1/x std, d mean, d std, 1/d std
    std::vector<float> norm_h;
    bool have_norm = false;
    // activations
    bf16* x0 = nullptr;
    std::vector<bf16*> h;
    std::vector<float*> pre;
    std::vector<bf16*> Ahat;
    bf16 *A1 = nullptr, *Yh = nullptr, *Z = nullptr, *q1 = nullptr;
    float *Kv = nullptr, *q1pre = nullptr, *out = nullptr, *target = nullptr, *xf = nullptr;
    // backward
    bf16 *gA = nullptr, *gB = nullptr, *dZ = nullptr, *dY = nullptr, *dAh = nullptr, *dA1 = nullptr;
    float *dhs = nullptr, *wpart = nullptr, *cpart = nullptr, *lpart = nullptr;
    size_t wpart_n = 0;
    int nsplit_max = 0, ncol_blocks = 0, nloss_blocks = 0;
    double* dloss = nullptr;
    int dloss_n = 0;
    float* skbuf = nullptr;   // split-K slices of one-batch GEMMs
    size_t skcap = 0;
    int* tc_err = nullptr;    // error word of the tensor-core GEMMs (null: mma.sync tiles only)
    // solver coupling
    double *basis = nullptr, *proj = nullptr;
    void* dec = nullptr;
    void* backup = nullptr;
    size_t dec_bytes = 0, backup_bytes = 0;
    float *xcol = nullptr, *delta = nullptr;
    // snapshot store
    float* store = nullptr;
    int nslots = 0;
    int *src_d = nullptr, *dst_d = nullptr, *sym_d = nullptr;
    int *aslot_d = nullptr, *zslot_d = nullptr, *pfslot_d = nullptr, *usepred_d = nullptr;
    int augment = 0;          // training with the box's horizontal symmetries
    float noise_rel = 0.0f;   // input noise, relative to each channel's increment std
    int pushforward = 0;      // every other iteration: inputs are the network's own predictions
    double* trace = nullptr;  // per-interval Nu_wall of a rollout (device)
    int trace_n = 0;
    // mean modes advanced by the plain recursion: forcing now / one interval earlier, start values
    double *g_now = nullptr, *g_prev = nullptr, *y0 = nullptr;
    bool have_prev = false;
    // executable graphs of one surrogate interval, per (solver, forcing buffers)
    struct AdvGraph {
        unsigned long long solver;
        const double* g_now;
        bool prev;
        cudaGraphExec_t exec;
    };
    std::vector<AdvGraph> graphs;
    bool use_graphs = true;
    double* stat_part = nullptr;
    int nstat_blocks = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

template <typename T> T* falloc(rbc_fno* f, size_t n)
{
    void* p = nullptr;
    FNO_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    f->owned.push_back(p);
    return static_cast<T*>(p);
}

rbc_status ffail(rbc_fno* f, rbc_status s, const std::string& m)
{
    if (f) f->last_error = m;
    return s;
}

// Reads (and clears) the error word of the tensor-core GEMMs after the caller's stream
// has been synchronised: a bounded wait inside one of them gave up.
rbc_status tc_check(rbc_fno* f)
{
    if (!f->tc_err) return RBC_OK;
    int e = 0;
    if (cudaMemcpy(&e, f->tc_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return ffail(f, RBC_ERR_CUDA, "reading the tensor-core GEMM error word failed");
    if (!e) return RBC_OK;
    cudaMemset(f->tc_err, 0, sizeof(int));
    return ffail(f, RBC_ERR_CUDA, "a tensor-core GEMM wait gave up (accumulator not committed)");
}

#define FNO_GUARD(f)                                                                     \
    if (!f) return RBC_ERR_INVALID_ARG;                                                  \
    try {                                                                                \
        FNO_CUDA(cudaSetDevice(f->p.device));
#define FNO_GUARD_END(f)                                                                 \
    }                                                                                    \
    catch (const CudaErr& e) {                                                           \
        return ffail(f, e.e == cudaErrorMemoryAllocation ? RBC_ERR_OUT_OF_MEMORY : RBC_ERR_CUDA, \
                     std::string(e.what) + ": " + cudaGetErrorString(e.e));              \
    }                                                                                    \
    catch (const ArgErr& e) {                                                            \
        return ffail(f, RBC_ERR_INVALID_ARG, e.msg);                                     \
    }

int load_mode(const bf16* base, long long rs, long long cs, long long bs, int rows, long long K)
{
    const bool al = ((uintptr_t)base % 16) == 0;
    if (cs == 1 && rs % 8 == 0 && bs % 8 == 0 && K % 8 == 0 && al) return 2;
    if (rs == 1 && cs % 8 == 0 && bs % 8 == 0 && rows % 8 == 0 && al) return 3;
    return rs == 1 ? 1 : 0;
}

constexpr int kSMs = 148;

// The tensor-core (tcgen05) GEMM serves products whose A rows are K-contiguous (load mode
// 2), with one B for all batches, N <= 256, K <= 256 (B^T held in shared memory: at most
// 64 KB), no split-K, and at least two waves of 128-row tiles (smaller products keep more
// CTAs in flight on the mma.sync tiles); tc_err null selects the mma.sync tiles for every
// product.
bool tc_shape_ok(const GemmOp& op)
{
    const int n16 = (op.N + 15) & ~15, nchunk = (op.K + kTcKC - 1) / kTcKC;
    return op.amode == 2 && op.N <= kTcNmax && op.K <= kTcKmax && op.ktot == 0 &&
           (op.batch == 1 || op.b_bs == 0) && (size_t)nchunk * n16 * 128 <= 65536;
}
bool tc_eligible(const GemmOp& op, const int* tc_err)
{
    // products with N < 16 or K < 32 stay on the mma.sync tiles: measured faster there (their
    // cost is the epilogue's stores, which the many CTAs of the tiles spread wider)
    const long long tiles = (long long)((op.M + kTcM - 1) / kTcM) * op.batch;
    return tc_err && tc_shape_ok(op) && tiles >= 2 * kSMs && op.N >= 16 && op.K >= 32;
}

int tc_cols(int N)
{
    const int n16 = (N + 15) & ~15;
    return n16 <= 32 ? 32 : n16 <= 64 ? 64 : n16 <= 128 ? 128 : 256;
}

// One CTA per SM where two would not fit the TMEM (2 x 2 x 256 columns): the dynamic
// shared memory asked for is then at least this much.
constexpr size_t kTcSmemFloor = 116 * 1024;

void set_tc_attributes()
{
    const int mx = (int)std::max<size_t>(kTcSmemFloor, gemm_tc_smem(kTcKmax / kTcKC, 128));
    FNO_CUDA(cudaFuncSetAttribute(k_gemm_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FNO_CUDA(cudaFuncSetAttribute(k_gemm_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FNO_CUDA(cudaFuncSetAttribute(k_gemm_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    FNO_CUDA(cudaFuncSetAttribute(k_gemm_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
}

// cuTensorMapEncodeTiled, from the driver through the runtime's entry-point query (no link
// against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Launches the tensor-core GEMM; false (nothing launched) when the tensor map of A cannot be
// encoded, and the caller uses the mma.sync tiles.
bool launch_gemm_tc(cudaStream_t s, const GemmOp& op, int* tc_err)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    CUtensorMap map;
    const long long bs = op.batch > 1 ? op.a_bs : (long long)op.M * op.a_rs;
    const cuuint64_t dims[3] = {(cuuint64_t)op.K, (cuuint64_t)op.M, (cuuint64_t)op.batch};
    const cuuint64_t strides[2] = {(cuuint64_t)op.a_rs * sizeof(bf16), (cuuint64_t)bs * sizeof(bf16)};
    const cuuint32_t box[3] = {(cuuint32_t)kTcKC, (cuuint32_t)kTcM, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16*>(op.A), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    TcArgs a;
    a.op = op;
    a.err = tc_err;
    a.mtiles = (op.M + kTcM - 1) / kTcM;
    a.ntiles = a.mtiles * op.batch;
    a.nchunk = (op.K + kTcKC - 1) / kTcKC;
    a.n16 = (op.N + 15) & ~15;
    auto al = [](const void* p, int b) { return p == nullptr || (uintptr_t)p % b == 0; };
    a.vec4 = (op.c_cs == 1 && op.c_rs % 4 == 0 && op.c_bs % 4 == 0 && al(op.outf, 16) && al(op.pre, 16) &&
              al(op.add, 16) && al(op.aux, 16) && al(op.bias, 16) && al(op.outb, 8)) ? 1 : 0;
    // two CTAs per SM when their accumulators fit the TMEM together and their shared memory too
    const bool two = tc_cols(op.N) <= 128 && gemm_tc_smem(a.nchunk, a.n16) <= 113 * 1024;
    const size_t sm = two ? gemm_tc_smem(a.nchunk, a.n16) : std::max(kTcSmemFloor, gemm_tc_smem(a.nchunk, a.n16));
    const int grid = std::min(a.ntiles, (two ? 2 : 1) * kSMs);
    switch (tc_cols(op.N)) {
    case 32: k_gemm_tc<32><<<grid, kTcThreads, sm, s>>>(map, a); break;
    case 64: k_gemm_tc<64><<<grid, kTcThreads, sm, s>>>(map, a); break;
    case 128: k_gemm_tc<128><<<grid, kTcThreads, sm, s>>>(map, a); break;
    default: k_gemm_tc<256><<<grid, kTcThreads, sm, s>>>(map, a); break;
    }
    FNO_CUDA(cudaGetLastError());
    return true;
}

void launch_gemm(cudaStream_t s, const GemmOp& op, int BM, int BN, int* tc_err = nullptr)
{
    if (tc_eligible(op, tc_err) && launch_gemm_tc(s, op, tc_err)) return;
    dim3 grid((op.M + BM - 1) / BM, (op.N + BN - 1) / BN, op.batch);
    if (grid.y > 65535) throw ArgErr{"gemm N too large"};
    if (BM == 32 && BN == 32) k_gemm<32, 32><<<grid, 128, 0, s>>>(op);
    else if (BM == 32) k_gemm<32, 64><<<grid, 128, 0, s>>>(op);
    else if (BM == 64 && BN == 32) k_gemm<64, 32><<<grid, 128, 0, s>>>(op);
    else if (BM == 64) k_gemm<64, 64><<<grid, 128, 0, s>>>(op);
    else k_gemm<128, 32><<<grid, 128, 0, s>>>(op);
    FNO_CUDA(cudaGetLastError());
}

// Tile choice: the largest tile that still gives one full wave of CTAs (148 SMs), else
// the one with the most CTAs. A one-batch product with too few CTAs and a plain store
// epilogue is split along K into FP32 slices (scratch splitk, cap floats) summed in order
// by k_splitk_finish.
void gemm_on(cudaStream_t s, GemmOp op, float* splitk, size_t cap, int* tc_err = nullptr)
{
    if (op.batch < 1 || op.batch > 65535 || op.M < 1 || op.N < 1 || op.K < 1) throw ArgErr{"gemm shape"};
    // split-K chunks start at multiples of K: 16-byte loads along k need K and ktot % 8 == 0
    long long kchk = op.K;
    if (op.ktot > 0) kchk = (op.K % 8 == 0 && op.ktot % 8 == 0) ? 8 : 1;
    op.amode = load_mode(op.A, op.a_rs, op.a_cs, op.a_bs, op.M, kchk);
    op.bmode = load_mode(op.B, op.b_cs, op.b_rs, op.b_bs, op.N, kchk);
    op.vec2 = (op.c_cs == 1 && op.c_rs % 2 == 0 && op.c_bs % 2 == 0 && op.N % 2 == 0) ? 1 : 0;
    static const int tiles[5][2] = {{128, 32}, {64, 64}, {64, 32}, {32, 64}, {32, 32}};
    auto ctas = [&](int bm, int bn) {
        return (long long)((op.M + bm - 1) / bm) * ((op.N + bn - 1) / bn) * op.batch;
    };
    int BM = 32, BN = 32;
    bool found = false;
    for (auto& t : tiles) {
        // no tile more than half empty along M or N; the 128-row tile only for N <= 32
        if ((t[0] > 32 && t[0] >= 2 * op.M) || (t[1] > 32 && t[1] >= 2 * op.N) || (t[0] == 128 && op.N > 32))
            continue;
        if (ctas(t[0], t[1]) >= kSMs) {
            BM = t[0];
            BN = t[1];
            found = true;
            break;
        }
    }
    if (!found) {
        BM = 32;
        BN = 32;
    }
    const bool plain = !op.bias && !op.add && !op.aux && !op.pre && op.act == ACT_NONE && op.alpha == 1.0f;
    const long long n_ctas = ctas(BM, BN);
    if (!found && plain && op.batch == 1 && op.ktot == 0 && op.K >= 128 && splitk) {
        int S = (int)std::min<long long>(op.K / 32, (2 * kSMs + n_ctas - 1) / n_ctas);
        const int Kc = ((op.K + S - 1) / S + 31) / 32 * 32;
        S = (op.K + Kc - 1) / Kc;
        if (S > 1 && (size_t)S * op.M * op.N <= cap) {
            GemmOp p = op;
            p.K = Kc;
            p.ktot = op.K;
            p.batch = S;
            p.a_bs = (long long)Kc * op.a_cs;
            p.b_bs = (long long)Kc * op.b_rs;
            p.c_rs = op.N;
            p.c_cs = 1;
            p.c_bs = (long long)op.M * op.N;
            p.outf = splitk;
            p.outb = nullptr;
            p.vec2 = op.N % 2 == 0 ? 1 : 0;
            const long long kc8 = (Kc % 8 == 0 && op.K % 8 == 0) ? 8 : 1;
            p.amode = load_mode(p.A, p.a_rs, p.a_cs, p.a_bs, p.M, kc8);
            p.bmode = load_mode(p.B, p.b_cs, p.b_rs, p.b_bs, p.N, kc8);
            launch_gemm(s, p, BM, BN, tc_err);
            const long long mn = (long long)op.M * op.N;
            k_splitk_finish<<<(int)std::min<long long>((mn + 255) / 256, 4 * kSMs), 256, 0, s>>>(
                splitk, S, op.M, op.N, op.c_rs, op.c_cs, op.outf, op.outb);
            FNO_CUDA(cudaGetLastError());
            return;
        }
    }
    launch_gemm(s, op, BM, BN, tc_err);
}

void gemm(rbc_fno* f, cudaStream_t s, const GemmOp& op) { gemm_on(s, op, f->skbuf, f->skcap, f->tc_err); }

int grid_1d(long long n, int threads = 256, int cap = 148 * 8)
{
    long long b = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(b, cap));
}

// dW[o][i] (grad + off) = sum_m G[m][o] X[m][i] over M rows: split-K GEMM into slices,
// then the slices summed in order.
void wgrad(rbc_fno* f, cudaStream_t s, const bf16* G, int No, const bf16* X, int Ni, long long M, long long off)
{
    long long Kc = (M + f->nsplit_max - 1) / f->nsplit_max;
    Kc = std::max<long long>(256, (Kc + 31) / 32 * 32);
    const int ns = (int)((M + Kc - 1) / Kc);
    if ((size_t)ns * No * Ni > f->wpart_n) throw ArgErr{"weight-gradient scratch too small"};
    GemmOp op;
    op.A = G;
    op.a_rs = 1;
    op.a_cs = No;
    op.a_bs = Kc * No;
    op.B = X;
    op.b_rs = Ni;
    op.b_cs = 1;
    op.b_bs = Kc * Ni;
    op.M = No;
    op.N = Ni;
    op.K = (int)Kc;
    op.ktot = M;
    op.batch = ns;
    op.c_rs = Ni;
    op.c_cs = 1;
    op.c_bs = (long long)No * Ni;
    op.outf = f->wpart;
    gemm(f, s, op);
    k_sum_slices<<<(int)(((long long)No * Ni + 31) / 32), dim3(32, 32), 0, s>>>(f->wpart, ns, (long long)No * Ni,
                                                                                f->grad + off, 0);
    FNO_CUDA(cudaGetLastError());
}

// grad[off + n] = sum_m X[m][n].
void colsum(rbc_fno* f, cudaStream_t s, const bf16* X, long long M, int N, long long off)
{
    if (N > 256) throw ArgErr{"column sum wider than a block"};
    const int nb = f->ncol_blocks;
    const long long rpb = (M + nb - 1) / nb;
    k_colsum_part<<<nb, 256, 0, s>>>(X, M, N, rpb, f->cpart);
    FNO_CUDA(cudaGetLastError());
    k_sum_slices<<<(N + 31) / 32, dim3(32, 32), 0, s>>>(f->cpart, nb, N, f->grad + off, 0);
    FNO_CUDA(cudaGetLastError());
}

const bf16* pb(const rbc_fno* f, long long off) { return f->pbf + off; }

// Forward pass of B samples from f->x0 into f->out (FP32 [B P C]).
void forward(rbc_fno* f, int B, cudaStream_t s)
{
    const int W = f->W, m = f->m, my = f->my, nx = f->nx, ny = f->ny, C = f->C, H = f->H;
    const long long M = (long long)B * f->P, mW = (long long)m * W;
    GemmOp op;
    // lift
    op = GemmOp();
    op.A = f->x0; op.a_rs = C; op.a_cs = 1;
    op.B = pb(f, f->oPw); op.b_rs = 1; op.b_cs = C;
    op.M = (int)M; op.N = W; op.K = C;
    op.c_rs = W; op.bias = f->param + f->oPb; op.outb = f->h[0];
    gemm(f, s, op);
    for (int l = 0; l < f->nl; ++l) {
        // x-DFT: per (b, y): A1[kr][c] = sum_x Fx[kr][x] h[x][c]
        op = GemmOp();
        op.A = f->FxT; op.a_rs = nx; op.a_cs = 1;
        op.B = f->h[l]; op.b_rs = W; op.b_cs = 1; op.b_bs = (long long)nx * W;
        op.M = 2 * m; op.N = W; op.K = nx; op.batch = B * ny;
        op.c_rs = W; op.c_bs = 2LL * m * W; op.outb = f->A1;
        gemm(f, s, op);
        // y-DFT: per b: Ahat[(ky, ri)][(kx, c)] = sum_(y, ri') Fy A1
        op = GemmOp();
        op.A = f->FyB; op.a_rs = 2 * ny; op.a_cs = 1;
        op.B = f->A1; op.b_rs = mW; op.b_cs = 1; op.b_bs = 2LL * ny * mW;
        op.M = 2 * my; op.N = (int)mW; op.K = 2 * ny; op.batch = B;
        op.c_rs = mW; op.c_bs = 2LL * my * mW; op.outb = f->Ahat[l];
        gemm(f, s, op);
        // per-mode channel mixing
        const size_t smf = (size_t)(2 * W * W + (128 / W) * 2 * W) * sizeof(float);
        k_modemix_fwd<<<my * m, 128, smf, s>>>(f->Ahat[l], pb(f, f->oR[l]), f->Yh, B, m, W);
        FNO_CUDA(cudaGetLastError());
        // inverse y
        op = GemmOp();
        op.A = f->GyB; op.a_rs = 2 * my; op.a_cs = 1;
        op.B = f->Yh; op.b_rs = mW; op.b_cs = 1; op.b_bs = 2LL * my * mW;
        op.M = 2 * ny; op.N = (int)mW; op.K = 2 * my; op.batch = B;
        op.c_rs = mW; op.c_bs = 2LL * ny * mW; op.outb = f->Z;
        gemm(f, s, op);
        // inverse x (FP32 result, added in the pointwise epilogue)
        op = GemmOp();
        op.A = f->GxT; op.a_rs = 2 * m; op.a_cs = 1;
        op.B = f->Z; op.b_rs = W; op.b_cs = 1; op.b_bs = 2LL * m * W;
        op.M = nx; op.N = W; op.K = 2 * m; op.batch = B * ny;
        op.c_rs = W; op.c_bs = (long long)nx * W; op.outf = f->Kv;
        gemm(f, s, op);
        // pointwise map + spectral part + bias, activation
        op = GemmOp();
        op.A = f->h[l]; op.a_rs = W; op.a_cs = 1;
        op.B = pb(f, f->oW[l]); op.b_rs = 1; op.b_cs = W;
        op.M = (int)M; op.N = W; op.K = W;
        op.c_rs = W; op.bias = f->param + f->ob[l]; op.add = f->Kv; op.pre = f->pre[l];
        op.act = l + 1 < f->nl ? ACT_GELU : ACT_NONE; op.outb = f->h[l + 1];
        gemm(f, s, op);
    }
    op = GemmOp();
    op.A = f->h[f->nl]; op.a_rs = W; op.a_cs = 1;
    op.B = pb(f, f->oQ1w); op.b_rs = 1; op.b_cs = W;
    op.M = (int)M; op.N = H; op.K = W;
    op.c_rs = H; op.bias = f->param + f->oQ1b; op.pre = f->q1pre; op.act = ACT_GELU; op.outb = f->q1;
    gemm(f, s, op);
    op = GemmOp();
    op.A = f->q1; op.a_rs = H; op.a_cs = 1;
    op.B = pb(f, f->oQ2w); op.b_rs = 1; op.b_cs = H;
    op.M = (int)M; op.N = C; op.K = H;
    op.c_rs = C; op.bias = f->param + f->oQ2b; op.outf = f->out;
    gemm(f, s, op);
}

// Loss of f->out against f->target (B samples) into dloss[idx]; gradient into f->grad.
void loss_backward(rbc_fno* f, int B, cudaStream_t s, int idx)
{
    const int W = f->W, m = f->m, my = f->my, nx = f->nx, ny = f->ny, C = f->C, H = f->H;
    const long long M = (long long)B * f->P, mW = (long long)m * W, n = M * C;
    k_mse<<<f->nloss_blocks, 256, 0, s>>>(f->out, f->target, n, f->gA, f->lpart);
    FNO_CUDA(cudaGetLastError());
    k_loss_final<<<1, 32, 0, s>>>(f->lpart, f->nloss_blocks, n, f->dloss, idx);
    FNO_CUDA(cudaGetLastError());
    // projection
    wgrad(f, s, f->gA, C, f->q1, H, M, f->oQ2w);
    colsum(f, s, f->gA, M, C, f->oQ2b);
    GemmOp op;
    op.A = f->gA; op.a_rs = C; op.a_cs = 1;
    op.B = pb(f, f->oQ2w); op.b_rs = H; op.b_cs = 1;
    op.M = (int)M; op.N = H; op.K = C;
    op.c_rs = H; op.act = ACT_GELU_BWD; op.aux = f->q1pre; op.outb = f->gB;
    gemm(f, s, op);
    wgrad(f, s, f->gB, H, f->h[f->nl], W, M, f->oQ1w);
    colsum(f, s, f->gB, M, H, f->oQ1b);
    op = GemmOp();
    op.A = f->gB; op.a_rs = H; op.a_cs = 1;
    op.B = pb(f, f->oQ1w); op.b_rs = W; op.b_cs = 1;
    op.M = (int)M; op.N = W; op.K = H;
    op.c_rs = W; op.outb = f->gA;
    gemm(f, s, op);
    bf16* gp = f->gA;
    bf16* gn = f->gB;
    for (int l = f->nl - 1; l >= 0; --l) {
        wgrad(f, s, gp, W, f->h[l], W, M, f->oW[l]);
        colsum(f, s, gp, M, W, f->ob[l]);
        // adjoint of the inverse x transform
        op = GemmOp();
        op.A = f->GxT; op.a_rs = 1; op.a_cs = 2 * m;
        op.B = gp; op.b_rs = W; op.b_cs = 1; op.b_bs = (long long)nx * W;
        op.M = 2 * m; op.N = W; op.K = nx; op.batch = B * ny;
        op.c_rs = W; op.c_bs = 2LL * m * W; op.outb = f->dZ;
        gemm(f, s, op);
        // adjoint of the inverse y transform
        op = GemmOp();
        op.A = f->GyB; op.a_rs = 1; op.a_cs = 2 * my;
        op.B = f->dZ; op.b_rs = mW; op.b_cs = 1; op.b_bs = 2LL * ny * mW;
        op.M = 2 * my; op.N = (int)mW; op.K = 2 * ny; op.batch = B;
        op.c_rs = mW; op.c_bs = 2LL * my * mW; op.outb = f->dY;
        gemm(f, s, op);
        const size_t smb = (size_t)(2 * W * W + 4 * W) * sizeof(float);
        k_modemix_bwd<<<my * m, 256, smb, s>>>(f->Ahat[l], pb(f, f->oR[l]), f->dY, f->dAh, f->grad + f->oR[l], B,
                                                m, W);
        FNO_CUDA(cudaGetLastError());
        // adjoint of the forward y transform
        op = GemmOp();
        op.A = f->FyB; op.a_rs = 1; op.a_cs = 2 * ny;
        op.B = f->dAh; op.b_rs = mW; op.b_cs = 1; op.b_bs = 2LL * my * mW;
        op.M = 2 * ny; op.N = (int)mW; op.K = 2 * my; op.batch = B;
        op.c_rs = mW; op.c_bs = 2LL * ny * mW; op.outb = f->dA1;
        gemm(f, s, op);
        // adjoint of the forward x transform (FP32)
        op = GemmOp();
        op.A = f->FxT; op.a_rs = 1; op.a_cs = nx;
        op.B = f->dA1; op.b_rs = W; op.b_cs = 1; op.b_bs = 2LL * m * W;
        op.M = nx; op.N = W; op.K = 2 * m; op.batch = B * ny;
        op.c_rs = W; op.c_bs = (long long)nx * W; op.outf = f->dhs;
        gemm(f, s, op);
        // adjoint of the pointwise map, plus the spectral part, times GELU' of the layer below
        op = GemmOp();
        op.A = gp; op.a_rs = W; op.a_cs = 1;
        op.B = pb(f, f->oW[l]); op.b_rs = W; op.b_cs = 1;
        op.M = (int)M; op.N = W; op.K = W;
        op.c_rs = W; op.add = f->dhs;
        if (l > 0) {
            op.act = ACT_GELU_BWD;
            op.aux = f->pre[l - 1];
        }
        op.outb = gn;
        gemm(f, s, op);
        std::swap(gp, gn);
    }
    wgrad(f, s, gp, W, f->x0, C, M, f->oPw);
    colsum(f, s, gp, M, W, f->oPb);
}

void cast_params(rbc_fno* f, cudaStream_t s)
{
    k_cast_bf16<<<grid_1d(f->nparam), 256, 0, s>>>(f->param, f->pbf, f->nparam);
    FNO_CUDA(cudaGetLastError());
}

void check_solver(const rbc_fno* f, const rbc_handle* h)
{
    const rbcint::GridDesc g = rbcint::grid(h);
    if (g.nx != f->nx || g.ny != f->ny || g.L != f->p.nz) throw ArgErr{"solver grid does not match the surrogate"};
    if (g.device != f->p.device) throw ArgErr{"solver and surrogate are on different devices"};
}

void check_status(rbc_status st, rbc_handle* h)
{
    if (st != RBC_OK) throw ArgErr{std::string("solver: ") + rbc_last_error(h)};
}

// One surrogate interval on the solver's stream (advance_body: device work only; host
// bookkeeping in advance_once): encode, network, decode into the state.
// With physics_mean the horizontal-mean modes (theta_k(q=0), F_k, G_k, which set Nu_wall)
// are then replaced by interval_steps recursions of the plain step's own q = 0 update,
// forced by the solver's nonlinear operator at this and the previous interval's start.
void advance_body(rbc_fno* f, rbc_handle* h)
{
    cudaStream_t s = rbcint::stream(h);
    if (f->p.physics_mean)
        check_status(rbcint::colloc_encode_forcing(h, f->p.nq, f->basis, f->xcol, f->g_now, f->y0), h);
    else
        check_status(rbcint::colloc_encode(h, f->p.nq, f->basis, f->xcol), h);
    const int C = f->C;
    k_normalize<<<grid_1d((long long)f->P * C), 256, 0, s>>>(f->xcol, f->P, C, f->norm, f->norm + C, f->x0);
    FNO_CUDA(cudaGetLastError());
    forward(f, 1, s);
    k_denormalize<<<grid_1d((long long)f->P * C), 256, 0, s>>>(f->out, f->P, C, f->norm + 2 * C, f->norm + 3 * C,
                                                               f->delta);
    FNO_CUDA(cudaGetLastError());
    check_status(rbcint::colloc_add(h, f->p.nq, f->proj, f->delta, f->dec), h);
    if (f->p.physics_mean)
        check_status(rbcint::mean_advance(h, f->y0, f->g_now, f->have_prev ? f->g_prev : nullptr, f->p.interval_steps),
                     h);
}

void drop_graphs(rbc_fno* f)
{
    for (auto& g : f->graphs) cudaGraphExecDestroy(g.exec);
    f->graphs.clear();
}

void advance_once(rbc_fno* f, rbc_handle* h)
{
    cudaStream_t s = rbcint::stream(h);
    // one interval is ~40 kernel launches: replayed from an executable graph captured
    // the first time for this solver and forcing-buffer order (a solver with tracers, or
    // the legacy default stream, runs them directly)
    if (f->use_graphs && s != nullptr && !rbcint::has_tracers(h)) {
        const unsigned long long id = rbcint::uid(h);
        cudaGraphExec_t exec = nullptr;
        for (auto& g : f->graphs)
            if (g.solver == id && g.g_now == f->g_now && g.prev == f->have_prev) exec = g.exec;
        if (!exec) {
            if (f->graphs.size() >= 16) drop_graphs(f);
            cudaGraph_t graph = nullptr;
            FNO_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                advance_body(f, h);
            } catch (...) {
                cudaStreamEndCapture(s, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            FNO_CUDA(cudaStreamEndCapture(s, &graph));
            const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            FNO_CUDA(e);
            f->graphs.push_back({id, f->g_now, f->have_prev, exec});
        }
        FNO_CUDA(cudaGraphLaunch(exec, s));
        rbcint::state_changed(h);
    } else {
        advance_body(f, h);
    }
    if (f->p.physics_mean) {
        std::swap(f->g_now, f->g_prev);
        f->have_prev = true;
    }
}

void build_dft(rbc_fno* f)
{
    const int m = f->m, my = f->my, nx = f->nx, ny = f->ny;
    std::vector<uint16_t> Fx((size_t)2 * m * nx), Fy((size_t)2 * my * 2 * ny), Gy((size_t)2 * ny * 2 * my),
        Gx((size_t)nx * 2 * m);
    auto bb = [](double v) { return bf16_bits((float)v); };
    for (int kx = 0; kx < m; ++kx)
        for (int x = 0; x < nx; ++x) {
            const double a = kTwoPi * (double)((long long)kx * x % nx) / nx;
            Fx[(size_t)kx * nx + x] = bb(std::cos(a));
            Fx[(size_t)(m + kx) * nx + x] = bb(-std::sin(a));
            const double w = (kx == 0 ? 1.0 : 2.0) / ((double)nx * ny);
            Gx[(size_t)x * 2 * m + kx] = bb(w * std::cos(a));
            Gx[(size_t)x * 2 * m + m + kx] = bb(-w * std::sin(a));
        }
    for (int ki = 0; ki < my; ++ki) {
        const int ky = ki < m ? ki : ki - my;
        for (int y = 0; y < ny; ++y) {
            const long long e = (((long long)ky * y) % ny + ny) % ny;
            const double a = kTwoPi * (double)e / ny, c = std::cos(a), sn = std::sin(a);
            // forward: rows (ky, ri'), columns (y, ri)
            Fy[(size_t)(2 * ki) * 2 * ny + 2 * y] = bb(c);
            Fy[(size_t)(2 * ki) * 2 * ny + 2 * y + 1] = bb(sn);
            Fy[(size_t)(2 * ki + 1) * 2 * ny + 2 * y] = bb(-sn);
            Fy[(size_t)(2 * ki + 1) * 2 * ny + 2 * y + 1] = bb(c);
            // inverse: rows (y, ri), columns (ky, ri')
            Gy[(size_t)(2 * y) * 2 * my + 2 * ki] = bb(c);
            Gy[(size_t)(2 * y) * 2 * my + 2 * ki + 1] = bb(-sn);
            Gy[(size_t)(2 * y + 1) * 2 * my + 2 * ki] = bb(sn);
            Gy[(size_t)(2 * y + 1) * 2 * my + 2 * ki + 1] = bb(c);
        }
    }
    f->FxT = falloc<bf16>(f, Fx.size());
    f->FyB = falloc<bf16>(f, Fy.size());
    f->GyB = falloc<bf16>(f, Gy.size());
    f->GxT = falloc<bf16>(f, Gx.size());
    FNO_CUDA(cudaMemcpy(f->FxT, Fx.data(), Fx.size() * 2, cudaMemcpyHostToDevice));
    FNO_CUDA(cudaMemcpy(f->FyB, Fy.data(), Fy.size() * 2, cudaMemcpyHostToDevice));
    FNO_CUDA(cudaMemcpy(f->GyB, Gy.data(), Gy.size() * 2, cudaMemcpyHostToDevice));
    FNO_CUDA(cudaMemcpy(f->GxT, Gx.data(), Gx.size() * 2, cudaMemcpyHostToDevice));
}

void init_params(rbc_fno* f, std::vector<float>& v)
{
    v.assign(f->nparam, 0.0f);
    uint64_t k = 0;
    auto uni = [&](float bound) {
        return (float)((2.0 * rbcrng::unit_open(rbcrng::stream_at(f->p.seed, k++)) - 1.0) * bound);
    };
    auto lin = [&](long long ow, long long ob, int out, int in) {
        const float b = 1.0f / std::sqrt((float)in);
        for (long long i = 0; i < (long long)out * in; ++i) v[ow + i] = uni(b);
        for (int i = 0; i < out; ++i) v[ob + i] = uni(b);
    };
    lin(f->oPw, f->oPb, f->W, f->C);
    for (int l = 0; l < f->nl; ++l) {
        lin(f->oW[l], f->ob[l], f->W, f->W);
        const float sc = 1.0f / ((float)f->W * f->W);
        const long long nr = (long long)f->my * f->m * 2 * f->W * f->W;
        for (long long i = 0; i < nr; ++i) v[f->oR[l] + i] = sc * (0.5f * (uni(1.0f) + 1.0f));
    }
    lin(f->oQ1w, f->oQ1b, f->H, f->W);
    lin(f->oQ2w, f->oQ2b, f->C, f->H);
}

} // namespace

extern "C" {

rbc_status rbc_fno_create(const rbc_fno_params* p, rbc_fno** out)
{
    if (!p || !out) return RBC_ERR_INVALID_ARG;
    *out = nullptr;
    if (p->nx < 8 || p->ny < 8 || p->nq < 1 || p->nz < 1 || p->nq < p->nz || p->width < 8 || p->width > 64 ||
        p->width % 8 || p->modes < 1 || 2 * p->modes > p->nx - 2 || 2 * p->modes > p->ny || p->layers < 1 ||
        p->hidden < 8 || p->hidden > 256 || p->max_batch < 1 || 4 * p->nq > 256 || p->interval_steps < 1 ||
        3 * p->nz > 64 || p->gemm_path < 0 || p->gemm_path > 1)
        return RBC_ERR_INVALID_ARG;
    rbc_fno* f = new rbc_fno;
    f->p = *p;
    f->C = 4 * p->nq;
    f->W = p->width;
    f->m = p->modes;
    f->my = 2 * p->modes;
    f->H = p->hidden;
    f->nl = p->layers;
    f->nx = p->nx;
    f->ny = p->ny;
    f->P = p->nx * p->ny;
    f->B = p->max_batch;
    try {
        FNO_CUDA(cudaSetDevice(p->device));
        FNO_CUDA(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
        FNO_CUDA(cudaEventCreate(&f->ev0));
        FNO_CUDA(cudaEventCreate(&f->ev1));
        const int W = f->W, C = f->C, H = f->H;
        long long o = 0;
        f->oPw = o; o += (long long)W * C;
        f->oPb = o; o += W;
        for (int l = 0; l < f->nl; ++l) {
            f->oW.push_back(o); o += (long long)W * W;
            f->ob.push_back(o); o += W;
            f->oR.push_back(o); o += (long long)f->my * f->m * 2 * W * W;
        }
        f->oQ1w = o; o += (long long)H * W;
        f->oQ1b = o; o += H;
        f->oQ2w = o; o += (long long)C * H;
        f->oQ2b = o; o += C;
        f->nparam = o;
        f->param = falloc<float>(f, o);
        f->grad = falloc<float>(f, o);
        f->am = falloc<float>(f, o);
        f->av = falloc<float>(f, o);
        f->pbf = falloc<bf16>(f, o);
        std::vector<float> v;
        init_params(f, v);
        FNO_CUDA(cudaMemcpy(f->param, v.data(), o * sizeof(float), cudaMemcpyHostToDevice));
        FNO_CUDA(cudaMemset(f->grad, 0, o * sizeof(float)));
        FNO_CUDA(cudaMemset(f->am, 0, o * sizeof(float)));
        FNO_CUDA(cudaMemset(f->av, 0, o * sizeof(float)));
        cast_params(f, f->stream);
        build_dft(f);
        f->norm = falloc<float>(f, 5 * C);
        f->norm_h.assign(5 * (size_t)C, 0.0f);
        for (int c = 0; c < C; ++c) f->norm_h[C + c] = f->norm_h[3 * C + c] = f->norm_h[4 * C + c] = 1.0f;
        FNO_CUDA(cudaMemcpy(f->norm, f->norm_h.data(), 5 * C * sizeof(float), cudaMemcpyHostToDevice));
        // activations for max_batch samples
        const long long M = (long long)f->B * f->P, mW = (long long)f->m * W;
        f->x0 = falloc<bf16>(f, M * C);
        f->xf = falloc<float>(f, M * C);
        for (int l = 0; l <= f->nl; ++l) f->h.push_back(falloc<bf16>(f, M * W));
        for (int l = 0; l < f->nl; ++l) {
            f->pre.push_back(falloc<float>(f, M * W));
            f->Ahat.push_back(falloc<bf16>(f, (long long)f->B * 2 * f->my * mW));
        }
        f->A1 = falloc<bf16>(f, (long long)f->B * 2 * f->ny * mW);
        f->Yh = falloc<bf16>(f, (long long)f->B * 2 * f->my * mW);
        f->Z = falloc<bf16>(f, (long long)f->B * 2 * f->ny * mW);
        f->Kv = falloc<float>(f, M * W);
        f->q1pre = falloc<float>(f, M * H);
        f->q1 = falloc<bf16>(f, M * H);
        f->out = falloc<float>(f, M * C);
        f->target = falloc<float>(f, M * C);
        const int gw = std::max({W, H, C});
        f->gA = falloc<bf16>(f, M * gw);
        f->gB = falloc<bf16>(f, M * gw);
        f->dhs = falloc<float>(f, M * W);
        f->dZ = falloc<bf16>(f, (long long)f->B * 2 * f->ny * mW);
        f->dY = falloc<bf16>(f, (long long)f->B * 2 * f->my * mW);
        f->dAh = falloc<bf16>(f, (long long)f->B * 2 * f->my * mW);
        f->dA1 = falloc<bf16>(f, (long long)f->B * 2 * f->ny * mW);
        f->nsplit_max = 148 * 2;
        f->wpart_n = (size_t)(f->nsplit_max + 1) * std::max({(long long)W * C, (long long)W * W, (long long)H * W,
                                                              (long long)C * H});
        f->wpart = falloc<float>(f, f->wpart_n);
        f->ncol_blocks = 148 * 2;
        f->cpart = falloc<float>(f, (size_t)f->ncol_blocks * 256);
        f->nloss_blocks = 148 * 4;
        f->lpart = falloc<float>(f, f->nloss_blocks);
        f->skcap = (size_t)1 << 20;
        f->skbuf = falloc<float>(f, f->skcap);
        if (p->gemm_path == 0) {
            set_tc_attributes();
            f->tc_err = falloc<int>(f, 1);
            FNO_CUDA(cudaMemset(f->tc_err, 0, sizeof(int)));
        }
        f->dloss_n = 1 << 16;
        f->dloss = falloc<double>(f, f->dloss_n);
        // solver coupling (grids with nz vertical modes)
        rbchost::CollocTables ct;
        if (!rbchost::colloc_tables(p->nz, p->nq, ct)) throw ArgErr{"collocation tables"};
        std::vector<double> bas((size_t)p->nq * 3 * p->nz), prj((size_t)2 * p->nz * p->nq);
        for (int q = 0; q < p->nq; ++q)
            for (int mm = 0; mm < p->nz; ++mm) {
                bas[((size_t)q * 3 + 0) * p->nz + mm] = ct.C[q * p->nz + mm];
                bas[((size_t)q * 3 + 1) * p->nz + mm] = ct.Cp[q * p->nz + mm];
                bas[((size_t)q * 3 + 2) * p->nz + mm] = ct.S[q * p->nz + mm];
            }
        std::copy(ct.Ps.begin(), ct.Ps.end(), prj.begin());
        std::copy(ct.Pc.begin(), ct.Pc.end(), prj.begin() + (size_t)p->nz * p->nq);
        f->basis = falloc<double>(f, bas.size());
        f->proj = falloc<double>(f, prj.size());
        FNO_CUDA(cudaMemcpy(f->basis, bas.data(), bas.size() * sizeof(double), cudaMemcpyHostToDevice));
        FNO_CUDA(cudaMemcpy(f->proj, prj.data(), prj.size() * sizeof(double), cudaMemcpyHostToDevice));
        const size_t mox = (size_t)p->nx / 2 + 1, ckp = ((mox + 3) / 4) * 4;
        f->dec_bytes = (size_t)4 * p->nz * f->P * sizeof(double) + (size_t)4 * p->nz * mox * p->ny * 16;
        f->dec = falloc<unsigned char>(f, f->dec_bytes);
        f->backup_bytes = ((size_t)3 * p->nz * ckp * p->ny + 2 * (size_t)p->nz) * 16;
        f->backup = falloc<unsigned char>(f, f->backup_bytes);
        f->g_now = falloc<double>(f, 3 * (size_t)p->nz);
        f->g_prev = falloc<double>(f, 3 * (size_t)p->nz);
        f->y0 = falloc<double>(f, 3 * (size_t)p->nz);
        f->trace_n = 1 << 16;
        f->trace = falloc<double>(f, f->trace_n);
        f->xcol = falloc<float>(f, (size_t)f->P * C);
        f->delta = falloc<float>(f, (size_t)f->P * C);
        FNO_CUDA(cudaStreamSynchronize(f->stream));
    } catch (const CudaErr& e) {
        for (void* q : f->owned) cudaFree(q);
        const bool oom = e.e == cudaErrorMemoryAllocation;
        delete f;
        return oom ? RBC_ERR_OUT_OF_MEMORY : RBC_ERR_CUDA;
    } catch (const ArgErr&) {
        for (void* q : f->owned) cudaFree(q);
        delete f;
        return RBC_ERR_INVALID_ARG;
    }
    *out = f;
    return RBC_OK;
}

void rbc_fno_destroy(rbc_fno* f)
{
    if (!f) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(f->p.device);
    if (f->stream) cudaStreamSynchronize(f->stream);
    cudaDeviceSynchronize();
    drop_graphs(f);
    for (void* q : f->owned) cudaFree(q);
    if (f->stream) cudaStreamDestroy(f->stream);
    if (f->ev0) cudaEventDestroy(f->ev0);
    if (f->ev1) cudaEventDestroy(f->ev1);
    cudaSetDevice(cur);
    delete f;
}

const char* rbc_fno_last_error(const rbc_fno* f) { return f ? f->last_error.c_str() : "null surrogate"; }

long long rbc_fno_num_params(const rbc_fno* f) { return f ? f->nparam : 0; }

rbc_status rbc_fno_get_params(rbc_fno* f, float* out, long long n)
{
    if (!out || (f && n != f->nparam)) return ffail(f, RBC_ERR_INVALID_ARG, "parameter count");
    FNO_GUARD(f)
    FNO_CUDA(cudaStreamSynchronize(f->stream));
    FNO_CUDA(cudaMemcpy(out, f->param, n * sizeof(float), cudaMemcpyDeviceToHost));
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_set_params(rbc_fno* f, const float* in, long long n)
{
    if (!in || (f && n != f->nparam)) return ffail(f, RBC_ERR_INVALID_ARG, "parameter count");
    FNO_GUARD(f)
    FNO_CUDA(cudaStreamSynchronize(f->stream));
    FNO_CUDA(cudaMemcpy(f->param, in, n * sizeof(float), cudaMemcpyHostToDevice));
    FNO_CUDA(cudaMemset(f->am, 0, n * sizeof(float)));
    FNO_CUDA(cudaMemset(f->av, 0, n * sizeof(float)));
    f->adam_t = 0;
    cast_params(f, f->stream);
    FNO_CUDA(cudaStreamSynchronize(f->stream));
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_get_norm(rbc_fno* f, float* out)
{
    if (!out) return ffail(f, RBC_ERR_INVALID_ARG, "null output");
    FNO_GUARD(f)
    const int C = f->C;
    for (int c = 0; c < C; ++c) {
        out[c] = f->norm_h[c];
        out[C + c] = 1.0f / f->norm_h[C + c];
        out[2 * C + c] = f->norm_h[2 * C + c];
        out[3 * C + c] = f->norm_h[3 * C + c];
    }
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_set_norm(rbc_fno* f, const float* in)
{
    if (!in) return ffail(f, RBC_ERR_INVALID_ARG, "null input");
    FNO_GUARD(f)
    const int C = f->C;
    for (int c = 0; c < C; ++c)
        if (!(in[C + c] > 0) || !(in[3 * C + c] > 0)) throw ArgErr{"standard deviations must be positive"};
    for (int c = 0; c < C; ++c) {
        f->norm_h[c] = in[c];
        f->norm_h[C + c] = 1.0f / in[C + c];
        f->norm_h[2 * C + c] = in[2 * C + c];
        f->norm_h[3 * C + c] = in[3 * C + c];
        f->norm_h[4 * C + c] = 1.0f / in[3 * C + c];
    }
    FNO_CUDA(cudaMemcpyAsync(f->norm, f->norm_h.data(), 5 * C * sizeof(float), cudaMemcpyHostToDevice, f->stream));
    FNO_CUDA(cudaStreamSynchronize(f->stream));
    f->have_norm = true;
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_forward(rbc_fno* f, const float* x, int batch, float* y)
{
    if (!x || !y || (f && (batch < 1 || batch > f->B))) return ffail(f, RBC_ERR_INVALID_ARG, "bad forward arguments");
    FNO_GUARD(f)
    const long long n = (long long)batch * f->P * f->C;
    FNO_CUDA(cudaMemcpyAsync(f->xf, x, n * sizeof(float), cudaMemcpyHostToDevice, f->stream));
    k_cast_bf16<<<grid_1d(n), 256, 0, f->stream>>>(f->xf, f->x0, n);
    FNO_CUDA(cudaGetLastError());
    forward(f, batch, f->stream);
    FNO_CUDA(cudaMemcpyAsync(y, f->out, n * sizeof(float), cudaMemcpyDeviceToHost, f->stream));
    FNO_CUDA(cudaStreamSynchronize(f->stream));
    return tc_check(f);
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_loss_grad(rbc_fno* f, const float* x, const float* target, int batch, double* loss, float* grad)
{
    if (!x || !target || !loss || !grad || (f && (batch < 1 || batch > f->B)))
        return ffail(f, RBC_ERR_INVALID_ARG, "bad gradient arguments");
    FNO_GUARD(f)
    const long long n = (long long)batch * f->P * f->C;
    FNO_CUDA(cudaMemcpyAsync(f->xf, x, n * sizeof(float), cudaMemcpyHostToDevice, f->stream));
    FNO_CUDA(cudaMemcpyAsync(f->target, target, n * sizeof(float), cudaMemcpyHostToDevice, f->stream));
    k_cast_bf16<<<grid_1d(n), 256, 0, f->stream>>>(f->xf, f->x0, n);
    FNO_CUDA(cudaGetLastError());
    forward(f, batch, f->stream);
    loss_backward(f, batch, f->stream, 0);
    FNO_CUDA(cudaMemcpyAsync(loss, f->dloss, sizeof(double), cudaMemcpyDeviceToHost, f->stream));
    FNO_CUDA(cudaMemcpyAsync(grad, f->grad, f->nparam * sizeof(float), cudaMemcpyDeviceToHost, f->stream));
    FNO_CUDA(cudaStreamSynchronize(f->stream));
    return tc_check(f);
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_colloc_get(rbc_fno* f, rbc_handle* h, float* out)
{
    if (!h || !out) return ffail(f, RBC_ERR_INVALID_ARG, "null argument");
    FNO_GUARD(f)
    check_solver(f, h);
    check_status(rbcint::colloc_encode(h, f->p.nq, f->basis, f->xcol), h);
    cudaStream_t s = rbcint::stream(h);
    FNO_CUDA(cudaMemcpyAsync(out, f->xcol, (size_t)f->P * f->C * sizeof(float), cudaMemcpyDeviceToHost, s));
    FNO_CUDA(cudaStreamSynchronize(s));
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_colloc_add(rbc_fno* f, rbc_handle* h, const float* delta)
{
    if (!h || !delta) return ffail(f, RBC_ERR_INVALID_ARG, "null argument");
    FNO_GUARD(f)
    check_solver(f, h);
    cudaStream_t s = rbcint::stream(h);
    FNO_CUDA(cudaMemcpyAsync(f->delta, delta, (size_t)f->P * f->C * sizeof(float), cudaMemcpyHostToDevice, s));
    check_status(rbcint::colloc_add(h, f->p.nq, f->proj, f->delta, f->dec), h);
    FNO_CUDA(cudaStreamSynchronize(s));
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_dataset_reserve(rbc_fno* f, int nslots)
{
    if (nslots < 2) return ffail(f, RBC_ERR_INVALID_ARG, "need at least two slots");
    FNO_GUARD(f)
    if (f->store) throw ArgErr{"the snapshot store is already reserved"};
    f->store = falloc<float>(f, (size_t)nslots * f->P * f->C);
    f->nslots = nslots;
    f->src_d = falloc<int>(f, nslots);
    f->dst_d = falloc<int>(f, nslots);
    f->sym_d = falloc<int>(f, nslots);
    f->aslot_d = falloc<int>(f, nslots);
    f->zslot_d = falloc<int>(f, nslots);
    f->pfslot_d = falloc<int>(f, nslots);
    f->usepred_d = falloc<int>(f, nslots);
    f->nstat_blocks = 148 * 4;
    f->stat_part = falloc<double>(f, (size_t)f->nstat_blocks * 4 * f->C);
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_dataset_capture(rbc_fno* f, rbc_handle* h, int slot)
{
    if (!h || (f && (slot < 0 || slot >= f->nslots))) return ffail(f, RBC_ERR_INVALID_ARG, "bad slot");
    FNO_GUARD(f)
    check_solver(f, h);
    float* dst = f->store + (size_t)slot * f->P * f->C;
    check_status(rbcint::colloc_encode(h, f->p.nq, f->basis, dst), h);
    FNO_CUDA(cudaStreamSynchronize(rbcint::stream(h)));
    return RBC_OK;
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_train(rbc_fno* f, const int* src, const int* dst, int npairs, int epochs, int batch, double lr,
                         unsigned long long seed, int fit_norm, double* epoch_loss)
{
    if (!src || !dst || !epoch_loss || npairs < 1 || epochs < 0 || batch < 1 || !(lr > 0))
        return ffail(f, RBC_ERR_INVALID_ARG, "bad training arguments");
    FNO_GUARD(f)
    if (!f->store || npairs > f->nslots) throw ArgErr{"pairs exceed the snapshot store"};
    if (batch > f->B || batch > npairs) throw ArgErr{"batch larger than max_batch or the pair count"};
    for (int i = 0; i < npairs; ++i)
        if (src[i] < 0 || src[i] >= f->nslots || dst[i] < 0 || dst[i] >= f->nslots) throw ArgErr{"slot out of range"};
    cudaStream_t s = f->stream;
    const int C = f->C;
    const long long P = f->P;
    FNO_CUDA(cudaMemcpyAsync(f->src_d, src, npairs * sizeof(int), cudaMemcpyHostToDevice, s));
    FNO_CUDA(cudaMemcpyAsync(f->dst_d, dst, npairs * sizeof(int), cudaMemcpyHostToDevice, s));
    if (fit_norm || !f->have_norm) {
        const long long rows = (long long)npairs * P;
        const long long rpb = (rows + f->nstat_blocks - 1) / f->nstat_blocks;
        k_pair_stats<<<f->nstat_blocks, 256, 0, s>>>(f->store, P, C, f->src_d, f->dst_d, npairs, rpb, f->stat_part);
        FNO_CUDA(cudaGetLastError());
        std::vector<double> part((size_t)f->nstat_blocks * 4 * C);
        FNO_CUDA(cudaMemcpyAsync(part.data(), f->stat_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        FNO_CUDA(cudaStreamSynchronize(s));
        std::vector<double> sum(4 * (size_t)C, 0.0);
        for (int b = 0; b < f->nstat_blocks; ++b)
            for (int k = 0; k < 4 * C; ++k) sum[k] += part[(size_t)b * 4 * C + k];
        // per-channel mean and std; with symmetry augmentation the velocity channels have
        // mean 0 (a flip reverses them) and, with the transpose, u and v share one std
        const int nq = f->p.nq;
        const double n = (double)rows;
        std::vector<double> mean(2 * (size_t)C), sec(2 * (size_t)C);
        for (int c = 0; c < C; ++c) {
            mean[c] = sum[c] / n;
            sec[c] = sum[C + c] / n;
            mean[C + c] = sum[2 * C + c] / n;
            sec[C + c] = sum[3 * C + c] / n;
        }
        if (f->augment)
            for (int q = 0; q < nq; ++q)
                for (int k = 0; k < 2; ++k) {
                    const int cu = k * C + nq + q, cv = k * C + 2 * nq + q;
                    mean[cu] = mean[cv] = 0.0;
                    if (f->augment == 2) sec[cu] = sec[cv] = 0.5 * (sec[cu] + sec[cv]);
                }
        for (int c = 0; c < C; ++c) {
            const double xv = std::max(0.0, sec[c] - mean[c] * mean[c]);
            const double dv = std::max(0.0, sec[C + c] - mean[C + c] * mean[C + c]);
            const double xs = xv > 0 ? std::sqrt(xv) : 1.0, ds = dv > 0 ? std::sqrt(dv) : 1.0;
            f->norm_h[c] = (float)mean[c];
            f->norm_h[C + c] = (float)(1.0 / xs);
            f->norm_h[2 * C + c] = (float)mean[C + c];
            f->norm_h[3 * C + c] = (float)ds;
            f->norm_h[4 * C + c] = (float)(1.0 / ds);
        }
        FNO_CUDA(cudaMemcpyAsync(f->norm, f->norm_h.data(), 5 * C * sizeof(float), cudaMemcpyHostToDevice, s));
        f->have_norm = true;
    }
    const int iters = npairs / batch;
    if (iters > f->dloss_n) throw ArgErr{"too many iterations per epoch"};
    const long long total = (long long)iters * epochs;
    // the pair that ends where pair i starts (same run), for pushforward inputs
    std::vector<int> prev(npairs, -1);
    {
        std::vector<int> by_dst(f->nslots, -1);
        for (int i = 0; i < npairs; ++i) by_dst[dst[i]] = i;
        for (int i = 0; i < npairs; ++i) prev[i] = by_dst[src[i]];
    }
    std::vector<int> perm(npairs), symv(npairs, 0), aslot(npairs), zslot(npairs), pfslot(npairs), usepred(npairs);
    std::vector<double> lh(iters);
    long long it_glob = 0;
    const long long nel = (long long)batch * P * C;
    for (int e = 0; e < epochs; ++e) {
        for (int i = 0; i < npairs; ++i) perm[i] = i;
        for (int i = npairs - 1; i > 0; --i) {
            const uint64_t r = rbcrng::stream_at(seed + 0x9E37ULL * (uint64_t)(e + 1), (uint64_t)i);
            const int j = (int)(r % (uint64_t)(i + 1));
            std::swap(perm[i], perm[j]);
        }
        for (int i = 0; i < npairs; ++i) {
            const int pi = perm[i];
            aslot[i] = src[pi];
            zslot[i] = dst[pi];
            pfslot[i] = prev[pi] >= 0 ? src[prev[pi]] : src[pi];
            usepred[i] = prev[pi] >= 0 ? 1 : 0;
            if (f->augment) {
                const int nsym = f->augment == 2 ? 8 : 4;
                const uint64_t r = rbcrng::stream_at(seed ^ 0x5EEDULL, (uint64_t)e * npairs + i);
                symv[i] = nsym == 8 ? (int)(r % 8) : (int)(r % 4) * 2;
            }
        }
        FNO_CUDA(cudaMemcpyAsync(f->aslot_d, aslot.data(), npairs * sizeof(int), cudaMemcpyHostToDevice, s));
        FNO_CUDA(cudaMemcpyAsync(f->zslot_d, zslot.data(), npairs * sizeof(int), cudaMemcpyHostToDevice, s));
        FNO_CUDA(cudaMemcpyAsync(f->pfslot_d, pfslot.data(), npairs * sizeof(int), cudaMemcpyHostToDevice, s));
        FNO_CUDA(cudaMemcpyAsync(f->usepred_d, usepred.data(), npairs * sizeof(int), cudaMemcpyHostToDevice, s));
        if (f->augment)
            FNO_CUDA(cudaMemcpyAsync(f->sym_d, symv.data(), npairs * sizeof(int), cudaMemcpyHostToDevice, s));
        for (int it = 0; it < iters; ++it, ++it_glob) {
            const size_t o = (size_t)it * batch;
            const int* symp = f->augment ? f->sym_d + o : nullptr;
            const unsigned long long nseed = rbcrng::mix64(seed ^ (0xA5A5ULL + (uint64_t)it_glob));
            const bool pf = f->pushforward && (it & 1);
            if (pf) {
                // the network's prediction from the previous snapshot of each pair's run
                k_gather_slots<<<grid_1d(nel), 256, 0, s>>>(f->store, f->nx, f->ny, f->p.nq, f->pfslot_d + o, nullptr,
                                                            symp, nullptr, nullptr, batch, f->norm, f->norm + C,
                                                            f->norm + 2 * C, f->norm + 3 * C, f->norm + 4 * C, 0.0f, 0,
                                                            f->x0, nullptr);
                FNO_CUDA(cudaGetLastError());
                forward(f, batch, s);
            }
            k_gather_slots<<<grid_1d(nel), 256, 0, s>>>(f->store, f->nx, f->ny, f->p.nq,
                                                        pf ? f->pfslot_d + o : f->aslot_d + o, f->zslot_d + o, symp,
                                                        f->usepred_d + o, pf ? f->out : nullptr, batch, f->norm,
                                                        f->norm + C, f->norm + 2 * C, f->norm + 3 * C, f->norm + 4 * C,
                                                        f->noise_rel, nseed, f->x0, f->target);
            FNO_CUDA(cudaGetLastError());
            forward(f, batch, s);
            loss_backward(f, batch, s, it);
            // cosine decay from lr to lr / 50 over the run
            const double frac = total > 1 ? (double)it_glob / (double)(total - 1) : 0.0;
            const double lr_t = lr * (0.02 + 0.98 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * frac)));
            ++f->adam_t;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.0f - std::pow(b1, (float)f->adam_t), c2 = 1.0f - std::pow(b2, (float)f->adam_t);
            k_adam<<<grid_1d(f->nparam), 256, 0, s>>>(f->param, f->grad, f->am, f->av, f->nparam, (float)lr_t, b1,
                                                      b2, 1e-8f, c1, c2);
            FNO_CUDA(cudaGetLastError());
            cast_params(f, s);
        }
        FNO_CUDA(cudaMemcpyAsync(lh.data(), f->dloss, iters * sizeof(double), cudaMemcpyDeviceToHost, s));
        FNO_CUDA(cudaStreamSynchronize(s));
        double m = 0;
        for (double v : lh) m += v;
        epoch_loss[e] = m / iters;
    }
    FNO_CUDA(cudaStreamSynchronize(s));
    return tc_check(f);
    FNO_GUARD_END(f)
}

rbc_status rbc_fno_set_train_options(rbc_fno* f, int augment, double noise_rel, int pushforward)
{
    if (!f) return RBC_ERR_INVALID_ARG;
    if (augment < 0 || augment > 2 || (augment == 2 && f->nx != f->ny) || !(noise_rel >= 0) || noise_rel > 10 ||
        pushforward < 0 || pushforward > 1)
        return ffail(f, RBC_ERR_INVALID_ARG, "bad training options");
    f->augment = augment;
    f->noise_rel = (float)noise_rel;
    f->pushforward = pushforward;
    return RBC_OK;
}

rbc_status rbc_fno_advance(rbc_fno* f, rbc_handle* h, int n)
{
    if (!h || n < 0) return ffail(f, RBC_ERR_INVALID_ARG, "bad advance arguments");
    FNO_GUARD(f)
    check_solver(f, h);
    f->have_prev = false;
    for (int i = 0; i < n; ++i) advance_once(f, h);
    FNO_CUDA(cudaStreamSynchronize(rbcint::stream(h)));
    return tc_check(f);
    FNO_GUARD_END(f)
}

rbc_status rbc_surrogate_run(rbc_fno* f, rbc_handle* h, const rbc_surrogate_params* sp, rbc_surrogate_report* rep,
                             double* nu_trace)
{
    if (!h || !sp || !rep || sp->intervals < 0 || sp->judge_every < 1 ||
        !(sp->nu_tol > 0) || sp->spec_bins < 0 || sp->spec_bins > 4096 ||
        (f && nu_trace && sp->intervals > f->trace_n))
        return ffail(f, RBC_ERR_INVALID_ARG, "bad surrogate-run arguments");
    FNO_GUARD(f)
    check_solver(f, h);
    std::memset(rep, 0, sizeof(*rep));
    cudaStream_t s = rbcint::stream(h);
    const int nb = sp->spec_bins;
    std::vector<double> spec_s(nb), spec_p(nb);
    FNO_CUDA(cudaEventRecord(f->ev0, s));
    long long fallback_left = 0;
    const int nstep = f->p.interval_steps;
    f->have_prev = false;
    for (int t = 0; t < sp->intervals; ++t) {
        if (fallback_left != 0) {
            check_status(rbc_step_async(h, nstep), h);
            ++rep->plain_intervals;
            f->have_prev = false;
            if (fallback_left > 0) --fallback_left;
            if (nu_trace) check_status(rbcint::nu_wall_record(h, f->trace + t), h);
            continue;
        }
        if ((t + 1) % sp->judge_every != 0) {
            advance_once(f, h);
            ++rep->surrogate_intervals;
            if (nu_trace) check_status(rbcint::nu_wall_record(h, f->trace + t), h);
            continue;
        }
        // check: the surrogate and the plain step over the same interval from one state
        check_status(rbcint::state_save(h, f->backup), h);
        advance_once(f, h);
        double nu_s = 0, nu_p = 0;
        check_status(rbcint::nu_wall(h, &nu_s), h);
        if (nb > 0) check_status(rbc_spectrum(h, 0.0, spec_s.data(), nb), h);
        check_status(rbcint::state_load(h, f->backup), h);
        check_status(rbc_step_async(h, nstep), h);
        f->have_prev = false;
        check_status(rbcint::nu_wall(h, &nu_p), h);
        if (nb > 0) check_status(rbc_spectrum(h, 0.0, spec_p.data(), nb), h);
        const double enu = std::fabs(nu_s - nu_p) / std::max(std::fabs(nu_p), 1e-300);
        double num = 0, den = 0;
        for (int i = 0; i < nb; ++i) {
            num += (spec_s[i] - spec_p[i]) * (spec_s[i] - spec_p[i]);
            den += spec_p[i] * spec_p[i];
        }
        const double esp = nb > 0 && den > 0 ? std::sqrt(num / den) : 0.0;
        ++rep->checks;
        ++rep->plain_intervals;
        rep->last_nu_err = enu;
        rep->last_spec_err = esp;
        rep->max_nu_err = std::max(rep->max_nu_err, enu);
        rep->max_spec_err = std::max(rep->max_spec_err, esp);
        const bool bad = !(enu <= sp->nu_tol) || (sp->spec_tol > 0 && nb > 0 && !(esp <= sp->spec_tol));
        if (bad) {
            ++rep->fallbacks;
            fallback_left = sp->fallback_intervals < 0 ? -1 : sp->fallback_intervals;
        }
        if (nu_trace) check_status(rbcint::nu_wall_record(h, f->trace + t), h);
    }
    FNO_CUDA(cudaEventRecord(f->ev1, s));
    FNO_CUDA(cudaEventSynchronize(f->ev1));
    float ms = 0;
    FNO_CUDA(cudaEventElapsedTime(&ms, f->ev0, f->ev1));
    rep->ms = ms;
    check_status(rbc_synchronize(h), h);
    if (nu_trace && sp->intervals > 0)
        FNO_CUDA(cudaMemcpy(nu_trace, f->trace, sp->intervals * sizeof(double), cudaMemcpyDeviceToHost));
    return tc_check(f);
    FNO_GUARD_END(f)
}

rbc_status rbc_gemm_bf16(int device, const void* A, const void* B, float* C, int M, int N, int K, int path,
                         void* stream)
{
    if (!A || !B || !C || M < 1 || N < 1 || K < 1 || path < 0 || path > 1) return RBC_ERR_INVALID_ARG;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return RBC_ERR_CUDA;
    rbc_status st = RBC_OK;
    static int* err_words[64] = {nullptr}; // one error word per device, kept for the process
    int* err = nullptr;
    try {
        cudaStream_t s = (cudaStream_t)stream;
        GemmOp op;
        op.A = static_cast<const bf16*>(A);
        op.a_rs = K;
        op.a_cs = 1;
        op.B = static_cast<const bf16*>(B);
        op.b_rs = N;
        op.b_cs = 1;
        op.M = M;
        op.N = N;
        op.K = K;
        op.c_rs = N;
        op.c_cs = 1;
        op.outf = C;
        if (path == 0) {
            // the tensor-core kernel for every size it can take (partial tiles included)
            op.amode = load_mode(op.A, op.a_rs, op.a_cs, op.a_bs, op.M, op.K);
            if (!tc_shape_ok(op)) throw ArgErr{"shape not supported by the tensor-core GEMM"};
            if (device < 0 || device >= 64) throw ArgErr{"device ordinal"};
            set_tc_attributes();
            if (!err_words[device]) FNO_CUDA(cudaMalloc(&err_words[device], sizeof(int)));
            err = err_words[device];
            FNO_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
            if (!launch_gemm_tc(s, op, err)) throw ArgErr{"the tensor map of A could not be encoded"};
        } else {
            gemm_on(s, op, nullptr, 0, nullptr);
        }
        FNO_CUDA(cudaStreamSynchronize(s));
        if (err) {
            int e = 0;
            FNO_CUDA(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
            if (e) st = RBC_ERR_CUDA;
        }
    } catch (const CudaErr&) {
        st = RBC_ERR_CUDA;
    } catch (const ArgErr&) {
        st = RBC_ERR_INVALID_ARG;
    }
    cudaSetDevice(prev);
    return st;
}

} // extern "C"
