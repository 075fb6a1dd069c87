// update_kernel.cuh -- fused per-wavenumber update of the IMEX step (sm_100a, FP64).
//
// One team of T = next_pow2(L) lanes per kept wavenumber (c, r); lane k owns vertical
// mode k and the team exchanges its mode vectors through a per-warp shared-memory slot.
// Per wavenumber it does:
//   inverse B        (inverse_B_matrix.cu:199-328): theta x2, f by the L x L B_ff^-1 of
//                    its q^2 class, g x (-2 Pr / q^2) (0 at q = 0), F, G x 2 Pr (Im = 0)
//   AB2 / Euler      (implicit_explicit_stepping.cu:43-69): u += 1.5dt r - 0.5dt r_prev
//   implicit solve   (linear_implicit_operator.cu:350-490): [theta; f] <- M(q)[theta; f],
//                    g / (1 + dt Pr (q^2 + (m pi)^2)), F, G / (1 + dt Pr (m pi)^2)
//   make_real        (util.cu:184-209) on the kx = 0 column: the team of row Ny - r
//                    also writes conj() into row r, row 0 gets Im = 0
//   diagnostics      Nu_wall, Nu_vol, KE of the new state by Parseval (spectral, exact)
// The dealiased band is never touched: it stays zero.
#pragma once
#include "common.cuh"
#include "step_kernels.cuh"

namespace rbck {

// The operators couple only vertical modes of equal parity: the Chandrasekhar functions
// and sines of odd index m + 1 are even in z, those of even index odd, and every matrix
// here (B_ff^-1, the four blocks of the implicit operator, the diagnostics' integrals) has
// exact zeros where the row and column parities differ. Row k of each is therefore kept
// as its OP_H(L) entries in columns m = (k & 1) + 2 i (0 past column L - 1), and the
// products skip the zeros, which leaves every sum bit for bit unchanged.
RBC_HD constexpr int op_half(int L) { return (L + 1) / 2; }
// Doubles per packed row: B_ff^-1, then the (tt, tf, ft, ff) blocks, padded to even.
RBC_HD constexpr int op_row(int L) { return (5 * op_half(L) + 1) & ~1; }

struct UpdateArgs {
    Geom G;
    const int* cls;            // CM [ckp][Ny] q^2 class (-1: not kept)
    const double* optab;       // [nclass][L][op_row(L)] parity-packed rows (see above)
    const double* diag_tab;    // [3][L*L]: int C'_i C'_j, int C_i C_j, int C_i S_j
    const void* N;             // CM [3][L][ckp][Ny] complex (R)
    const double* NFG;         // [2][L]
    double2* th; double2* f; double2* g;   // CM state
    double2* FG;               // [2][L]
    double2* hist;             // CM [3][L][ckp][Ny]
    double2* hFG;              // [2][L]
    int first;                 // 1: Euler step (no history yet)
    // diagnostics
    double* partial;           // [gridDim.x][2]
    unsigned int* ticket;      // last-block counter (self-resetting)
    double* th00;              // [L] Re theta(q=0) after the step
    double* ring;              // [cap + 1][4] = nu_wall, nu_vol, ke, step; entry cap = newest
    int ring_cap;
    long long* step_counter;
    int* err;
    // kept rows (2/3 rule): r < nlow or r >= nlow + (ny - nkr); teams cover only these
    int nlow, nkr;
};

template <int L> struct TeamSize { static constexpr int value = L <= 2 ? 2 : L <= 4 ? 4 : L <= 8 ? 8 : 16; };

RBC_D double2 shfl2(double2 v, int src, int width)
{
    return make_double2(__shfl_sync(0xffffffffu, v.x, src, width), __shfl_sync(0xffffffffu, v.y, src, width));
}

template <typename R, int L>
__global__ void __launch_bounds__(kThreads, 2) k_update(UpdateArgs A)
{
    typedef typename cplx_t<R>::type C;
    constexpr int T = TeamSize<L>::value;
    constexpr int TPW = 32 / T;                 // teams per warp
    // per-warp staging of the team vectors: [team][mode] (instead of shuffles)
    __shared__ double2 stg[kThreads / 32][2][TPW][T];
    const double* dtab = A.diag_tab;            // [3][L*L], read through the L1 cache
    const Geom& G = A.G;
    const int ny = G.ny;
    const size_t plane = (size_t)G.ckp * ny;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int tm = lane / T;                    // team within the warp
    const int k = lane - tm * T;                // this lane's vertical mode
    const C* Nc = reinterpret_cast<const C*>(A.N);
    const double dt = G.dt, pr = G.pr;
    const double a1 = A.first ? dt : 1.5 * dt, a2 = -0.5 * dt;
    const double mpi = (k + 1) * kPi;
    double esum = 0.0, wsum = 0.0;
    const long long nwave = (long long)G.ckeep * A.nkr; // kept wavenumbers
    pdl_trigger();
    {
        // kept wavenumber e = c * nkr + j, j the kept-row index (the removed rows stay zero
        // and get no team)
        const long long e = (long long)blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
        const int c = (int)(e / A.nkr), j = (int)(e - (long long)c * A.nkr);
        const int r = j < A.nlow ? j : j + (ny - A.nkr);
        const size_t o = (size_t)c * ny + r;           // CM offset in a plane
        // the class index is constant and is fetched before the wait; after it the
        // vectors and the class's table rows are fetched together (the vector loads are
        // predicated on the kept band by its formula, always in bounds)
        const int cl = (e < nwave) ? __ldg(A.cls + o) : -1;   // uniform over the team
        pdl_wait(); // N and the mean-flow terms come from the column pass
        const bool geo = e < nwave && k < L && c < G.ckeep && row_kept(r, ny);
        const int ry = wrap_row(r, ny);
        const double mx = (kPi + kPi) * (c / G.lx), my = (kPi + kPi) * (ry / G.ly);
        const double q2d = mx * mx + my * my;       // device formula of the reference kernels
        const bool mirror = (c == 0 && r > 0 && r < ny / 2);
        double2 nt = make_double2(0, 0), nf = nt, ng = nt, ut = nt, uf = nt, ug = nt, ht = nt, hf = nt, hg = nt;
        if (geo) {
            const C t0 = ld_cg(Nc + (0 * L + k) * plane + o), t1 = ld_cg(Nc + (1 * L + k) * plane + o),
                    t2 = ld_cg(Nc + (2 * L + k) * plane + o);
            nt = make_double2(t0.x, t0.y);
            nf = make_double2(t1.x, t1.y);
            ng = make_double2(t2.x, t2.y);
            if (!mirror) {
                ut = ld_cg(A.th + k * plane + o);
                uf = ld_cg(A.f + k * plane + o);
                ug = ld_cg(A.g + k * plane + o);
                if (!A.first) {
                    ht = ld_cg(A.hist + (0 * L + k) * plane + o);
                    hf = ld_cg(A.hist + (1 * L + k) * plane + o);
                    hg = ld_cg(A.hist + (2 * L + k) * plane + o);
                }
            }
        }
        const bool act = cl >= 0;
        const bool kact = act && k < L;
        constexpr int H = op_half(L), RW = op_row(L);
        const int par = k & 1;                      // columns m = par + 2 i of row k
        double tv[RW];                              // bi = tv[0, H), block b at tv[(b + 1) H ...]
        if (kact) {
            // rows start on even doubles: 16-byte loads
            const double2* row = reinterpret_cast<const double2*>(A.optab + ((size_t)cl * L + k) * RW);
#pragma unroll
            for (int i = 0; i < RW / 2; ++i) {
                const double2 v = __ldg(row + i);
                tv[2 * i] = v.x;
                tv[2 * i + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < RW; ++i) tv[i] = 0;
        }
        // ---------------- inverse B (f needs the team's N_f)
        stg[wid][0][tm][k] = nf;
        __syncwarp();
        const double2 bt = nt * 2.0;
        double2 bf = make_double2(0, 0);
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const double2 v = stg[wid][0][tm][par + 2 * i]; // past L - 1: a zero slot and a zero entry
            bf = make_double2(bf.x + tv[i] * v.x, bf.y + tv[i] * v.y);
        }
        const double2 bg = (q2d != 0.0) ? ng * ((-2.0) * pr / q2d) : make_double2(0, 0);
        // ---------------- AB2 and history
        if (kact) {
            if (!mirror) {
                ut = make_double2(fma(bt.x, a1, ut.x), fma(bt.y, a1, ut.y));
                uf = make_double2(fma(bf.x, a1, uf.x), fma(bf.y, a1, uf.y));
                ug = make_double2(fma(bg.x, a1, ug.x), fma(bg.y, a1, ug.y));
                if (!A.first) {
                    ut = make_double2(fma(ht.x, a2, ut.x), fma(ht.y, a2, ut.y));
                    uf = make_double2(fma(hf.x, a2, uf.x), fma(hf.y, a2, uf.y));
                    ug = make_double2(fma(hg.x, a2, ug.x), fma(hg.y, a2, ug.y));
                }
            }
            A.hist[(0 * L + k) * plane + o] = bt;
            A.hist[(1 * L + k) * plane + o] = bf;
            A.hist[(2 * L + k) * plane + o] = bg;
        }
        // ---------------- implicit solve
        __syncwarp();
        stg[wid][0][tm][k] = ut;
        stg[wid][1][tm][k] = uf;
        __syncwarp();
        double2 to = make_double2(0, 0), fo = to;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const int m = par + 2 * i;
            const double2 vt = stg[wid][0][tm][m], vf = stg[wid][1][tm][m];
            const double m0 = tv[H + i], m1 = tv[2 * H + i], m2 = tv[3 * H + i], m3 = tv[4 * H + i];
            to = make_double2(to.x + (m0 * vt.x + m1 * vf.x), to.y + (m0 * vt.y + m1 * vf.y));
            fo = make_double2(fo.x + (m2 * vt.x + m3 * vf.x), fo.y + (m2 * vt.y + m3 * vf.y));
        }
        double2 go = (q2d != 0.0) ? ug * (1.0 / (1.0 + dt * pr * (q2d + mpi * mpi))) : make_double2(0, 0);
        if (c == 0 && r == 0) { to.y = 0; fo.y = 0; go.y = 0; }
        if (kact && !mirror) {
            A.th[k * plane + o] = to;
            A.f[k * plane + o] = fo;
            A.g[k * plane + o] = go;
            if (c == 0 && r > ny / 2) {
                const size_t om = (size_t)(ny - r);
                A.th[k * plane + om] = cconj(to);
                A.f[k * plane + om] = cconj(fo);
                A.g[k * plane + om] = cconj(go);
            }
            if (!isfinite(to.x + to.y + fo.x + fo.y + go.x + go.y)) atomicOr(A.err, RBC_DEVERR_NAN);
        }
        // ---------------- diagnostics: Parseval over the full spectrum; columns c > 0
        // stand for +-kx (weight 2), the kx = 0 team of row Ny - r also for row r.
        __syncwarp();
        stg[wid][0][tm][k] = to;
        stg[wid][1][tm][k] = fo;
        __syncwarp();
        if (kact && !mirror) {
            const double wq = (c > 0 || r > ny / 2) ? 2.0 : 1.0;
            const double qx = 2 * kPi * c / G.lx, qy = 2 * kPi * ry / G.ly, q2 = qx * qx + qy * qy;
            double eff = 0, ecc = 0, wt = 0;
#pragma unroll
            for (int i = 0; i < H; ++i) {
                const int j = par + 2 * i;
                if (j >= L) break;
                const double2 tj = stg[wid][0][tm][j], fj = stg[wid][1][tm][j];
                const double ff = fo.x * fj.x + fo.y * fj.y;
                eff += __ldg(dtab + k + j * L) * ff;
                ecc += __ldg(dtab + L * L + k + j * L) * ff;
                wt += __ldg(dtab + 2 * L * L + k + j * L) * (fo.x * tj.x + fo.y * tj.y);
            }
            const double egg = go.x * go.x + go.y * go.y;
            esum += wq * (q2 * eff + 0.5 * q2 * egg + q2 * q2 * ecc);
            wsum += wq * q2 * wt;
            if (c == 0 && r == 0) {
                const double fac = 1.0 / (1.0 + dt * pr * mpi * mpi);
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const double b = 2.0 * pr * ld_cg(A.NFG + s * L + k);
                    double2 u = ld_cg(A.FG + s * L + k);
                    u.x = fma(b, a1, u.x);
                    if (!A.first) u.x = fma(ld_cg(A.hFG + s * L + k).x, a2, u.x);
                    A.hFG[s * L + k] = make_double2(b, 0.0);
                    u = make_double2(fac * u.x, 0.0);
                    A.FG[s * L + k] = u;
                    esum += 0.5 * u.x * u.x;
                }
                A.th00[k] = to.x;
            }
        }
    }
    // deterministic two-level reduction: block partials, then the last block
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        esum += __shfl_down_sync(0xffffffffu, esum, s);
        wsum += __shfl_down_sync(0xffffffffu, wsum, s);
    }
    __shared__ double red[2][kThreads / 32];
    if (lane == 0) { red[0][wid] = esum; red[1][wid] = wsum; }
    __syncthreads();
    if (wid != 0) return; // warp 0 publishes the block partial and, in the last block, reduces
    bool last = false;
    if (lane == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) { a += red[0][w]; b += red[1][w]; }
        A.partial[2 * blockIdx.x] = a;
        A.partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        last = atomicAdd(A.ticket, 1u) == gridDim.x - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    // fixed partition (lane l sums blocks l, l + 32, ...) and a fixed shuffle tree:
    // the result does not depend on the order in which blocks finished. The partials are
    // read through L2 (the fence above orders them after the other blocks' writes), eight
    // loads in flight per lane before they are added in that order.
    double a = 0, b = 0;
    const int nb = (int)gridDim.x;
    for (int i0 = lane; i0 < nb; i0 += 32 * 8) {
        double pa[8], pb[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int i = i0 + 32 * j;
            pa[j] = i < nb ? ld_cg(A.partial + 2 * i) : 0.0;
            pb[j] = i < nb ? ld_cg(A.partial + 2 * i + 1) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (i0 + 32 * j < nb) {
                a += pa[j];
                b += pb[j];
            }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, s);
        b += __shfl_down_sync(0xffffffffu, b, s);
    }
    if (lane == 0) {
        double t00[L];
#pragma unroll
        for (int kk = 0; kk < L; ++kk) t00[kk] = ld_cg(A.th00 + kk);
        double nuw = 1.0;
#pragma unroll
        for (int kk = 0; kk < L; ++kk) nuw -= (kk + 1) * kPi * t00[kk];
        const long long s = *A.step_counter + 1;
        *A.step_counter = s;
        double* slot = A.ring + 4 * (size_t)((s - 1) % A.ring_cap);
        slot[0] = nuw;
        slot[1] = 1.0 + b;
        slot[2] = 0.5 * a;
        slot[3] = (double)s;
        // the newest entry again, after the ring: one read gives the latest diagnostics
        double* last = A.ring + 4 * (size_t)A.ring_cap;
        last[0] = nuw;
        last[1] = 1.0 + b;
        last[2] = 0.5 * a;
        last[3] = (double)s;
        *A.ticket = 0u;
    }
}

// One team per kept wavenumber (ckeep columns x nkr kept rows).
template <int L> inline int update_blocks(int ckeep, int nkr)
{
    const long long threads = (long long)ckeep * nkr * TeamSize<L>::value;
    return (int)((threads + kThreads - 1) / kThreads);
}

} // namespace rbck
