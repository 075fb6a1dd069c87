// update_kernel.cuh -- fused per-wavenumber update of the IMEX step (sm_100a, FP64).
//
// One thread per kept wavenumber (c, r) does, for all vertical modes at once:
//   inverse B        (inverse_B_matrix.cu:199-328): theta x2, f by the L x L B_ff^-1 of
//                    its q^2 class, g x (-2 Pr / q^2) (0 at q = 0), F, G x 2 Pr (Im = 0)
//   AB2 / Euler      (implicit_explicit_stepping.cu:43-69): u += 1.5dt r - 0.5dt r_prev
//   implicit solve   (linear_implicit_operator.cu:350-490): [theta; f] <- M(q)[theta; f],
//                    g / (1 + dt Pr (q^2 + (m pi)^2)), F, G / (1 + dt Pr (m pi)^2)
//   make_real        (util.cu:184-209) on the kx = 0 column: the thread of row Ny - r
//                    also writes conj() into row r, rows 0 get Im = 0
//   diagnostics      Nu_wall, Nu_vol, KE of the new state by Parseval (spectral, exact)
// The dealiased band is never touched: it stays zero.
#pragma once
#include "common.cuh"
#include "step_kernels.cuh"

namespace rbck {

struct UpdateArgs {
    Geom G;
    const int* cls;            // CM [ckp][Ny] q^2 class (-1: not kept)
    const double* binv;        // [nclass][L*L]
    const double* imp;         // [nclass][4][L*L]
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
    double* ring;              // [cap][4] = nu_wall, nu_vol, ke, step
    int ring_cap;
    long long* step_counter;
    int* err;
};

template <typename R, int L>
__global__ void __launch_bounds__(kThreads) k_update(UpdateArgs A)
{
    typedef typename cplx_t<R>::type C;
    const Geom& G = A.G;
    const int ny = G.ny;
    const size_t plane = (size_t)G.ckp * ny;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = e / ny, r = e - c * ny;
    double esum = 0.0, wsum = 0.0;
    const C* Nc = reinterpret_cast<const C*>(A.N);
    const int cl = (c < G.ckeep) ? A.cls[e] : -1;
    if (cl >= 0) {
        const size_t o = e; // (c, r) offset inside one CM plane
        const int ry = wrap_row(r, ny);
        const double mx = (kPi + kPi) * (c / G.lx), my = (kPi + kPi) * (ry / G.ly);
        const double q2d = mx * mx + my * my;       // device formula of the reference kernels
        const bool mirror = (c == 0 && r > 0 && r < ny / 2);
        const double dt = G.dt, pr = G.pr;
        const double a1 = A.first ? dt : 1.5 * dt, a2 = -0.5 * dt;
        // ---------------- g: independent per mode
        double2 gn[L];
#pragma unroll
        for (int k = 0; k < L; ++k) {
            const C nv = Nc[(2 * L + k) * plane + o];
            double2 b = make_double2(0, 0);
            if (q2d != 0.0) b = make_double2(nv.x, nv.y) * ((-2.0) * pr / q2d);
            double2* hp = A.hist + (2 * L + k) * plane + o;
            if (!mirror) {
                double2 u = A.g[k * plane + o];
                if (A.first) u = make_double2(fma(b.x, a1, u.x), fma(b.y, a1, u.y));
                else {
                    const double2 h = *hp;
                    u = make_double2(fma(b.x, a1, u.x), fma(b.y, a1, u.y));
                    u = make_double2(fma(h.x, a2, u.x), fma(h.y, a2, u.y));
                }
                const double mpi = (k + 1) * kPi;
                const double fac = q2d != 0.0 ? 1.0 / (1.0 + dt * pr * (q2d + mpi * mpi)) : 0.0;
                gn[k] = q2d != 0.0 ? u * fac : make_double2(0, 0);
            }
            *hp = b;
        }
        // ---------------- theta, f
        double2 bt[L], bf[L];
        {
            double2 nf[L];
#pragma unroll
            for (int k = 0; k < L; ++k) {
                const C nt = Nc[(0 * L + k) * plane + o];
                const C nfk = Nc[(1 * L + k) * plane + o];
                bt[k] = make_double2(nt.x, nt.y) * 2.0;
                nf[k] = make_double2(nfk.x, nfk.y);
            }
            const double* bi = A.binv + (size_t)cl * L * L;
#pragma unroll
            for (int k = 0; k < L; ++k) {
                double2 s = make_double2(0, 0);
#pragma unroll
                for (int m = 0; m < L; ++m) {
                    const double op = bi[k * L + m];
                    s = make_double2(s.x + op * nf[m].x, s.y + op * nf[m].y);
                }
                bf[k] = s;
            }
        }
        double2 tn[L], fn[L];
        if (!mirror) {
#pragma unroll
            for (int k = 0; k < L; ++k) {
                double2 ut = A.th[k * plane + o], uf = A.f[k * plane + o];
                ut = make_double2(fma(bt[k].x, a1, ut.x), fma(bt[k].y, a1, ut.y));
                uf = make_double2(fma(bf[k].x, a1, uf.x), fma(bf[k].y, a1, uf.y));
                if (!A.first) {
                    const double2 ht = A.hist[(0 * L + k) * plane + o], hf = A.hist[(1 * L + k) * plane + o];
                    ut = make_double2(fma(ht.x, a2, ut.x), fma(ht.y, a2, ut.y));
                    uf = make_double2(fma(hf.x, a2, uf.x), fma(hf.y, a2, uf.y));
                }
                tn[k] = ut;
                fn[k] = uf;
            }
        }
#pragma unroll
        for (int k = 0; k < L; ++k) {
            A.hist[(0 * L + k) * plane + o] = bt[k];
            A.hist[(1 * L + k) * plane + o] = bf[k];
        }
        if (!mirror) {
            const double* M = A.imp + (size_t)cl * 4 * L * L;
            double2 to[L], fo[L];
#pragma unroll
            for (int k = 0; k < L; ++k) {
                double2 st = make_double2(0, 0), sf = make_double2(0, 0);
#pragma unroll
                for (int m = 0; m < L; ++m) {
                    const double tt = M[k * L + m], tf = M[L * L + k * L + m];
                    const double ft = M[2 * L * L + k * L + m], ff = M[3 * L * L + k * L + m];
                    st = make_double2(st.x + (tt * tn[m].x + tf * fn[m].x), st.y + (tt * tn[m].y + tf * fn[m].y));
                    sf = make_double2(sf.x + (ft * tn[m].x + ff * fn[m].x), sf.y + (ft * tn[m].y + ff * fn[m].y));
                }
                to[k] = st;
                fo[k] = sf;
            }
            if (c == 0 && r == 0) {
#pragma unroll
                for (int k = 0; k < L; ++k) { to[k].y = 0; fo[k].y = 0; gn[k].y = 0; }
            }
            bool bad = false;
#pragma unroll
            for (int k = 0; k < L; ++k) {
                A.th[k * plane + o] = to[k];
                A.f[k * plane + o] = fo[k];
                A.g[k * plane + o] = gn[k];
                bad |= !isfinite(to[k].x + to[k].y + fo[k].x + fo[k].y + gn[k].x + gn[k].y);
            }
            if (c == 0 && r > ny / 2) {
                const size_t om = (size_t)(ny - r);
#pragma unroll
                for (int k = 0; k < L; ++k) {
                    A.th[k * plane + om] = cconj(to[k]);
                    A.f[k * plane + om] = cconj(fo[k]);
                    A.g[k * plane + om] = cconj(gn[k]);
                }
            }
            if (bad) atomicOr(A.err, RBC_DEVERR_NAN);
            // Parseval over the full spectrum: columns c > 0 stand for +-kx (weight 2);
            // the kx = 0 thread of row Ny - r also stands for its mirror row r.
            const double wq = (c > 0 || r > ny / 2) ? 2.0 : 1.0;
            const double qx = 2 * kPi * c / G.lx, qy = 2 * kPi * ry / G.ly, q2 = qx * qx + qy * qy;
            const double* CpCp = A.diag_tab;
            const double* CC = A.diag_tab + L * L;
            const double* CS = A.diag_tab + 2 * L * L;
            double eff = 0, ecc = 0, egg = 0, wt = 0;
#pragma unroll
            for (int i = 0; i < L; ++i) {
                egg += gn[i].x * gn[i].x + gn[i].y * gn[i].y;
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    const double ff = fo[i].x * fo[j].x + fo[i].y * fo[j].y;
                    eff += CpCp[i + j * L] * ff;
                    ecc += CC[i + j * L] * ff;
                    wt += CS[i + j * L] * (fo[i].x * to[j].x + fo[i].y * to[j].y);
                }
            }
            esum = wq * (q2 * eff + 0.5 * q2 * egg + q2 * q2 * ecc);
            wsum = wq * q2 * wt;
            if (c == 0 && r == 0) {
                // mean flow F, G and the q = 0 temperature
                const double* nfg = A.NFG;
                double eFG = 0;
#pragma unroll
                for (int k = 0; k < L; ++k) {
                    const double mpi = (k + 1) * kPi;
                    const double fac = 1.0 / (1.0 + dt * pr * mpi * mpi);
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const double b = 2.0 * pr * nfg[s * L + k];
                        double2 u = A.FG[s * L + k];
                        u.x = fma(b, a1, u.x);
                        if (!A.first) u.x = fma(A.hFG[s * L + k].x, a2, u.x);
                        A.hFG[s * L + k] = make_double2(b, 0.0);
                        u = make_double2(fac * u.x, 0.0);
                        A.FG[s * L + k] = u;
                        eFG += 0.5 * u.x * u.x;
                    }
                    A.th00[k] = to[k].x;
                }
                esum += eFG;
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
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { red[0][wid] = esum; red[1][wid] = wsum; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) { a += red[0][w]; b += red[1][w]; }
        A.partial[2 * blockIdx.x] = a;
        A.partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        const unsigned int t = atomicAdd(A.ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double a = 0, b = 0;
        for (int i = 0; i < (int)gridDim.x; ++i) {
            a += ((volatile double*)A.partial)[2 * i];
            b += ((volatile double*)A.partial)[2 * i + 1];
        }
        double nuw = 1.0;
        for (int k = 0; k < L; ++k) nuw -= (k + 1) * kPi * ((volatile double*)A.th00)[k];
        const long long s = *A.step_counter + 1;
        *A.step_counter = s;
        double* slot = A.ring + 4 * (size_t)((s - 1) % A.ring_cap);
        slot[0] = nuw;
        slot[1] = 1.0 + b;
        slot[2] = 0.5 * a;
        slot[3] = (double)s;
        *A.ticket = 0u;
    }
}

} // namespace rbck
