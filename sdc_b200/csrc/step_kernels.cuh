// step_kernels.cuh -- sm_100a kernels of the Boussinesq RBC IMEX step.
//
// Internal HBM layout. Spectral arrays are column-major "CM": [plane][c][y] with the
// y (ky) index fastest and a column stride ckp >= Nx/2+1 (padded to the column block W);
// the reference layout [L][Ny][Nx/2+1] (matrix_device.h) is used only at the C ABI.
// A step only works on the columns c < ckeep kept by the 2/3 rule (ckw = ckeep padded
// to W); those columns' removed rows and all other columns are identically zero after
// every step (dealias_implicit, implicit_explicit_stepping.cu:163). The standalone
// nonlinear operator runs the analysis kernels with ckeep = Nx/2+1 to return every mode.
//   state theta, f, g   CM [L][ckp][Ny] double2,  F, G  [2][L] double2
//   AB2 history          CM [3][L][ckp][Ny] double2 + [2][L] double2
//   H    synthesis after the y pass      CM [8][L][ckp][Ny]  C
//   phys synthesised fields              [8][L][Ny][Nx]      R  (row-major)
//   grp  contracted groups               [13][L][Ny][Nx]     R
//   gh   groups after the x pass         CM [13][L][ckp][Ny] C
//   N    nonlinear term, scaled          CM [3][L][ckp][Ny]  C,   NFG [2][L] double
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace rbck {

constexpr double kPi = 3.14159265358979323846;
constexpr int kThreads = 256;
constexpr int kMaxB = 4; // butterflies per thread per FFT pass

RBC_HD int wrap_row(int r, int ny) { return r > ny / 2 ? r - ny : r; }
RBC_HD bool row_kept(int r, int ny) { return !(fabs(0.5 * ny - r) <= (1.0 / 3.0) * 0.5 * ny); }

// Transforms of length n processed per FFT call so that nb * n / 2 <= kMaxB * kThreads.
RBC_HD int fft_chunk(int n) { int c = (kMaxB * kThreads * 2) / n; return c < 1 ? 1 : c; }

template <typename R>
RBC_D void load_twiddles(typename cplx_t<R>::type* tw, const double2* twg, int n)
{
    typedef typename cplx_t<R>::type C;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = cmk<C>(twg[t].x, twg[t].y);
}

template <typename R>
RBC_D void fft_batched(typename cplx_t<R>::type* buf, const rbcfft::Plan& p, int nb,
                       const typename cplx_t<R>::type* tw, int sign)
{
    const int ch = fft_chunk(p.n);
    for (int b0 = 0; b0 < nb; b0 += ch) {
        const int cnt = nb - b0 < ch ? nb - b0 : ch;
        rbcfft::run<kMaxB, R>(buf + b0 * p.n, p, cnt, tw, sign);
    }
}

struct Geom {
    int nx, ny, mox, L, ckeep, ckw, ckp, P;
    double lx, ly, pr, dt;
};

// Spectral derivative factors with the reference's formulas (nonlinear operator
// derivative kernels, nonlinear_operator_rayleigh_noslip.cu:1428-1583).
struct Mult {
    double fx, fy, lap, xy;
    RBC_HD Mult(int c, int r, const Geom& G)
    {
        const int ry = wrap_row(r, G.ny);
        fx = c * (2 * kPi / G.lx);
        fy = ry * (2 * kPi / G.ly);
        const double a = c / G.lx, b = ry / G.ly;
        lap = (-4 * kPi * kPi) * (a * a + b * b);
        xy = -4 * kPi * kPi * (c * ry) / (G.lx * G.ly);
    }
};

// ---------------------------------------------------------------------------------
// K1: spectral multipliers and inverse y transform of the 8 synthesis fields.
// Grid (ckw / W, L); one CTA = W adjacent columns of one vertical mode k.
// Reference: nonlinear_operator_rayleigh_noslip.cu:112-233 (u11 = d_x f, u21 = d_y f,
// u31 = q^2 f, u12 = d_y g + F, u22 = -d_x g + G, theta, d_x theta, d_y theta).
template <typename R>
__global__ void __launch_bounds__(kThreads) k_synth_columns(
    Geom G, int W, rbcfft::Plan py, const double2* __restrict__ twy, const double2* __restrict__ th,
    const double2* __restrict__ f, const double2* __restrict__ g, const double2* __restrict__ FG,
    typename cplx_t<R>::type* __restrict__ H)
{
    typedef typename cplx_t<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + G.ny;
    const int k = blockIdx.y;
    const int c0 = blockIdx.x * W;
    load_twiddles<R>(tw, twy, G.ny);
    const size_t base = ((size_t)k * G.ckp + c0) * G.ny;
    for (int e = threadIdx.x; e < W * G.ny; e += blockDim.x) {
        const int cc = e / G.ny, r = e - cc * G.ny, c = c0 + cc;
        double2 vt = make_double2(0, 0), vf = vt, vg = vt;
        if (c < G.ckeep && row_kept(r, G.ny)) {
            vt = th[base + e];
            vf = f[base + e];
            vg = g[base + e];
        }
        const Mult m(c, r, G);
        double2 u12 = cmul_is<double2, double>(vg, m.fy);
        double2 u22 = cmul_is<double2, double>(vg, m.fx) * (-1.0);
        if (c == 0 && r == 0) {
            u12 = u12 + FG[k];
            u22 = u22 + FG[G.L + k];
        }
        const double2 vals[8] = {cmul_is<double2, double>(vf, m.fx), cmul_is<double2, double>(vf, m.fy),
                                 vf * (-m.lap), u12, u22, vt,
                                 cmul_is<double2, double>(vt, m.fx), cmul_is<double2, double>(vt, m.fy)};
#pragma unroll
        for (int fld = 0; fld < 8; ++fld) buf[(fld * W + cc) * G.ny + r] = cmk<C>(vals[fld].x, vals[fld].y);
    }
    __syncthreads();
    fft_batched<R>(buf, py, 8 * W, tw, +1);
    for (int e = threadIdx.x; e < 8 * W * G.ny; e += blockDim.x) {
        const int fld = e / (W * G.ny);
        const int rem = e - fld * W * G.ny;
        H[(((size_t)fld * G.L + k) * G.ckp + c0) * G.ny + rem] = buf[fld * W * G.ny + rem];
    }
}

// ---------------------------------------------------------------------------------
// K2: inverse x transform (C2R) of pairs of rows y, y+1 of one plane:
// z = IFFT(A + iB) with the Hermitian extension, a = Re z, b = Im z. The imaginary
// parts of the DC entries are dropped, as a C2R does. NP pairs per CTA, all in one
// plane (NP divides Ny/2).
template <typename R>
__global__ void __launch_bounds__(kThreads) k_rows_c2r(
    Geom G, int NP, rbcfft::Plan px, const double2* __restrict__ twx,
    const typename cplx_t<R>::type* __restrict__ H, R* __restrict__ phys)
{
    typedef typename cplx_t<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + G.nx;
    load_twiddles<R>(tw, twx, G.nx);
    const int nx = G.nx;
    const int row0 = 2 * NP * blockIdx.x;           // first row (plane * Ny + y)
    const int plane = row0 / G.ny, y0 = row0 - plane * G.ny;
    for (int e = threadIdx.x; e < NP * nx; e += blockDim.x) {
        const int pp = e / nx, n = e - pp * nx;
        if (n >= G.ckeep && n <= nx - G.ckeep) buf[pp * nx + n] = cmk<C>(0, 0);
    }
    const C* src = H + (size_t)plane * G.ckp * G.ny + y0;
    for (int e = threadIdx.x; e < NP * G.ckeep; e += blockDim.x) {
        const int n = e / NP, pp = e - n * NP;
        C A = src[(size_t)n * G.ny + 2 * pp], B = src[(size_t)n * G.ny + 2 * pp + 1];
        if (n == 0) { A.y = 0; B.y = 0; }
        C z; z.x = A.x - B.y; z.y = A.y + B.x;       // A + iB
        buf[pp * nx + n] = z;
        if (n > 0) {
            C zm; zm.x = A.x + B.y; zm.y = B.x - A.y; // conj(A) + i conj(B)
            buf[pp * nx + nx - n] = zm;
        }
    }
    __syncthreads();
    fft_batched<R>(buf, px, NP, tw, +1);
    R* dst = phys + (size_t)row0 * nx;
    for (int e = threadIdx.x; e < NP * nx; e += blockDim.x) {
        const int pp = e / nx, x = e - pp * nx;
        const C z = buf[pp * nx + x];
        dst[(size_t)(2 * pp) * nx + x] = z.x;
        dst[(size_t)(2 * pp + 1) * nx + x] = z.y;
    }
}

// ---------------------------------------------------------------------------------
// K4: forward x transform (R2C) of pairs of rows: Z = FFT(a + ib),
// A[n] = (Z[n] + conj Z[-n]) / 2, B[n] = (Z[n] - conj Z[-n]) / 2i, columns n < ckw
// (zero for n >= ckeep). Output CM.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_rows_r2c(
    Geom G, int NP, rbcfft::Plan px, const double2* __restrict__ twx,
    const R* __restrict__ grp, typename cplx_t<R>::type* __restrict__ gh)
{
    typedef typename cplx_t<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + G.nx;
    load_twiddles<R>(tw, twx, G.nx);
    const int nx = G.nx;
    const int row0 = 2 * NP * blockIdx.x;
    const int plane = row0 / G.ny, y0 = row0 - plane * G.ny;
    const R* src = grp + (size_t)row0 * nx;
    for (int e = threadIdx.x; e < NP * nx; e += blockDim.x) {
        const int pp = e / nx, x = e - pp * nx;
        buf[pp * nx + x] = cmk<C>(src[(size_t)(2 * pp) * nx + x], src[(size_t)(2 * pp + 1) * nx + x]);
    }
    __syncthreads();
    fft_batched<R>(buf, px, NP, tw, -1);
    const R half = (R)0.5;
    C* dst = gh + (size_t)plane * G.ckp * G.ny + y0;
    for (int e = threadIdx.x; e < NP * G.ckw; e += blockDim.x) {
        const int n = e / NP, pp = e - n * NP;
        C A = cmk<C>(0, 0), B = A;
        if (n < G.ckeep) {
            const C z = buf[pp * nx + n];
            const C zm = buf[pp * nx + (n == 0 ? 0 : nx - n)];
            A.x = half * (z.x + zm.x);
            A.y = half * (z.y - zm.y);
            B.x = half * (z.y + zm.y);
            B.y = half * (zm.x - z.x);
        }
        dst[(size_t)n * G.ny + 2 * pp] = A;
        dst[(size_t)n * G.ny + 2 * pp + 1] = B;
    }
}

// ---------------------------------------------------------------------------------
// K5: forward y transform of the 13 group planes of one mode k and W columns, the
// derivative multiplier of each group, and the reference's final scaling
// (nonlinear_operator_rayleigh_noslip.cu:1366-1370) with the 1/P of its products:
//   N_theta = -(1/P) sum,  N_f = N_g = -(1/(Pr P)) sum.
// F_k and G_k (reference :950-1003) are the q = 0 entries of the g-y group and of
// the negated g-x group, scaled like f.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_columns_combine(
    Geom G, int W, rbcfft::Plan py, const double2* __restrict__ twy,
    const typename cplx_t<R>::type* __restrict__ gh, typename cplx_t<R>::type* __restrict__ N,
    double* __restrict__ NFG)
{
    typedef typename cplx_t<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + G.ny;
    const int k = blockIdx.y;
    const int c0 = blockIdx.x * W;
    load_twiddles<R>(tw, twy, G.ny);
    const int nel = W * G.ny;
    // accumulators of theta, f, g for this tile (each element owned by one thread)
    double2* acc = reinterpret_cast<double2*>(buf + nel);
    for (int e = threadIdx.x; e < 3 * nel; e += blockDim.x) acc[e] = make_double2(0, 0);
    const double invP = 1.0 / ((double)G.nx * G.ny);
    for (int grpi = 0; grpi < 13; ++grpi) {
        const C* src = gh + (((size_t)grpi * G.L + k) * G.ckp + c0) * G.ny;
        __syncthreads();
        for (int e = threadIdx.x; e < nel; e += blockDim.x) buf[e] = src[e];
        __syncthreads();
        fft_batched<R>(buf, py, W, tw, -1);
        double2* at = acc + (grpi < 8 ? 1 : (grpi < 12 ? 2 : 0)) * nel;
        for (int e = threadIdx.x; e < nel; e += blockDim.x) {
            const int cc = e / G.ny, r = e - cc * G.ny, c = c0 + cc;
            const C zv = buf[e];
            const double2 v = make_double2(zv.x, zv.y);
            if (c == 0 && r == 0) {
                if (grpi == 10) NFG[k] = v.x * (-invP / G.pr);           // F
                if (grpi == 11) NFG[G.L + k] = -v.x * (-invP / G.pr);    // G
            }
            const Mult m(c, r, G);
            double2 o;
            switch (grpi) {
            case 0: o = v * (-(m.fx * m.fx)); break;                          // f: xx
            case 1: o = v * m.xy; break;                                      // f: xy
            case 2: o = v * (-(m.fy * m.fy)); break;                          // f: yy
            case 3: o = cmul_is<double2, double>(v, m.fx); break;             // f: x
            case 4: o = cmul_is<double2, double>(v, m.fy); break;             // f: y
            case 5: o = cmul_is<double2, double>(v, m.fx) * m.lap; break;     // f: lap o x
            case 6: o = cmul_is<double2, double>(v, m.fy) * m.lap; break;     // f: lap o y
            case 7: o = v * m.lap; break;                                     // f: lap
            case 8: o = v * m.xy; break;                                      // g: xy
            case 9: o = v * ((m.fx * m.fx) - (m.fy * m.fy)); break;           // g: yy - xx
            case 10: o = cmul_is<double2, double>(v, m.fy); break;            // g: y
            case 11: o = cmul_is<double2, double>(v, m.fx); break;            // g: x
            default: o = v; break;                                            // theta
            }
            at[e] = at[e] + o;
        }
    }
    const double sc[3] = {-invP, -invP / G.pr, -invP / G.pr};
    for (int a = 0; a < 3; ++a) {
        C* dst = N + (((size_t)a * G.L + k) * G.ckp + c0) * G.ny;
        for (int e = threadIdx.x; e < nel; e += blockDim.x) {
            const double2 v = acc[a * nel + e] * sc[a];
            dst[e] = cmk<C>(v.x, v.y);
        }
    }
}

} // namespace rbck
