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
#include "fft2p.cuh"

namespace rbck {

constexpr double kPi = 3.14159265358979323846;
constexpr int kThreads = rbcfft::kPlanThreads;

RBC_HD int wrap_row(int r, int ny) { return r > ny / 2 ? r - ny : r; }
RBC_HD bool row_kept(int r, int ny) { return !(fabs(0.5 * ny - r) <= (1.0 / 3.0) * 0.5 * ny); }


template <typename R>
RBC_D void load_twiddles(typename cplx_t<R>::type* tw, const double2* twg, int n)
{
    typedef typename cplx_t<R>::type C;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = cmk<C>(twg[t].x, twg[t].y);
}

// The same table copy issued asynchronously where no conversion is needed (FP64): it
// completes at the kernel's next cp_async_wait_all(), so its latency overlaps the data loads
// that follow (and the predecessor's tail under programmatic launch).
template <typename R>
RBC_D void load_twiddles_async(typename cplx_t<R>::type* tw, const double2* twg, int n)
{
    if constexpr (sizeof(typename cplx_t<R>::type) == sizeof(double2)) {
        for (int t = threadIdx.x; t < n; t += blockDim.x) cp_async<sizeof(double2)>(tw + t, twg + t);
    } else {
        load_twiddles<R>(tw, twg, n);
    }
}

template <typename R>
RBC_D void fft_batched(typename cplx_t<R>::type* buf, const rbcfft::Plan& p, int nb,
                       const typename cplx_t<R>::type* tw, int sign)
{
    const int ch = p.chunk;
    for (int b0 = 0; b0 < nb; b0 += ch) {
        const int cnt = nb - b0 < ch ? nb - b0 : ch;
        rbcfft::run<R>(buf + b0 * p.stride, p, cnt, tw, sign);
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
__global__ void __launch_bounds__(kThreads, 2) k_synth_columns(
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
    const int st = py.stride;
    pdl_trigger();
    load_twiddles<R>(tw, twy, G.ny);
    pdl_wait(); // the state is complete (K1 is a dependent launch inside multi-step graphs)
    const size_t base = ((size_t)k * G.ckp + c0) * G.ny;
    constexpr bool kStage = sizeof(C) == sizeof(double2);
    if constexpr (kStage) {
        // FP64: theta, f and g land in the slots of fields 5, 0 and 3 of their own
        // (column, row); the same thread reads them back below, so no barrier is needed.
        for (int e = threadIdx.x; e < W * G.ny; e += blockDim.x) {
            const int cc = e / G.ny, r = e - cc * G.ny, c = c0 + cc;
            if (c < G.ckeep && row_kept(r, G.ny)) {
                copy_cg<16>(buf + (5 * W + cc) * st + rbcfft::pad(r), th + base + e);
                copy_cg<16>(buf + (0 * W + cc) * st + rbcfft::pad(r), f + base + e);
                copy_cg<16>(buf + (3 * W + cc) * st + rbcfft::pad(r), g + base + e);
            }
        }
        cp_async_wait_all();
    }
    for (int e = threadIdx.x; e < W * G.ny; e += blockDim.x) {
        const int cc = e / G.ny, r = e - cc * G.ny, c = c0 + cc;
        double2 vt = make_double2(0, 0), vf = vt, vg = vt;
        if (c < G.ckeep && row_kept(r, G.ny)) {
            if constexpr (kStage) {
                const C a = buf[(5 * W + cc) * st + rbcfft::pad(r)], b = buf[(0 * W + cc) * st + rbcfft::pad(r)],
                        d = buf[(3 * W + cc) * st + rbcfft::pad(r)];
                vt = make_double2(a.x, a.y);
                vf = make_double2(b.x, b.y);
                vg = make_double2(d.x, d.y);
            } else {
                vt = ld_cg(th + base + e);
                vf = ld_cg(f + base + e);
                vg = ld_cg(g + base + e);
            }
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
        for (int fld = 0; fld < 8; ++fld) buf[(fld * W + cc) * st + rbcfft::pad(r)] = cmk<C>(vals[fld].x, vals[fld].y);
    }
    __syncthreads();
    fft_batched<R>(buf, py, 8 * W, tw, +1);
    for (int e = threadIdx.x; e < 8 * W * G.ny; e += blockDim.x) {
        const int fld = e / (W * G.ny);
        const int rem = e - fld * W * G.ny;
        const int cc = rem / G.ny, r = rem - cc * G.ny;
        H[(((size_t)fld * G.L + k) * G.ckp + c0) * G.ny + rem] = buf[(fld * W + cc) * st + rbcfft::pad(r)];
    }
}

// ---------------------------------------------------------------------------------
// K2: inverse x transform (C2R) of pairs of rows y, y+1 of one plane:
// z = IFFT(A + iB) with the Hermitian extension, a = Re z, b = Im z. The imaginary
// parts of the DC entries are dropped, as a C2R does. NP pairs per CTA, all in one
// plane (NP divides Ny/2).
template <typename R>
__global__ void __launch_bounds__(kThreads, 2) k_rows_c2r(
    Geom G, int NP, rbcfft::Plan px, const double2* __restrict__ twx,
    const typename cplx_t<R>::type* __restrict__ H, R* __restrict__ phys)
{
    typedef typename cplx_t<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + G.nx;
    pdl_trigger();
    load_twiddles<R>(tw, twx, G.nx);
    pdl_wait();
    const int nx = G.nx, st = px.stride;
    const int row0 = 2 * NP * blockIdx.x;           // first row (plane * Ny + y)
    const int plane = row0 / G.ny, y0 = row0 - plane * G.ny;
    // A[n] lands at n and B[n] at nx - n, where the Hermitian extension puts its values;
    // B[0] goes to the spare last slot of the padded row (st - 1 > pad(nx - 1)).
    const C* src = H + (size_t)plane * G.ckp * G.ny + y0;
    for (int e = threadIdx.x; e < NP * G.ckeep; e += blockDim.x) {
        const int n = e / NP, pp = e - n * NP;
        C* row = buf + pp * st;
        copy_cg<sizeof(C)>(row + rbcfft::pad(n), src + (size_t)n * G.ny + 2 * pp);
        copy_cg<sizeof(C)>(row + (n ? rbcfft::pad(nx - n) : st - 1), src + (size_t)n * G.ny + 2 * pp + 1);
    }
    for (int e = threadIdx.x; e < NP * nx; e += blockDim.x) {
        const int pp = e / nx, n = e - pp * nx;
        if (n >= G.ckeep && n <= nx - G.ckeep) buf[pp * st + rbcfft::pad(n)] = cmk<C>(0, 0);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int e = threadIdx.x; e < NP * G.ckeep; e += blockDim.x) {
        const int n = e / NP, pp = e - n * NP;
        C* row = buf + pp * st;
        C* pb = row + (n ? rbcfft::pad(nx - n) : st - 1);
        C A = row[rbcfft::pad(n)], B = *pb;
        if (n == 0) { A.y = 0; B.y = 0; }
        C z; z.x = A.x - B.y; z.y = A.y + B.x;       // A + iB
        row[rbcfft::pad(n)] = z;
        if (n > 0) {
            C zm; zm.x = A.x + B.y; zm.y = B.x - A.y; // conj(A) + i conj(B)
            *pb = zm;
        }
    }
    __syncthreads();
    fft_batched<R>(buf, px, NP, tw, +1);
    R* dst = phys + (size_t)row0 * nx;
    for (int e = threadIdx.x; e < NP * nx; e += blockDim.x) {
        const int pp = e / nx, x = e - pp * nx;
        const C z = buf[pp * st + rbcfft::pad(x)];
        dst[(size_t)(2 * pp) * nx + x] = z.x;
        dst[(size_t)(2 * pp + 1) * nx + x] = z.y;
    }
}

// ---------------------------------------------------------------------------------
// K4: forward x transform (R2C) of pairs of rows: Z = FFT(a + ib),
// A[n] = (Z[n] + conj Z[-n]) / 2, B[n] = (Z[n] - conj Z[-n]) / 2i, columns n < ckw
// (zero for n >= ckeep). Output CM.
template <typename R>
__global__ void __launch_bounds__(kThreads, 2) k_rows_r2c(
    Geom G, int NP, rbcfft::Plan px, const double2* __restrict__ twx,
    const R* __restrict__ grp, typename cplx_t<R>::type* __restrict__ gh)
{
    typedef typename cplx_t<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + G.nx;
    pdl_trigger();
    load_twiddles<R>(tw, twx, G.nx);
    pdl_wait();
    const int nx = G.nx, st = px.stride;
    const int row0 = 2 * NP * blockIdx.x;
    const int plane = row0 / G.ny, y0 = row0 - plane * G.ny;
    const R* src = grp + (size_t)row0 * nx;
    for (int e = threadIdx.x; e < NP * nx; e += blockDim.x) {
        const int pp = e / nx, x = e - pp * nx;
        R* d = reinterpret_cast<R*>(buf + pp * st + rbcfft::pad(x));
        copy_cg<sizeof(R)>(d, src + (size_t)(2 * pp) * nx + x);
        copy_cg<sizeof(R)>(d + 1, src + (size_t)(2 * pp + 1) * nx + x);
    }
    cp_async_wait_all();
    __syncthreads();
    fft_batched<R>(buf, px, NP, tw, -1);
    const R half = (R)0.5;
    C* dst = gh + (size_t)plane * G.ckp * G.ny + y0;
    for (int e = threadIdx.x; e < NP * G.ckw; e += blockDim.x) {
        const int n = e / NP, pp = e - n * NP;
        C A = cmk<C>(0, 0), B = A;
        if (n < G.ckeep) {
            const C z = buf[pp * st + rbcfft::pad(n)];
            const C zm = buf[pp * st + rbcfft::pad(n == 0 ? 0 : nx - n)];
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
// K5: forward y transform of the 13 group columns of one (column c, mode k), the
// derivative multiplier of each group, and the reference's final scaling
// (nonlinear_operator_rayleigh_noslip.cu:1366-1370) with the 1/P of its products:
//   N_theta = -(1/P) sum,  N_f = N_g = -(1/(Pr P)) sum.
// F_k and G_k (reference :950-1003) are the q = 0 entries of the g-y group and of
// the negated g-x group, scaled like f. Grid (ckw, L).
template <typename R>
__global__ void __launch_bounds__(kThreads, 2) k_columns_combine(
    Geom G, rbcfft::Plan py, const double2* __restrict__ twy,
    const typename cplx_t<R>::type* __restrict__ gh, typename cplx_t<R>::type* __restrict__ N,
    double* __restrict__ NFG)
{
    typedef typename cplx_t<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + G.ny;
    const int c = blockIdx.x, k = blockIdx.y, ny = G.ny;
    pdl_trigger();
    load_twiddles<R>(tw, twy, ny);
    pdl_wait();
    const size_t cstride = (size_t)G.L * G.ckp * ny; // between groups
    const C* src = gh + ((size_t)k * G.ckp + c) * ny;
    for (int e = threadIdx.x; e < 13 * ny; e += blockDim.x) {
        const int grpi = e / ny, r = e - grpi * ny;
        copy_cg<sizeof(C)>(buf + grpi * py.stride + rbcfft::pad(r), src + grpi * cstride + r);
    }
    cp_async_wait_all();
    __syncthreads();
    fft_batched<R>(buf, py, 13, tw, -1);
    const double invP = 1.0 / ((double)G.nx * ny);
    for (int r = threadIdx.x; r < ny; r += blockDim.x) {
        double2 v[13];
#pragma unroll
        for (int gi = 0; gi < 13; ++gi) {
            const C z = buf[gi * py.stride + rbcfft::pad(r)];
            v[gi] = make_double2(z.x, z.y);
        }
        if (c == 0 && r == 0) {
            NFG[k] = v[10].x * (-invP / G.pr);          // F: mean of the g-y group
            NFG[G.L + k] = -v[11].x * (-invP / G.pr);   // G: minus mean of the g-x group
        }
        const Mult m(c, r, G);
        const double xx = -(m.fx * m.fx), yy = -(m.fy * m.fy);
        double2 af = v[0] * xx + v[1] * m.xy + v[2] * yy + cmul_is<double2, double>(v[3], m.fx) +
                     cmul_is<double2, double>(v[4], m.fy) + cmul_is<double2, double>(v[5], m.fx) * m.lap +
                     cmul_is<double2, double>(v[6], m.fy) * m.lap + v[7] * m.lap;
        double2 ag = v[8] * m.xy + v[9] * (yy - xx) + cmul_is<double2, double>(v[10], m.fy) +
                     cmul_is<double2, double>(v[11], m.fx);
        const double2 at = v[12] * (-invP);
        af = af * (-invP / G.pr);
        ag = ag * (-invP / G.pr);
        const size_t o = ((size_t)k * G.ckp + c) * ny + r;
        const size_t pl = (size_t)G.L * G.ckp * ny;
        N[o] = cmk<C>(at.x, at.y);
        N[pl + o] = cmk<C>(af.x, af.y);
        N[2 * pl + o] = cmk<C>(ag.x, ag.y);
    }
}

// =================================================================================
// Register-FFT forms of K1, K2, K4 and K5 for the transform lengths N = 64, 128, 192, 256
// and 512 (fft2p.cuh): the CTA holds the same transforms as the Stockham forms; each transform
// is done by TL = reg_fft_lanes(N) consecutive lanes (8, 8, 16, 16, 32) holding VL = N / TL
// values each, so the block has (transforms x TL) threads. A transform's shared region has
// tp_stride(N) elements (the padded row of the Stockham forms, or the register FFT's tile
// if that is longer).
RBC_HD int tp_stride(int n)
{
    return rbcfft::padded_len(n) > rbcfft::reg_tile_len(n) ? rbcfft::padded_len(n) : rbcfft::reg_tile_len(n);
}

// Synthesis field fld (order of k_synth_columns) at (c, r) from theta, f, g.
RBC_D double2 synth_value(int fld, double2 vt, double2 vf, double2 vg, const Mult& m)
{
    switch (fld) {
    case 0: return cmul_is<double2, double>(vf, m.fx);
    case 1: return cmul_is<double2, double>(vf, m.fy);
    case 2: return vf * (-m.lap);
    case 3: return cmul_is<double2, double>(vg, m.fy);
    case 4: return cmul_is<double2, double>(vg, m.fx) * (-1.0);
    case 5: return vt;
    case 6: return cmul_is<double2, double>(vt, m.fx);
    default: return cmul_is<double2, double>(vt, m.fy);
    }
}

// K1, register FFT: grid (ckw / W, L), block 8 W TL threads (transform q = fld W + cc).
template <typename R, int N>
__global__ void __launch_bounds__(kThreads, 2) k_synth_columns_tp(
    Geom G, int W, const double2* __restrict__ twy, const double2* __restrict__ th,
    const double2* __restrict__ f, const double2* __restrict__ g, const double2* __restrict__ FG,
    typename cplx_t<R>::type* __restrict__ H)
{
    typedef typename cplx_t<R>::type C;
    constexpr int TL = rbcfft::reg_fft_lanes(N), VL = N / TL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    const int st = tp_stride(N);
    C* buf = tw + N;
    double2* stg = reinterpret_cast<double2*>(buf + 8 * W * st); // [3][W][N]: theta, f, g
    const int k = blockIdx.y;
    const int c0 = blockIdx.x * W;
    const size_t base = ((size_t)k * G.ckp + c0) * N;
    pdl_trigger();
    load_twiddles_async<R>(tw, twy, N);
    pdl_wait(); // the state is complete (K1 is a dependent launch inside multi-step graphs)
    for (int e = threadIdx.x; e < W * N; e += blockDim.x) {
        const int cc = e / N, r = e - cc * N;
        if (c0 + cc < G.ckeep && row_kept(r, N)) {
            copy_cg<16>(stg + e, th + base + e);
            copy_cg<16>(stg + W * N + e, f + base + e);
            copy_cg<16>(stg + 2 * W * N + e, g + base + e);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int q = threadIdx.x / TL, t = threadIdx.x - q * TL;
    const int fld = q / W, cc = q - fld * W, c = c0 + cc;
    // the multipliers of Mult, evaluated with the same expressions, only where a field
    // needs them (fx per column; fy and the Laplacian per row)
    const double fx = c * (2 * kPi / G.lx), ac = c / G.lx;
    const bool ckept = c < G.ckeep;
    const double2* in = stg + (fld < 3 ? W * N : fld < 5 ? 2 * W * N : 0) + cc * N; // f, g or theta
    C v[VL];
#pragma unroll
    for (int a = 0; a < VL; ++a) {
        const int r = t + TL * a;
        const double2 u = (ckept && row_kept(r, N)) ? in[r] : make_double2(0, 0);
        const int ry = wrap_row(r, N);
        double2 val;
        switch (fld) {
        case 0: case 4: case 6: val = cmul_is<double2, double>(u, fx); if (fld == 4) val = val * (-1.0); break;
        case 1: case 3: case 7: val = cmul_is<double2, double>(u, ry * (2 * kPi / G.ly)); break;
        case 2: {
            const double b = ry / G.ly;
            val = u * (-((-4 * kPi * kPi) * (ac * ac + b * b)));
            break;
        }
        default: val = u;
        }
        if (c == 0 && r == 0) {
            if (fld == 3) val = val + FG[k];
            else if (fld == 4) val = val + FG[G.L + k];
        }
        v[a] = cmk<C>(val.x, val.y);
    }
    rbcfft::reg_fft<N, R>(v, t, buf + q * st, tw, +1);
    C* dst = H + (((size_t)fld * G.L + k) * G.ckp + c) * N;
#pragma unroll
    for (int k2 = 0; k2 < VL; ++k2) dst[t + TL * k2] = v[k2];
}

// K2, register FFT: block NP TL threads, transform pp = row pair.
template <typename R, int N>
__global__ void __launch_bounds__(kThreads, 2) k_rows_c2r_tp(
    Geom G, int NP, const double2* __restrict__ twx, const typename cplx_t<R>::type* __restrict__ H,
    R* __restrict__ phys)
{
    typedef typename cplx_t<R>::type C;
    constexpr int TL = rbcfft::reg_fft_lanes(N), VL = N / TL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + N;
    const int st = tp_stride(N);
    const int row0 = 2 * NP * blockIdx.x;
    const int plane = row0 / G.ny, y0 = row0 - plane * G.ny;
    pdl_trigger();
    load_twiddles_async<R>(tw, twx, N);
    pdl_wait();
    // A[n] to slot n, B[n] to slot N - n (B[0] to the spare last slot st - 1 > pad(N - 1))
    const C* src = H + (size_t)plane * G.ckp * G.ny + y0;
    for (int e = threadIdx.x; e < NP * G.ckeep; e += blockDim.x) {
        const int n = e / NP, pp = e - n * NP;
        C* row = buf + pp * st;
        copy_cg<sizeof(C)>(row + rbcfft::pad(n), src + (size_t)n * G.ny + 2 * pp);
        copy_cg<sizeof(C)>(row + (n ? rbcfft::pad(N - n) : st - 1), src + (size_t)n * G.ny + 2 * pp + 1);
    }
    for (int e = threadIdx.x; e < NP * N; e += blockDim.x) {
        const int pp = e / N, n = e - pp * N;
        if (n >= G.ckeep && n <= N - G.ckeep) buf[pp * st + rbcfft::pad(n)] = cmk<C>(0, 0);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int e = threadIdx.x; e < NP * G.ckeep; e += blockDim.x) {
        const int n = e / NP, pp = e - n * NP;
        C* row = buf + pp * st;
        C* pb = row + (n ? rbcfft::pad(N - n) : st - 1);
        C A = row[rbcfft::pad(n)], B = *pb;
        if (n == 0) { A.y = 0; B.y = 0; }
        C z; z.x = A.x - B.y; z.y = A.y + B.x;       // A + iB
        row[rbcfft::pad(n)] = z;
        if (n > 0) {
            C zm; zm.x = A.x + B.y; zm.y = B.x - A.y; // conj(A) + i conj(B)
            *pb = zm;
        }
    }
    __syncthreads();
    const int pp = threadIdx.x / TL, t = threadIdx.x - pp * TL;
    C* S = buf + pp * st;
    C v[VL];
#pragma unroll
    for (int a = 0; a < VL; ++a) v[a] = S[rbcfft::pad(t + TL * a)];
    __syncwarp(rbcfft::team_mask<TL>()); // every lane has read before the tile is overwritten
    rbcfft::reg_fft<N, R>(v, t, S, tw, +1);
    R* dst = phys + (size_t)(row0 + 2 * pp) * N;
#pragma unroll
    for (int k2 = 0; k2 < VL; ++k2) {
        dst[t + TL * k2] = v[k2].x;
        dst[N + t + TL * k2] = v[k2].y;
    }
}

// K4, register FFT: block NP TL threads; item i = row pairs [NP i, NP (i + 1)) of the 13 L
// group planes. A CTA takes items blockIdx.x, blockIdx.x + gridDim.x, ... and loads the next
// item's rows into registers as soon as the current item's spectra are in shared memory, so
// the loads are in flight during the current item's output stage.
template <typename R, int N>
__global__ void __launch_bounds__(kThreads, 2) k_rows_r2c_tp(
    Geom G, int NP, int nitems, const double2* __restrict__ twx, const R* __restrict__ grp,
    typename cplx_t<R>::type* __restrict__ gh)
{
    typedef typename cplx_t<R>::type C;
    constexpr int TL = rbcfft::reg_fft_lanes(N), VL = N / TL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + N;
    const int st = tp_stride(N);
    const int pp = threadIdx.x / TL, t = threadIdx.x - pp * TL;
    C* S = buf + pp * st;
    C v[VL];
    auto load = [&](int item) {
        const R* src = grp + (size_t)(2 * NP * item + 2 * pp) * N;
#pragma unroll
        for (int a = 0; a < VL; ++a) {
            v[a].x = ld_cg(src + t + TL * a);
            v[a].y = ld_cg(src + N + t + TL * a);
        }
    };
    pdl_trigger();
    load_twiddles_async<R>(tw, twx, N);
    pdl_wait();
    int it = blockIdx.x; // < nitems: the grid is never larger than the item count
    load(it);
    cp_async_wait_all();
    __syncthreads();
    const R half = (R)0.5;
    for (;;) {
        rbcfft::reg_fft<N, R>(v, t, S, tw, -1);
#pragma unroll
        for (int k2 = 0; k2 < VL; ++k2) S[rbcfft::pad(t + TL * k2)] = v[k2];
        const int nxt = it + gridDim.x;
        if (nxt < nitems) load(nxt);
        __syncthreads();
        const int row0 = 2 * NP * it;
        const int plane = row0 / G.ny, y0 = row0 - plane * G.ny;
        C* dst = gh + (size_t)plane * G.ckp * G.ny + y0;
        for (int e = threadIdx.x; e < NP * G.ckw; e += blockDim.x) {
            const int n = e / NP, q = e - n * NP;
            C A = cmk<C>(0, 0), B = A;
            if (n < G.ckeep) {
                const C z = buf[q * st + rbcfft::pad(n)];
                const C zm = buf[q * st + rbcfft::pad(n == 0 ? 0 : N - n)];
                A.x = half * (z.x + zm.x);
                A.y = half * (z.y - zm.y);
                B.x = half * (z.y + zm.y);
                B.y = half * (zm.x - z.x);
            }
            dst[(size_t)n * G.ny + 2 * q] = A;
            dst[(size_t)n * G.ny + 2 * q + 1] = B;
        }
        it = nxt;
        if (it >= nitems) break;
        __syncthreads(); // the spectra are read before the next transform reuses the tiles
    }
}

// K5, register FFT: grid (ckw, L), block min(13 TL, kThreads) threads; team q (TL lanes)
// transforms groups q, q + teams, ... (one group each for TL <= 16, up to two for TL = 32).
template <typename R, int N>
__global__ void __launch_bounds__(kThreads, 2) k_columns_combine_tp(
    Geom G, const double2* __restrict__ twy, const typename cplx_t<R>::type* __restrict__ gh,
    typename cplx_t<R>::type* __restrict__ N_out, double* __restrict__ NFG)
{
    typedef typename cplx_t<R>::type C;
    constexpr int TL = rbcfft::reg_fft_lanes(N), VL = N / TL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf = tw + N;
    const int st = tp_stride(N);
    const int c = blockIdx.x, k = blockIdx.y;
    const size_t cstride = (size_t)G.L * G.ckp * N; // between groups
    const int teams = blockDim.x / TL, team = threadIdx.x / TL, t = threadIdx.x - team * TL;
    const C* src = gh + ((size_t)k * G.ckp + c) * N + t;
    pdl_trigger();
    load_twiddles_async<R>(tw, twy, N);
    pdl_wait();
    int gq = team;
    C v[VL];
#pragma unroll
    for (int a = 0; a < VL; ++a) v[a] = ld_cg(src + gq * cstride + TL * a);
    cp_async_wait_all();
    __syncthreads();
    for (;;) {
        C* S = buf + gq * st;
        rbcfft::reg_fft<N, R>(v, t, S, tw, -1);
#pragma unroll
        for (int k2 = 0; k2 < VL; ++k2) S[rbcfft::pad(t + TL * k2)] = v[k2];
        gq += teams;
        if (gq >= 13) break;
#pragma unroll
        for (int a = 0; a < VL; ++a) v[a] = ld_cg(src + gq * cstride + TL * a);
    }
    __syncthreads();
    const double invP = 1.0 / ((double)G.nx * N);
    for (int r = threadIdx.x; r < N; r += blockDim.x) {
        double2 vv[13];
#pragma unroll
        for (int gi = 0; gi < 13; ++gi) {
            const C z = buf[gi * st + rbcfft::pad(r)];
            vv[gi] = make_double2(z.x, z.y);
        }
        if (c == 0 && r == 0) {
            NFG[k] = vv[10].x * (-invP / G.pr);          // F: mean of the g-y group
            NFG[G.L + k] = -vv[11].x * (-invP / G.pr);   // G: minus mean of the g-x group
        }
        const Mult m(c, r, G);
        const double xx = -(m.fx * m.fx), yy = -(m.fy * m.fy);
        double2 af = vv[0] * xx + vv[1] * m.xy + vv[2] * yy + cmul_is<double2, double>(vv[3], m.fx) +
                     cmul_is<double2, double>(vv[4], m.fy) + cmul_is<double2, double>(vv[5], m.fx) * m.lap +
                     cmul_is<double2, double>(vv[6], m.fy) * m.lap + vv[7] * m.lap;
        double2 ag = vv[8] * m.xy + vv[9] * (yy - xx) + cmul_is<double2, double>(vv[10], m.fy) +
                     cmul_is<double2, double>(vv[11], m.fx);
        const double2 at = vv[12] * (-invP);
        af = af * (-invP / G.pr);
        ag = ag * (-invP / G.pr);
        const size_t o = ((size_t)k * G.ckp + c) * N + r;
        const size_t pl = (size_t)G.L * G.ckp * N;
        N_out[o] = cmk<C>(at.x, at.y);
        N_out[pl + o] = cmk<C>(af.x, af.y);
        N_out[2 * pl + o] = cmk<C>(ag.x, ag.y);
    }
}

} // namespace rbck
