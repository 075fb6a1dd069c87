// mask_kernels.cuh -- physical-space field operators of the reference on the spectral
// state: freeze_operator (gpu_flow/code/operator/freeze_operator.cu) and masktemp
// (gpu_flow/code/operator/masktemp.cu), both wired into the iteration loop by main.cu:569-590.
//
// Each operator takes the horizontal planes of the selected fields (theta, f, g for the
// freeze, theta for the heating; every vertical mode on its own) to the Nx x Ny grid with
// the unnormalised C2R, changes the values where a mask is 0, multiplies everything by
// 1/(Nx Ny) and returns with the unnormalised R2C:
//   freeze   v = mask ? v : frozen        (freeze_operator.cu:242-257)
//   heating  v = mask ? v : v + increment (masktemp.cu:191-208, increment 1.5/100)
//   scaling  v = mask ? v : v factor      (masking.cu:43-58, factor 1.1 by default)
// The frozen planes are the C2R of the state when the freeze was taken
// (freeze_operator.cu:60-111).
//
// FP64 throughout, three launches over the planes (S = the CM scratch [plane][ckp][Ny]):
//   KM1 k_mask_cols<+1>  inverse y transforms of the kept columns c < ckeep      state -> S
//   KM2 k_mask_rows      two rows as one complex transform: Hermitian extension, inverse
//                        x transform, the mask operation, forward x transform, split  S -> S
//   KM3 k_mask_cols<-1>  forward y transforms, rows outside the 2/3 band zeroed     S -> state
// Columns c >= ckeep are zero in the state and stay zero. The reference leaves the R2C
// output undealiased and its next step starts with dealias_data
// (implicit_explicit_stepping.cu:39); both operators are affine, so dropping the removed
// modes here gives the same state at the start of that step.
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "step_kernels.cuh"

namespace rbck {

enum MaskOp { MASK_SNAPSHOT = 0, MASK_FREEZE = 1, MASK_HEAT = 2, MASK_SCALE = 3 };

// Up to three fields of L planes each; plane pl is vertical mode pl % L of field pl / L.
struct MaskFields {
    double2* p[3];
};

// Masks of the reference (init_mask_physical_space_circle / _rectangle,
// freeze_operator.cu:261-308, masktemp.cu:211-259): 1 keeps the current value.
//   circle     (col - cx Nx)^2 + (row - cy Ny)^2 > (size 0.5 min(Nx, Ny))^2
//   rectangle  col < size Nx || col > (1 - size) Nx || row < size Ny || row > (1 - size) Ny
// Rounded operations without contraction, as the host restatement evaluates them.
__global__ void k_field_mask(unsigned char* __restrict__ mask, int nx, int ny, int shape, double cx, double cy,
                             double size)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return;
    const int col = i % nx, row = i / nx;
    unsigned char m = 0;
    if (shape == 0) {
        const double a = __dsub_rn((double)col, __dmul_rn(cx, (double)nx));
        const double b = __dsub_rn((double)row, __dmul_rn(cy, (double)ny));
        const double d2 = __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b));
        const double rmax = __dmul_rn(__dmul_rn(size, 0.5), (double)(ny < nx ? ny : nx));
        m = d2 > __dmul_rn(rmax, rmax);
    } else {
        const double wx = __dmul_rn(size, (double)nx), wy = __dmul_rn(size, (double)ny);
        const double ux = __dmul_rn(__dsub_rn(1.0, size), (double)nx);
        const double uy = __dmul_rn(__dsub_rn(1.0, size), (double)ny);
        m = (col < wx) || (col > ux) || (row < wy) || (row > uy);
    }
    mask[i] = m;
}

// KM1 / KM3. Grid (ceil(ckeep / W), planes); W <= py.chunk columns of one plane per CTA
// and at least W Ny / (smallest radix) threads (every butterfly of a pass has a thread).
// Shared: twiddles [Ny] + W padded transforms.
template <int SIGN>
__global__ void __launch_bounds__(kThreads, 2) k_mask_cols(Geom G, int W, rbcfft::Plan py, const double2* __restrict__ twy,
                                                        MaskFields fl, double2* __restrict__ S)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* buf = tw + G.ny;
    const int ny = G.ny, pl = blockIdx.y, c0 = blockIdx.x * W;
    const int nc = G.ckeep - c0 < W ? G.ckeep - c0 : W;
    load_twiddles<double>(tw, twy, ny);
    double2* state = fl.p[pl / G.L] + (size_t)(pl % G.L) * G.ckp * ny;
    double2* scr = S + (size_t)pl * G.ckp * ny;
    const double2* src = SIGN > 0 ? state : scr;
    for (int e = threadIdx.x; e < nc * ny; e += blockDim.x) {
        const int j = e / ny, r = e - j * ny;
        cp_async<sizeof(double2)>(buf + j * py.stride + rbcfft::pad(r), src + (size_t)(c0 + j) * ny + r);
    }
    cp_async_wait_all();
    __syncthreads();
    fft_batched<double>(buf, py, nc, tw, SIGN);
    double2* dst = SIGN > 0 ? scr : state;
    for (int e = threadIdx.x; e < nc * ny; e += blockDim.x) {
        const int j = e / ny, r = e - j * ny;
        double2 v = buf[j * py.stride + rbcfft::pad(r)];
        if (SIGN < 0 && !row_kept(r, ny)) v = make_double2(0.0, 0.0);
        dst[(size_t)(c0 + j) * ny + r] = v;
    }
}

// KM2. Grid (ceil(Ny / (2 NB)), planes), kThreads threads. Transform t of the CTA holds
// rows ya = 2 (blockIdx.x NB + t) and ya + 1 as z = x_a + i x_b. Shared: twiddles [Nx],
// NB padded transforms, and the staged kept coefficients [ckeep][2 NB].
// op: MASK_SNAPSHOT writes the C2R of the planes to `frozen` and leaves S alone;
// MASK_FREEZE / MASK_HEAT / MASK_SCALE apply the operation (increment is the factor of
// MASK_SCALE) and write the R2C back into S.
__global__ void __launch_bounds__(kThreads, 2) k_mask_rows(Geom G, int NB, rbcfft::Plan px, const double2* __restrict__ twx,
                                                        double2* __restrict__ S, int op,
                                                        const unsigned char* __restrict__ mask,
                                                        double* __restrict__ frozen, double increment)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* buf = tw + G.nx;
    double2* stg = buf + NB * px.stride;
    const int nx = G.nx, ny = G.ny, ck = G.ckeep, pl = blockIdx.y;
    const int y0 = blockIdx.x * 2 * NB;
    const int nrow = ny - y0 < 2 * NB ? ny - y0 : 2 * NB; // even: Ny is even
    const int nt = nrow / 2;
    load_twiddles<double>(tw, twx, nx);
    double2* scr = S + (size_t)pl * G.ckp * ny;
    for (int e = threadIdx.x; e < ck * nrow; e += blockDim.x) {
        const int c = e / nrow, y = e - c * nrow;
        cp_async<sizeof(double2)>(stg + c * 2 * NB + y, scr + (size_t)c * ny + y0 + y);
    }
    cp_async_wait_all();
    __syncthreads();
    // Hermitian extension of rows a and b, packed: Z[j] = A[j] + i B[j] and
    // Z[Nx - j] = conj(A[j]) + i conj(B[j]); the imaginary parts of A and B at j = 0
    // and j = Nx/2 are ignored, as by a C2R transform.
    const int half = nx / 2;
    for (int e = threadIdx.x; e < nt * nx; e += blockDim.x) {
        const int t = e / nx, j = e - t * nx;
        const int m = j <= half ? j : nx - j;
        double2 A = make_double2(0.0, 0.0), B = A;
        if (m < ck) {
            A = stg[m * 2 * NB + 2 * t];
            B = stg[m * 2 * NB + 2 * t + 1];
        }
        double2 z;
        if (j == 0 || j == half) z = make_double2(A.x, B.x);
        else if (j < half) z = make_double2(A.x - B.y, A.y + B.x);
        else z = make_double2(A.x + B.y, B.x - A.y);
        buf[t * px.stride + rbcfft::pad(j)] = z;
    }
    __syncthreads();
    fft_batched<double>(buf, px, nt, tw, +1);
    const double invP = 1.0 / ((double)nx * ny);
    double* fr = frozen ? frozen + (size_t)pl * G.P : nullptr;
    // four elements per thread and round: their mask and frozen values are loaded before
    // any of them is used
    const int tot = nt * nx;
    for (int e0 = threadIdx.x; e0 < tot; e0 += 4 * blockDim.x) {
        unsigned char ma[4], mb[4];
        double fa[4], fb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = e0 + u * blockDim.x;
            ma[u] = mb[u] = 1;
            fa[u] = fb[u] = 0.0;
            if (e < tot && op != MASK_SNAPSHOT) {
                const int t = e / nx, x = e - t * nx;
                const size_t ia = (size_t)(y0 + 2 * t) * nx + x;
                ma[u] = mask[ia];
                mb[u] = mask[ia + nx];
                if (op == MASK_FREEZE) {
                    fa[u] = fr[ia];
                    fb[u] = fr[ia + nx];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e >= tot) continue;
            const int t = e / nx, x = e - t * nx;
            const size_t ia = (size_t)(y0 + 2 * t) * nx + x;
            double2& z = buf[t * px.stride + rbcfft::pad(x)];
            if (op == MASK_SNAPSHOT) {
                fr[ia] = z.x;
                fr[ia + nx] = z.y;
                continue;
            }
            double va = z.x, vb = z.y;
            if (op == MASK_SCALE) { // masking.cu:49-56: (1/P) v factor inside the circle
                va = ma[u] ? invP * va : invP * va * increment;
                vb = mb[u] ? invP * vb : invP * vb * increment;
            } else {
                if (!ma[u]) va = op == MASK_FREEZE ? fa[u] : va + increment;
                if (!mb[u]) vb = op == MASK_FREEZE ? fb[u] : vb + increment;
                va *= invP;
                vb *= invP;
            }
            z = make_double2(va, vb);
        }
    }
    if (op == MASK_SNAPSHOT) return; // uniform over the CTA
    __syncthreads();
    fft_batched<double>(buf, px, nt, tw, -1);
    // split: A[c] = (Z[c] + conj(Z[-c])) / 2, B[c] = (Z[c] - conj(Z[-c])) / (2 i)
    for (int e = threadIdx.x; e < ck * nrow; e += blockDim.x) {
        const int c = e / nrow, y = e - c * nrow;
        const int t = y >> 1;
        const double2 P = buf[t * px.stride + rbcfft::pad(c)];
        const double2 Q = buf[t * px.stride + rbcfft::pad(c == 0 ? 0 : nx - c)];
        double2 v;
        if ((y & 1) == 0) v = make_double2(0.5 * (P.x + Q.x), 0.5 * (P.y - Q.y));
        else v = make_double2(0.5 * (P.y + Q.y), -0.5 * (P.x - Q.x));
        scr[(size_t)c * ny + y0 + y] = v;
    }
}

} // namespace rbck
