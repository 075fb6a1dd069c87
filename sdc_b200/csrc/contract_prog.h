// contract_prog.h -- the nonlinear operator as a physical-space Galerkin contraction.
//
// The reference (gpu_flow/code/operator/nonlinear_operator_rayleigh_noslip.cu:263-1095)
// forms, for every vertical mode pair (i,j), 20 pointwise products a_i(x) b_j(x),
// transforms each with an R2C FFT and adds D(q) * C(i,j,k) * FFT[a_i b_j] into the
// outputs f_k, g_k, theta_k, F_k, G_k, where D is a spectral derivative multiplier
// (xx, xy, yy, x, y, Laplacian o x, Laplacian o y, Laplacian, identity).
//
// Because the FFT is linear, all terms that share one output mode k and one multiplier
// D can be summed in physical space first:
//     out_k(q) = sum_D D(q) * FFT[ Q_{D,k}(x) ],  Q_{D,k} = sum_{terms,i,j} C a_i b_j.
// This needs 13 L transforms per step instead of 20 L^2. The 13 groups are the 8 f
// multipliers, 4 g multipliers (the reference's g terms under Dyy and Dxx carry opposite
// signs and merge into one group with multiplier Dyy - Dxx) and theta. F and G are the
// q = 0 entries of the g "y" and g "x" groups before their multipliers are applied
// (reference :950-1003 adds exactly those products' DC parts).
//
// Per physical point the contraction is organised as 20 units. A unit contracts one
// input field with one coefficient matrix T'(o,s) (for fixed k) into a vector
// w_o = sum_s T'(o,s) field_s, and each of its edges adds weight * sum_o w_o other_o to
// one group. "Right" units contract the b (second) index, "left" units the a index.
// The tensors and index orders are the reference's; the unit/edge grouping is a minimum
// vertex cover of the (a-field, b-field) pairs that share a tensor.
#pragma once

#ifdef __CUDACC__
#define RBCP_HD __host__ __device__
#else
#define RBCP_HD
#endif

namespace rbcprog {

enum Field { U11 = 0, U21, U31, U12, U22, TH, THX, THY, NFIELD };
// U11 = d_x f, U21 = d_y f, U31 = -lap_h f (= q^2 f), U12 = d_y g + F, U22 = -d_x g + G,
// TH = theta, THX = d_x theta, THY = d_y theta -- each synthesised per vertical mode.

enum Group { FXX = 0, FXY, FYY, FX, FY, FLX, FLY, FL, GXY, GD, GY, GX, TQ, NGROUP };

// Tensor families with the index order the reference uses; T'(i,j) at fixed k is
// the listed getter with (i, j, k) substituted.
enum Family {
    IBBB_IJK = 0, // Ibbb(i,j,k) = -Iabc(i,j,k) - Iabc(i,k,j)
    IBB1_IKJ,     // Ibb1(i,k,j)
    IB11_KIJ,     // Ib11(k,i,j)
    IABC_JIK,     // Iabc(j,i,k)
    IAC1_IKJ,     // Iac1(i,k,j)
    IAAB_JKI,     // Iaab(j,k,i)
    IAA1_IKJ,     // Iaa1(i,k,j)
    IAAB_IJK,     // Iaab(i,j,k)
    IBB1_IJK,     // Ibb1(i,j,k)
    IB11_IJK,     // Ib11(i,j,k)
    I111_IJK,     // I111(i,j,k)
    IAB2_JIK,     // Iab2(j,i,k)
    IA12_IJK,     // Ia12(i,j,k)
    IA12_IKJ,     // Ia12(i,k,j)
    NFAMILY
};

// z-parity of each family's integrand: the number of z-derivatives mod 2. An entry
// T'(i,j) at output k is zero unless (i + j + k + parity) is even.
RBCP_HD constexpr int family_parity(int f)
{
    return (f == IBBB_IJK || f == IB11_KIJ || f == IABC_JIK || f == IAAB_JKI || f == IAAB_IJK ||
            f == IB11_IJK || f == IA12_IJK || f == IA12_IKJ) ? 1 : 0;
}

struct Edge {
    int other;  // field contracted against w
    int group;  // output group
    int weight; // +-1 or +-2
};

struct Unit {
    int family;
    int left;   // 0: w_i = sum_j T'(i,j) fixed_j (fixed = b field, other = a field)
                // 1: w_j = sum_i T'(i,j) fixed_i (fixed = a field, other = b field)
    int fixed;
    int nedge;
    Edge e[3];
};

constexpr int NUNIT = 20;

// Each line: reference summand(s) covered (f_n / g_n numbering of the reference file).
RBCP_HD constexpr Unit unit_at(int u)
{
    return u == 0 ? Unit{IBBB_IJK, 0, U11, 2, {{U11, FXX, -1}, {U21, FXY, -2}, {0, 0, 0}}}      // f1, f4
         : u == 1 ? Unit{IBBB_IJK, 0, U21, 1, {{U21, FYY, -1}, {0, 0, 0}, {0, 0, 0}}}          // f14
         : u == 2 ? Unit{IBB1_IKJ, 0, U12, 2, {{U11, FXX, -2}, {U21, FXY, -2}, {0, 0, 0}}}     // f2, f5
         : u == 3 ? Unit{IBB1_IKJ, 0, U22, 2, {{U11, FXY, -2}, {U21, FYY, -2}, {0, 0, 0}}}     // f6, f15
         : u == 4 ? Unit{IB11_KIJ, 1, U12, 2, {{U12, FXX, -1}, {U22, FXY, -2}, {0, 0, 0}}}     // f3, f7
         : u == 5 ? Unit{IB11_KIJ, 0, U22, 1, {{U22, FYY, -1}, {0, 0, 0}, {0, 0, 0}}}          // f16
         : u == 6 ? Unit{IABC_JIK, 0, U31, 2, {{U11, FX, 1}, {U21, FY, 1}, {0, 0, 0}}}         // f8, f17
         : u == 7 ? Unit{IAC1_IKJ, 1, U31, 2, {{U12, FX, 1}, {U22, FY, 1}, {0, 0, 0}}}         // f9, f18
         : u == 8 ? Unit{IAAB_JKI, 0, U31, 2, {{U11, FLX, -1}, {U21, FLY, -1}, {0, 0, 0}}}     // f19, f22
         : u == 9 ? Unit{IAA1_IKJ, 1, U31, 2, {{U12, FLX, -1}, {U22, FLY, -1}, {0, 0, 0}}}     // f21, f23
         : u == 10 ? Unit{IAAB_IJK, 0, U31, 1, {{U31, FL, 1}, {0, 0, 0}, {0, 0, 0}}}           // f24
         : u == 11 ? Unit{IBB1_IJK, 1, U11, 2, {{U11, GXY, 1}, {U21, GD, 1}, {0, 0, 0}}}       // g1, g4/g10
         : u == 12 ? Unit{IBB1_IJK, 0, U21, 1, {{U21, GXY, -1}, {0, 0, 0}, {0, 0, 0}}}         // g14
         : u == 13 ? Unit{IB11_IJK, 1, U11, 3, {{U12, GXY, 2}, {U22, GD, 1}, {THX, TQ, 1}}}    // g2, g6/g12, t1
         : u == 14 ? Unit{IB11_IJK, 1, U21, 3, {{U22, GXY, -2}, {U12, GD, 1}, {THY, TQ, 1}}}   // g15, g5/g11, t3
         : u == 15 ? Unit{I111_IJK, 1, U12, 3, {{U12, GXY, 1}, {U22, GD, 1}, {THX, TQ, 1}}}    // g3, g7/g13, t2
         : u == 16 ? Unit{I111_IJK, 1, U22, 2, {{U22, GXY, -1}, {THY, TQ, 1}, {0, 0, 0}}}      // g16, t4
         : u == 17 ? Unit{IAB2_JIK, 0, U31, 2, {{U11, GY, -1}, {U21, GX, 1}, {0, 0, 0}}}       // g8, g17 (F, G)
         : u == 18 ? Unit{IA12_IJK, 1, U31, 2, {{U12, GY, -1}, {U22, GX, 1}, {0, 0, 0}}}       // g9, g18 (F, G)
                   : Unit{IA12_IKJ, 0, TH, 1, {{U31, TQ, 1}, {0, 0, 0}, {0, 0, 0}}};           // t5
}

// Number of stored coefficients per (unit, k, o) row: the parity-nonzero s values
// s0, s0+2, ... < L with s0 = (o + k + parity) & 1, padded to H = (L+1)/2.
RBCP_HD constexpr int half_len(int L) { return (L + 1) / 2; }

} // namespace rbcprog
