// colloc_prog.h -- the nonlinear operator's contraction as products on collocation levels.
//
// Every term of the exact contraction (contract_prog.h) is C(i,j,k) a_i b_j with a Galerkin
// tensor C(i,j,k) = int phi_i(z) psi_j(z) chi_k(z) dz of three basis functions (kinds C, C',
// C'', S, S'; the reference's coefficient getters, gpu_flow/code/util/coeff.h:22-47). With a
// quadrature rule of Q levels z_q, weights w_q, in place of the integral, the term becomes
//     sum_q w_q chi_k(z_q) A(z_q) B(z_q),   A(z) = sum_i a_i phi_i(z),  B(z) = sum_j b_j psi_j(z),
// i.e. the two fields synthesised on the levels (a mode -> level product), multiplied there,
// and projected back (a level -> mode product). On the step's fields that needs:
//   - 12 synthesised pairs (field, kind): u11 and u21 with C, C', C''; u31 with C; u12, u22,
//     theta_x, theta_y with S; theta with S';
//   - 41 products per level, each adding weight * A * B to one of
//   - 16 projected pairs (group, kind), whose level sums against w_q chi_k(z_q) give the 13
//     contracted groups of contract_prog.h.
// The list is derived here at compile time from the unit program of contract_prog.h and the
// kinds of each tensor's arguments, so both contractions come from one description of the
// reference's summands. With Q levels of Gauss-Legendre the result equals the exact
// contraction with the Q-level sums in place of the tensors (rbchost::build_tables with
// colloc_nq = Q).
#pragma once
#include "contract_prog.h"

namespace rbccol {

enum Kind { KC = 0, KCP, KCPP, KS, KSP, NKIND }; // C, C', C'', S, S' (galerkin.cpp's basis kinds)

// Kinds of the three arguments of each Galerkin tensor (coeff.h definitions).
enum Tensor { T_IABC = 0, T_IBB1, T_IB11, T_I111, T_IAC1, T_IAAB, T_IAA1, T_IAB2, T_IA12 };
RBCP_HD constexpr int tensor_kind(int t, int arg)
{
    constexpr int k[9][3] = {{KC, KCP, KCPP}, {KCP, KCP, KS}, {KCP, KS, KS},   {KS, KS, KS},   {KC, KCPP, KS},
                             {KC, KC, KCP},   {KC, KC, KS},   {KC, KCP, KSP}, {KC, KS, KSP}};
    return k[t][arg];
}

// One term of a contraction family: sign * tensor(args), the arguments given as roles
// (0: i, the a-field index; 1: j, the b-field index; 2: k, the output mode).
struct Term {
    int sign, tensor, role[3];
};
RBCP_HD constexpr int family_terms(int f) { return f == rbcprog::IBBB_IJK ? 2 : 1; }
RBCP_HD constexpr Term family_term(int f, int n)
{
    using namespace rbcprog;
    return f == IBBB_IJK ? (n == 0 ? Term{-1, T_IABC, {0, 1, 2}} : Term{-1, T_IABC, {0, 2, 1}})
         : f == IBB1_IKJ ? Term{1, T_IBB1, {0, 2, 1}}
         : f == IB11_KIJ ? Term{1, T_IB11, {2, 0, 1}}
         : f == IABC_JIK ? Term{1, T_IABC, {1, 0, 2}}
         : f == IAC1_IKJ ? Term{1, T_IAC1, {0, 2, 1}}
         : f == IAAB_JKI ? Term{1, T_IAAB, {1, 2, 0}}
         : f == IAA1_IKJ ? Term{1, T_IAA1, {0, 2, 1}}
         : f == IAAB_IJK ? Term{1, T_IAAB, {0, 1, 2}}
         : f == IBB1_IJK ? Term{1, T_IBB1, {0, 1, 2}}
         : f == IB11_IJK ? Term{1, T_IB11, {0, 1, 2}}
         : f == I111_IJK ? Term{1, T_I111, {0, 1, 2}}
         : f == IAB2_JIK ? Term{1, T_IAB2, {1, 0, 2}}
         : f == IA12_IJK ? Term{1, T_IA12, {0, 1, 2}}
                         : Term{1, T_IA12, {0, 2, 1}}; // IA12_IKJ
}
RBCP_HD constexpr int role_kind(const Term& t, int role)
{
    return t.role[0] == role ? tensor_kind(t.tensor, 0) : t.role[1] == role ? tensor_kind(t.tensor, 1)
                                                                              : tensor_kind(t.tensor, 2);
}

// Synthesised pairs, grouped by field (one tensor-core product per field).
struct SPair {
    int field, kind;
};
constexpr int NSPAIR = 12;
RBCP_HD constexpr SPair spair_at(int p)
{
    using namespace rbcprog;
    constexpr SPair t[NSPAIR] = {{U11, KC}, {U11, KCP}, {U11, KCPP}, {U21, KC}, {U21, KCP}, {U21, KCPP},
                                 {U31, KC}, {U12, KS},  {U22, KS},   {TH, KSP}, {THX, KS},  {THY, KS}};
    return t[p];
}
RBCP_HD constexpr int spair_index(int field, int kind)
{
    for (int p = 0; p < NSPAIR; ++p)
        if (spair_at(p).field == field && spair_at(p).kind == kind) return p;
    return -1;
}
// First pair and pair count of each field.
RBCP_HD constexpr int field_first_pair(int f)
{
    for (int p = 0; p < NSPAIR; ++p)
        if (spair_at(p).field == f) return p;
    return -1;
}
RBCP_HD constexpr int field_pairs(int f)
{
    int n = 0;
    for (int p = 0; p < NSPAIR; ++p) n += spair_at(p).field == f;
    return n;
}

// Projected pairs (group, kind).
struct PPair {
    int group, kind;
};
constexpr int NPPAIR = 16;
RBCP_HD constexpr PPair ppair_at(int p)
{
    using namespace rbcprog;
    constexpr PPair t[NPPAIR] = {{FXX, KCP}, {FXX, KCPP}, {FXY, KCP}, {FXY, KCPP}, {FYY, KCP}, {FYY, KCPP},
                                 {FX, KCPP}, {FY, KCPP},  {FLX, KC},  {FLY, KC},   {FL, KCP},  {GXY, KS},
                                 {GD, KS},   {GY, KSP},   {GX, KSP},  {TQ, KS}};
    return t[p];
}
RBCP_HD constexpr int ppair_index(int group, int kind)
{
    for (int p = 0; p < NPPAIR; ++p)
        if (ppair_at(p).group == group && ppair_at(p).kind == kind) return p;
    return -1;
}

// One product on a level: weight * A[a] * B[b] added to projected pair `to`.
struct Prod {
    int a, b, to, weight;
};
constexpr int NPROD = 41;
// The n-th product, walking units, edges and family terms in order.
RBCP_HD constexpr Prod prod_at(int n)
{
    int c = 0;
    for (int u = 0; u < rbcprog::NUNIT; ++u) {
        const rbcprog::Unit un = rbcprog::unit_at(u);
        for (int e = 0; e < un.nedge; ++e) {
            const int fa = un.left == 0 ? un.e[e].other : un.fixed; // field at index i
            const int fb = un.left == 0 ? un.fixed : un.e[e].other; // field at index j
            for (int t = 0; t < family_terms(un.family); ++t, ++c) {
                if (c != n) continue;
                const Term tm = family_term(un.family, t);
                return Prod{spair_index(fa, role_kind(tm, 0)), spair_index(fb, role_kind(tm, 1)),
                            ppair_index(un.e[e].group, role_kind(tm, 2)), tm.sign * un.e[e].weight};
            }
        }
    }
    return Prod{-1, -1, -1, 0};
}
RBCP_HD constexpr bool program_complete()
{
    for (int n = 0; n < NPROD; ++n) {
        const Prod p = prod_at(n);
        if (p.a < 0 || p.b < 0 || p.to < 0 || p.weight == 0) return false;
    }
    return prod_at(NPROD).a < 0; // and no product beyond NPROD
}
static_assert(program_complete(), "every product maps to a synthesised and a projected pair");

} // namespace rbccol
