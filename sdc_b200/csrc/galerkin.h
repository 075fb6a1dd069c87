// galerkin.h -- host-side precomputation for the RBC step (library side).
#pragma once
#include <cstdint>
#include <vector>

namespace rbchost {

// Galerkin integrals over z in (-1/2, 1/2) of Chandrasekhar functions C_m and sines
// S_m (m 0-based). 2-index tables at i + j*L, 3-index tables at i + j*L + k*L*L, the
// index order of the reference getters (gpu_flow/code/util/coeff.cu:1151-1222).
struct Tables {
    int L = 0;
    std::vector<double> lambda;                 // lambda_{m+1}
    std::vector<double> Iac, Ia1, Ia2;          // as the reference uses them (Iac closed forms)
    std::vector<double> Ibb1, Ib11, I111, Iabc, Iac1, Iaab, Iaa1, Iab2, Ia12;
    std::vector<double> CpCp, CC, CS;           // exact int C'_i C'_j, int C_i C_j, int C_i S_j (diagnostics)
    double t3(const std::vector<double>& t, int i, int j, int k) const { return t[i + j * L + k * L * L]; }
    double ibbb(int i, int j, int k) const { return -t3(Iabc, i, j, k) - t3(Iabc, i, k, j); }
};

// colloc_nq > 0: the 3-index tensors (the nonlinear term's) are the colloc_nq-point
// Gauss-Legendre sums sum_q w_q a_i(z_q) b_j(z_q) c_k(z_q) instead of the exact integrals,
// i.e. the tensors of a step that forms its products on colloc_nq collocation levels and
// projects them back with the same rule; the 2-index tables (linear operators,
// diagnostics) stay exact.
void build_tables(int L, Tables& T, int colloc_nq = 0);

// Value of the contraction matrix T'(i,j) of family f at output mode k.
double family_value(const Tables& T, int family, int i, int j, int k);

// Packed contraction coefficients coef[u][k][o][h] (see contract_prog.h).
void pack_contraction(const Tables& T, std::vector<double>& coef);

// Partial-pivot LU inverse of a row-major n x n matrix; false if singular.
bool lu_invert(int n, const std::vector<double>& A, std::vector<double>& inv);

// Per-wavenumber operators, deduplicated by the exact bit pattern of q^2 as the
// reference computes it on the host (inverse_B_matrix.cu:108-118,
// linear_implicit_operator.cu:46-59).
struct OperatorTables {
    int nclass = 0;
    std::vector<int> cls;         // [Ny][mox] class of each wavenumber (-1: dealiased)
    std::vector<double> binv;     // [nclass][L*L]  B_ff^-1 (row-major m*L+m1)
    std::vector<double> imp;      // [nclass][4][L*L]  (tt, tf, ft, ff) blocks of (I - dt B^-1 L)^-1
};

struct GridInfo {
    int nx, ny, L, mox;
    double lx, ly, ra, pr, dt;
    int ckeep;                    // columns c < ckeep survive the 2/3 rule
    std::vector<uint8_t> row_kept;// [Ny]
};

void grid_info(int nx, int ny, int L, double lx, double ly, double ra, double pr, double dt, GridInfo& g);
void build_operator_tables(const GridInfo& g, const Tables& T, OperatorTables& op);

// Seeded initial temperature (SplitMix64 + Box-Muller) into theta [L][Ny][mox]
// (interleaved complex), followed by the Hermitian fix on the kx = 0 column.
void seeded_theta(const GridInfo& g, uint64_t seed, double amp, double kmax, double* theta);
void seeded_positions(uint64_t seed, int n, double lx, double ly, double* xyz);
// Pattern initial temperature (rbc_init_pattern types) into theta [L][Ny][mox]
// (interleaved complex): the reference's real-space pattern R2C-transformed into the
// lowest vertical mode, uniform noise in the others, the Hermitian fix. For the TEST
// pattern f and F are filled too (f [L][Ny][mox], F [L] interleaved complex).
void pattern_theta(const GridInfo& g, int type, double mode, double amp, uint64_t seed, double noise, double* theta,
                   double* f, double* F);
// Forward real 2-D FFT (unnormalised, e^{-i}) of real[ny][nx] into out[ny][nx/2+1]
// (interleaved complex); nx, ny = 2^a 3^b.
void rfft2(int nx, int ny, const double* real, double* out);
// Collocation levels of the surrogate: the nq Gauss-Legendre nodes z_q on (-1/2, 1/2),
// the basis values there (C, C', S at [q][m]) and the least-squares inverses of the
// S and C samples (Ps, Pc at [m][q]: (B^T B)^-1 B^T for B[q][m] = S_m(z_q) or C_m(z_q)),
// which recover the L mode amplitudes of any field that lies in the span exactly.
struct CollocTables {
    int L = 0, nq = 0;
    std::vector<double> z, C, Cp, S, Ps, Pc;
};
bool colloc_tables(int L, int nq, CollocTables& t);
// The collocation form's contraction (colloc_prog.h) on Q Gauss-Legendre levels of
// (-1/2, 1/2): z[q], w[q], basis[(kind * L + i) * Q + q] = kind's function i at z_q (kinds
// C, C', C'', S, S') and proj[(kind * Q + q) * L + k] = w_q times kind's function k at z_q.
struct CollocContract {
    int L = 0, Q = 0;
    std::vector<double> z, w, basis, proj;
};
void colloc_contract_tables(int L, int Q, CollocContract& t);
// Tracer start patterns of particle_tracer::init_positions (rbc_tracer_init types).
void tracer_pattern(int type, uint64_t seed, int n, double lx, double ly, double cx, double cy, double cz,
                    double sigma, double* xyz);

} // namespace rbchost
