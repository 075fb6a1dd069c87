// galerkin.cpp -- Galerkin integrals, per-wavenumber operators and seeded inputs.
//
// The integrals follow the definitions of gpu_flow/code/util/coeff.h:22-47 (basis
// C_k, S_k on z in (-1/2,1/2), lambda table coeff.cu:1232-1257). They are evaluated
// here by composite Gauss-Legendre quadrature (8 panels), which reproduces the
// reference's closed forms (coeff.cu:60-1083) to ~1e-15 of each table's scale for all
// 3-index tensors the step uses. Iac uses the analytic closed forms (see build_tables).
// The implicit and inverse-B operators follow linear_implicit_operator.cu:46-197 and
// inverse_B_matrix.cu:108-160 with a partial-pivot LU in place of GSL.
#include "galerkin.h"
#include "contract_prog.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <algorithm>

namespace rbchost {

static const double kPi = 3.14159265358979323846;

static double lambda_k(int k) // k >= 1
{
    static const double r[] = {0.0, 1.505618731142, 2.499752670074, 3.500010679436, 4.499999538484,
                               5.500000019944, 6.499999999138, 7.500000000037, 8.499999999998};
    return k > 8 ? kPi * (k + 0.5) : kPi * r[k];
}

// Basis function values: kind 0 = C, 1 = C', 2 = C'', 3 = S, 4 = S'.
static double basis(int kind, int m, double z)
{
    const int k = m + 1;
    if (kind >= 3) {
        const double a = k * kPi;
        return kind == 3 ? std::sin(a * (z + 0.5)) : a * std::cos(a * (z + 0.5));
    }
    const double l = lambda_k(k);
    if (k & 1) {
        const double ich = 1.0 / std::cosh(0.5 * l), ic = 1.0 / std::cos(0.5 * l);
        if (kind == 0) return std::cosh(l * z) * ich - std::cos(l * z) * ic;
        if (kind == 1) return l * (std::sinh(l * z) * ich + std::sin(l * z) * ic);
        return l * l * (std::cosh(l * z) * ich + std::cos(l * z) * ic);
    }
    const double ish = 1.0 / std::sinh(0.5 * l), is = 1.0 / std::sin(0.5 * l);
    if (kind == 0) return std::sinh(l * z) * ish - std::sin(l * z) * is;
    if (kind == 1) return l * (std::cosh(l * z) * ish - std::cos(l * z) * is);
    return l * l * (std::sinh(l * z) * ish + std::sin(l * z) * is);
}

static bool basis_odd(int kind, int m)
{
    const int nder = kind == 1 ? 1 : kind == 2 ? 2 : kind == 4 ? 1 : 0;
    return ((m & 1) + nder) & 1;
}

// Composite Gauss-Legendre rule: `panels` panels of n nodes on (-1/2, 1/2).
static void composite_gl(int panels, int n, std::vector<double>& z, std::vector<double>& w)
{
    std::vector<long double> xs(n), ws(n);
    for (int i = 0; i < n; ++i) {
        long double t = std::cos(kPi * (i + 0.75) / (n + 0.5)), p1 = 0, p0 = 0, d = 0;
        for (int it = 0; it < 60; ++it) {
            p0 = 1;
            p1 = t;
            for (int k = 2; k <= n; ++k) {
                long double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            d = n * (t * p1 - p0) / (t * t - 1);
            long double step = p1 / d;
            t -= step;
            if (std::fabs((double)step) < 1e-20) break;
        }
        xs[i] = t;
        ws[i] = 2.0L / ((1 - t * t) * d * d);
    }
    z.clear();
    w.clear();
    const long double h = 1.0L / panels;
    for (int p = 0; p < panels; ++p) {
        const long double a = -0.5L + p * h;
        for (int i = 0; i < n; ++i) {
            z.push_back((double)(a + 0.5L * h * (xs[i] + 1)));
            w.push_back((double)(0.5L * h * ws[i]));
        }
    }
}

void build_tables(int L, Tables& T, int colloc_nq)
{
    T.L = L;
    T.lambda.resize(L);
    for (int m = 0; m < L; ++m) T.lambda[m] = lambda_k(m + 1);
    std::vector<double> z, w;
    composite_gl(8, 24 + 2 * L, z, w);
    const int nq = (int)z.size();
    std::vector<double> v(5 * L * nq);
    for (int kind = 0; kind < 5; ++kind)
        for (int m = 0; m < L; ++m)
            for (int q = 0; q < nq; ++q) v[(kind * L + m) * nq + q] = basis(kind, m, z[q]);
    auto col = [&](int kind, int m) { return &v[(kind * L + m) * nq]; };
    auto int2 = [&](int ka, int kb, std::vector<double>& out) {
        out.assign(L * L, 0.0);
        for (int j = 0; j < L; ++j)
            for (int i = 0; i < L; ++i) {
                if (basis_odd(ka, i) != basis_odd(kb, j)) continue;
                const double *a = col(ka, i), *b = col(kb, j);
                long double s = 0;
                for (int q = 0; q < nq; ++q) s += (long double)w[q] * a[q] * b[q];
                out[i + j * L] = (double)s;
            }
    };
    // the rule of the 3-index tensors: the exact one, or the collocation levels' rule
    std::vector<double> z3 = z, w3 = w, v3 = v;
    if (colloc_nq > 0) {
        composite_gl(1, colloc_nq, z3, w3);
        v3.assign((size_t)5 * L * colloc_nq, 0.0);
        for (int kind = 0; kind < 5; ++kind)
            for (int m = 0; m < L; ++m)
                for (int q = 0; q < colloc_nq; ++q) v3[((size_t)kind * L + m) * colloc_nq + q] = basis(kind, m, z3[q]);
    }
    const int nq3 = (int)z3.size();
    auto int3 = [&](int ka, int kb, int kc, std::vector<double>& out) {
        out.assign(L * L * L, 0.0);
        double mx = 0;
        auto col3 = [&](int kind, int m) { return &v3[((size_t)kind * L + m) * nq3]; };
        for (int k = 0; k < L; ++k)
            for (int j = 0; j < L; ++j)
                for (int i = 0; i < L; ++i) {
                    if ((basis_odd(ka, i) + basis_odd(kb, j) + basis_odd(kc, k)) & 1) continue;
                    const double *a = col3(ka, i), *b = col3(kb, j), *c = col3(kc, k);
                    long double s = 0;
                    for (int q = 0; q < nq3; ++q) s += (long double)w3[q] * a[q] * b[q] * c[q];
                    out[i + j * L + k * L * L] = (double)s;
                    mx = std::max(mx, std::fabs((double)s));
                }
        // integrals that cancel to quadrature noise are exact zeros
        for (double& e : out)
            if (std::fabs(e) < 1e-13 * mx) e = 0.0;
    };
    int2(0, 3, T.Ia1);
    // Ia2 = int C_i S'_j (penalization terms only), in the closed form that follows from
    // C(+-1/2) = 0, evaluated with the tabulated lambda as the reference does (coeff.cu:143-180):
    // with z = lambda_i / pi and tau = 2 z tan(lambda_i/2) (odd 1-based i) or 2 z cot(lambda_i/2)
    // (even i), Ia2(i, j) = 2 j z^2 tau / (j^4 - z^4) for i, j of opposite parity, else 0.
    T.Ia2.assign(L * L, 0.0);
    for (int i = 0; i < L; ++i) {
        const int mi = i + 1;
        const double li = T.lambda[i], zi = li / kPi, zi2 = zi * zi;
        const double tau = (mi & 1) ? zi * 2.0 * std::tan(0.5 * li) : zi * 2.0 / std::tan(0.5 * li);
        for (int j = 0; j < L; ++j) {
            const int mj = j + 1;
            if ((mi & 1) == (mj & 1)) continue;
            const int j2 = mj * mj;
            T.Ia2[i + j * L] = 2.0 * mj * zi2 * tau / (j2 * j2 - zi2 * zi2);
        }
    }
    T.CS = T.Ia1;
    int2(1, 1, T.CpCp);
    int2(0, 0, T.CC);
    // Iac = int C_i C_j'': the analytic values implied by C = C' = 0 at the walls,
    // evaluated with the tabulated lambda as the reference does (coeff.cu:76-122):
    // t_m = lambda tan(lambda/2) (odd 1-based m) or lambda cot(lambda/2) (even m);
    // diagonal -2t - t^2 (odd) / 2t - t^2 (even); odd-odd off-diagonal
    // 8 l_i^2 l_j^2 (t_j - t_i) / (l_i^4 - l_j^4). Even-even off-diagonal entries are
    // exactly 0 in the reference (its formula subtracts a term from itself,
    // coeff.cu:112); that value is kept so the operators match the reference.
    T.Iac.assign(L * L, 0.0);
    for (int j = 0; j < L; ++j)
        for (int i = 0; i < L; ++i) {
            const int mi = i + 1, mj = j + 1;
            if ((mi & 1) != (mj & 1)) continue;
            const double li = T.lambda[i], lj = T.lambda[j];
            const bool odd = mi & 1;
            const double ti = odd ? li * std::tan(0.5 * li) : li / std::tan(0.5 * li);
            const double tj = odd ? lj * std::tan(0.5 * lj) : lj / std::tan(0.5 * lj);
            if (i == j) T.Iac[i + j * L] = odd ? (-2.0 * ti - ti * ti) : (2.0 * ti - ti * ti);
            else if (odd) {
                const double a = li * li, b = lj * lj;
                T.Iac[i + j * L] = 8.0 * a * b * (tj - ti) / (a * a - b * b);
            }
        }
    // kinds: 0 C, 1 C', 2 C'', 3 S, 4 S'
    int3(1, 1, 3, T.Ibb1);
    int3(1, 3, 3, T.Ib11);
    int3(3, 3, 3, T.I111);
    int3(0, 1, 2, T.Iabc);
    int3(0, 2, 3, T.Iac1);
    int3(0, 0, 1, T.Iaab);
    int3(0, 0, 3, T.Iaa1);
    int3(0, 1, 4, T.Iab2);
    int3(0, 3, 4, T.Ia12);
}

static bool ls_inverse(int nq, int L, const std::vector<double>& B, std::vector<double>& P)
{
    std::vector<double> N((size_t)L * L, 0.0), Ni;
    for (int a = 0; a < L; ++a)
        for (int b = 0; b < L; ++b) {
            long double s = 0;
            for (int q = 0; q < nq; ++q) s += (long double)B[q * L + a] * B[q * L + b];
            N[a * L + b] = (double)s;
        }
    if (!lu_invert(L, N, Ni)) return false;
    P.assign((size_t)L * nq, 0.0);
    for (int m = 0; m < L; ++m)
        for (int q = 0; q < nq; ++q) {
            long double s = 0;
            for (int a = 0; a < L; ++a) s += (long double)Ni[m * L + a] * B[q * L + a];
            P[m * nq + q] = (double)s;
        }
    return true;
}

void colloc_contract_tables(int L, int Q, CollocContract& t)
{
    t.L = L;
    t.Q = Q;
    composite_gl(1, Q, t.z, t.w);
    t.basis.assign((size_t)5 * L * Q, 0.0);
    t.proj.assign((size_t)5 * Q * L, 0.0);
    for (int kind = 0; kind < 5; ++kind)
        for (int i = 0; i < L; ++i)
            for (int q = 0; q < Q; ++q) {
                const double v = basis(kind, i, t.z[q]);
                t.basis[((size_t)kind * L + i) * Q + q] = v;
                t.proj[((size_t)kind * Q + q) * L + i] = t.w[q] * v;
            }
}

bool colloc_tables(int L, int nq, CollocTables& t)
{
    if (L < 1 || nq < L) return false;
    t.L = L;
    t.nq = nq;
    std::vector<double> w;
    composite_gl(1, nq, t.z, w);
    std::sort(t.z.begin(), t.z.end());
    t.C.resize((size_t)nq * L);
    t.Cp.resize((size_t)nq * L);
    t.S.resize((size_t)nq * L);
    for (int q = 0; q < nq; ++q)
        for (int m = 0; m < L; ++m) {
            t.C[q * L + m] = basis(0, m, t.z[q]);
            t.Cp[q * L + m] = basis(1, m, t.z[q]);
            t.S[q * L + m] = basis(3, m, t.z[q]);
        }
    return ls_inverse(nq, L, t.S, t.Ps) && ls_inverse(nq, L, t.C, t.Pc);
}

double family_value(const Tables& T, int f, int i, int j, int k)
{
    using namespace rbcprog;
    switch (f) {
    case IBBB_IJK: return T.ibbb(i, j, k);
    case IBB1_IKJ: return T.t3(T.Ibb1, i, k, j);
    case IB11_KIJ: return T.t3(T.Ib11, k, i, j);
    case IABC_JIK: return T.t3(T.Iabc, j, i, k);
    case IAC1_IKJ: return T.t3(T.Iac1, i, k, j);
    case IAAB_JKI: return T.t3(T.Iaab, j, k, i);
    case IAA1_IKJ: return T.t3(T.Iaa1, i, k, j);
    case IAAB_IJK: return T.t3(T.Iaab, i, j, k);
    case IBB1_IJK: return T.t3(T.Ibb1, i, j, k);
    case IB11_IJK: return T.t3(T.Ib11, i, j, k);
    case I111_IJK: return T.t3(T.I111, i, j, k);
    case IAB2_JIK: return T.t3(T.Iab2, j, i, k);
    case IA12_IJK: return T.t3(T.Ia12, i, j, k);
    default: return T.t3(T.Ia12, i, k, j);
    }
}

void pack_contraction(const Tables& T, std::vector<double>& coef)
{
    using namespace rbcprog;
    const int L = T.L, H = half_len(L);
    coef.assign((size_t)NUNIT * L * L * H, 0.0);
    for (int u = 0; u < NUNIT; ++u) {
        const Unit U = unit_at(u);
        const int par = family_parity(U.family);
        for (int k = 0; k < L; ++k)
            for (int o = 0; o < L; ++o) {
                const int s0 = (o + k + par) & 1;
                for (int h = 0; h < H; ++h) {
                    const int s = s0 + 2 * h;
                    if (s >= L) continue;
                    const int i = U.left ? s : o, j = U.left ? o : s;
                    coef[(((size_t)u * L + k) * L + o) * H + h] = family_value(T, U.family, i, j, k);
                }
            }
    }
}

bool lu_invert(int n, const std::vector<double>& Ain, std::vector<double>& inv)
{
    std::vector<double> A(Ain);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (A[piv * n + c] == 0.0) return false;
        if (piv != c) {
            for (int j = 0; j < n; ++j) std::swap(A[c * n + j], A[piv * n + j]);
            std::swap(perm[c], perm[piv]);
        }
        const double d = A[c * n + c];
        for (int r = c + 1; r < n; ++r) {
            const double l = A[r * n + c] / d;
            A[r * n + c] = l;
            for (int j = c + 1; j < n; ++j) A[r * n + j] -= l * A[c * n + j];
        }
    }
    inv.assign(n * n, 0.0);
    std::vector<double> x(n);
    for (int e = 0; e < n; ++e) {
        for (int i = 0; i < n; ++i) {
            double s = perm[i] == e ? 1.0 : 0.0;
            for (int j = 0; j < i; ++j) s -= A[i * n + j] * x[j];
            x[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = x[i];
            for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * x[j];
            x[i] = s / A[i * n + i];
        }
        for (int i = 0; i < n; ++i) inv[i * n + e] = x[i];
    }
    return true;
}

void grid_info(int nx, int ny, int L, double lx, double ly, double ra, double pr, double dt, GridInfo& g)
{
    g.nx = nx;
    g.ny = ny;
    g.L = L;
    g.mox = nx / 2 + 1;
    g.lx = lx;
    g.ly = ly;
    g.ra = ra;
    g.pr = pr;
    g.dt = dt;
    // 2/3 rule exactly as dealias_implicit (implicit_explicit_stepping.cu:173-180)
    g.ckeep = 0;
    while (g.ckeep < g.mox && !(g.mox - g.ckeep <= (1.0 / 3.0) * g.mox)) ++g.ckeep;
    g.row_kept.assign(ny, 0);
    for (int r = 0; r < ny; ++r) g.row_kept[r] = !(std::fabs(0.5 * ny - r) <= (1.0 / 3.0) * 0.5 * ny);
}

void build_operator_tables(const GridInfo& g, const Tables& T, OperatorTables& op)
{
    const int L = g.L, mox = g.mox, ny = g.ny, n2 = 2 * L;
    op.cls.assign((size_t)ny * mox, -1);
    std::map<uint64_t, int> seen;
    std::vector<double> q2s;
    for (int l = 0; l < ny; ++l) {
        if (!g.row_kept[l]) continue;
        for (int k = 0; k < g.ckeep; ++k) {
            const double mx = k * 2.0 * kPi / g.lx;
            double my = 2.0 * kPi / g.ly;
            if (l < ny / 2 + 1) my *= l;
            else my *= (l - ny);
            const double q2 = mx * mx + my * my;
            uint64_t key;
            std::memcpy(&key, &q2, 8);
            if (k == 0 && l == 0) key = ~0ULL; // the q = 0 mode has its own operator
            auto it = seen.find(key);
            int c;
            if (it == seen.end()) {
                c = (int)q2s.size();
                seen[key] = c;
                q2s.push_back(q2);
            } else {
                c = it->second;
            }
            op.cls[(size_t)l * mox + k] = c;
        }
    }
    op.nclass = (int)q2s.size();
    op.binv.assign((size_t)op.nclass * L * L, 0.0);
    op.imp.assign((size_t)op.nclass * 4 * L * L, 0.0);
    for (const auto& kv : seen) {
        const int c = kv.second;
        const bool zero = kv.first == ~0ULL;
        const double q2 = zero ? 0.0 : q2s[c];
        double* bi = &op.binv[(size_t)c * L * L];
        double* im = &op.imp[(size_t)c * 4 * L * L];
        // B_ff = q^2 (q^2 delta - Iac) / Pr, inverted (inverse_B_matrix.cu:128-141); 0 at q = 0
        if (!zero) {
            std::vector<double> B(L * L), Bi;
            for (int m = 0; m < L; ++m)
                for (int m1 = 0; m1 < L; ++m1)
                    B[m * L + m1] = q2 * (q2 * (m == m1 ? 1.0 : 0.0) - T.Iac[m + m1 * L]) / g.pr;
            lu_invert(L, B, Bi);
            std::memcpy(bi, Bi.data(), sizeof(double) * L * L);
        }
        // (I - dt B^-1 L)^-1 (linear_implicit_operator.cu:60-197)
        std::vector<double> I(n2 * n2, 0.0), Bi2(n2 * n2, 0.0), Lm(n2 * n2, 0.0), C(n2 * n2), M;
        for (int m = 0; m < n2; ++m) I[m * n2 + m] = 1.0;
        if (zero) {
            for (int m = L; m < n2; ++m) I[m * n2 + m] = 0.0;
            for (int m = 0; m < L; ++m) Bi2[m * n2 + m] = 2.0;
        } else {
            std::vector<double> B2(n2 * n2, 0.0);
            for (int m = 0; m < L; ++m) {
                B2[m * n2 + m] = 0.5;
                for (int m1 = 0; m1 < L; ++m1)
                    B2[(m + L) * n2 + m1 + L] = q2 * (q2 * (m == m1 ? 1.0 : 0.0) - T.Iac[m + m1 * L]) / g.pr;
            }
            lu_invert(n2, B2, Bi2);
        }
        for (int m = 0; m < L; ++m)
            for (int m1 = 0; m1 < L; ++m1) {
                const double d = m == m1 ? 1.0 : 0.0;
                const double mp = (m + 1) * kPi;
                const double l4 = std::pow(T.lambda[m], 4.0);
                Lm[m * n2 + m1] = -0.5 * (q2 + mp * mp) * d;
                Lm[m * n2 + m1 + L] = q2 * T.Ia1[m1 + m * L];
                Lm[(m + L) * n2 + m1] = g.ra * q2 * T.Ia1[m + m1 * L];
                Lm[(m + L) * n2 + m1 + L] = -q2 * ((l4 + q2 * q2) * d - 2.0 * q2 * T.Iac[m + m1 * L]);
            }
        for (int a = 0; a < n2; ++a)
            for (int b = 0; b < n2; ++b) {
                double s = 0.0;
                for (int c2 = 0; c2 < n2; ++c2) s += Bi2[a * n2 + c2] * Lm[c2 * n2 + b];
                C[a * n2 + b] = I[a * n2 + b] - g.dt * s;
            }
        if (zero) {
            std::vector<double> up(L * L), upi;
            for (int m = 0; m < L; ++m)
                for (int m1 = 0; m1 < L; ++m1) up[m * L + m1] = C[m * n2 + m1];
            lu_invert(L, up, upi);
            M.assign(n2 * n2, 0.0);
            for (int m = 0; m < L; ++m)
                for (int m1 = 0; m1 < L; ++m1) M[m * n2 + m1] = upi[m * L + m1];
        } else {
            lu_invert(n2, C, M);
        }
        for (int m = 0; m < L; ++m)
            for (int m1 = 0; m1 < L; ++m1) {
                im[0 * L * L + m * L + m1] = M[m * n2 + m1];
                im[1 * L * L + m * L + m1] = M[m * n2 + m1 + L];
                im[2 * L * L + m * L + m1] = M[(m + L) * n2 + m1];
                im[3 * L * L + m * L + m1] = M[(m + L) * n2 + m1 + L];
            }
    }
}

// SplitMix64 (Steele, Lea & Flood, OOPSLA 2014) and Box-Muller.
static inline uint64_t sm64(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static inline double unit_open(uint64_t& s) { return ((sm64(s) >> 11) + 0.5) * 0x1.0p-53; }

void seeded_theta(const GridInfo& g, uint64_t seed, double amp, double kmax, double* th)
{
    const int mox = g.mox, ny = g.ny;
    std::memset(th, 0, sizeof(double) * 2 * (size_t)mox * ny * g.L);
    uint64_t s = seed;
    for (int r = 0; r < ny; ++r) {
        const int rr = r > ny / 2 ? r - ny : r;
        for (int c = 0; c < mox; ++c) {
            if ((double)(c * c + rr * rr) > kmax * kmax) continue;
            const double u1 = unit_open(s), u2 = unit_open(s);
            const double rad = std::sqrt(-2.0 * std::log(u1)), ang = 2.0 * kPi * u2;
            th[2 * ((size_t)r * mox + c)] = amp * rad * std::cos(ang);
            th[2 * ((size_t)r * mox + c) + 1] = amp * rad * std::sin(ang);
        }
    }
    // Hermitian fix on the kx = 0 column (util.cu:184-209) for every mode
    for (int k = 0; k < g.L; ++k) {
        double* a = th + 2 * (size_t)k * mox * ny;
        for (int r = 0; r < ny; ++r) {
            double* e = a + 2 * (size_t)r * mox;
            if (r == 0 || r == ny / 2) e[1] = 0.0;
            else if (r < ny / 2) {
                const double* src = a + 2 * (size_t)(ny - r) * mox;
                e[0] = src[0];
                e[1] = -src[1];
            }
        }
    }
}

void seeded_positions(uint64_t seed, int n, double lx, double ly, double* xyz)
{
    uint64_t s = seed;
    for (int i = 0; i < n; ++i) {
        xyz[i] = lx * unit_open(s);
        xyz[n + i] = ly * unit_open(s);
        xyz[2 * n + i] = unit_open(s) - 0.5;
    }
}

// particle_tracer.cu:58-137 (patterns) and 376-450 (device initialisers); the reference's
// cuRAND draws are replaced by the SplitMix64 stream of `seed`.
void tracer_pattern(int type, uint64_t seed, int n, double lx, double ly, double cx, double cy, double cz,
                    double sigma, double* xyz)
{
    double* x = xyz;
    double* y = xyz + n;
    double* z = xyz + 2 * (size_t)n;
    uint64_t s = seed;
    auto normal = [&s]() {
        const double u1 = unit_open(s), u2 = unit_open(s);
        return std::cos(2.0 * kPi * u2) * std::sqrt(-2.0 * std::log(u1));
    };
    switch (type) {
    case 0: // random
        seeded_positions(seed, n, lx, ly, xyz);
        return;
    case 3: // diagonal
        for (int i = 0; i < n; ++i) {
            x[i] = (lx * i) / (double)n;
            y[i] = (ly * i) / (double)n;
            z[i] = 0.0;
        }
        return;
    case 4: // pairs
        for (int i = 0; i + 1 < n; i += 2) {
            const double px = lx * unit_open(s), py = ly * unit_open(s);
            x[i] = x[i + 1] = px;
            y[i] = y[i + 1] = py;
            z[i] = z[i + 1] = 0.0;
        }
        return;
    default: break;
    }
    // center, center_sigma, coord_sigma: a point, then sigma N(0,1) per coordinate
    if (type == 1 || type == 2) { cx = 0.5 * lx; cy = 0.5 * ly; cz = 0.0; }
    if (type == 1) sigma = 0.0;
    for (int i = 0; i < n; ++i) {
        x[i] = cx;
        y[i] = cy;
        z[i] = cz;
        if (sigma > 0.0) {
            x[i] += sigma * normal();
            y[i] += sigma * normal();
            z[i] += sigma * normal();
        }
    }
}

// ------------------------------------------------------------------ pattern init
typedef std::complex<double> cplx;

// Recursive mixed-radix (2, 3) DFT, y[k] = sum_j x[j s] exp(-2 pi i j k / n); twiddles
// from long double.
static void dft23(const cplx* x, int s, int n, cplx* y)
{
    if (n == 1) {
        y[0] = x[0];
        return;
    }
    const int r = (n % 2 == 0) ? 2 : 3, m = n / r;
    for (int p = 0; p < r; ++p) dft23(x + (size_t)p * s, s * r, m, y + (size_t)p * m);
    cplx t[3], u[3];
    for (int k = 0; k < m; ++k) {
        for (int p = 0; p < r; ++p) {
            const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)(p * k) / n;
            t[p] = y[(size_t)p * m + k] * cplx((double)std::cos(a), (double)std::sin(a));
        }
        for (int q = 0; q < r; ++q) {
            cplx acc = 0;
            for (int p = 0; p < r; ++p) {
                const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)(p * q) / r;
                acc += t[p] * cplx((double)std::cos(a), (double)std::sin(a));
            }
            u[q] = acc;
        }
        for (int q = 0; q < r; ++q) y[k + (size_t)q * m] = u[q];
    }
}

void rfft2(int nx, int ny, const double* real, double* out)
{
    const int mox = nx / 2 + 1;
    std::vector<cplx> row(nx), rowo(nx), half((size_t)ny * mox), col(ny), colo(ny);
    for (int y = 0; y < ny; ++y) {
        for (int x = 0; x < nx; ++x) row[x] = real[(size_t)y * nx + x];
        dft23(row.data(), 1, nx, rowo.data());
        for (int c = 0; c < mox; ++c) half[(size_t)y * mox + c] = rowo[c];
    }
    for (int c = 0; c < mox; ++c) {
        for (int y = 0; y < ny; ++y) col[y] = half[(size_t)y * mox + c];
        dft23(col.data(), 1, ny, colo.data());
        for (int y = 0; y < ny; ++y) {
            out[2 * ((size_t)y * mox + c)] = colo[y].real();
            out[2 * ((size_t)y * mox + c) + 1] = colo[y].imag();
        }
    }
}

// Real-space patterns of matrix_device_init (gpu_flow/code/util/init.cu:22-261) on the
// Nx x Ny grid of the unit square, in FP64. `mode` is passed to the reference's int
// parameter, so it is truncated; the rectangle pattern takes x_mode from Lx and Nx as
// main.cu:330 does; sv and cr use x_frac 0.2 and 0.8 (main.cu:339-342). The reference's
// rand() draws (rectangle noise strip, isr phase) come from the SplitMix64 stream.
static void pattern_real(const GridInfo& g, int type, double mode, double amp, uint64_t& s, std::vector<double>& v)
{
    const int nx = g.nx, ny = g.ny;
    const double PI = kPi;
    v.assign((size_t)nx * ny, 0.0);
    const int im = (int)mode;
    auto at = [&](int i, int j) -> double& { return v[(size_t)j * nx + i]; };
    switch (type) {
    case 1: { // isr (init.cu:102-128)
        const double phase = 2 * PI * unit_open(s);
        const double dx = double(im) / nx, dy = 0.0 / ny;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) at(i, j) = amp * std::cos(2.0 * PI * (i * dx + j * dy) + phase);
        break;
    }
    case 2: { // dislocation (init.cu:22-67), y_mode 0
        const double dx = 1.0 / nx, dy = 1.0 / ny;
        const double x1 = (nx / 2.0) * dx + dx / 2.0, x2 = x1;
        const double y1 = (ny / 4.0) * dy + dy / 2.0, y2 = (3.0 * ny / 4.0) * dy + dy / 2.0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double p1 = std::atan2(j * dy - y1, i * dx - x1), p2 = std::atan2(j * dy - y2, i * dx - x2);
                at(i, j) = amp * std::cos(im * 2.0 * PI * (i * dx) + 0 * 2.0 * PI * (j * dy) - p1 + p2);
            }
        break;
    }
    case 3: { // rectangle (init.cu:69-100) with x_mode = (Lx / (Nx - 1)) (Nx - 5) / 2 (main.cu:330)
        const int xm = (int)((g.lx / (nx - 1.0)) * (nx - 5.0) / 2.0);
        const double dx = double(xm) / nx, dy = 0.0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                at(i, j) = (i < nx / 8) ? (2.0 * unit_open(s) - 1.0) * amp : amp * std::cos(2.0 * PI * (i * dx + j * dy));
        break;
    }
    case 4: { // sv (init.cu:130-163), x_frac 0.2
        const double x_frac = 0.2, dy = double(im) / ny;
        const double xl = 0.5 * (1.0 - x_frac), xr = 1.0 - xl;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double x = i / double(nx), y = j / double(ny);
                double ph = -0.5 * std::sin(2 * PI * y) - x * x;
                if (x > xr) ph += 1.0;
                else if (x > xl) ph += 0.5 * (1.0 - std::cos(PI * (x - xl) / x_frac));
                at(i, j) = amp * std::cos(2.0 * PI * (j * dy + ph));
            }
        break;
    }
    case 5: { // cr (init.cu:165-207), x_frac 0.8
        const double x_frac = 0.8, dx = 1.0 / nx, dy = 1.0 / ny;
        const double x1 = 0.5 * ((1.0 - x_frac) * nx + 1) * dx, x2 = 1.0 - x1;
        const double y1 = 0.5 * (ny + 1) * dy, y2 = y1;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double p1 = std::atan2(j * dy - y1, i * dx - x1), p2 = std::atan2(j * dy - y2, i * dx - x2);
                at(i, j) = amp * std::cos(im * 2.0 * PI * (j * dy) - p1 + p2);
            }
        break;
    }
    case 6: { // giantspiral (init.cu:209-248)
        const double dx = 1.0 / nx, dy = 1.0 / ny;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double ax = i * dx - 0.5, ay = j * dy - 0.5, bx = i * dx - 0.8, by = j * dy - 0.5;
                const double r = std::sqrt(ax * ax + ay * ay);
                at(i, j) = amp * std::cos(2.0 * PI * im * r - std::atan2(ay, ax) + std::atan2(by, bx));
            }
        break;
    }
    default: break;
    }
}

void pattern_theta(const GridInfo& g, int type, double mode, double amp, uint64_t seed, double noise, double* theta,
                   double* f, double* F)
{
    const int mox = g.mox, ny = g.ny, L = g.L;
    const size_t plane = (size_t)mox * ny;
    std::memset(theta, 0, sizeof(double) * 2 * plane * L);
    uint64_t s = seed;
    if (type == 7) {
        // init_test (init.cu:250-310): row 0, columns c > 0 of every mode get amp sin(c)
        // in f and theta; F_k = amp cos(k)
        std::memset(f, 0, sizeof(double) * 2 * plane * L);
        for (int k = 0; k < L; ++k) {
            for (int c = 1; c < mox; ++c) {
                theta[2 * ((size_t)k * plane + c)] = amp * std::sin((double)c);
                f[2 * ((size_t)k * plane + c)] = amp * std::sin((double)c);
            }
            F[2 * k] = amp * std::cos((double)k);
            F[2 * k + 1] = 0.0;
        }
    } else {
        std::vector<double> v;
        pattern_real(g, type, mode, amp, s, v);
        rfft2(g.nx, ny, v.data(), theta);
        // modes k >= 1: uniform noise in [-noise, noise) (init_random, init.cu:350-365)
        if (noise > 0)
            for (int k = 1; k < L; ++k)
                for (size_t e = 0; e < plane; ++e) {
                    theta[2 * ((size_t)k * plane + e)] = noise * (2.0 * unit_open(s) - 1.0);
                    theta[2 * ((size_t)k * plane + e) + 1] = noise * (2.0 * unit_open(s) - 1.0);
                }
    }
    // Hermitian fix on the kx = 0 column (make_real_signal, util.cu:184-224)
    auto fix = [&](double* a) {
        for (int k = 0; k < L; ++k) {
            double* b = a + 2 * (size_t)k * plane;
            for (int r = 0; r < ny; ++r) {
                double* e = b + 2 * (size_t)r * mox;
                if (r == 0 || r == ny / 2) e[1] = 0.0;
                else if (r < ny / 2) {
                    const double* src = b + 2 * (size_t)(ny - r) * mox;
                    e[0] = src[0];
                    e[1] = -src[1];
                }
            }
        }
    };
    fix(theta);
    if (type == 7) fix(f);
}

} // namespace rbchost
