// CPU check of the collocation form's program (colloc_prog.h) and tables: on random point
// values of the 8 synthesised fields, the level products (synthesis on Q Gauss-Legendre
// levels, the 41 products, projection with the weighted basis) must equal the exact
// contraction program (contract_prog.h) evaluated with the Q-level tensors of
// rbchost::build_tables(L, T, Q). Prints the largest relative difference over the 13 groups.
// Built and run by tests/test_colloc_cpu.py.
#include "colloc_prog.h"
#include "galerkin.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

int main(int argc, char** argv)
{
    const int L = argc > 1 ? std::atoi(argv[1]) : 8, Q = argc > 2 ? std::atoi(argv[2]) : 16;
    rbchost::Tables T;
    rbchost::build_tables(L, T, Q);
    rbchost::CollocContract C;
    rbchost::colloc_contract_tables(L, Q, C);
    std::mt19937_64 rng(7);
    std::normal_distribution<double> N01;
    double worst = 0.0;
    for (int pt = 0; pt < 20; ++pt) {
        std::vector<double> a(8 * L);
        for (double& v : a) v = N01(rng);
        // exact program with the Q-level tensors
        std::vector<double> ex(rbcprog::NGROUP * L, 0.0);
        for (int u = 0; u < rbcprog::NUNIT; ++u) {
            const rbcprog::Unit un = rbcprog::unit_at(u);
            for (int e = 0; e < un.nedge; ++e)
                for (int k = 0; k < L; ++k) {
                    double s = 0.0;
                    for (int i = 0; i < L; ++i)
                        for (int j = 0; j < L; ++j) {
                            const double t = rbchost::family_value(T, un.family, i, j, k);
                            const double ai = un.left == 0 ? a[un.e[e].other * L + i] : a[un.fixed * L + i];
                            const double bj = un.left == 0 ? a[un.fixed * L + j] : a[un.e[e].other * L + j];
                            s += t * ai * bj;
                        }
                    ex[un.e[e].group * L + k] += un.e[e].weight * s;
                }
        }
        // level products
        std::vector<double> co(rbcprog::NGROUP * L, 0.0);
        for (int q = 0; q < Q; ++q) {
            double S[rbccol::NSPAIR], G[rbccol::NPPAIR] = {0};
            for (int p = 0; p < rbccol::NSPAIR; ++p) {
                const rbccol::SPair sp = rbccol::spair_at(p);
                double v = 0.0;
                for (int i = 0; i < L; ++i) v += C.basis[((size_t)sp.kind * L + i) * Q + q] * a[sp.field * L + i];
                S[p] = v;
            }
            for (int n = 0; n < rbccol::NPROD; ++n) {
                const rbccol::Prod pr = rbccol::prod_at(n);
                G[pr.to] += pr.weight * S[pr.a] * S[pr.b];
            }
            for (int p = 0; p < rbccol::NPPAIR; ++p) {
                const rbccol::PPair pp = rbccol::ppair_at(p);
                for (int k = 0; k < L; ++k) co[pp.group * L + k] += C.proj[((size_t)pp.kind * Q + q) * L + k] * G[p];
            }
        }
        for (int g = 0; g < rbcprog::NGROUP; ++g) {
            double num = 0.0, den = 0.0;
            for (int k = 0; k < L; ++k) {
                num = std::fmax(num, std::fabs(co[g * L + k] - ex[g * L + k]));
                den = std::fmax(den, std::fabs(ex[g * L + k]));
            }
            if (den > 0) worst = std::fmax(worst, num / den);
        }
    }
    std::printf("%.3e\n", worst);
    return 0;
}
