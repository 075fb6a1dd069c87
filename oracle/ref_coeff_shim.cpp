// Test-only shim: exposes the reference's own Galerkin coefficient class
// (gpu_flow/code/util/coeff.{h,cu}, compiled from the reference sources in place)
// through a C ABI so the oracle's quadrature tables can be pinned against it.
// Built into oracle/_ref/ by oracle/build_ref.sh; never linked by the product.
#include "coeff.h"
#include <cstring>

extern "C" {

// Fill out[] with one table of the reference Coeff<double>(moz).
// name: "Iac","Ia1" (moz*moz, index i+j*moz) or a 3-index getter name
// ("Ibbb","Ibb1","Ib11","I111","Iabc","Iac1","Iaab","Iaa1","Iab2","Ia12",
//  "Ia11","Iaad") with index i+j*moz+k*moz*moz. "lambda" gives lambda(1..moz).
// Returns the number of values written, or -1 for an unknown name.
int ref_coeff_table(int moz, const char* name, double* out)
{
    Coeff<double> c(moz);
    const int n = moz;
    if (!strcmp(name, "lambda")) {
        for (int i = 0; i < n; ++i) out[i] = c.lambda(i + 1);
        return n;
    }
    if (!strcmp(name, "Iac") || !strcmp(name, "Ia1") || !strcmp(name, "Iab") || !strcmp(name, "Ia2")) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double v = 0;
                if (!strcmp(name, "Iac")) v = c.Iac(i, j);
                else if (!strcmp(name, "Ia1")) v = c.Ia1(i, j);
                else if (!strcmp(name, "Iab")) v = c.Iab(i, j);
                else v = c.Ia2(i, j);
                out[i + j * n] = v;
            }
        return n * n;
    }
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double v;
                if (!strcmp(name, "Ibbb")) v = c.Ibbb(i, j, k);
                else if (!strcmp(name, "Ibb1")) v = c.Ibb1(i, j, k);
                else if (!strcmp(name, "Ib11")) v = c.Ib11(i, j, k);
                else if (!strcmp(name, "I111")) v = c.I111(i, j, k);
                else if (!strcmp(name, "Iabc")) v = c.Iabc(i, j, k);
                else if (!strcmp(name, "Iac1")) v = c.Iac1(i, j, k);
                else if (!strcmp(name, "Iaab")) v = c.Iaab(i, j, k);
                else if (!strcmp(name, "Iaa1")) v = c.Iaa1(i, j, k);
                else if (!strcmp(name, "Iab2")) v = c.Iab2(i, j, k);
                else if (!strcmp(name, "Ia12")) v = c.Ia12(i, j, k);
                else if (!strcmp(name, "Ia11")) v = c.Ia11(i, j, k);
                else if (!strcmp(name, "Iaad")) v = c.Iaad(i, j, k);
                else return -1;
                out[i + j * n + k * n * n] = v;
            }
    return n * n * n;
}

}
