// Host check of the storage-shift table (make_shift in mt_lattice.cuh):
// s_k = feq_k(1, u_s) sums to 1, its first moment is u_s, u_s = 0 gives the
// weights exactly, and the FP32 / difference tables are the FP64 values
// rounded once.
#define MT_HD inline
#include <cmath>
#include <cstdio>
#include <initializer_list>

#include "../../mortontrie_amr_b200/csrc/mt_lattice.cuh"

using namespace mt;

static int fails = 0;
static void check(bool ok, const char *what, int q, double a, double b)
{
    if (!ok) {
        std::printf("FAIL %s q=%d %.17g %.17g\n", what, q, a, b);
        ++fails;
    }
}

int main()
{
    const double us[4][3] = {{0, 0, 0}, {0.1, 0, 0}, {0.04, -0.02, 0.01}, {-0.3, 0.2, 0.1}};
    for (int q : {19, 27}) {
        for (const auto &u : us) {
            const Shift s = make_shift(q, u);
            double m0 = 0, m1[3] = {0, 0, 0};
            for (int k = 0; k < q; ++k) {
                const double wk = q == 19 ? w<19>(k) : w<27>(k);
                m0 += s.d[k];
                m1[0] += ex(k) * s.d[k];
                m1[1] += ey(k) * s.d[k];
                m1[2] += ez(k) * s.d[k];
                check(s.v[k] == (float)s.d[k], "v is d rounded", q, s.v[k], s.d[k]);
                check(s.dw[k] == (float)(s.d[k] - wk) || std::fabs(s.dw[k] - (s.d[k] - wk)) <= 1e-7 * wk,
                      "dw is d - w", q, s.dw[k], s.d[k] - wk);
                if (u[0] == 0 && u[1] == 0 && u[2] == 0) {
                    check(s.d[k] == wk, "zero shift is w", q, s.d[k], wk);
                    check(s.dw[k] == 0.0f, "zero shift dw", q, s.dw[k], 0);
                }
            }
            check(std::fabs(m0 - 1.0) < 1e-14, "sum", q, m0, 1.0);
            for (int a = 0; a < 3; ++a) check(std::fabs(m1[a] - u[a]) < 1e-14, "first moment", q, m1[a], u[a]);
            for (int a = 0; a < 3; ++a) check(s.u[a] == (float)u[a], "u", q, s.u[a], u[a]);
        }
    }
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
