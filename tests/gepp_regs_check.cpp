// Host check of the register GEPP of the Newton fast path (gepp_regs, row
// swaps as bitwise blends) against the full-matrix GEPP of the generic path
// (gepp_full, the statement-by-statement form of SourceStep.hpp:211-242), on
// seeded random systems whose pivot searches swap rows.  Built and run by
// tests/test_gepp_regs.py; prints "swaps <n> singular <n> systems <n>" and
// exits 0 when every solution agrees bit for bit.
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "gepp_regs.h"

namespace {

uint64_t state = 0x9e3779b97f4a7c15ull;
double uniform() {   // xorshift64*, in [-1, 1)
    state ^= state >> 12;
    state ^= state << 25;
    state ^= state >> 27;
    const uint64_t v = state * 0x2545f4914f6cdd1dull;
    return (double)(v >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

bool same(double a, double b) { return std::memcmp(&a, &b, sizeof a) == 0; }

template <int NB>
int check(int systems, long& swaps, long& singular) {
    for (int s = 0; s < systems; ++s) {
        double A[NB][NB], b[NB], x[NB], J[NB * NB], bv[NB], xv[NB];
        const int kind = s % 4;   // 0, 1: dense; 2: diagonally dominant; 3: a zero or tiny column
        const int zc = s % NB;
        for (int i = 0; i < NB; ++i) {
            for (int j = 0; j < NB; ++j) {
                double v = uniform();
                if (kind == 2 && i == j) v += 4.0;
                if (kind == 3 && j == zc) v = (s / 4) % 2 ? 0.0 : 1e-16 * v;
                A[i][j] = v;
                J[i * NB + j] = v;
            }
            b[i] = bv[i] = uniform();
            x[i] = xv[i] = 0.0;
        }
        for (int k = 0; k < NB; ++k) {   // count the pivot searches that pick another row
            int mr = k;
            for (int i = k + 1; i < NB; ++i)
                if (std::fabs(J[i * NB + k]) > std::fabs(J[mr * NB + k])) mr = i;
            swaps += mr != k;
            break;
        }
        const bool ok_r = zsme::gepp_regs<NB>(A, b, x);
        const bool ok_f = zsme::gepp_full<NB>(J, bv, xv);
        if (!ok_f) {
            ++singular;
            if (ok_r) {
                std::printf("NB %d system %d: register form missed a small pivot\n", NB, s);
                return 1;
            }
            continue;
        }
        if (!ok_r) {
            std::printf("NB %d system %d: register form flagged a pivot the full form took\n", NB, s);
            return 1;
        }
        for (int i = 0; i < NB; ++i)
            if (!same(x[i], xv[i])) {
                std::printf("NB %d system %d: x[%d] %.17g vs %.17g\n", NB, s, i, x[i], xv[i]);
                return 1;
            }
    }
    return 0;
}

}  // namespace

// blend moves bits: NaN payloads, signed zeros and infinities come through
int check_blend() {
    const uint64_t pats[] = {0x7ff8000000000123ull, 0xfff0000000000001ull, 0x8000000000000000ull, 0ull,
                             0x7ff0000000000000ull, 0xfff0000000000000ull, 0x0000000000000001ull,
                             0x3ff0000000000000ull};
    for (uint64_t a : pats)
        for (uint64_t b : pats) {
            double da, db;
            std::memcpy(&da, &a, 8);
            std::memcpy(&db, &b, 8);
            const double r1 = zsme::blend(true, da, db), r0 = zsme::blend(false, da, db);
            uint64_t u1, u0;
            std::memcpy(&u1, &r1, 8);
            std::memcpy(&u0, &r0, 8);
            if (u1 != a || u0 != b) {
                std::printf("blend %016llx %016llx\n", (unsigned long long)a, (unsigned long long)b);
                return 1;
            }
        }
    return 0;
}

int main() {
    if (check_blend()) return 1;
    long swaps = 0, singular = 0;
    const int n = 20000;
    if (check<2>(n, swaps, singular) || check<3>(n, swaps, singular) || check<4>(n, swaps, singular) ||
        check<5>(n, swaps, singular) || check<6>(n, swaps, singular))
        return 1;
    std::printf("swaps %ld singular %ld systems %d\n", swaps, singular, 5 * n);
    return 0;
}
