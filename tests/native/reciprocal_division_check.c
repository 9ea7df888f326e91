// The division sequence of norm4 (joint_bp_plus_pp_b200/csrc/kernels_bp.cuh: recip_for_div,
// div_by_recip) against IEEE division: y = RN(1/s), q = RN(m y), r = fma(-s, q, m),
// q' = fma(r, y, q) must equal m / s (x86 SSE2 divsd, correctly rounded) for every pair the
// kernel sends down that path -- 0 <= m <= s with m >= 2^-900 and s <= 2^900 -- including
// divisors with all-ones significands, m = s, m just below s and m at the 2^-900 edge.  Pairs
// outside the guard, which the kernel divides directly, are counted as skipped.
//
//     reciprocal_division_check N lo hi    (N pairs, exponents of s in [lo, hi]); exit 0 = all equal
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t st = 88172645463325252ull;
static uint64_t xr(void) { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return st; }
static double bits(uint64_t b) { double d; memcpy(&d, &b, 8); return d; }

static long long bad = 0, tot = 0, skipped = 0;

static void one(double m, double s) {
    if (!(m >= 0x1p-900 && s <= 0x1p900)) { skipped++; return; }   // the kernel divides directly
    const double y = 1.0 / s;
    const double q = m * y;
    const double r = fma(-s, q, m);
    const double q2 = fma(r, y, q);
    const double t = m / s;
    tot++;
    if (memcmp(&q2, &t, 8) != 0) {
        if (bad < 10) printf("mismatch m=%a s=%a got %a want %a\n", m, s, q2, t);
        bad++;
    }
}

int main(int argc, char **argv) {
    const long long N = argc > 1 ? atoll(argv[1]) : 100000000LL;
    const int lo = argc > 2 ? atoi(argv[2]) : -960, hi = argc > 3 ? atoi(argv[3]) : 900;
    for (long long i = 0; i < N; ++i) {
        const int e = lo + (int)(xr() % (uint64_t)(hi - lo + 1));
        const double s = bits(((uint64_t)(e + 1023) << 52) | (xr() & ((1ull << 52) - 1)));
        double m;
        switch (i & 7) {
        case 0: m = s; break;
        case 1: m = s * bits(0x3ff0000000000000ull | (xr() & ((1ull << 52) - 1))) * 0.5; break;   // [s/2, s)
        case 2: m = nextafter(s, 0.0); break;
        case 3: m = ldexp(s, -(int)(xr() % 60)) * bits(0x3ff0000000000000ull | (xr() & 0xfffffffffffffull)) * 0.5; break;
        case 6: m = ldexp(bits(0x3ff0000000000000ull | (xr() & 0xfffffffffffffull)), -900 + (int)(xr() % 8)); break;
        default: m = s * ((double)(xr() >> 11) * 0x1.0p-53); break;   // uniform in [0, s)
        }
        if (m > s) m = s;
        one(m, s);
        if ((i & 1023) == 0) {   // all-ones significands of s
            const double s1 = bits(((uint64_t)(e + 1023) << 52) | ((1ull << 52) - 1));
            one(s1 * ((double)(xr() >> 11) * 0x1.0p-53), s1);
            one(nextafter(s1, 0.0), s1);
        }
    }
    printf("skipped %lld pairs %lld mismatches %lld (exponents of s in [%d, %d])\n", skipped, tot, bad, lo, hi);
    return bad != 0;
}
