// The branch-free reciprocal of the FP64 kernels (recip_rn_fast in
// joint_bp_plus_pp_b200/csrc/kernels_bp.cuh) against IEEE division: from a starting
// approximation y0 of 1/s with relative error up to 2^-16 (the device starts from the hardware
// approximation rcp.approx.ftz.f64, measured within 2^-19.9), two Newton steps
// y <- fma(y, fma(-s, y, 1), y) and the final choice between y and its two neighbours by the
// exact remainder 1 - s y must give 1.0 / s (x86 SSE2 divsd, correctly rounded) for every s of
// the fast path's domain [2^-900, 2^900]: random significands, all-ones significands, powers of
// two and their neighbours, each from several starting errors (both signs, the extremes).
//
//     reciprocal_rn_check N lo hi    (N divisors, exponents in [lo, hi]); exit 0 = all equal
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t st = 0x9E3779B97F4A7C15ull;
static uint64_t xr(void) { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return st; }
static double bits(uint64_t b) { double d; memcpy(&d, &b, 8); return d; }
static uint64_t ubits(double d) { uint64_t b; memcpy(&b, &d, 8); return b; }

static double recip_seq(double s, double y) {
    double e;
    e = fma(-s, y, 1.0); y = fma(y, e, y);
    e = fma(-s, y, 1.0); y = fma(y, e, y);
    const double r = fma(-s, y, 1.0);
    const uint64_t yb = ubits(y);
    const double ulp = bits((yb & 0x7FF0000000000000ull) - (52ull << 52));
    const int pow2 = (yb & 0x000FFFFFFFFFFFFFull) == 0;
    const double t_up = s * ulp * 0.5;
    const double t_dn = pow2 ? t_up * 0.5 : t_up;
    if (r > t_up) return bits(yb + 1);
    if (r < -t_dn) return bits(yb - 1);
    return y;
}

static long long bad = 0, tot = 0;

static void one(double s) {
    const double want = 1.0 / s;
    static const double starts[] = {0.0, 0x1p-16, -0x1p-16, 0x1p-30, -0x1p-30, 0x1p-52, -0x1p-52};
    for (int k = 0; k < 8; ++k) {
        const double d = k < 7 ? starts[k] : ((double)(xr() >> 11) * 0x1.0p-53 * 2.0 - 1.0) * 0x1p-16;
        const double y0 = want * (1.0 + d);
        const double got = recip_seq(s, y0);
        tot++;
        if (ubits(got) != ubits(want)) {
            if (bad < 10) printf("mismatch s=%a y0=%a got %a want %a\n", s, y0, got, want);
            bad++;
        }
    }
}

int main(int argc, char **argv) {
    const long long N = argc > 1 ? atoll(argv[1]) : 10000000LL;
    const int lo = argc > 2 ? atoi(argv[2]) : -900, hi = argc > 3 ? atoi(argv[3]) : 899;
    for (long long i = 0; i < N; ++i) {
        const int e = lo + (int)(xr() % (uint64_t)(hi - lo + 1));
        const uint64_t ex = (uint64_t)(e + 1023) << 52;
        switch (i & 7) {
        case 0: one(bits(ex | ((1ull << 52) - 1))); break;                 // all-ones significand
        case 1: one(bits(ex)); break;                                        // power of two
        case 2: one(bits(ex | 1)); break;                                    // just above it
        case 3: one(bits(ex | ((1ull << 52) - 1 - (xr() & 0xFFFF)))); break; // near all ones
        default: one(bits(ex | (xr() & ((1ull << 52) - 1)))); break;        // random significand
        }
    }
    printf("divisors %lld cases %lld mismatches %lld (exponents in [%d, %d])\n", N, tot, bad, lo, hi);
    return bad != 0;
}
