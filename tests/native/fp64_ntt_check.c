// Test of the arithmetic of the forward NTT's FP64 butterflies (shmoai_b200/csrc/ntt.cuh: ct_bf_dbl,
// dbl_centre, the kBfF64 and kBfF64R passes) restated with IEEE double fma / add / mul, the
// operations the GPU code uses (__fma_rn, __dadd_rn, __dmul_rn; compiled without contraction), against
// exact integer arithmetic: all 16 Cooley-Tukey stages on N = 2^16 with random twiddles, at primes at
// the edges of each family.  It also counts every quotient outside the range in which the rounding
// through 1.5 2^52 is exact and every value at or above 2^53.  Exit status 0 when all match.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
#define N (1 << 16)
static uint64_t rng = 88172645463325252ull;
static uint64_t xs(void) { rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17; return rng; }

static double centre(double v, double q, double qinv) {
    const double magic = 6755399441055744.0;
    double Q = (fma(v, qinv, magic)) - magic;
    return fma(-Q, q, v);
}
static int bad_range = 0;
static void bf_dbl(double *x, double *y, double w, double wq, double q) {
    const double magic = 6755399441055744.0;
    double z = *y * wq;  // only for the range check
    if (fabs(z) >= 2251799813685248.0) bad_range++;
    double Q = fma(*y, wq, magic) - magic;
    double hi = *y * w;
    double lo = fma(*y, w, -hi);
    double t = fma(-Q, q, hi) + lo;
    double a = *x;
    *x = a + t;
    *y = a - t;
    if (fabs(*x) >= 9007199254740992.0 || fabs(*y) >= 9007199254740992.0) bad_range++;
}

int run(uint64_t q, int centred) {
    static uint64_t a[N], w[N];
    static double d[N], wd[N], wq[N];
    const double qd = (double)q, qinv = 1.0 / qd;
    for (int i = 0; i < N; i++) {
        a[i] = xs() % q;
        w[i] = xs() % q;
        d[i] = (double)a[i];
        // the centred family keeps its twiddles within q/2 of zero
        wd[i] = centred && w[i] > q / 2 ? (double)w[i] - qd : (double)w[i];
        wq[i] = wd[i] / qd;
    }
    if (centred) for (int i = 0; i < N; i++) d[i] = centre(d[i], qd, qinv);
    double maxabs = 0;
    for (int s = 0; s < 16; s++) {
        int m = 1 << s, t = N >> (s + 1);
        for (int i = 0; i < m; i++) {
            uint64_t W = w[m + i - (m + i >= N ? N : 0)];
            double Wd = wd[m + i - (m + i >= N ? N : 0)], Wq = wq[m + i - (m + i >= N ? N : 0)];
            for (int j = 2 * i * t; j < 2 * i * t + t; j++) {
                uint64_t x = a[j], y = (uint64_t)(((u128)a[j + t] * W) % q);
                a[j] = (x + y) % q;
                a[j + t] = (x + q - y) % q;
                if (centred && (s & 3) == 3) d[j + t] = centre(d[j + t], qd, qinv);  // a pass's fourth stage
                bf_dbl(&d[j], &d[j + t], Wd, Wq, qd);
                if (fabs(d[j]) > maxabs) maxabs = fabs(d[j]);
                if (fabs(d[j + t]) > maxabs) maxabs = fabs(d[j + t]);
            }
        }
        if (centred && (s & 3) == 3) for (int k = 0; k < N; k++) d[k] = centre(d[k], qd, qinv);
    }
    int bad = 0;
    for (int k = 0; k < N; k++) {
        double v = d[k];
        double Q = fma(v, qinv, 6755399441055744.0) - 6755399441055744.0;
        double r = fma(-Q, qd, v);
        if (r < 0) r += qd;
        if ((uint64_t)r != a[k]) bad++;
    }
    printf("q=%llu (2^%.3f) %s: mismatches %d, range violations %d, max |v| / q = %.2f\n", (unsigned long long)q,
           log2((double)q), centred ? "centred" : "plain  ", bad, bad_range, maxabs / qd);
    bad_range = 0;
    return bad;
}

int main(void) {
    int bad = 0;
    const uint64_t lim = (1ull << 52) / 36;
    bad += run(lim - 1 - ((lim - 1) % 2 == 0), 0);
    bad += run((1ull << 46) - (1ull << 17) + 1, 0);
    bad += run((1ull << 51) - 1, 1);
    bad += run((1ull << 51) - (1ull << 17) * 3 + 1, 1);
    bad += run((1ull << 50) + (1ull << 17) + 1, 1);
    bad += run(lim + 1 + (lim % 2), 1);
    printf(bad ? "FAIL\n" : "OK\n");
    return bad != 0;
}
