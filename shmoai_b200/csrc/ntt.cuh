// Batched negacyclic NTT / INTT over RNS limbs.
//
// Definition (bit-identical to the reference, thirdparty/phantom-fhe/src/ntt/fntt_2d.cu
// and intt_2d.cu): forward = Cooley-Tukey with root_powers[bitrev(i)] = psi^i, natural
// order in, bit-reversed order out, fully reduced to [0, q); inverse = Gentleman-Sande
// with psi^-i, including N^-1.
//
// Decomposition: N = M * M (M = 2^(2R)).  The first log M forward stages only
// combine elements of one "column" {c + M*p : p < M}; the last log M stages only
// combine elements of one contiguous "block" {b*M + p : p < M}.  Each phase is one
// kernel in which a CTA owns S columns (or S blocks) of one limb (S = 16 or 8, the tile
// variant); a thread owns 2^R elements and runs R radix-2 stages in registers, twice, with
// one shared-memory exchange in between.  Global loads and stores move S consecutive words
// per column row / per block segment (128 bytes at S = 16).  Values between the two
// phases are lazy: below 36q (grow butterflies, q < 2^57), in [0, 4q) (Harvey), or signed
// doubles below 7q in magnitude (the forward's FP64 butterflies, q < 2^52 / 36).
//
// The inverse's last stage folds a per-limb scale c (N^-1, or N^-1 times the
// ModUp digit factor) into both outputs: (X+Y)*c and (X-Y)*psi^-(N/2)*c.
#pragma once
#include <cstdint>

#include "modarith.cuh"

namespace shm {

// Tile variants of the NTT kernels (columns or blocks per CTA, minimum resident CTAs per SM,
// which caps the registers a thread may use); the autotuner picks one per context.
struct NttVariant {
    int subs, min_blocks;
};
constexpr NttVariant kNttVariants[] = {{16, 4}, {16, 3}, {8, 8}, {8, 6}};
constexpr int kNttVariantCount = 4;

struct LimbMap {
    uint8_t prime[512];  // limb slot within a polynomial -> prime index; 255 = leave untouched
};

// The rescale's forward NTT (ntt_forward_rescale): rows (poly, j < L-1) are read as
// last[poly] mod q_j and written as (in[poly][j] - NTT(...)) * q_{L-1}^-1 into out[poly][j]
struct RescaleIO {
    const uint64_t *last = nullptr;  // [polys][N], c_{L-1} in coefficient form
    const uint64_t *in = nullptr;    // [polys][L][N]
    uint64_t *out = nullptr;         // [polys][L-1][N]
    const uint64_t *inv = nullptr;   // [L-1][2]: q_{L-1}^-1 mod q_j and its Shoup companion
};

// The ModDown's forward NTT (ntt_forward_moddown): rows (poly, j < L) of the delta buffer are
// read as the base conversion sum_k z_k (phat_k mod q_j) of the INTT'd special-prime limbs
// z_k = acc[poly][L + k], and written as (acc[poly][j] - NTT(...)) P^-1 (+ add, or
// + add * add_mul[j]) into out;
// poly = ct * H + h.  The add term of rows h < n_add is read at perm[pos] for rows h < n_perm.
struct ModDownIO {
    const uint64_t *acc = nullptr;   // [polys][L + np][N]
    const uint64_t *conv = nullptr;  // [nq][np]: phat_k mod q_j
    const uint64_t *pinv = nullptr;  // [nq][2]: P^-1 mod q_j and its Shoup companion
    uint64_t *out = nullptr;
    const uint64_t *add = nullptr;
    const uint64_t *add_mul = nullptr;  // [nq][2]: the add term times this per-limb constant; null: as is
    const uint32_t *perm = nullptr;
    // exact conversion: the conversion sum minus vs[j][v] (v S mod q_j) with v = vrow[poly][k],
    // the overflow count floor(sum_k z_k / s_k); null: the approximate conversion
    const uint8_t *vrow = nullptr;
    const uint64_t *vs = nullptr;  // [slots][16]
    long long out_ct = 0, out_h = 0, add_ct = 0, add_h = 0;  // word strides
    uint32_t H = 2, np = 0, n_add = 0, n_perm = 0;
    int s52 = 0;  // every prime below 2^52: Acc<true>
};

// ModUp's forward NTT (ntt_forward_modup): row (ct, b, j) of up [n_cts][beta][LP][N].  For j
// outside digit b (limbs [b alpha, min((b+1) alpha, L))) the column kernel reads the base
// conversion sum_i y_i (qhat_i mod t_j) of the digit's INTT'd, qhat^-1-scaled limbs
// y = x[ct][b alpha ..] (coefficient form) and the row is transformed; for j inside the digit it
// copies d[ct][j] (already NTT form) and the block kernel leaves the row alone (map 255).  The
// converted digits are never stored in coefficient form.
struct ModUpIO {
    const uint64_t *x = nullptr;     // [n_cts][L][N]
    const uint64_t *d = nullptr;     // ciphertext ct's polynomial at d + ct * d_stride, [L][N]
    const uint64_t *conv = nullptr;  // [beta][LP][np]: qhat_i mod t_j of the level's digits
    long long d_stride = 0;
    uint32_t L = 0, np = 0, LP = 0;
    int s52 = 0;
};

// the optional load / store transforms of the forward NTT kernels
struct NttIO {
    RescaleIO rs;
    ModDownIO md;
    ModUpIO mu;
};
constexpr int kIoPlain = 0, kIoRescale = 1, kIoModDown = 2, kIoModUp = 3;

// scale constants of the inverse's last stage, per limb slot: c, c', c*psi^-(N/2), (c*psi^-(N/2))'
struct InvScale {
    const uint64_t *c;  // [slots][4]
};

__device__ __forceinline__ void ct_bf(uint64_t &x, uint64_t &y, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t q2 = 2 * q;
    uint64_t a = csub(x, q2);
    uint64_t t = shoup_lazy(y, w, ws, q);
    x = a + t;
    y = a - t + q2;
}

// Cooley-Tukey butterfly without the reduction of x: outputs exceed the inputs by less
// than 4q (shoup_lazy4 is below 4q for any 64-bit multiplicand).  From inputs below 4q,
// 16 stages stay below 68q < 2^(k+7), so this is exact for primes q < 2^57 and the last
// stage's output is reduced by reduce_small.
constexpr uint64_t kGrowPrimeLimit = 1ull << 57;

__device__ __forceinline__ void ct_bf_grow(uint64_t &x, uint64_t &y, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t t = shoup_lazy4(y, w, ws, q);
    uint64_t a = x;
    x = a + t;
    y = a - t + 4 * q;
}

// Primes below kF64GrowLimit take the twiddle product's quotient from the FP64 pipe instead of the
// integer multipliers (the quotient estimate of Shoup's NTL MulMod, with the product's remainder
// formed by the 64-bit low products): with wq = w / q rounded to the nearest double and y < 2^52,
// y is exact as a double (its bits under the exponent of 2^52, minus 2^52), and
// Q = round(y wq) comes from the mantissa of fma(y, wq, 2^52).  |Q - y w / q| <= 1/2 + y 2^-54 < 3/4,
// so Q is floor(y w / q) or one more and r = y w - Q q lies in [-q, q) (as a wrapped 64-bit value);
// the inverse's butterflies add q to it.  The integer pipe keeps the two low products only.
constexpr uint64_t kF64GrowLimit = (1ull << 52) / 36;

__device__ __forceinline__ uint64_t mulmod_f64_centred(uint64_t y, uint64_t w, double wq, uint64_t q) {
    const double two52 = 4503599627370496.0;
    const double yd = __dsub_rn(__longlong_as_double((long long)(0x4330000000000000ull | y)), two52);
    const uint64_t Q = (uint64_t)__double_as_longlong(__fma_rn(yd, wq, two52)) & 0x000FFFFFFFFFFFFFull;
    return y * w - Q * q;
}

// The forward transform of the primes below kF64GrowLimit runs entirely on the FP64 pipe, on values
// held as doubles (signed exact integers, stored in the uint64_t registers as their bit patterns;
// the column phase's output keeps that form in memory for the block phase).  Cooley-Tukey:
// t = y w - Q q with Q = round(y wq), |Q - y w / q| < 3/4 (|y| < 16q, so |y| 2^-53 < 1/4), hence
// |t| < q; y w = hi + lo exactly (hi = y w rounded, lo from an fma), hi - Q q is exact by a second
// fma (an integer below 2^47 in magnitude), and t = (hi - Q q) + lo exactly.  From inputs below q in
// magnitude, values grow by less than 3q/4 per stage: below 13q < 2^51 after 16 stages.  Eight FP64
// operations and no integer multiply per butterfly.
__device__ __forceinline__ void ct_bf_dbl(uint64_t &xb, uint64_t &yb, double w, double wq, double q) {
    const double magic = 6755399441055744.0;  // 1.5 2^52
    const double x = __longlong_as_double((long long)xb), y = __longlong_as_double((long long)yb);
    const double Q = __dsub_rn(__fma_rn(y, wq, magic), magic);
    const double hi = __dmul_rn(y, w);
    const double lo = __fma_rn(y, w, -hi);
    const double t = __dadd_rn(__fma_rn(-Q, q, hi), lo);
    xb = (uint64_t)__double_as_longlong(__dadd_rn(x, t));
    yb = (uint64_t)__double_as_longlong(__dsub_rn(x, t));
}

// x < 2^52 as the bit pattern of the double x
__device__ __forceinline__ uint64_t to_dbl_bits(uint64_t x) {
    const double two52 = 4503599627370496.0;
    return (uint64_t)__double_as_longlong(__dsub_rn(__longlong_as_double((long long)(0x4330000000000000ull | x)), two52));
}

// Primes in [kF64GrowLimit, 2^51) run the same butterfly on twiddles kept within q/2 of zero
// (|wq| <= 1/2, |wq - w / q| <= 2^-55), with every value centred (dbl_centre) at the start and
// after every pass of four stages, and the multiplicands of a pass's fourth stage centred before
// their products.  |Q - y w / q| <= 1/2 + |y| 2^-55, so from |v| <= q/2 the multiplicands of the
// first three stages stay below q/2, 1.03q and 1.6q (|y wq| < 2^51: the rounding through
// 1.5 2^52 is exact), |t| below 0.53q, 0.57q and 0.6q, the fourth stage's below 0.53q, and every
// value below 2.73q < 2^53: exact; |y w| < 2^102, so |lo| <= 2^48 and hi - Q q stays below 2^52.
constexpr uint64_t kF64CentreLimit = 1ull << 51;

// v (|v| < 2^52, a signed integer) -> v - round(v / q) q, within q/2 + 1 of zero (exact: an integer
// below q); qinv = 1 / q rounded
__device__ __forceinline__ uint64_t dbl_centre(uint64_t vb, double q, double qinv) {
    const double magic = 6755399441055744.0;
    const double v = __longlong_as_double((long long)vb);
    const double Q = __dsub_rn(__fma_rn(v, qinv, magic), magic);
    return (uint64_t)__double_as_longlong(__fma_rn(-Q, q, v));
}

// a centred double (|v| <= q/2 + 1) -> v mod q in [0, q) as an integer
__device__ __forceinline__ uint64_t dbl_bits_canon(uint64_t vb, double q) {
    const double two52 = 4503599627370496.0;
    double v = __longlong_as_double((long long)vb);
    v = v < 0.0 ? __dadd_rn(v, q) : v;
    return (uint64_t)__double_as_longlong(__dadd_rn(v, two52)) & 0x000FFFFFFFFFFFFFull;
}

// a double holding a signed integer v (|v| < 2^51) -> v mod q in [0, q): v - round(v / q) q is exact
// and within q/2 + 1 of zero, one conditional addition of q finishes it
__device__ __forceinline__ uint64_t dbl_bits_mod(uint64_t vb, double q, double qinv) {
    const double magic = 6755399441055744.0, two52 = 4503599627370496.0;
    const double v = __longlong_as_double((long long)vb);
    const double Q = __dsub_rn(__fma_rn(v, qinv, magic), magic);
    double r = __fma_rn(-Q, q, v);
    r = r < 0.0 ? __dadd_rn(r, q) : r;
    return (uint64_t)__double_as_longlong(__dadd_rn(r, two52)) & 0x000FFFFFFFFFFFFFull;
}

// Gentleman-Sande butterfly on [0, 4q) with the FP64 quotient: x - y + 4q < 8q < 2^52
__device__ __forceinline__ void gs_bf_f64(uint64_t &x, uint64_t &y, uint64_t w, double wq, uint64_t q) {
    const uint64_t q4 = 4 * q;
    const uint64_t a = x + y, d = x - y + q4;
    x = csub(a, q4);
    y = mulmod_f64_centred(d, w, wq, q) + q;
}

__device__ __forceinline__ void gs_bf(uint64_t &x, uint64_t &y, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t q2 = 2 * q;
    uint64_t a = x + y;
    uint64_t d = x - y + q2;
    x = csub(a, q2);
    y = shoup_lazy(d, w, ws, q);
}

// Gentleman-Sande butterfly on [0, 4q) with the cheaper quotient of shoup_lazy4 (needs 8q < 2^64)
__device__ __forceinline__ void gs_bf4(uint64_t &x, uint64_t &y, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t q4 = 4 * q;
    uint64_t a = x + y;
    uint64_t d = x - y + q4;
    x = csub(a, q4);
    y = shoup_lazy4(d, w, ws, q);
}

// R forward stages on E = 2^R registers.  Stage r of the pass is global stage
// s0 + r; the twiddle of the pair starting at m is tw[(tb << (s0 + r)) + (g << r) + (m >> (R - r))].
// MODE kBfHarvey: Harvey butterflies that keep values in [0, 4q) (any prime); kBfGrow: ct_bf_grow
// (primes below kGrowPrimeLimit); kBfF64: ct_bf_dbl (forward, primes below kF64GrowLimit) on values
// held as doubles, with the twiddles wd (w as doubles) and wq (w / q as doubles); kBfF64R: the same
// on centred twiddles, with the last stage's multiplicands centred before their products and
// every value centred after the pass (forward, primes below kF64CentreLimit).  The inverse's kBfF64 is gs_bf_f64 (integer values,
// FP64 quotient).
constexpr int kBfHarvey = 0, kBfGrow = 1, kBfF64 = 2, kBfF64R = 3;

// the inverse's butterfly family of a limb's prime
__host__ __device__ __forceinline__ int bf_mode_of(uint64_t q) {
    return q < kF64GrowLimit ? kBfF64 : q < kGrowPrimeLimit ? kBfGrow : kBfHarvey;
}

// the forward's butterfly family of a limb's prime
__host__ __device__ __forceinline__ int fwd_mode_of(uint64_t q) {
    return q < kF64GrowLimit ? kBfF64 : q < kF64CentreLimit ? kBfF64R : q < kGrowPrimeLimit ? kBfGrow : kBfHarvey;
}

// The families a kernel instantiation carries (a bit per family, forward and inverse together).
// Every unrolled family adds a full copy of the transform's butterflies to the kernel, so a
// context's launches use the instantiation with just the families its primes need: kFamSmall
// (every prime below 2^57: the bootstrapping chains), kFamLarge (none below kF64GrowLimit),
// kFamAll otherwise.
constexpr int kFamSmall = (1 << kBfF64) | (1 << kBfF64R) | (1 << kBfGrow),
              kFamLarge = (1 << kBfF64R) | (1 << kBfGrow) | (1 << kBfHarvey), kFamAll = kFamSmall | kFamLarge;

template <int R, int MODE = kBfHarvey>
__device__ __forceinline__ void fwd_pass(uint64_t (&a)[1 << R], const uint64_t *__restrict__ w,
                                         const uint64_t *__restrict__ ws, const double *__restrict__ wq,
                                         const double *__restrict__ wd, uint32_t tb, uint32_t s0, uint32_t g,
                                         uint64_t q) {
    const double qd = (double)q;
    const double qinv = MODE == kBfF64R ? __ldg(wq) : 0.0;  // wq[0] = 1 / q (the twiddle at index 0 is 1)
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int half = (1 << R) >> (r + 1);
        const uint32_t base = (tb << (s0 + r)) + (g << r);
#pragma unroll
        for (int m = 0; m < (1 << R); m++) {
            if (m & half) continue;
            uint32_t idx = base + (m >> (R - r));
            if (MODE == kBfF64)
                ct_bf_dbl(a[m], a[m + half], __ldg(wd + idx), __ldg(wq + idx), qd);
            else if (MODE == kBfF64R) {
                if (r == R - 1) a[m + half] = dbl_centre(a[m + half], qd, qinv);
                ct_bf_dbl(a[m], a[m + half], __ldg(wd + idx), __ldg(wq + idx), qd);
            }
            else if (MODE == kBfGrow)
                ct_bf_grow(a[m], a[m + half], __ldg(w + idx), __ldg(ws + idx), q);
            else
                ct_bf(a[m], a[m + half], __ldg(w + idx), __ldg(ws + idx), q);
        }
    }
    if (MODE == kBfF64R) {
#pragma unroll
        for (int m = 0; m < (1 << R); m++) a[m] = dbl_centre(a[m], qd, qinv);
    }
}

// fwd_pass in the butterfly family `mode` (uniform per CTA: one limb), one of the families FAM carries
template <int R, int FAM>
__device__ __forceinline__ void fwd_pass_any(int mode, uint64_t (&a)[1 << R], const uint64_t *__restrict__ w,
                                             const uint64_t *__restrict__ ws, const double *__restrict__ wq,
                                             const double *__restrict__ wd, uint32_t tb, uint32_t s0, uint32_t g,
                                             uint64_t q) {
    if ((FAM & (1 << kBfF64)) && mode == kBfF64)
        fwd_pass<R, kBfF64>(a, w, ws, wq, wd, tb, s0, g, q);
    else if ((FAM & (1 << kBfF64R)) && mode == kBfF64R)
        fwd_pass<R, kBfF64R>(a, w, ws, wq, wd, tb, s0, g, q);
    else if (!(FAM & (1 << kBfHarvey)) || mode == kBfGrow)
        fwd_pass<R, kBfGrow>(a, w, ws, wq, wd, tb, s0, g, q);
    else
        fwd_pass<R, kBfHarvey>(a, w, ws, wq, wd, tb, s0, g, q);
}

// MODE kBfGrow: gs_bf4 on [0, 4q) (primes below kGrowPrimeLimit); kBfF64: gs_bf_f64 on [0, 4q);
// kBfHarvey: gs_bf on [0, 2q)
template <int R, int MODE = kBfHarvey>
__device__ __forceinline__ void inv_pass(uint64_t (&a)[1 << R], const uint64_t *__restrict__ w,
                                         const uint64_t *__restrict__ ws, const double *__restrict__ wq, uint32_t tb,
                                         uint32_t s0, uint32_t g, uint64_t q, int skip_stage0) {
#pragma unroll
    for (int r = R - 1; r >= 0; r--) {
        if (r == 0 && skip_stage0) break;
        const int half = (1 << R) >> (r + 1);
        const uint32_t base = (tb << (s0 + r)) + (g << r);
#pragma unroll
        for (int m = 0; m < (1 << R); m++) {
            if (m & half) continue;
            uint32_t idx = base + (m >> (R - r));
            if (MODE == kBfF64)
                gs_bf_f64(a[m], a[m + half], __ldg(w + idx), __ldg(wq + idx), q);
            else if (MODE == kBfGrow)
                gs_bf4(a[m], a[m + half], __ldg(w + idx), __ldg(ws + idx), q);
            else
                gs_bf(a[m], a[m + half], __ldg(w + idx), __ldg(ws + idx), q);
        }
    }
}

template <int R, int FAM>
__device__ __forceinline__ void inv_pass_any(int mode, uint64_t (&a)[1 << R], const uint64_t *__restrict__ w,
                                             const uint64_t *__restrict__ ws, const double *__restrict__ wq,
                                             uint32_t tb, uint32_t s0, uint32_t g, uint64_t q, int skip_stage0) {
    if ((FAM & (1 << kBfF64)) && mode == kBfF64)
        inv_pass<R, kBfF64>(a, w, ws, wq, tb, s0, g, q, skip_stage0);
    else if (!(FAM & (1 << kBfHarvey)) || mode == kBfGrow)
        inv_pass<R, kBfGrow>(a, w, ws, wq, tb, s0, g, q, skip_stage0);
    else
        inv_pass<R, kBfHarvey>(a, w, ws, wq, tb, s0, g, q, skip_stage0);
}

}  // namespace shm
