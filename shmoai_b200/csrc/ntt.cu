// Batched NTT / INTT kernels (see ntt.cuh for the decomposition).
#include "core.hpp"

namespace shm {

namespace {

template <int R, int S>
struct Geo {
    static constexpr int LOGM = 2 * R;
    static constexpr uint32_t M = 1u << LOGM;  // sub-transform length
    static constexpr int LOGN = 2 * LOGM;
    static constexpr uint32_t N = 1u << LOGN;
    static constexpr int E = 1 << R;  // elements per thread
    static constexpr uint32_t THREADS = S * E;
    static constexpr uint32_t CHUNKS = M / S;  // CTAs per limb
    static constexpr uint32_t PAD_M = M + M / 16;     // padded block row in shared memory
};

__device__ __forceinline__ uint32_t padded(uint32_t p) { return p + (p >> 4); }

// sum_{i < n} x[i << log_n] c[i] mod p (a base conversion's term for one coefficient; n <= 16).  The
// first eight terms' loads are issued together before any product, so one load latency is exposed
// per coefficient instead of one per term.
template <bool S52>
__device__ __forceinline__ uint64_t conv_sum(const uint64_t *__restrict__ x, const uint64_t *c, uint32_t n,
                                             int log_n, const PrimeConst &p) {
    constexpr uint32_t kBatch = 8;
    uint64_t v[kBatch];
#pragma unroll
    for (uint32_t i = 0; i < kBatch; i++) v[i] = i < n ? x[(size_t)i << log_n] : 0;
    Acc<S52> acc;
#pragma unroll
    for (uint32_t i = 0; i < kBatch; i++)
        if (i < n) acc.add(v[i], c[i]);
    for (uint32_t i = kBatch; i < n; i++) acc.add(x[(size_t)i << log_n], c[i]);
    return barrett(acc.get(), p);
}

// CTAs are issued limb-major: consecutive CTAs work on the same limb slot (one prime) of
// successive polynomials, so the CTAs in flight share one prime's twiddle table in L2.
// rows = polys * slots; CTA index t -> (poly = t % polys, slot = t / polys).
__device__ __forceinline__ uint32_t limb_major_row(uint32_t t, uint32_t slots, uint32_t rows) {
    const uint32_t polys = rows / slots;
    return (t % polys) * slots + t / polys;
}

// ---------------- forward, phase 1: columns (global stages 0 .. LOGM-1)
// IOK = kIoRescale: row (poly, j) is read as c_last[poly] mod q_j from the coefficient-form
// last limbs; kIoModDown: as the base conversion of the special-prime limbs (ModDownIO);
// kIoPlain: from `data`
template <int R, int S, int MINB, int IOK, int FAM>
__global__ void __launch_bounds__(Geo<R, S>::THREADS, MINB) fwd_col(uint64_t *__restrict__ data, uint32_t slots, LimbMap map,
                                                            const uint64_t *__restrict__ tw,
                                                            const double *__restrict__ twq,
                                                            const PrimeConst *__restrict__ pc, NttIO io) {
    using G = Geo<R, S>;
    __shared__ uint64_t sm[G::M * S];
    const uint32_t chunk = blockIdx.x % G::CHUNKS;
    // ModUp rows go ct-major instead: the rows of one digit are consecutive CTAs, so the digit's
    // coefficient-form limbs that every one of its rows reads stay in L2 while they run
    const uint32_t row = IOK == kIoModUp ? blockIdx.x / G::CHUNKS
                                         : limb_major_row(blockIdx.x / G::CHUNKS, slots, gridDim.x / G::CHUNKS);
    const uint32_t pidx = map.prime[row % slots];
    const uint32_t sig = threadIdx.x % S, lane = threadIdx.x / S;
    if constexpr (IOK == kIoModUp) {
        if (pidx == 255) {  // a limb of the digit itself: the NTT-form input, copied
            const ModUpIO &mu = io.mu;
            const uint32_t ct = row / slots, j = (row % slots) % mu.LP;
            if (j >= mu.L) return;  // rows past the extended basis (none in a ModUp map)
            const uint64_t *src = mu.d + ct * mu.d_stride + ((size_t)j << G::LOGN) + chunk * S;
            uint64_t *dst = data + ((size_t)row << G::LOGN) + chunk * S;
#pragma unroll
            for (int m = 0; m < G::E; m++) {
                const size_t pos = sig + (size_t)G::M * (lane + m * G::E);
                dst[pos] = src[pos];
            }
            return;
        }
    }
    if (pidx == 255) return;
    const uint64_t q = pc[pidx].q;
    const uint64_t *w = tw + ((size_t)pidx * 4 << G::LOGN), *ws = w + G::N;
    const double *wq = twq + ((size_t)pidx * 3 << G::LOGN), *wd = wq + 2 * G::N;
    uint64_t *x = data + ((size_t)row << G::LOGN) + chunk * S;

    const int mode = fwd_mode_of(q);  // uniform per CTA (one limb)
    uint64_t a[G::E];
    if constexpr (IOK == kIoModUp) {
        const ModUpIO &mu = io.mu;
        __shared__ uint64_t sconv[16];
        const uint32_t ct = row / slots, slot = row % slots, b = slot / mu.LP, j = slot % mu.LP;
        const uint32_t s0 = b * mu.np, na = min(mu.np, mu.L - s0);
        if (threadIdx.x < na) sconv[threadIdx.x] = mu.conv[((size_t)b * mu.LP + j) * mu.np + threadIdx.x];
        __syncthreads();
        const PrimeConst p = pc[pidx];
        const uint64_t *y = mu.x + (((size_t)ct * mu.L + s0) << G::LOGN) + chunk * S;
#pragma unroll
        for (int m = 0; m < G::E; m++) {
            const size_t pos = sig + (size_t)G::M * (lane + m * G::E);
            a[m] = mu.s52 ? conv_sum<true>(y + pos, sconv, na, G::LOGN, p)
                          : conv_sum<false>(y + pos, sconv, na, G::LOGN, p);
        }
    } else if constexpr (IOK == kIoRescale) {
        const PrimeConst p = pc[pidx];
        const uint64_t *src = io.rs.last + ((size_t)(row / slots) << G::LOGN) + chunk * S;
#pragma unroll
        for (int m = 0; m < G::E; m++) a[m] = barrett({src[sig + (size_t)G::M * (lane + m * G::E)], 0}, p);
    } else if constexpr (IOK == kIoModDown) {
        __shared__ uint64_t sconv[16], svs[16];
        const uint32_t np = io.md.np, j = row % slots;
        if (threadIdx.x < np) sconv[threadIdx.x] = io.md.conv[(size_t)j * np + threadIdx.x];
        if (io.md.vrow && threadIdx.x < 16) svs[threadIdx.x] = io.md.vs[(size_t)j * 16 + threadIdx.x];
        __syncthreads();
        const PrimeConst p = pc[pidx];
        const uint64_t *z = io.md.acc + ((size_t)((row / slots) * (slots + np) + slots) << G::LOGN) + chunk * S;
#pragma unroll
        for (int m = 0; m < G::E; m++) {
            const size_t pos = sig + (size_t)G::M * (lane + m * G::E);
            a[m] = io.md.s52 ? conv_sum<true>(z + pos, sconv, np, G::LOGN, p)
                             : conv_sum<false>(z + pos, sconv, np, G::LOGN, p);
        }
        if (io.md.vrow) {
            const uint8_t *vr = io.md.vrow + ((size_t)(row / slots) << G::LOGN) + chunk * S;
#pragma unroll
            for (int m = 0; m < G::E; m++) a[m] = sub_mod(a[m], svs[vr[sig + (size_t)G::M * (lane + m * G::E)] & 15], q);
        }
    } else {
#pragma unroll
        for (int m = 0; m < G::E; m++) a[m] = x[sig + (size_t)G::M * (lane + m * G::E)];
    }
    if ((FAM & (1 << kBfF64)) && mode == kBfF64) {  // [0, q) -> doubles for the FP64 butterflies
#pragma unroll
        for (int m = 0; m < G::E; m++) a[m] = to_dbl_bits(a[m]);
    } else if ((FAM & (1 << kBfF64R)) && mode == kBfF64R) {  // [0, q) -> doubles within q/2 of zero
        const double qd = (double)q, qinv = __ldg(wq);
#pragma unroll
        for (int m = 0; m < G::E; m++) a[m] = dbl_centre(to_dbl_bits(a[m]), qd, qinv);
    }
    fwd_pass_any<R, FAM>(mode, a, w, ws, wq, wd, 1, 0, 0, q);
#pragma unroll
    for (int m = 0; m < G::E; m++) sm[(lane + m * G::E) * S + sig] = a[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < G::E; m++) a[m] = sm[(lane * G::E + m) * S + sig];
    fwd_pass_any<R, FAM>(mode, a, w, ws, wq, wd, 1, R, lane, q);
#pragma unroll
    for (int m = 0; m < G::E; m++) x[sig + (size_t)G::M * (lane * G::E + m)] = a[m];
}

// ---------------- forward, phase 2: blocks (global stages LOGM .. 2*LOGM-1), fully reduced output
// IOK = kIoRescale: instead of storing t = NTT(...) of row (poly, j), write (c_j - t) q_last^-1
// to io.rs.out; kIoModDown: write (acc_j - t) P^-1 (+ add) to io.md.out
template <int R, int S, int MINB, int IOK, int FAM>
__global__ void __launch_bounds__(Geo<R, S>::THREADS, MINB) fwd_blk(uint64_t *__restrict__ data, uint32_t slots, LimbMap map,
                                                            const uint64_t *__restrict__ tw,
                                                            const double *__restrict__ twq,
                                                            const PrimeConst *__restrict__ pc, NttIO io) {
    using G = Geo<R, S>;
    __shared__ uint64_t sm[S * G::PAD_M];
    const uint32_t chunk = blockIdx.x % G::CHUNKS;
    const uint32_t row = limb_major_row(blockIdx.x / G::CHUNKS, slots, gridDim.x / G::CHUNKS);
    const uint32_t pidx = map.prime[row % slots];
    if (pidx == 255) return;
    const uint64_t q = pc[pidx].q;
    const uint64_t *w = tw + ((size_t)pidx * 4 << G::LOGN), *ws = w + G::N;
    const double *wq = twq + ((size_t)pidx * 3 << G::LOGN), *wd = wq + 2 * G::N;
    uint64_t *xc = data + ((size_t)row << G::LOGN) + (size_t)chunk * S * G::M;
    const uint32_t sig = threadIdx.x / G::E, lane = threadIdx.x % G::E;
    const uint32_t b = chunk * S + sig;
    uint64_t *x = xc + (size_t)sig * G::M;
    uint64_t *s = sm + sig * G::PAD_M;

    const int mode = fwd_mode_of(q);  // the same choice fwd_col made for this limb
    uint64_t a[G::E];
#pragma unroll
    for (int m = 0; m < G::E; m++) a[m] = x[lane + m * G::E];
    fwd_pass_any<R, FAM>(mode, a, w, ws, wq, wd, G::M + b, 0, 0, q);
#pragma unroll
    for (int m = 0; m < G::E; m++) s[padded(lane + m * G::E)] = a[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < G::E; m++) a[m] = s[padded(lane * G::E + m)];
    if ((FAM & (1 << kBfF64)) && mode == kBfF64) {
        fwd_pass<R, kBfF64>(a, w, ws, wq, wd, G::M + b, R, lane, q);
        const double qd = (double)q, qinv = __ldg(wq);  // wq[0] = 1 / q
#pragma unroll
        for (int m = 0; m < G::E; m++) s[padded(lane * G::E + m)] = dbl_bits_mod(a[m], qd, qinv);  // |v| < 13q -> [0, q)
    } else if ((FAM & (1 << kBfF64R)) && mode == kBfF64R) {
        fwd_pass<R, kBfF64R>(a, w, ws, wq, wd, G::M + b, R, lane, q);  // centred by the pass
        const double qd = (double)q;
#pragma unroll
        for (int m = 0; m < G::E; m++) s[padded(lane * G::E + m)] = dbl_bits_canon(a[m], qd);
    } else if (!(FAM & (1 << kBfHarvey)) || mode != kBfHarvey) {
        fwd_pass<R, kBfGrow>(a, w, ws, wq, wd, G::M + b, R, lane, q);
        const PrimeConst p = pc[pidx];
#pragma unroll
        for (int m = 0; m < G::E; m++) s[padded(lane * G::E + m)] = reduce_small(a[m], p);  // < 68q -> [0, q)
    } else {
        fwd_pass<R, kBfHarvey>(a, w, ws, wq, wd, G::M + b, R, lane, q);
        const uint64_t q2 = 2 * q;
#pragma unroll
        for (int m = 0; m < G::E; m++) s[padded(lane * G::E + m)] = csub(csub(a[m], q2), q);
    }
    __syncthreads();
    if constexpr (IOK == kIoRescale) {
        const uint32_t poly = row / slots, j = row % slots;
        const size_t off = (size_t)chunk * S * G::M;
        const uint64_t *cin = io.rs.in + (((size_t)poly * (slots + 1) + j) << G::LOGN) + off;
        uint64_t *o = io.rs.out + ((size_t)row << G::LOGN) + off;
        const uint64_t iw = io.rs.inv[2 * j], iws = io.rs.inv[2 * j + 1];
#pragma unroll
        for (int i = 0; i < G::E; i++) {
            uint32_t e = threadIdx.x + i * G::THREADS;
            const uint64_t t = sm[(e / G::M) * G::PAD_M + padded(e % G::M)];
            o[e] = shoup(sub_mod(cin[e], t, q), iw, iws, q);
        }
    } else if constexpr (IOK == kIoModDown) {
        const ModDownIO &md = io.md;
        const uint32_t poly = row / slots, j = row % slots, ct = poly / md.H, h = poly % md.H;
        const size_t off = (size_t)chunk * S * G::M;
        const uint64_t *ain = md.acc + (((size_t)poly * (slots + md.np) + j) << G::LOGN) + off;
        uint64_t *o = md.out + ct * md.out_ct + h * md.out_h + ((size_t)j << G::LOGN) + off;
        const uint64_t iw = md.pinv[2 * j], iws = md.pinv[2 * j + 1];
        const bool add = h < md.n_add, perm = add && h < md.n_perm && md.perm;
        const uint64_t *ad = add ? md.add + ct * md.add_ct + h * md.add_h + ((size_t)j << G::LOGN) : nullptr;
        if (md.add_mul) {
            const uint64_t mw = md.add_mul[2 * j], mws = md.add_mul[2 * j + 1];
#pragma unroll
            for (int i = 0; i < G::E; i++) {
                uint32_t e = threadIdx.x + i * G::THREADS;
                const uint64_t t = sm[(e / G::M) * G::PAD_M + padded(e % G::M)];
                uint64_t r = shoup(sub_mod(ain[e], t, q), iw, iws, q);
                if (add) r = add_mod(r, shoup(ad[perm ? __ldg(md.perm + off + e) : off + e], mw, mws, q), q);
                o[e] = r;
            }
        } else {
#pragma unroll
            for (int i = 0; i < G::E; i++) {
                uint32_t e = threadIdx.x + i * G::THREADS;
                const uint64_t t = sm[(e / G::M) * G::PAD_M + padded(e % G::M)];
                uint64_t r = shoup(sub_mod(ain[e], t, q), iw, iws, q);
                if (add) r = add_mod(r, ad[perm ? __ldg(md.perm + off + e) : off + e], q);
                o[e] = r;
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < G::E; i++) {
            uint32_t e = threadIdx.x + i * G::THREADS;
            xc[e] = sm[(e / G::M) * G::PAD_M + padded(e % G::M)];
        }
    }
}

// ---------------- inverse, phase 1: blocks (global stages 2*LOGM-1 .. LOGM)
template <int R, int S, int MINB, int FAM>
__global__ void __launch_bounds__(Geo<R, S>::THREADS, MINB) inv_blk(uint64_t *__restrict__ data, uint32_t slots, LimbMap map,
                                                            const uint64_t *__restrict__ tw,
                                                            const double *__restrict__ twq,
                                                            const PrimeConst *__restrict__ pc) {
    using G = Geo<R, S>;
    __shared__ uint64_t sm[S * G::PAD_M];
    const uint32_t chunk = blockIdx.x % G::CHUNKS;
    const uint32_t row = limb_major_row(blockIdx.x / G::CHUNKS, slots, gridDim.x / G::CHUNKS);
    const uint32_t pidx = map.prime[row % slots];
    if (pidx == 255) return;
    const uint64_t q = pc[pidx].q;
    const uint64_t *w = tw + ((size_t)pidx * 4 << G::LOGN) + 2 * G::N, *ws = w + G::N;
    const double *wq = twq + ((size_t)pidx * 3 << G::LOGN) + G::N;
    uint64_t *xc = data + ((size_t)row << G::LOGN) + (size_t)chunk * S * G::M;
    const uint32_t sig = threadIdx.x / G::E, lane = threadIdx.x % G::E;
    const uint32_t b = chunk * S + sig;
    uint64_t *s = sm + sig * G::PAD_M;

#pragma unroll
    for (int i = 0; i < G::E; i++) {
        uint32_t e = threadIdx.x + i * G::THREADS;
        sm[(e / G::M) * G::PAD_M + padded(e % G::M)] = xc[e];
    }
    __syncthreads();
    uint64_t a[G::E];
#pragma unroll
    for (int m = 0; m < G::E; m++) a[m] = s[padded(lane * G::E + m)];
    const int mode = bf_mode_of(q);  // uniform per CTA (one limb)
    inv_pass_any<R, FAM>(mode, a, w, ws, wq, G::M + b, R, lane, q, 0);
#pragma unroll
    for (int m = 0; m < G::E; m++) s[padded(lane * G::E + m)] = a[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < G::E; m++) a[m] = s[padded(lane + m * G::E)];
    inv_pass_any<R, FAM>(mode, a, w, ws, wq, G::M + b, 0, 0, q, 0);
    uint64_t *x = xc + (size_t)sig * G::M;
#pragma unroll
    for (int m = 0; m < G::E; m++) x[lane + m * G::E] = a[m];
}

// ---------------- inverse, phase 2: columns (global stages LOGM-1 .. 0) with the folded scale
template <int R, int S, int MINB, int FAM>
__global__ void __launch_bounds__(Geo<R, S>::THREADS, MINB) inv_col(uint64_t *__restrict__ data, uint32_t slots, LimbMap map,
                                                            const uint64_t *__restrict__ tw,
                                                            const double *__restrict__ twq,
                                                            const PrimeConst *__restrict__ pc,
                                                            const uint64_t *__restrict__ scale, int scale_by_prime,
                                                            uint32_t scale_base) {
    using G = Geo<R, S>;
    __shared__ uint64_t sm[G::M * S];
    const uint32_t chunk = blockIdx.x % G::CHUNKS;
    const uint32_t row = limb_major_row(blockIdx.x / G::CHUNKS, slots, gridDim.x / G::CHUNKS);
    const uint32_t slot = row % slots;
    const uint32_t pidx = map.prime[slot];
    if (pidx == 255) return;
    const uint64_t q = pc[pidx].q;
    const uint64_t *w = tw + ((size_t)pidx * 4 << G::LOGN) + 2 * G::N, *ws = w + G::N;
    const double *wq = twq + ((size_t)pidx * 3 << G::LOGN) + G::N;
    const uint64_t *sc = scale + 4 * (scale_by_prime ? pidx : slot - scale_base);
    uint64_t *x = data + ((size_t)row << G::LOGN) + chunk * S;
    const uint32_t sig = threadIdx.x % S, lane = threadIdx.x / S;

    uint64_t a[G::E];
#pragma unroll
    for (int m = 0; m < G::E; m++) a[m] = x[sig + (size_t)G::M * (lane * G::E + m)];
    const int mode = bf_mode_of(q);  // the same choice inv_blk made for this limb
    inv_pass_any<R, FAM>(mode, a, w, ws, wq, 1, R, lane, q, 0);
#pragma unroll
    for (int m = 0; m < G::E; m++) sm[(lane * G::E + m) * S + sig] = a[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < G::E; m++) a[m] = sm[(lane + m * G::E) * S + sig];
    inv_pass_any<R, FAM>(mode, a, w, ws, wq, 1, 0, 0, q, 1);
    // values in [0, 4q) (grow, FP64) or [0, 2q) (Harvey)
    const uint64_t c0 = sc[0], c0s = sc[1], c1 = sc[2], c1s = sc[3], q2 = (mode != kBfHarvey ? 4 : 2) * q;
#pragma unroll
    for (int m = 0; m < G::E / 2; m++) {
        uint64_t u = a[m], v = a[m + G::E / 2];
        a[m] = shoup(u + v, c0, c0s, q);
        a[m + G::E / 2] = shoup(u - v + q2, c1, c1s, q);
    }
#pragma unroll
    for (int m = 0; m < G::E; m++) x[sig + (size_t)G::M * (lane + m * G::E)] = a[m];
}

template <int R, int S, int MINB, int IOK, int FAM>
void launch_fwd_v(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                  cudaStream_t st, const NttIO &io) {
    using G = Geo<R, S>;
    dim3 grid(rows * G::CHUNKS);
    constexpr int BLK = IOK == kIoModUp ? kIoPlain : IOK;  // ModUp's block phase is a plain one
    SHM_LAUNCHED(1);
    fwd_col<R, S, MINB, IOK, FAM><<<grid, G::THREADS, 0, st>>>(data, slots, map, c.tw, c.twq, c.pc, io);
    SHM_LAUNCHED(1);
    fwd_blk<R, S, MINB, BLK, FAM><<<grid, G::THREADS, 0, st>>>(data, slots, map, c.tw, c.twq, c.pc, io);
}

template <int R, int S, int MINB, int FAM>
void launch_inv_v(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                  const uint64_t *scale, uint32_t scale_base, cudaStream_t st) {
    using G = Geo<R, S>;
    dim3 grid(rows * G::CHUNKS);
    SHM_LAUNCHED(1);
    inv_blk<R, S, MINB, FAM><<<grid, G::THREADS, 0, st>>>(data, slots, map, c.tw, c.twq, c.pc);
    SHM_LAUNCHED(1);
    inv_col<R, S, MINB, FAM><<<grid, G::THREADS, 0, st>>>(data, slots, map, c.tw, c.twq, c.pc,
                                                          scale ? scale : c.inv_scale_plain, scale ? 0 : 1, scale_base);
}

// the tile variants of kNttVariants (ntt.cuh), selected per context by c.ntt_variant, in the
// butterfly families of the context's primes (c.ntt_families)
template <int R, int IOK, int FAM>
void launch_fwd_f(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                  cudaStream_t st, const NttIO &io) {
    switch (c.ntt_variant) {
        case 1: launch_fwd_v<R, 16, 3, IOK, FAM>(c, data, rows, slots, map, st, io); break;
        case 2: launch_fwd_v<R, 8, 8, IOK, FAM>(c, data, rows, slots, map, st, io); break;
        case 3: launch_fwd_v<R, 8, 6, IOK, FAM>(c, data, rows, slots, map, st, io); break;
        default: launch_fwd_v<R, 16, 4, IOK, FAM>(c, data, rows, slots, map, st, io); break;
    }
}

template <int R, int IOK = kIoPlain>
void launch_fwd(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                cudaStream_t st, const NttIO &io = NttIO{}) {
    switch (c.ntt_families) {
        case kFamSmall: launch_fwd_f<R, IOK, kFamSmall>(c, data, rows, slots, map, st, io); break;
        case kFamLarge: launch_fwd_f<R, IOK, kFamLarge>(c, data, rows, slots, map, st, io); break;
        default: launch_fwd_f<R, IOK, kFamAll>(c, data, rows, slots, map, st, io); break;
    }
}

template <int R, int FAM>
void launch_inv_f(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                  const uint64_t *scale, uint32_t scale_base, cudaStream_t st) {
    switch (c.ntt_variant) {
        case 1: launch_inv_v<R, 16, 3, FAM>(c, data, rows, slots, map, scale, scale_base, st); break;
        case 2: launch_inv_v<R, 8, 8, FAM>(c, data, rows, slots, map, scale, scale_base, st); break;
        case 3: launch_inv_v<R, 8, 6, FAM>(c, data, rows, slots, map, scale, scale_base, st); break;
        default: launch_inv_v<R, 16, 4, FAM>(c, data, rows, slots, map, scale, scale_base, st); break;
    }
}

template <int R>
void launch_inv(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                const uint64_t *scale, uint32_t scale_base, cudaStream_t st) {
    switch (c.ntt_families) {
        case kFamSmall: launch_inv_f<R, kFamSmall>(c, data, rows, slots, map, scale, scale_base, st); break;
        case kFamLarge: launch_inv_f<R, kFamLarge>(c, data, rows, slots, map, scale, scale_base, st); break;
        default: launch_inv_f<R, kFamAll>(c, data, rows, slots, map, scale, scale_base, st); break;
    }
}

}  // namespace

LimbMap q_map(uint32_t L) {
    LimbMap m;
    for (int i = 0; i < 512; i++) m.prime[i] = (uint32_t)i < L ? (uint8_t)i : 255;
    return m;
}

void ntt_forward(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                 cudaStream_t st) {
    if (rows == 0) return;
    if (c.log_n == 16) launch_fwd<4>(c, data, rows, slots, map, st);
    else if (c.log_n == 12) launch_fwd<3>(c, data, rows, slots, map, st);
    else throw std::invalid_argument("NTT supports N = 2^12 and 2^16");
    SHM_CUDA(cudaGetLastError());
}

void ntt_forward_rescale(const Context &c, const RescaleIO &rs, uint64_t *t, uint32_t n_polys, uint32_t L,
                         cudaStream_t st) {
    if (n_polys == 0) return;
    NttIO io;
    io.rs = rs;
    if (c.log_n == 16) launch_fwd<4, kIoRescale>(c, t, n_polys * (L - 1), L - 1, q_map(L - 1), st, io);
    else if (c.log_n == 12) launch_fwd<3, kIoRescale>(c, t, n_polys * (L - 1), L - 1, q_map(L - 1), st, io);
    else throw std::invalid_argument("NTT supports N = 2^12 and 2^16");
    SHM_CUDA(cudaGetLastError());
}

void ntt_forward_moddown(const Context &c, const ModDownIO &md, uint64_t *delta, uint32_t n_polys, uint32_t L,
                         cudaStream_t st) {
    if (n_polys == 0) return;
    if (md.np > 16 || md.H == 0) throw std::invalid_argument("ModDown: shape out of range");
    NttIO io;
    io.md = md;
    if (c.log_n == 16) launch_fwd<4, kIoModDown>(c, delta, n_polys * L, L, q_map(L), st, io);
    else if (c.log_n == 12) launch_fwd<3, kIoModDown>(c, delta, n_polys * L, L, q_map(L), st, io);
    else throw std::invalid_argument("NTT supports N = 2^12 and 2^16");
    SHM_CUDA(cudaGetLastError());
}

void ntt_forward_modup(const Context &c, const ModUpIO &mu, uint64_t *up, uint32_t n_cts, uint32_t beta,
                       const LimbMap &map, cudaStream_t st) {
    if (n_cts == 0) return;
    if (mu.np > 16 || mu.np == 0 || mu.LP != mu.L + mu.np) throw std::invalid_argument("ModUp: shape out of range");
    NttIO io;
    io.mu = mu;
    const uint32_t slots = beta * mu.LP;
    if (c.log_n == 16) launch_fwd<4, kIoModUp>(c, up, n_cts * slots, slots, map, st, io);
    else if (c.log_n == 12) launch_fwd<3, kIoModUp>(c, up, n_cts * slots, slots, map, st, io);
    else throw std::invalid_argument("NTT supports N = 2^12 and 2^16");
    SHM_CUDA(cudaGetLastError());
}

void ntt_inverse(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                 const uint64_t *scale, cudaStream_t st, uint32_t scale_base) {
    if (rows == 0) return;
    if (c.log_n == 16) launch_inv<4>(c, data, rows, slots, map, scale, scale_base, st);
    else if (c.log_n == 12) launch_inv<3>(c, data, rows, slots, map, scale, scale_base, st);
    else throw std::invalid_argument("NTT supports N = 2^12 and 2^16");
    SHM_CUDA(cudaGetLastError());
}

}  // namespace shm
