// Rotation-free ct-pt matmul on the INT8 tensor cores (tcgen05.mma kind::i8), exact.
//
// Y[o][r] = sum_i X[i][r] * W[i][o] mod q_limb(r): X rows r of the n_in input
// ciphertexts (2 L N residues each), W the signed integer weights.  This is the
// reference's multiply_plain + add_inplace loop over constant plaintexts
// (src/include/source/matrix_mul/Ct_pt_matrix_mul.cuh:112-158) computed as one
// dense contraction.
//
// Exactness by a small-modulus residue system: the integer S = sum_i x_i w_i
// (|S| <= (q_l - 1) max_o sum_i |w_io|) is computed modulo T pairwise-coprime moduli
// m_t <= 251 whose product exceeds 2.02 |S|, each as an int8 GEMM with balanced
// residues in [-125, 125] (|acc| < n_in * 125^2 < 2^31), then rebuilt by the CRT:
//   S = sum_t r_t c_t - v M,  c_t = (M/m_t) [(M/m_t)^-1]_{m_t},  v = round(sum_t r_t inv_t / m_t),
// and reduced mod q_l with per-limb constants.  T GEMMs replace the 35 byte-slice
// products of a positional split; T is chosen per limb (a smaller prime needs fewer moduli)
// and each pass of columns runs with the largest T of its limbs.
//
// Pipeline per pass of columns: X residue planes [T][R][K] and W residue planes [T][N][K]
// (both K-major) -> tcgen05 GEMMs (weights as the M = 128 side, 256 X columns as N, s32
// accumulators in TMEM; operands by TMA where the X tile fits in shared memory) ->
// epilogue tcgen05.ld, acc mod m_t -> uint8 residue planes -> CRT kernel.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "core.hpp"
#include "host_math.hpp"

namespace shm {

namespace {

constexpr int kMaxMods = 20;
constexpr uint32_t kBM = 128;   // outputs per tile (MMA M: A = the weight residues)
constexpr uint32_t kBN = 256;   // X columns per tile (MMA N: B = the X residues)
constexpr uint32_t kKB = 64;    // K bytes per stage (two k32 MMAs)
constexpr int kStages = 4;
constexpr uint32_t kStageA = kBM * kKB;  // 8 KB
constexpr uint32_t kStageB = kBN * kKB;  // 16 KB
constexpr uint32_t kSmem = kStages * (kStageA + kStageB) + 1024;
constexpr uint32_t kThreads = 256;  // two warpgroups: loads shared, epilogue split by output columns
constexpr long long kSpinLimit = 1ll << 24;

// The constants of every candidate modulus, and the CRT fractions for every modulus count T
// (M = m_0 .. m_{T-1}): the table does not depend on the call, so concurrent calls that
// write it write the same bytes; each kernel takes its T as an argument.
struct ModTab {
    uint32_t m[kMaxMods];
    uint32_t fracq[kMaxMods + 1][kMaxMods];  // [T][t]: round(2^19 [(M/m_t)^-1]_{m_t} / m_t)
    uint32_t c24[kMaxMods];  // 2^20 mod m_t
    uint32_t c48[kMaxMods];  // 2^40 mod m_t
    uint32_t magic[kMaxMods];  // ceil(2^32 / m_t)
    double inv[kMaxMods];    // 1 / m_t
    float invf[kMaxMods];
};

__constant__ ModTab c_mods;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---------------------------------------------------------------- residues
__device__ __forceinline__ int8_t balanced(uint32_t r, uint32_t m) { return (int8_t)(r > m / 2 ? (int)r - (int)m : (int)r); }

// x mod m_t for x < 2^61 in 32-bit arithmetic: x = a 2^40 + b 2^20 + d (a < 2^21, b, d < 2^20)
// folds to s = a (2^40 mod m) + b (2^20 mod m) + d < 2^30; the quotient
// umulhi(s, ceil(2^32 / m)) is floor(s / m) or one more.
__device__ __forceinline__ uint32_t mod_small(uint64_t x, uint32_t t) {
    const uint32_t m = c_mods.m[t];
    const uint32_t a = (uint32_t)(x >> 40), b = (uint32_t)(x >> 20) & 0xFFFFF, d = (uint32_t)x & 0xFFFFF;
    const uint32_t s = a * c_mods.c48[t] + b * c_mods.c24[t] + d;
    int r = (int)(s - __umulhi(s, c_mods.magic[t]) * m);
    return (uint32_t)(r < 0 ? r + (int)m : r);
}

// a mod m_t in [0, m_t) for any int32 accumulator: a + m * 2^24 (a multiple of m above
// 2^31, the moduli being > 128) is non-negative and below 2^33, then the 32-bit fold above
// a mod m_t for |a| < 2^24 (every accumulator: n_in * 125^2 < 2^24 up to n_in = 1073): a is
// exact in float, floor(a / m) from one float multiply is off by at most one (relative error
// ~2^-24 of a quotient below 2^17), and two conditional corrections finish it
__device__ __forceinline__ uint32_t mod_acc24(int a, uint32_t t) {
    const int m = (int)c_mods.m[t];
    const int q = __float2int_rd((float)a * c_mods.invf[t]);
    int r = a - q * m;
    r += r < 0 ? m : 0;
    r -= r >= m ? m : 0;
    return (uint32_t)r;
}

__device__ __forceinline__ uint32_t mod_acc(int a, uint32_t t) {
    const uint64_t x = (uint64_t)((int64_t)a + ((int64_t)c_mods.m[t] << 24));
    return mod_small(x, t);
}

// The balanced residue of x mod m_t (in (-m/2, m/2), m odd) for x < 2^51 given as the exact double
// xd and its low word xlo: q = round(x / m) from fma(xd, 1/m, 1.5 2^52) (the pre-rounding value is
// within (x / m) 2^-53 < 0.25 / m of x / m, and x / m lies at least 0.5 / m from a half-integer,
// so q is the nearest integer).  The fma's result 1.5 2^52 + q carries q in the low bits of its
// mantissa (2^51 is a multiple of 2^32), so (x - q m) mod 2^32 = xlo - q_lo m, whose low byte is
// the two's complement of the residue: one FP64 multiply-add and one integer multiply-add.
__device__ __forceinline__ uint32_t balanced_f64(double xd, uint32_t xlo, uint32_t t) {
    const double magic = 6755399441055744.0;  // 1.5 * 2^52
    const uint32_t q = (uint32_t)__double2loint(__fma_rn(xd, c_mods.inv[t], magic));
    return xlo - q * c_mods.m[t];
}

// the low bytes of four words as one word
__device__ __forceinline__ uint32_t pack_low_bytes(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3) {
    return __byte_perm(__byte_perm(b0, b1, 0x0040), __byte_perm(b2, b3, 0x0040), 0x5410);
}

// X [n_in][R] (uint64) -> XP [t][R][Kp] (int8), via 64 x 64 shared-memory transposes.  A block
// converts kXresTiles column tiles of one 64-input group: the next tile's rows are copied by
// cp.async (8-byte pieces; rows past n_in filled with zeros) while the current one is converted.
// Each thread writes four consecutive inputs' residues of one column as one 32-bit word, so a
// warp's store covers 64 contiguous bytes of each of two columns for every modulus.  F64 (every
// limb prime below 2^51): each residue from one FP64 and one integer multiply-add (balanced_f64),
// else in 32-bit integer arithmetic (mod_small).
constexpr uint32_t kXresTiles = 2;
constexpr uint32_t kXresSmem = 2 * 64 * 65 * 8;

template <bool F64>
__global__ void __launch_bounds__(256, 3) xres_kernel(const uint64_t *__restrict__ X, int8_t *__restrict__ XP,
                                                      uint32_t n_in, uint32_t Kp, uint64_t R, uint64_t r0,
                                                      uint64_t chunk, uint32_t T) {
    extern __shared__ uint64_t xres_smem[];
    uint64_t(*tile)[64][65] = reinterpret_cast<uint64_t(*)[64][65]>(xres_smem);
    const uint32_t i0 = blockIdx.y * 64;
    const uint32_t tx = threadIdx.x & 63, ty = threadIdx.x >> 6;  // 256 threads: 64 x 4
    const uint64_t rb0 = (uint64_t)blockIdx.x * kXresTiles * 64;
    auto fetch = [&](uint32_t buf, uint64_t rb) {
        for (uint32_t i = ty; i < 64; i += 4) {
            const uint32_t ii = i0 + i;
            const uint64_t *src = X + (uint64_t)(ii < n_in ? ii : 0) * R + r0 + rb + tx;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(&tile[buf][i][tx])), "l"(src),
                         "r"(ii < n_in ? 8 : 0));
        }
        asm volatile("cp.async.commit_group;\n");
    };
    fetch(0, rb0);
    const uint32_t kq = threadIdx.x & 15, cg = threadIdx.x >> 4;  // inputs 4 kq .. 4 kq + 3, columns 4 cg .. 4 cg + 3
    for (uint32_t k = 0; k < kXresTiles; k++) {
        const uint32_t buf = k & 1;
        const uint64_t rb = rb0 + (uint64_t)k * 64;
        if (k + 1 < kXresTiles) {
            fetch(buf ^ 1, rb + 64);
            asm volatile("cp.async.wait_group 1;\n");
        } else {
            asm volatile("cp.async.wait_group 0;\n");
        }
        __syncthreads();
#pragma unroll
        for (uint32_t c = 0; c < 4; c++) {
            const uint32_t col = 4 * cg + c;
            uint64_t x[4];
#pragma unroll
            for (uint32_t j = 0; j < 4; j++) x[j] = tile[buf][4 * kq + j][col];
            int8_t *dst = XP + (rb + col) * Kp + i0 + 4 * kq;
            if constexpr (F64) {
                const double two52 = 4503599627370496.0;
                double xd[4];
                uint32_t xl[4];
#pragma unroll
                for (uint32_t j = 0; j < 4; j++) {  // exact: x < 2^51
                    xd[j] = __dsub_rn(__longlong_as_double((long long)(0x4330000000000000ull | x[j])), two52);
                    xl[j] = (uint32_t)x[j];
                }
                // unrolled over every candidate modulus (a uniform guard): the constants become operands
#pragma unroll
                for (uint32_t t = 0; t < (uint32_t)kMaxMods; t++) {
                    if (t < T)
                        *reinterpret_cast<uint32_t *>(dst + (uint64_t)t * chunk * Kp) =
                            pack_low_bytes(balanced_f64(xd[0], xl[0], t), balanced_f64(xd[1], xl[1], t),
                                           balanced_f64(xd[2], xl[2], t), balanced_f64(xd[3], xl[3], t));
                }
            } else {
                for (uint32_t t = 0; t < T; t++) {
                    uint32_t w = 0;
#pragma unroll
                    for (uint32_t j = 0; j < 4; j++)
                        w |= (uint32_t)(uint8_t)balanced(mod_small(x[j], t), c_mods.m[t]) << (8 * j);
                    *reinterpret_cast<uint32_t *>(dst + (uint64_t)t * chunk * Kp) = w;
                }
            }
        }
        __syncthreads();  // the buffer is refilled by the tile after next
    }
}

// W [n_in][n_out] (int64) -> WP [t][Np][Kp] (int8)
__global__ void wres_kernel(const int64_t *__restrict__ W, int8_t *__restrict__ WP, uint32_t n_in, uint32_t n_out,
                            uint32_t Kp, uint32_t Np, uint32_t T) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // input index (K)
    const uint32_t o = blockIdx.y;
    if (i >= Kp) return;
    int64_t w = (i < n_in && o < n_out) ? W[(uint64_t)i * n_out + o] : 0;
    for (uint32_t t = 0; t < T; t++) {
        int64_t m = c_mods.m[t];
        int64_t r = w % m;
        if (r < 0) r += m;
        WP[((uint64_t)t * Np + o) * Kp + i] = balanced((uint32_t)r, (uint32_t)m);
    }
}

// ---------------------------------------------------------------- tcgen05 GEMM

// K-major, no-swizzle ("interleaved") operand: core matrices of 8 rows x 16 bytes,
// K-adjacent core matrices 128 B apart (LBO), 8-row groups (KB / 16) * 128 B apart (SBO).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)(128 >> 4) << 16;             // leading byte offset (K direction)
    d |= (uint64_t)((kKB / 16 * 128) >> 4) << 32;  // stride byte offset (M/N direction)
    d |= (uint64_t)1 << 46;                      // descriptor version for sm_100
    return d;                                    // base offset 0, lbo mode 0, layout SWIZZLE_NONE
}

// K-major operand written by TMA with the 64-byte swizzle (rows of kKB = 64 bytes, 8-row groups
// 512 bytes apart); the MMA over K bytes [32 k, 32 k + 32) starts 32 k bytes into the atom
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;           // leading byte offset: unused within one swizzle atom
    d |= (uint64_t)(512 >> 4) << 32;  // stride byte offset: 8 rows x 64 bytes
    d |= (uint64_t)1 << 46;           // descriptor version for sm_100
    d |= (uint64_t)4 << 61;           // layout: SWIZZLE_64B
    return d;
}

// byte offset of (row, k-chunk) inside one stage operand of `rows` x kKB bytes
__device__ __forceinline__ uint32_t core_off(uint32_t row, uint32_t kc) {
    return ((row >> 3) * (kKB / 16) + kc) * 128 + (row & 7) * 16;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long it = 0; it < kSpinLimit; it++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity));
        if (ok) return true;
    }
    return false;
}

// grid: (Np / 128, R_chunk / 256, T); one modulus per blockIdx.z.  D[o][r] = W[o] . X[r]: the
// weights are A (128 outputs, TMEM lanes), the X residues B (256 columns, TMEM columns), so an
// epilogue thread holds 32 consecutive columns of one output and writes them as two 16-byte
// stores.  The output tiles are the fastest grid dimension: the CTAs that share an X tile
// run together and read it from HBM once (then from L2).  Two CTAs per SM (2 x 97 KB shared
// memory, 2 x 256 TMEM columns).
//
// Warp-specialised: warps 0-3 fill a kStages-deep ring with cp.async (each producer thread
// waits for its own copies of the previous stage, fences them into the async proxy and
// arrives on that stage's `full` barrier); one thread of warp 4 issues the MMAs of a stage
// once it is full and frees it through tcgen05.commit on its `empty` barrier; after the
// last commit (`done`) all eight warps read the accumulators back.  No block-wide barrier
// inside the K loop; every wait is bounded (a timeout sets *err and skips the stores).
__global__ void __launch_bounds__(kThreads, 2) mma_kernel(const int8_t *__restrict__ XP, const int8_t *__restrict__ WP,
                                                          uint8_t *__restrict__ RES, uint32_t Kp, uint32_t Np,
                                                          uint32_t n_out, uint64_t chunk, int *__restrict__ err,
                                                          int acc24) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t t = blockIdx.z;
    const uint64_t rbase = (uint64_t)blockIdx.y * kBN;
    const uint32_t obase = blockIdx.x * kBM;
    const int8_t *A = WP + ((uint64_t)t * Np + obase) * Kp;     // [128][Kp]
    const int8_t *B = XP + ((uint64_t)t * chunk + rbase) * Kp;  // [256][Kp]
    uint8_t *sA = smem, *sB = smem + kStages * kStageA;
    constexpr uint32_t kProducers = 128;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base)),
                     "r"(kBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&full[s])), "r"(kProducers));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[s])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&done)));
        asm volatile("fence.mbarrier_init.release.cluster;\n");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    const uint32_t tmem = tmem_base;
    const uint32_t nkb = Kp / kKB;
    // instruction descriptor: s32 accumulate, A and B signed int8, both K-major, N = 256, M = 128
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((kBN >> 3) << 17) | ((kBM >> 4) << 24);

    if (tid < kProducers) {
        bool ok = true;
        for (uint32_t kb = 0; kb < nkb; kb++) {
            const uint32_t s = kb % kStages;
            if (kb >= (uint32_t)kStages && !mbar_wait(smem_u32(&empty[s]), ((kb / kStages) - 1) & 1)) ok = false;
            const uint32_t a_dst = smem_u32(sA + s * kStageA), b_dst = smem_u32(sB + s * kStageB);
            const uint64_t koff = (uint64_t)kb * kKB;
            if (ok) {
                for (uint32_t c = tid; c < kBM * (kKB / 16); c += kProducers) {
                    const uint32_t row = c / (kKB / 16), kc = c % (kKB / 16);
                    cp_async16(a_dst + core_off(row, kc), A + (uint64_t)row * Kp + koff + kc * 16);
                }
                for (uint32_t c = tid; c < kBN * (kKB / 16); c += kProducers) {
                    const uint32_t row = c / (kKB / 16), kc = c % (kKB / 16);
                    cp_async16(b_dst + core_off(row, kc), B + (uint64_t)row * Kp + koff + kc * 16);
                }
            }
            asm volatile("cp.async.commit_group;\n");
            if (kb >= 1) {  // this thread's copies of stage kb - 1 have landed
                asm volatile("cp.async.wait_group 1;\n");
                asm volatile("fence.proxy.async.shared::cta;\n");
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&full[(kb - 1) % kStages])));
            }
        }
        asm volatile("cp.async.wait_group 0;\n");
        asm volatile("fence.proxy.async.shared::cta;\n");
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&full[(nkb - 1) % kStages])));
        if (!ok) failed = 1;
    } else if (tid == kProducers) {
        bool ok = true;
        for (uint32_t kb = 0; kb < nkb; kb++) {
            const uint32_t s = kb % kStages;
            if (!mbar_wait(smem_u32(&full[s]), (kb / kStages) & 1)) ok = false;
            asm volatile("tcgen05.fence::after_thread_sync;\n");
            if (ok) {
                const uint32_t a0 = smem_u32(sA + s * kStageA), b0 = smem_u32(sB + s * kStageB);
#pragma unroll
                for (uint32_t k = 0; k < kKB / 32; k++) {
                    uint64_t ad = smem_desc(a0 + k * 256), bd = smem_desc(b0 + k * 256);
                    uint32_t acc = (kb | k) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                        "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                smem_u32(&empty[s])));
        }
        // completes once every MMA above has
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
            smem_u32(&done)));
        if (!ok) failed = 1;
    }
    // the idle warps wait here instead of spinning beside the producers and the MMA thread
    __syncthreads();  // also publishes `failed` from the producer and MMA roles
    const bool landed = mbar_wait(smem_u32(&done), 0);
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    if (!landed || failed) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (outputs); warpgroup w / 4 takes one
        // half of the 256 X columns, 32 at a time
        const uint32_t quarter = warp & 3, half = warp >> 2;
        const uint32_t o = obase + quarter * 32 + lane;
        for (uint32_t c0 = half * (kBN / 2); c0 < (half + 1) * (kBN / 2); c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((quarter * 32) << 16) + c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n");
            if (o < n_out) {
                uint32_t pk[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    uint32_t w = 0;
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        w |= (acc24 ? mod_acc24((int)v[4 * j + b], t) : mod_acc((int)v[4 * j + b], t)) << (8 * b);
                    pk[j] = w;
                }
                uint4 *dst = reinterpret_cast<uint4 *>(RES + ((uint64_t)t * n_out + o) * chunk + rbase + c0);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kBN));
}

// ---------------------------------------------------------------- persistent GEMM
// For K <= kResKp the 256-column X tile of one modulus stays resident in shared memory (Kp / 64
// blocks of 16 KB in the MMA's core-matrix layout) while the CTA runs every output tile of it:
// the weight tiles (A, 128 outputs x 64 K bytes) stream through a kAStages ring, and the
// accumulators alternate between two 256-column TMEM buffers so that the epilogue of one output
// tile overlaps the MMAs of the next.  One CTA per SM (all 512 TMEM columns), persistent over
// the (modulus, column tile) pairs.  Roles: warps 0-3 copy (cp.async; the X tile together, then
// the A stages, warp w filling ring slot w and arriving on its barrier once its copies land, the
// next X tile prefetched into L2 meanwhile), one thread of warp 4
// issues the MMAs, warps 5-12 read the accumulators back (two warps per 32-lane quarter, one
// per half of the columns).  Every wait is bounded; after a timeout a role waits no more and
// carries on without its work, still arriving on its barriers, so the other roles finish too,
// and the call reports the failure through *err.
constexpr uint32_t kResKp = 768;
constexpr int kAStages = 4;  // one ring slot per producer warp
constexpr uint32_t kXBlock = kBN * kKB;  // 16 KB
constexpr uint32_t kSmemP = (kResKp / kKB) * kXBlock + kAStages * kStageA + 1024;
constexpr uint32_t kEpiWarp0 = 5;
constexpr uint32_t kThreadsP = (kEpiWarp0 + 8) * 32;

// TMA_A: both operands come by TMA (one thread issues the X tile's and the weight stages' loads,
// 64-byte swizzle, completion on their mbarriers) instead of the producer warps' cp.async
template <bool TMA_A>
__global__ void __launch_bounds__(kThreadsP, 1) mma_persistent_kernel(const int8_t *__restrict__ XP,
                                                                      const int8_t *__restrict__ WP,
                                                                      uint8_t *__restrict__ RES, uint32_t Kp,
                                                                      uint32_t Np, uint32_t n_out, uint64_t chunk,
                                                                      uint32_t T, int *__restrict__ err, int acc24,
                                                                      const __grid_constant__ CUtensorMap tmA,
                                                                      const __grid_constant__ CUtensorMap tmX) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);  // swizzle atoms need 1 KB alignment
    __shared__ __align__(8) uint64_t full[kAStages], empty[kAStages], x_full, x_empty, acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint8_t *sX = smem, *sA = smem + (kResKp / kKB) * kXBlock;
    const uint32_t nkb = Kp / kKB, n_ot = Np / kBM;
    const uint64_t n_ct = chunk / kBN, n_tiles = (uint64_t)T * n_ct;
    constexpr uint32_t kProducers = 128, kEpi = 256;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base)),
                     "r"(2 * kBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (tid == 0) {
        for (int s = 0; s < kAStages; s++) {
            // the TMA issuer's expect-tx arrival, or the 32 threads of the slot's producer warp
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&full[s])), "r"(TMA_A ? 1 : 32));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[s])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&x_full)), "r"(TMA_A ? 1 : kProducers));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&x_empty)));
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&acc_full[b])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&acc_empty[b])), "r"(kEpi));
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((kBN >> 3) << 17) | ((kBM >> 4) << 24);
    auto arrive = [](uint32_t bar) { asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar)); };

    if (tid < kProducers && !(TMA_A && warp > 0)) {
        // cp.async: producer warp w fills ring slot w (A stages w, w + 4, ...): each warp waits for
        // its own copies only, so four stages are in flight; all four copy the X tile together.
        // TMA: thread 0 issues every load (the X tile as Kp / 64 boxes of 256 rows, then the A
        // stages), its warp prefetches the next X tile into L2
        bool ok = true;
        uint64_t g = 0;   // A stages so far (ring position)
        uint32_t ti = 0;  // column tiles of this CTA so far
        const uint32_t kx16 = Kp / 16;
        for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ti++) {
            const uint32_t t = (uint32_t)(tile / n_ct);
            const uint64_t rbase = (tile % n_ct) * kBN;
            if constexpr (TMA_A) {
                if (tid == 0) {
                    // every MMA of the previous column tile must have read the X tile
                    if (ok && ti > 0 && !mbar_wait(smem_u32(&x_empty), (ti - 1) & 1)) ok = false;
                    const uint32_t bar = smem_u32(&x_full);
                    if (ok) {
                        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                                     "r"(kBN * Kp));
                        for (uint32_t kb = 0; kb < nkb; kb++)  // x = kb * 64 bytes: 16-byte aligned
                            asm volatile(
                                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                                "[%0], [%1, {%2, %3}], [%4];\n" ::"r"(smem_u32(sX + kb * kXBlock)),
                                "l"(reinterpret_cast<uint64_t>(&tmX)), "r"((int)(kb * kKB)),
                                "r"((int)((uint64_t)t * chunk + rbase)), "r"(bar)
                                : "memory");
                    } else {
                        arrive(bar);
                    }
                }
                __syncwarp();
            } else {
                // every MMA of the previous column tile must have read the X tile
                if (ok && ti > 0 && !mbar_wait(smem_u32(&x_empty), (ti - 1) & 1)) ok = false;
                const int8_t *B = XP + ((uint64_t)t * chunk + rbase) * Kp;
                if (ok)
                    for (uint32_t c = tid; c < kBN * kx16; c += kProducers) {
                        const uint32_t row = c / kx16, k16 = c % kx16;
                        cp_async16(smem_u32(sX + (k16 >> 2) * kXBlock) + core_off(row, k16 & 3),
                                   B + (uint64_t)row * Kp + k16 * 16);
                    }
                asm volatile("cp.async.commit_group;\n");
                asm volatile("cp.async.wait_group 0;\n");
                asm volatile("fence.proxy.async.shared::cta;\n");
                arrive(smem_u32(&x_full));
            }
            // the next column tile's X into L2 while this one's MMAs run
            const uint64_t next = tile + gridDim.x;
            if (next < n_tiles) {
                const int8_t *Bn = XP + ((uint64_t)(next / n_ct) * chunk + (next % n_ct) * kBN) * Kp;
                const uint32_t nthr = TMA_A ? 32 : kProducers;
                for (uint32_t off = tid * 128; off < kBN * Kp; off += nthr * 128)
                    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(Bn + off));
            }
            for (uint32_t o = 0; o < n_ot; o++) {
                const int8_t *A = WP + ((uint64_t)t * Np + o * kBM) * Kp;
                for (uint32_t kb = 0; kb < nkb; kb++, g++) {
                    const uint32_t s = (uint32_t)(g % kAStages);
                    if constexpr (TMA_A) {
                        if (tid != 0) continue;
                        if (ok && g >= (uint64_t)kAStages && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((g / kAStages) - 1) & 1))
                            ok = false;
                        const uint32_t bar = smem_u32(&full[s]);
                        if (ok) {
                            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                                         "r"(kStageA));
                            // x = kb * 64 bytes: 16-byte aligned as a tiled TMA load requires
                            asm volatile(
                                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                                "[%0], [%1, {%2, %3}], [%4];\n" ::"r"(smem_u32(sA + s * kStageA)),
                                "l"(reinterpret_cast<uint64_t>(&tmA)), "r"((int)(kb * kKB)),
                                "r"((int)(t * Np + o * kBM)), "r"(bar)
                                : "memory");
                        } else {
                            arrive(bar);  // no copy: the barrier still completes
                        }
                        continue;
                    }
                    if (s != warp) continue;
                    if (ok && g >= (uint64_t)kAStages && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((g / kAStages) - 1) & 1))
                        ok = false;
                    if (ok)
                        for (uint32_t c = lane; c < kBM * (kKB / 16); c += 32) {
                            const uint32_t row = c / (kKB / 16), kc = c % (kKB / 16);
                            cp_async16(smem_u32(sA + s * kStageA) + core_off(row, kc),
                                       A + (uint64_t)row * Kp + (uint64_t)kb * kKB + kc * 16);
                        }
                    asm volatile("cp.async.commit_group;\n");
                    asm volatile("cp.async.wait_group 0;\n");
                    asm volatile("fence.proxy.async.shared::cta;\n");
                    arrive(smem_u32(&full[s]));
                }
            }
        }
        if (!ok) failed = 1;
    } else if (tid == kProducers) {
        bool ok = true;
        uint64_t g = 0;
        uint32_t ti = 0, ai = 0;  // column tiles, accumulator tiles
        for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ti++) {
            if (ok && !mbar_wait(smem_u32(&x_full), ti & 1)) ok = false;
            asm volatile("tcgen05.fence::after_thread_sync;\n");
            for (uint32_t o = 0; o < n_ot; o++, ai++) {
                const uint32_t buf = ai & 1;
                if (ok && ai >= 2 && !mbar_wait(smem_u32(&acc_empty[buf]), ((ai >> 1) - 1) & 1)) ok = false;
                asm volatile("tcgen05.fence::after_thread_sync;\n");
                for (uint32_t kb = 0; kb < nkb; kb++, g++) {
                    const uint32_t s = (uint32_t)(g % kAStages);
                    if (ok && !mbar_wait(smem_u32(&full[s]), (uint32_t)(g / kAStages) & 1)) ok = false;
                    asm volatile("tcgen05.fence::after_thread_sync;\n");
                    if (ok) {
                        const uint32_t a0 = smem_u32(sA + s * kStageA), b0 = smem_u32(sX + kb * kXBlock);
#pragma unroll
                        for (uint32_t k = 0; k < kKB / 32; k++) {
                            const uint64_t ad = TMA_A ? smem_desc_sw64(a0 + k * 32) : smem_desc(a0 + k * 256);
                            const uint64_t bd = TMA_A ? smem_desc_sw64(b0 + k * 32) : smem_desc(b0 + k * 256);
                            const uint32_t accum = (kb | k) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + buf * kBN),
                                "l"(ad), "l"(bd), "r"(idesc), "r"(accum));
                        }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                        smem_u32(&empty[s])));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                    smem_u32(&acc_full[buf])));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                smem_u32(&x_empty)));
        }
        if (!ok) failed = 1;
    } else if (warp >= kEpiWarp0) {
        bool ok = true;
        const uint32_t quarter = warp & 3, half = (warp - kEpiWarp0) >> 2;
        uint32_t ai = 0;
        for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
            const uint32_t t = (uint32_t)(tile / n_ct);
            const uint64_t rbase = (tile % n_ct) * kBN;
            for (uint32_t o = 0; o < n_ot; o++, ai++) {
                const uint32_t buf = ai & 1;
                if (ok && !mbar_wait(smem_u32(&acc_full[buf]), (ai >> 1) & 1)) ok = false;
                asm volatile("tcgen05.fence::after_thread_sync;\n");
                const uint32_t out = o * kBM + quarter * 32 + lane;
                if (ok) {
                    for (uint32_t c0 = half * (kBN / 2); c0 < (half + 1) * (kBN / 2); c0 += 32) {
                        uint32_t v[32];
                        const uint32_t taddr = tmem + ((quarter * 32) << 16) + buf * kBN + c0;
                        asm volatile(
                            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                              "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
                              "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
                              "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                            : "r"(taddr));
                        asm volatile("tcgen05.wait::ld.sync.aligned;\n");
                        if (out < n_out) {
                            uint32_t pk[8];
#pragma unroll
                            for (int j = 0; j < 8; j++) {
                                uint32_t w = 0;
#pragma unroll
                                for (int b = 0; b < 4; b++)
                                    w |= (acc24 ? mod_acc24((int)v[4 * j + b], t) : mod_acc((int)v[4 * j + b], t))
                                         << (8 * b);
                                pk[j] = w;
                            }
                            uint4 *dst = reinterpret_cast<uint4 *>(RES + ((uint64_t)t * n_out + out) * chunk + rbase + c0);
                            dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                            dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                        }
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;\n");
                arrive(smem_u32(&acc_empty[buf]));
            }
        }
        if (!ok) failed = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    if (tid == 0 && failed) atomicExch(err, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * kBN));
}

// ---------------------------------------------------------------- CRT fold
struct CrtLimb {
    uint64_t c[kMaxMods];  // c_t mod q_l
    uint64_t M;            // M mod q_l
    uint64_t Mneg;         // q_l - (M mod q_l), below q_l
};

// Fraction bits of the fixed-point CRT fractions F_t = round(2^19 [(M/m_t)^-1]_{m_t} / m_t): with
// r_t < 251 and T <= 20, sum_t r_t F_t + 2^18 < 2^32, and the sum's rounding error
// T 251 2^-20 < 0.005 keeps v = round(sum_t r_t frac_t) exact (M > 2.02 |S| leaves the true sum
// within 0.495 of an integer).
constexpr uint32_t kCrtFracBits = 19;

// workspace bytes before the residue planes: the error flag, then the CRT tables for every
// moduli count in use (at most kMaxMods counts of up to 64 limbs)
constexpr size_t kCrtTabBytes = 256 + sizeof(CrtLimb) * 64 * kMaxMods;

// One thread folds 4 consecutive columns r of one output (4-byte residue loads, two 16-byte
// stores).  The host sizes the block so that its 4 blockDim.x columns lie in one limb: the limb's
// constants (the 32-bit halves of c_t and the fixed-point fractions) are staged in shared memory
// once per block.  Per residue and column three integer multiply-adds:
//   lo += r_t (c_t mod 2^32),  hi += r_t (c_t >> 32)   (exact sums),
//   v  += r_t F_t                                        (32-bit fixed point),
// then S = lo + hi 2^32 - v M = lo + hi 2^32 + v (q - M mod q) mod q, one Barrett reduction
// (the sum is below 20 251 2^61 + 2^13 2^61 < 2^75).  HI32: the host has checked that
// T 250 max(c_t >> 32) < 2^32, so hi is summed in 32 bits.  The residue words (one per modulus,
// read once: streaming loads) are requested before the fold.
template <bool HI32>
__global__ void __launch_bounds__(256) crt_kernel(const uint8_t *__restrict__ RES, uint64_t *__restrict__ Y,
                                                  const CrtLimb *__restrict__ tab, uint32_t n_out, uint64_t chunk,
                                                  uint64_t r0, uint64_t R, uint32_t L, uint32_t log_n,
                                                  const PrimeConst *__restrict__ pc, uint32_t T) {
    __shared__ uint32_t s_lo[kMaxMods], s_hi[kMaxMods], s_f[kMaxMods];
    const uint64_t rb = (uint64_t)blockIdx.x * blockDim.x * 4;
    const uint32_t o = blockIdx.y;
    const uint32_t row = (uint32_t)((r0 + rb) >> log_n);  // h L + limb, below 2 L
    const uint32_t limb = row >= L ? row - L : row;
    if (threadIdx.x < (uint32_t)kMaxMods) {
        const uint32_t t = threadIdx.x;
        const uint64_t c = t < T ? tab[limb].c[t] : 0;
        s_lo[t] = (uint32_t)c;
        s_hi[t] = (uint32_t)(c >> 32);
        s_f[t] = t < T ? c_mods.fracq[T][t] : 0u;
    }
    __syncthreads();
    const uint64_t r = rb + (uint64_t)threadIdx.x * 4;
    if (r >= chunk) return;
    const uint64_t rg = r0 + r;
    const PrimeConst p = pc[limb];
    const uint64_t Mneg = tab[limb].Mneg;
    constexpr uint32_t kAhead = 16;  // residue words requested before the fold
    uint32_t res[kAhead];
#pragma unroll
    for (uint32_t t = 0; t < kAhead; t++)
        res[t] = t < T ? __ldcs(reinterpret_cast<const uint32_t *>(RES + ((uint64_t)t * n_out + o) * chunk + r)) : 0u;
    using HiT = typename std::conditional<HI32, uint32_t, uint64_t>::type;
    uint64_t lo[4] = {0, 0, 0, 0};
    HiT hi[4] = {0, 0, 0, 0};
    uint32_t v[4];
#pragma unroll
    for (int e = 0; e < 4; e++) v[e] = 1u << (kCrtFracBits - 1);
#pragma unroll
    for (uint32_t t = 0; t < (uint32_t)kMaxMods; t++) {
        if (t < T) {
            const uint32_t r4 =
                t < kAhead ? res[t]
                           : __ldcs(reinterpret_cast<const uint32_t *>(RES + ((uint64_t)t * n_out + o) * chunk + r));
            const uint32_t cl = s_lo[t], ch = s_hi[t], f = s_f[t];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const uint32_t rt = (r4 >> (8 * e)) & 0xFF;
                lo[e] += (uint64_t)rt * cl;
                hi[e] += (HiT)rt * ch;
                v[e] += rt * f;
            }
        }
    }
    uint64_t y[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const uint64_t h = hi[e];
        const uint64_t plo = lo[e] + (h << 32);
        u128 pos = {plo, (h >> 32) + (plo < lo[e] ? 1ull : 0ull)};
        mac(pos, v[e] >> kCrtFracBits, Mneg);
        y[e] = barrett(pos, p);
    }
    ulonglong2 *out = reinterpret_cast<ulonglong2 *>(Y + (uint64_t)o * R + rg);
    out[0] = make_ulonglong2(y[0], y[1]);
    out[1] = make_ulonglong2(y[2], y[3]);
}

}  // namespace

// ------------------------------------------------------------------ host side

namespace {

struct Plan {
    ModTab mods;
    uint32_t T_min = 0, T_max = 0;   // the moduli counts the limbs need
    std::vector<uint32_t> limb_T;    // per limb
    std::vector<CrtLimb> limbs;      // [T - T_min][L]: the CRT constants for each count in use
    bool hi32 = false;               // T_max 250 max(c_t >> 32) < 2^32: the CRT's high sums in 32 bits
};

// The moduli count of each limb: |S| = |sum_i x_i w_io| <= (q_l - 1) max_o sum_i |w_io| = B_l, and
// the CRT with the fixed-point v (error below 0.005) is exact while M > 2 B_l / (1 - 0.01); the
// product of the first T candidates must exceed that (log2 M >= log2 B_l + 1.05).
Plan make_plan(const Context &c, uint32_t L, uint64_t max_l1) {
    static const uint32_t cand[kMaxMods] = {251, 241, 239, 233, 229, 227, 223, 211, 199, 197,
                                            193, 191, 181, 179, 173, 167, 163, 157, 151, 149};
    Plan p{};
    p.limb_T.resize(L);
    p.T_min = kMaxMods;
    uint64_t max_hi = 0;
    for (uint32_t l = 0; l < L; l++) {
        const uint64_t q = c.primes[l];
        const double need = std::log2((double)(q - 1)) + std::log2((double)std::max<uint64_t>(max_l1, 1)) + 1.05;
        double have = 0;
        uint32_t T = 0;
        while (have < need) {
            if (T >= (uint32_t)kMaxMods) throw std::invalid_argument("ct-pt matmul: weights or inputs too large");
            have += std::log2((double)cand[T]);
            T++;
        }
        p.limb_T[l] = T;
        p.T_min = std::min(p.T_min, T);
        p.T_max = std::max(p.T_max, T);
        max_hi = std::max(max_hi, (q - 1) >> 32);
    }
    p.hi32 = (uint64_t)p.T_max * 250 * max_hi < (1ull << 32);
    for (uint32_t t = 0; t < (uint32_t)kMaxMods; t++) {
        const uint32_t m = cand[t];
        p.mods.m[t] = m;
        p.mods.c24[t] = (1u << 20) % m;
        p.mods.c48[t] = (uint32_t)((uint64_t)p.mods.c24[t] * p.mods.c24[t] % m);
        p.mods.magic[t] = (uint32_t)(((1ull << 32) + m - 1) / m);
        p.mods.inv[t] = 1.0 / m;
        p.mods.invf[t] = 1.0f / (float)m;
    }
    // CRT fractions [(M/m_t)^-1 mod m_t] / m_t in fixed point, for every modulus count
    for (uint32_t n = 1; n <= (uint32_t)kMaxMods; n++)
        for (uint32_t t = 0; t < n; t++) {
            const uint32_t m = cand[t];
            uint32_t Mt_mod_m = 1;
            for (uint32_t u = 0; u < n; u++)
                if (u != t) Mt_mod_m = (uint32_t)((uint64_t)Mt_mod_m * (cand[u] % m) % m);
            const uint32_t inv = (uint32_t)host::powmod(Mt_mod_m, m - 2, m);  // m prime
            p.mods.fracq[n][t] = (uint32_t)((((uint64_t)inv << kCrtFracBits) + m / 2) / m);
        }
    // CRT constants for each count T in use: c_t = (M/m_t) * [(M/m_t)^-1 mod m_t] mod q_l
    p.limbs.resize((size_t)(p.T_max - p.T_min + 1) * L);
    for (uint32_t T = p.T_min; T <= p.T_max; T++)
        for (uint32_t l = 0; l < L; l++) {
            CrtLimb &cl = p.limbs[(size_t)(T - p.T_min) * L + l];
            uint64_t q = c.primes[l], M = 1;
            for (uint32_t u = 0; u < T; u++) M = host::mulmod(M, cand[u], q);
            cl.M = M;
            cl.Mneg = (q - M) % q;
            for (uint32_t t = 0; t < T; t++) {
                uint32_t m = cand[t], Mt_mod_m = 1;
                uint64_t Mt = 1;
                for (uint32_t u = 0; u < T; u++)
                    if (u != t) {
                        Mt = host::mulmod(Mt, cand[u], q);
                        Mt_mod_m = (uint32_t)((uint64_t)Mt_mod_m * (cand[u] % m) % m);
                    }
                uint32_t inv = (uint32_t)host::powmod(Mt_mod_m, m - 2, m);
                cl.c[t] = host::mulmod(Mt, inv, q);
            }
        }
    return p;
}

}  // namespace

// Residue planes [rows][Kp] (the weights' or X's) as a 2D tensor map for TMA: 64-byte K boxes of
// box_rows rows with the 64-byte swizzle.  False when the driver's encoder is unavailable or
// refuses, or when the environment sets SHMOAI_CTPT_TMA=0 (then the producer warps copy the
// operand tiles with cp.async).
bool operand_tensor_map(CUtensorMap *map, const int8_t *P, uint32_t Kp, uint64_t rows, uint32_t box_rows) {
    static PFN_cuTensorMapEncodeTiled encode = [] {
        const char *off = std::getenv("SHMOAI_CTPT_TMA");
        if (off && off[0] == '0') return (PFN_cuTensorMapEncodeTiled) nullptr;
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        cudaGetLastError();
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
    }();
    if (!encode) return false;
    const cuuint64_t dims[2] = {Kp, rows}, strides[1] = {Kp};
    const cuuint32_t box[2] = {kKB, box_rows}, estr[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t *>(P), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// columns of X processed per pass (bounds the residue workspaces); the environment variable
// SHMOAI_CTPT_CHUNK (a multiple of 256) replaces the default, read once per process
constexpr uint64_t kChunkCols = 131072;

static uint64_t chunk_cols() {
    static const uint64_t v = [] {
        const char *s = std::getenv("SHMOAI_CTPT_CHUNK");
        const uint64_t c = s ? std::strtoull(s, nullptr, 10) : 0;
        return (c >= kBN && c % kBN == 0) ? c : kChunkCols;
    }();
    return v;
}

size_t ctpt_tc_ws_bytes(const Context &c, uint32_t n_in, uint32_t n_out, uint32_t L) {
    const uint64_t R = 2ull * L * c.n;
    const uint64_t chunk = std::min<uint64_t>(R, chunk_cols());
    const uint32_t Kp = (n_in + kKB - 1) / kKB * kKB, Np = (n_out + kBM - 1) / kBM * kBM;
    return (size_t)kMaxMods * (chunk * Kp + (uint64_t)Np * Kp + (uint64_t)n_out * chunk) + kCrtTabBytes;
}

// Chunks of 131,072 columns run one after the other on `st`.  (Alternating them over two
// streams, so that one chunk's residue and CRT kernels could run beside the other's GEMM,
// measured no faster: the GEMM's grid fills every SM.)
void ctpt_matmul_tc(const Context &c, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in, uint32_t n_out,
                    uint32_t L, void *ws, uint64_t max_l1, cudaStream_t st) {
    if (n_in == 0 || n_out == 0) return;
    const uint64_t R = 2ull * L * c.n;
    if (R % kBN) throw std::invalid_argument("ct-pt matmul: 2 L N must be a multiple of 256");
    const uint64_t chunk = std::min<uint64_t>(R, chunk_cols());
    const uint32_t Kp = (n_in + kKB - 1) / kKB * kKB, Np = (n_out + kBM - 1) / kBM * kBM;
    Plan plan = make_plan(c, L, max_l1);
    const uint32_t T = plan.T_max;  // the weight planes and the workspaces hold T_max moduli
    SHM_CUDA(cudaMemcpyToSymbolAsync(c_mods, &plan.mods, sizeof(ModTab), 0, cudaMemcpyHostToDevice, st));
    // workspace carve-up
    uint8_t *base = static_cast<uint8_t *>(ws);
    int *err = reinterpret_cast<int *>(base);
    CrtLimb *tab = reinterpret_cast<CrtLimb *>(base + 256);
    int8_t *XP = reinterpret_cast<int8_t *>(base + kCrtTabBytes);
    int8_t *WP = XP + (size_t)T * chunk * Kp;
    uint8_t *RES = reinterpret_cast<uint8_t *>(WP + (size_t)T * Np * Kp);
    if (plan.limbs.size() > (size_t)64 * kMaxMods) throw std::invalid_argument("ct-pt matmul: too many limbs");
    SHM_CUDA(cudaMemcpyAsync(tab, plan.limbs.data(), sizeof(CrtLimb) * plan.limbs.size(), cudaMemcpyHostToDevice, st));
    SHM_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    // zero-padded K tail of the X planes stays zero: clear once per call
    if (Kp != n_in) SHM_CUDA(cudaMemsetAsync(XP, 0, (size_t)T * chunk * Kp, st));
    SHM_LAUNCHED(1);
    wres_kernel<<<dim3((Kp + 255) / 256, Np), 256, 0, st>>>(W, WP, n_in, n_out, Kp, Np, T);
    SHM_CUDA(cudaGetLastError());
    const bool resident = Kp <= kResKp;  // the X tile fits in shared memory: the persistent kernel
    CUtensorMap tmA, tmX;
    std::memset(&tmA, 0, sizeof tmA);
    std::memset(&tmX, 0, sizeof tmX);
    const bool tma_a = resident && operand_tensor_map(&tmA, WP, Kp, (uint64_t)T * Np, kBM);
    if (resident)
        SHM_CUDA(cudaFuncSetAttribute(tma_a ? mma_persistent_kernel<true> : mma_persistent_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemP));
    else
        SHM_CUDA(cudaFuncSetAttribute(mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem));
    int sms = 0;
    SHM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
    const int acc24 = (uint64_t)Kp * 125 * 125 < (1ull << 24) ? 1 : 0;  // accumulators exact in float
    bool f64_res = true;  // every limb prime below 2^51: the X residues on the FP64 pipe
    for (uint32_t l = 0; l < L; l++) f64_res = f64_res && c.primes[l] < (1ull << 51);
    SHM_CUDA(cudaFuncSetAttribute(f64_res ? xres_kernel<true> : xres_kernel<false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, kXresSmem));
    for (uint64_t r0 = 0; r0 < R; r0 += chunk) {
        // a shorter last pass (2 L N not a multiple of the chunk, e.g. at N = 2^12) lays its planes out
        // with its own column count; every count here is a multiple of 256
        const uint64_t cur = std::min<uint64_t>(chunk, R - r0);
        // the pass's moduli count: the largest its limbs (rows h L + l, h = 0, 1) need
        uint32_t Tc = 0;
        for (uint64_t row = r0 >> c.log_n; row <= (r0 + cur - 1) >> c.log_n; row++)
            Tc = std::max(Tc, plan.limb_T[row % L]);
        const CrtLimb *tab_c = tab + (size_t)(Tc - plan.T_min) * L;
        SHM_LAUNCHED(1);
        const dim3 xgrid((uint32_t)(cur / (64 * kXresTiles)), (n_in + 63) / 64);
        if (f64_res)
            xres_kernel<true><<<xgrid, 256, kXresSmem, st>>>(X, XP, n_in, Kp, R, r0, cur, Tc);
        else
            xres_kernel<false><<<xgrid, 256, kXresSmem, st>>>(X, XP, n_in, Kp, R, r0, cur, Tc);
        SHM_CUDA(cudaGetLastError());
        SHM_LAUNCHED(1);
        if (resident) {
            const uint64_t tiles = (uint64_t)Tc * (cur / kBN);
            const uint32_t grid = (uint32_t)std::min<uint64_t>(tiles, (uint64_t)sms);
            // the X planes of this pass, [T * cur][Kp], as 256-row boxes (a pass's planes have its own
            // column count)
            const bool tma = tma_a && operand_tensor_map(&tmX, XP, Kp, (uint64_t)Tc * cur, kBN);
            if (tma)
                mma_persistent_kernel<true>
                    <<<grid, kThreadsP, kSmemP, st>>>(XP, WP, RES, Kp, Np, n_out, cur, Tc, err, acc24, tmA, tmX);
            else
                mma_persistent_kernel<false>
                    <<<grid, kThreadsP, kSmemP, st>>>(XP, WP, RES, Kp, Np, n_out, cur, Tc, err, acc24, tmA, tmX);
        } else {
            mma_kernel<<<dim3(Np / kBM, (uint32_t)(cur / kBN), Tc), kThreads, kSmem, st>>>(XP, WP, RES, Kp, Np, n_out,
                                                                                          cur, err, acc24);
        }
        SHM_CUDA(cudaGetLastError());
        SHM_LAUNCHED(1);
        // 4 columns a thread; a block's columns within one limb (N and r0 are multiples of the block's)
        const uint32_t crt_threads = chunk % 1024 == 0 ? 256 : 64;
        const dim3 cgrid((uint32_t)((cur / 4 + crt_threads - 1) / crt_threads), n_out);
        if (plan.hi32)
            crt_kernel<true><<<cgrid, crt_threads, 0, st>>>(RES, Y, tab_c, n_out, cur, r0, R, L, c.log_n, c.pc, Tc);
        else
            crt_kernel<false><<<cgrid, crt_threads, 0, st>>>(RES, Y, tab_c, n_out, cur, r0, R, L, c.log_n, c.pc, Tc);
        SHM_CUDA(cudaGetLastError());
    }
}

int ctpt_tc_error(void *ws, cudaStream_t st) {
    int h = 0;
    SHM_CUDA(cudaMemcpyAsync(&h, ws, sizeof(int), cudaMemcpyDeviceToHost, st));
    SHM_CUDA(cudaStreamSynchronize(st));
    return h;
}

}  // namespace shm
