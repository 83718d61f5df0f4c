// Canonical-embedding encode and decode on the GPU in FP64 (the only floating-point work of
// the library): a batched radix-2 FFT of M = 2N points per slot vector.  The reference encodes
// one vector at a time with a host round trip per call (thirdparty/phantom-fhe/src/ckks.cu:89-246,
// fft.cu:358-439); here a whole batch is one sequence of launches.
//
// The arithmetic is the host encoder's (shmoai::Encoder::encode_float / decode, host_core.cpp)
// operation for operation: the same twiddles (cos / sin of 2 pi k / M, computed on the host),
// the same butterflies with every multiply and add rounded on its own (__dmul_rn, __dadd_rn,
// no contraction), so the coefficients are identical to the host's bit for bit.
#include <cmath>

#include "core.hpp"

namespace shm {

namespace {

constexpr int kT = 256;

struct EncTables {
    double2 *roots = nullptr;  // [M]: (cos, sin)(2 pi k / M)
    uint32_t *exps = nullptr;  // [N/2]: 5^j mod M
};

std::mutex g_tab_mu;
std::map<const Context *, EncTables> g_tabs;

const EncTables &tables(const Context &c) {
    std::lock_guard<std::mutex> g(g_tab_mu);
    auto it = g_tabs.find(&c);
    if (it != g_tabs.end()) return it->second;
    const uint32_t M = 2 * c.n, slots = c.n / 2;
    std::vector<double2> r(M);
    for (uint32_t k = 0; k < M; k++) {
        const double ang = 2.0 * M_PI * (double)k / (double)M;
        r[k] = make_double2(std::cos(ang), std::sin(ang));
    }
    std::vector<uint32_t> e(slots);
    uint64_t v = 1;
    for (uint32_t j = 0; j < slots; j++) {
        e[j] = (uint32_t)v;
        v = (v * 5) % M;
    }
    EncTables t;
    SHM_CUDA(cudaMalloc(&t.roots, M * sizeof(double2)));
    SHM_CUDA(cudaMemcpy(t.roots, r.data(), M * sizeof(double2), cudaMemcpyHostToDevice));
    SHM_CUDA(cudaMalloc(&t.exps, slots * sizeof(uint32_t)));
    SHM_CUDA(cudaMemcpy(t.exps, e.data(), slots * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return g_tabs.emplace(&c, t).first->second;
}

__device__ __forceinline__ uint32_t brev(uint32_t x, uint32_t logm) { return __brev(x) >> (32 - logm); }

// A[p][brev(5^j)] = z_j (the rest zero, cleared before): the forward FFT's input in bit-reversed order
__global__ void enc_scatter(const double *__restrict__ re, const double *__restrict__ im, double2 *__restrict__ A,
                            const uint32_t *__restrict__ exps, uint32_t n_values, uint32_t logm) {
    const uint32_t p = blockIdx.y, j = blockIdx.x * kT + threadIdx.x;
    if (j >= n_values) return;
    A[((size_t)p << logm) + brev(exps[j], logm)] = make_double2(re[(size_t)p * n_values + j], im[(size_t)p * n_values + j]);
}

// one radix-2 stage of length `len` over every point: u = a[i+k], v = a[i+k+h] * w,
// a[i+k] = u + v, a[i+k+h] = u - v; w = roots[k M / len], conjugated for the forward transform
__global__ void fft_stage(double2 *__restrict__ A, const double2 *__restrict__ roots, uint32_t len, uint32_t logm,
                          int forward) {
    const uint32_t p = blockIdx.y, b = blockIdx.x * kT + threadIdx.x, half = len >> 1;
    const uint32_t M = 1u << logm;
    if (b >= (M >> 1)) return;
    const uint32_t k = b % half, i = (b / half) * len;
    double2 w = roots[(size_t)k * (M / len)];
    if (forward) w.y = -w.y;
    double2 *a = A + ((size_t)p << logm);
    const double2 u = a[i + k], x = a[i + k + half];
    const double2 v = make_double2(__dsub_rn(__dmul_rn(x.x, w.x), __dmul_rn(x.y, w.y)),
                                   __dadd_rn(__dmul_rn(x.x, w.y), __dmul_rn(x.y, w.x)));
    a[i + k] = make_double2(__dadd_rn(u.x, v.x), __dadd_rn(u.y, v.y));
    a[i + k + half] = make_double2(__dsub_rn(u.x, v.x), __dsub_rn(u.y, v.y));
}

// coeffs[p][k] = round-half-even(f * Re A[p][k]), k < N; *bad = 1 when a value reaches 2^62
__global__ void enc_round(const double2 *__restrict__ A, int64_t *__restrict__ coeffs, double f, uint32_t n,
                          uint32_t logm, int *__restrict__ bad) {
    const uint32_t p = blockIdx.y, k = blockIdx.x * kT + threadIdx.x;
    if (k >= n) return;
    const double r = rint(__dmul_rn(f, A[((size_t)p << logm) + k].x));
    if (!(fabs(r) < 4611686018427387904.0)) {
        *bad = 1;
        coeffs[(size_t)p * n + k] = 0;
        return;
    }
    coeffs[(size_t)p * n + k] = (int64_t)r;
}

// B[p][brev(k)] = (coeffs[p][k], 0), k < N (the rest zero, cleared before)
__global__ void dec_scatter(const double *__restrict__ coeffs, double2 *__restrict__ B, uint32_t n, uint32_t logm) {
    const uint32_t p = blockIdx.y, k = blockIdx.x * kT + threadIdx.x;
    if (k >= n) return;
    B[((size_t)p << logm) + brev(k, logm)] = make_double2(coeffs[(size_t)p * n + k], 0.0);
}

// z_j = B[p][5^j] / scale
__global__ void dec_gather(const double2 *__restrict__ B, const uint32_t *__restrict__ exps, double *__restrict__ re,
                           double *__restrict__ im, uint32_t slots, uint32_t logm, double scale) {
    const uint32_t p = blockIdx.y, j = blockIdx.x * kT + threadIdx.x;
    if (j >= slots) return;
    const double2 v = B[((size_t)p << logm) + exps[j]];
    re[(size_t)p * slots + j] = __ddiv_rn(v.x, scale);
    im[(size_t)p * slots + j] = __ddiv_rn(v.y, scale);
}

void run_fft(const Context &c, double2 *A, uint32_t n_pts, bool forward, cudaStream_t st) {
    const uint32_t M = 2 * c.n, logm = c.log_n + 1;
    const EncTables &t = tables(c);
    for (uint32_t len = 2; len <= M; len <<= 1) {
        SHM_LAUNCHED(1);
        fft_stage<<<dim3((M / 2 + kT - 1) / kT, n_pts), kT, 0, st>>>(A, t.roots, len, logm, forward ? 1 : 0);
        SHM_CUDA(cudaGetLastError());
    }
}

}  // namespace

size_t encode_ws_bytes(const Context &c, uint32_t n_pts) { return (size_t)n_pts * 2 * c.n * sizeof(double2) + 256; }

bool encode(const Context &c, const double *re, const double *im, uint32_t n_pts, uint32_t n_values, double scale,
            int64_t *coeffs, void *ws, cudaStream_t st) {
    if (n_values > c.n / 2) throw std::invalid_argument("more values than slots");
    if (!n_pts) return true;
    const uint32_t M = 2 * c.n, logm = c.log_n + 1;
    const EncTables &t = tables(c);
    int *bad = static_cast<int *>(ws);
    double2 *A = reinterpret_cast<double2 *>(static_cast<uint8_t *>(ws) + 256);
    SHM_CUDA(cudaMemsetAsync(ws, 0, encode_ws_bytes(c, n_pts), st));
    if (n_values) {
        SHM_LAUNCHED(1);
        enc_scatter<<<dim3((n_values + kT - 1) / kT, n_pts), kT, 0, st>>>(re, im, A, t.exps, n_values, logm);
        SHM_CUDA(cudaGetLastError());
    }
    run_fft(c, A, n_pts, true, st);
    SHM_LAUNCHED(1);
    enc_round<<<dim3(c.n / kT, n_pts), kT, 0, st>>>(A, coeffs, 2.0 * scale / (double)c.n, c.n, logm, bad);
    SHM_CUDA(cudaGetLastError());
    int h = 0;
    SHM_CUDA(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    SHM_CUDA(cudaStreamSynchronize(st));
    (void)M;
    return h == 0;
}

void decode(const Context &c, const double *coeffs, uint32_t n_pts, double scale, double *re, double *im, void *ws,
            cudaStream_t st) {
    if (!n_pts) return;
    const uint32_t logm = c.log_n + 1, slots = c.n / 2;
    const EncTables &t = tables(c);
    double2 *B = reinterpret_cast<double2 *>(static_cast<uint8_t *>(ws) + 256);
    SHM_CUDA(cudaMemsetAsync(ws, 0, encode_ws_bytes(c, n_pts), st));
    SHM_LAUNCHED(1);
    dec_scatter<<<dim3(c.n / kT, n_pts), kT, 0, st>>>(coeffs, B, c.n, logm);
    SHM_CUDA(cudaGetLastError());
    run_fft(c, B, n_pts, false, st);
    SHM_LAUNCHED(1);
    dec_gather<<<dim3((slots + kT - 1) / kT, n_pts), kT, 0, st>>>(B, t.exps, re, im, slots, logm, scale);
    SHM_CUDA(cudaGetLastError());
}

void release_encode_tables(const Context &c) {
    std::lock_guard<std::mutex> g(g_tab_mu);
    auto it = g_tabs.find(&c);
    if (it == g_tabs.end()) return;
    cudaFree(it->second.roots);
    cudaFree(it->second.exps);
    g_tabs.erase(it);
}

}  // namespace shm
