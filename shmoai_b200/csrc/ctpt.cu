// Rotation-free ct-pt matmul, CUDA-core path.
//
// Y[o][h][l][k] = sum_i X[i][h][l][k] * W[i][o]  (mod q_l), the exact result of the
// reference's multiply_plain(X_i, Enc(W_io)) + add_inplace loop
// (src/include/source/matrix_mul/Ct_pt_matrix_mul.cuh:112-158), where a constant
// plaintext in NTT form is the residue of the signed integer W_io in every slot.
//
// The signed weights are small (|W| < 2^40), so each thread accumulates the
// positive and the negative part of sum_i x_i * |W_io| exactly in two 128-bit
// registers and reduces once at the end.
#include <algorithm>

#include "core.hpp"

namespace shm {

namespace {

constexpr int kCtThreads = 128;
constexpr int kOutTile = 8;
constexpr int kInTile = 64;

// grid: (N/128, 2L, n_out/8); each thread owns one coefficient of one limb row and 8 outputs
__global__ void __launch_bounds__(kCtThreads) ctpt_cuda_core(const uint64_t *__restrict__ X,
                                                             const int64_t *__restrict__ W, uint64_t *__restrict__ Y,
                                                             uint32_t n_in, uint32_t n_out, uint32_t L, uint32_t log_n,
                                                             const PrimeConst *__restrict__ pc) {
    __shared__ uint64_t s_mag[kInTile][kOutTile];
    __shared__ uint8_t s_neg[kInTile][kOutTile];
    const uint32_t r = blockIdx.y;  // row within a ciphertext: h * L + l
    const uint32_t l = r % L;
    const uint32_t o0 = blockIdx.z * kOutTile;
    const size_t n = (size_t)1 << log_n;
    const size_t ctw = 2 * (size_t)L * n;
    const size_t k = (size_t)r * n + blockIdx.x * kCtThreads + threadIdx.x;
    u128 pos[kOutTile], neg[kOutTile];
#pragma unroll
    for (int o = 0; o < kOutTile; o++) pos[o] = neg[o] = {0, 0};
    for (uint32_t i0 = 0; i0 < n_in; i0 += kInTile) {
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < kInTile * kOutTile; t += kCtThreads) {
            uint32_t ii = t / kOutTile, oo = t % kOutTile;
            int64_t w = (i0 + ii < n_in && o0 + oo < n_out) ? W[(size_t)(i0 + ii) * n_out + o0 + oo] : 0;
            s_neg[ii][oo] = w < 0;
            s_mag[ii][oo] = w < 0 ? (uint64_t)(-(w + 1)) + 1 : (uint64_t)w;
        }
        __syncthreads();
        const uint32_t iend = min(kInTile, n_in - i0);
        for (uint32_t ii = 0; ii < iend; ii++) {
            const uint64_t x = X[(size_t)(i0 + ii) * ctw + k];
#pragma unroll
            for (int o = 0; o < kOutTile; o++) {
                if (s_neg[ii][o]) mac(neg[o], x, s_mag[ii][o]);
                else mac(pos[o], x, s_mag[ii][o]);
            }
        }
    }
    const PrimeConst p = pc[l];
#pragma unroll
    for (int o = 0; o < kOutTile; o++) {
        if (o0 + o >= n_out) break;
        Y[(size_t)(o0 + o) * ctw + k] = sub_mod(barrett(pos[o], p), barrett(neg[o], p), p.q);
    }
}

}  // namespace

void ctpt_matmul_cuda_core(const Context &c, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in,
                           uint32_t n_out, uint32_t L, cudaStream_t st) {
    if (n_in == 0 || n_out == 0) return;
    if (L < 1 || L > c.nq) throw std::invalid_argument("level out of range");
    dim3 grid(c.n / kCtThreads, 2 * L, (n_out + kOutTile - 1) / kOutTile);
    SHM_LAUNCHED(1); ctpt_cuda_core<<<grid, kCtThreads, 0, st>>>(X, W, Y, n_in, n_out, L, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
}

size_t ctpt_ws_words(const Context &c, uint32_t n_in, uint32_t n_out, uint32_t L) {
    return (ctpt_tc_ws_bytes(c, n_in, n_out, L) + 7) / 8;
}

void ctpt_matmul(const Context &c, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in, uint32_t n_out,
                 uint32_t L, uint64_t *ws, cudaStream_t st) {
    if (n_in == 0 || n_out == 0) return;
    if (L < 1 || L > c.nq) throw std::invalid_argument("level out of range");
    // the residue system is sized from the largest column sum of |W| (one small device-to-host copy
    // of the weights); every |W| must be below 2^40
    std::vector<int64_t> hw((size_t)n_in * n_out);
    SHM_CUDA(cudaMemcpyAsync(hw.data(), W, hw.size() * 8, cudaMemcpyDeviceToHost, st));
    SHM_CUDA(cudaStreamSynchronize(st));
    std::vector<uint64_t> l1(n_out, 0);
    uint64_t mx = 0;
    for (uint32_t i = 0; i < n_in; i++)
        for (uint32_t o = 0; o < n_out; o++) {
            const int64_t w = hw[(size_t)i * n_out + o];
            const uint64_t a = w < 0 ? (uint64_t)(-(w + 1)) + 1 : (uint64_t)w;
            mx = std::max(mx, a);
            l1[o] += a;  // below n_in 2^40: no overflow for n_in < 2^24
        }
    if (mx >= (1ull << 40)) throw std::invalid_argument("ct-pt matmul: |W| must be below 2^40");
    if (n_in >= (1u << 24)) throw std::invalid_argument("ct-pt matmul: too many inputs");
    ctpt_matmul_tc(c, X, W, Y, n_in, n_out, L, ws, *std::max_element(l1.begin(), l1.end()), st);
    if (ctpt_tc_error(ws, st)) throw CudaError("ct-pt matmul: tensor-core pipeline wait timed out");
}

}  // namespace shm
