// Autotuning of the kernel tile knobs (no reference counterpart: the reference's launch
// shapes are fixed).  Each tuner times every candidate with CUDA events on scratch data
// shaped like the caller's workload, on a private stream, and keeps the fastest in the
// context; the device is synchronised before and after.
#include <algorithm>

#include "core.hpp"

namespace shm {

namespace {

// median of `reps` timed runs of f after two untimed ones
template <typename F>
float time_ms(cudaStream_t st, int reps, F &&f) {
    cudaEvent_t a, b;
    SHM_CUDA(cudaEventCreate(&a));
    SHM_CUDA(cudaEventCreate(&b));
    for (int i = 0; i < 2; i++) f();
    std::vector<float> t;
    for (int i = 0; i < reps; i++) {
        SHM_CUDA(cudaEventRecord(a, st));
        f();
        SHM_CUDA(cudaEventRecord(b, st));
        SHM_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        SHM_CUDA(cudaEventElapsedTime(&ms, a, b));
        t.push_back(ms);
    }
    SHM_CUDA(cudaEventDestroy(a));
    SHM_CUDA(cudaEventDestroy(b));
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

struct Scratch {
    std::vector<uint64_t *> p;
    cudaStream_t st;
    uint64_t *get(size_t words) {
        uint64_t *q = nullptr;
        SHM_CUDA(cudaMallocAsync(&q, words * 8, st));
        p.push_back(q);
        return q;
    }
    ~Scratch() {
        for (uint64_t *q : p) cudaFreeAsync(q, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
};

cudaStream_t new_stream() {
    SHM_CUDA(cudaDeviceSynchronize());
    cudaStream_t st;
    SHM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    return st;
}

uint32_t argmin(const std::vector<float> &ms) {
    return (uint32_t)(std::min_element(ms.begin(), ms.end()) - ms.begin());
}

}  // namespace

// forward + inverse NTT of `rows` limbs (cycling through the chain's primes) per candidate
uint32_t tune_ntt_tile(Context &c, uint32_t rows, std::vector<float> &ms) {
    if (rows == 0) throw std::invalid_argument("autotune: empty workload");
    Scratch s{{}, new_stream()};
    const uint32_t L = std::min(rows, c.nq);
    const uint32_t polys = (rows + L - 1) / L;
    uint64_t *x = s.get((size_t)polys * L * c.n);
    sample_uniform(c, x, polys, L, 0x7E57, s.st);
    ms.clear();
    for (int v = 0; v < kNttVariantCount; v++) {
        c.ntt_variant = v;
        ms.push_back(time_ms(s.st, 5, [&] {
            ntt_forward(c, x, polys * L, L, q_map(L), s.st);
            ntt_inverse(c, x, polys * L, L, q_map(L), nullptr, s.st);
        }));
    }
    c.ntt_variant = (int)argmin(ms);
    return (uint32_t)c.ntt_variant;
}

// the Sh-Rot inner product of `groups` groups of `members` at L primes per candidate
uint32_t tune_ip_chunk(Context &c, uint32_t groups, uint32_t L, uint32_t members, std::vector<float> &ms) {
    if (groups == 0 || members == 0) throw std::invalid_argument("autotune: empty workload");
    if (c.np == 0 || L < 1 || L > c.nq) throw std::invalid_argument("autotune: level out of range");
    const uint32_t np = c.np, beta = (L + np - 1) / np, LP = L + np, QP = c.nq + np, H = members + 1;
    if (beta > 16 || H > 64) throw std::invalid_argument("autotune: shape too large");
    Scratch s{{}, new_stream()};
    uint64_t *up = s.get((size_t)groups * beta * LP * c.n);
    uint64_t *key = s.get((size_t)beta * H * QP * c.n);
    uint64_t *acc = s.get((size_t)groups * H * LP * c.n);
    sample_uniform(c, up, groups * beta, LP, 0x7E58, s.st);
    sample_uniform(c, key, beta * H, QP, 0x7E59, s.st);
    ms.clear();
    for (uint32_t b : kIpChunkCandidates) {
        c.ip_chunk_bytes = b;
        ms.push_back(time_ms(s.st, 5, [&] { ip_multi(c, up, key, acc, groups, L, beta, H, nullptr, s.st); }));
    }
    const uint32_t best = argmin(ms);
    c.ip_chunk_bytes = kIpChunkCandidates[best];
    return best;
}

}  // namespace shm
