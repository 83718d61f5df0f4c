// CUDA graphs of host-level operation sequences (include/shmoai/host.hpp, class Graph).
#include "internal.hpp"

namespace shmoai {

Graph::Graph(const Evaluator &base, const std::function<void(const Evaluator &ev)> &fn) : base_(base.context()) {
    const Context &c = base_;
    c.synchronize();  // inputs written on the base stream are complete before the private stream reads them
    c.check(shm_stream_create(c.handle(), &stream_));
    view_.reset(new Context(c, stream_));
    enc_.reset(new Encoder(*view_));
    ev_.reset(new Evaluator(*view_, *enc_));
    ev_->relin_key = base.relin_key;
    ev_->galois_keys = base.galois_keys;
    ev_->shared_keys = base.shared_keys;
    fn(*ev_);  // uncaptured: workspaces and lazily built tables reach their final size
    view_->check(shm_graph_begin(c.handle(), stream_));
    try {
        fn(*ev_);
    } catch (...) {
        shm_graph *partial = nullptr;
        shm_graph_end(c.handle(), stream_, &partial);  // leave capture mode before reporting
        shm_graph_destroy(partial);
        throw;
    }
    view_->check(shm_graph_end(c.handle(), stream_, &g_));
}

Graph::~Graph() {
    shm_graph_destroy(g_);
    ev_.reset();
    enc_.reset();
    view_.reset();  // synchronises the private stream
    if (stream_) shm_stream_destroy(base_.handle(), stream_);
}

void Graph::launch() const { base_.check(shm_graph_launch(g_, base_.stream())); }

uint64_t Graph::kernels() const { return shm_graph_kernels(g_); }

std::unique_ptr<Graph> BatchBootstrapper::capture(const Ciphertext &in, uint32_t members, Ciphertext &out) const {
    auto run = [this, &in, members](const Evaluator &ev) {
        return members ? bootstrap_shared_a_s2c_first(in, members, &ev) : bootstrap_ordinary_s2c_first(in, &ev);
    };
    // the output's shape from one run on the base evaluator; the buffer belongs to the base context
    Ciphertext shape = run(ev_);
    const Context &c = ev_.context();
    out.data = DeviceBuffer(c, shape.data.words());
    out.count = shape.count;
    out.size = shape.size;
    out.L = shape.L;
    out.scale_ = shape.scale_;
    out.shared = shape.shared;
    c.synchronize();
    uint64_t *dst = out.data.data();
    const size_t bytes = shape.data.words() * 8;
    return std::unique_ptr<Graph>(new Graph(ev_, [run, dst, bytes](const Evaluator &ev) {
        Ciphertext r = run(ev);
        const Context &v = ev.context();
        v.check(shm_memcpy(v.handle(), dst, r.data.data(), bytes, SHM_COPY_D2D, v.stream()));
    }));
}

}  // namespace shmoai
