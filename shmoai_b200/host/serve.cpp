// The serving loop of the C++ host library (Server, include/shmoai/host.hpp): HBM-budget
// admission, one worker thread + stream + evaluator per slot, continuous batching of
// queued jobs of the same kind and shape.  The reference has no serving loop (its driver
// runs operators one after the other, src/include/test/bootstrapping/test_shared_a.cuh);
// this is the request loop the north-star workload asks for.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>

#include "internal.hpp"

namespace shmoai {

struct Server::Job {
    uint64_t id = 0;
    JobKind kind = JobKind::Rotate;
    Ciphertext input;
    int step = 0;
    std::vector<int64_t> W;
    uint32_t n_out = 0;
    double w_scale = 1.0;
    uint32_t members = 0;
    size_t bytes = 0;
    ServeResult result;
    bool done = false;
};

struct Server::Slot {
    void *stream = nullptr;
    std::unique_ptr<Context> view;
    std::unique_ptr<Encoder> enc;
    std::unique_ptr<Evaluator> ev;
};

struct Server::State {
    mutable std::mutex mu;
    std::condition_variable work, done;
    std::deque<Job *> queue;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    uint64_t next_id = 1;
    size_t admitted = 0;
    uint32_t inflight = 0;
    bool stop = false, paused = false;
    ServeStats stats;
    std::vector<Slot> slots;
    std::vector<std::thread> threads;
};

double Server::now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

Server::Server(const Evaluator &base, const BatchBootstrapper *boot, const std::map<uint32_t, SharedAKeys> *shared,
               size_t hbm_budget, uint32_t slots, uint32_t max_merge)
    : base_(base), boot_(boot), shared_(shared), budget_(hbm_budget), max_merge_(max_merge ? max_merge : 1),
      st_(new State) {
    if (!slots) throw Error("a server needs at least one slot");
    const Context &c = base.context();
    c.synchronize();  // keys and plaintexts made on the base stream are complete
    st_->stats.budget = budget_;
    st_->slots.resize(slots);
    for (auto &s : st_->slots) {
        c.check(shm_stream_create(c.handle(), &s.stream));
        s.view.reset(new Context(c, s.stream));
        s.enc.reset(new Encoder(*s.view));
        s.ev.reset(new Evaluator(*s.view, *s.enc));
        s.ev->relin_key = base.relin_key;
        s.ev->galois_keys = base.galois_keys;
    }
    for (uint32_t i = 0; i < slots; i++) st_->threads.emplace_back([this, i] { worker(i); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> g(st_->mu);
        st_->stop = true;
        st_->paused = false;
    }
    st_->work.notify_all();
    for (auto &t : st_->threads) t.join();
    const Context &c = base_.context();
    for (auto &s : st_->slots) {
        s.ev.reset();
        s.enc.reset();
        s.view.reset();
        shm_stream_destroy(c.handle(), s.stream);
    }
}

// device bytes a job keeps live while it runs (input, output, intermediates, workspace)
size_t Server::estimate(const Job &j) const {
    const Context &c = base_.context();
    const size_t word = (size_t)c.n * 8, L = j.input.L, cnt = j.input.count;
    const size_t ct = 2 * L * word;
    switch (j.kind) {
        case JobKind::Rotate:
            return cnt * 3 * ct + shm_keyswitch_workspace_bytes(c.handle(), (uint32_t)cnt, (uint32_t)L);
        case JobKind::Matmul:
            return (cnt + 2 * (size_t)j.n_out) * ct + j.W.size() * 8 +
                   shm_ctpt_matmul_workspace_bytes(c.handle(), (uint32_t)cnt, j.n_out, (uint32_t)L);
        case JobKind::Bootstrap: {
            // CoeffToSlot at nq primes: ~8 polynomials per input polynomial (baby steps, sums)
            // plus the hoisted ModUp digits (dnum x (nq + np) limbs) per ciphertext or group.
            // EvalMod on 2 x cnt ciphertexts (real and imaginary parts) near nq - 4 primes:
            // ~24 ciphertexts each (Chebyshev basis, products, partial sums, dropped copies)
            // plus two sets of relinearisation digits -- calibrated on the pool's high-water
            // mark (~60 GB for 32 ciphertexts at the reference parameters).  The two phases
            // do not overlap; the larger one sets the peak.
            const size_t top_poly = (size_t)c.nq * word, digits = (size_t)c.dnum * (c.nq + c.np) * word;
            const size_t units = j.members ? cnt / j.members : cnt;
            const size_t polys_per_unit = j.members ? j.members + 1 : 2;
            const size_t c2s = units * (polys_per_unit * 8 * top_poly + digits);
            const size_t evalmod = 2 * cnt * (24 * 2 * (size_t)(c.nq - 4) * word + 2 * digits);
            return std::max(c2s, evalmod) + 2 * cnt * 2 * top_poly;
        }
    }
    return 0;
}

uint64_t Server::enqueue(std::unique_ptr<Job> j) {
    j->bytes = estimate(*j);
    if (j->bytes > budget_)
        throw Error("job needs ~" + std::to_string(j->bytes >> 20) + " MiB, above the HBM budget of " +
                    std::to_string(budget_ >> 20) + " MiB");
    j->result.t_submit = now();
    // The input was produced on the base context's stream; the slots' streams do not wait for
    // it (they are non-blocking), so the input must be complete before a slot can pick it up.
    base_.context().synchronize();
    std::lock_guard<std::mutex> g(st_->mu);
    if (st_->stop) throw Error("server is stopping");
    j->id = st_->next_id++;
    Job *p = j.get();
    const uint64_t id = j->id;
    st_->jobs.emplace(id, std::move(j));
    st_->queue.push_back(p);
    st_->work.notify_one();
    return id;
}

uint64_t Server::submit_rotate(Ciphertext &&ct, int step) {
    if (ct.shared || ct.size != 2) throw Error("rotation jobs take ordinary ciphertexts");
    std::unique_ptr<Job> j(new Job);
    j->kind = JobKind::Rotate;
    j->input = std::move(ct);
    j->step = step;
    return enqueue(std::move(j));
}

uint64_t Server::submit_matmul(Ciphertext &&X, std::vector<int64_t> W, uint32_t n_out, double w_scale) {
    std::unique_ptr<Job> j(new Job);
    j->kind = JobKind::Matmul;
    j->input = std::move(X);
    j->W = std::move(W);
    j->n_out = n_out;
    j->w_scale = w_scale;
    return enqueue(std::move(j));
}

uint64_t Server::submit_bootstrap(Ciphertext &&ct, uint32_t members) {
    if (!boot_) throw Error("server has no bootstrapper");
    if (members && (!shared_ || !shared_->count(members))) throw Error("no shared-a keys for this group size");
    if (members && ct.count % members) throw Error("batch is not a multiple of the group size");
    std::unique_ptr<Job> j(new Job);
    j->kind = JobKind::Bootstrap;
    j->input = std::move(ct);
    j->members = members;
    return enqueue(std::move(j));
}

namespace {

constexpr double kReserveAfter = 0.5;  // seconds the head may be passed by smaller jobs

bool mergeable(const Ciphertext &a, const Ciphertext &b) {
    return a.L == b.L && a.size == b.size && a.shared == b.shared && Evaluator::same_scale(a.scale_, b.scale_);
}

}  // namespace

void Server::worker(uint32_t slot) {
    State &S = *st_;
    for (;;) {
        std::vector<Job *> batch;
        {
            std::unique_lock<std::mutex> lk(S.mu);
            // Admission: the head of the queue when it fits the budget; while it does not, a later
            // job that fits may start in its place (backfill), until the head has waited
            // kReserveAfter seconds: from then on nothing else starts, so the budget the running
            // jobs release is kept for the head (a large bootstrap is not starved by small jobs)
            auto pick = [&]() -> std::deque<Job *>::iterator {
                if (S.paused || S.queue.empty()) return S.queue.end();
                Job *h0 = S.queue.front();
                if (S.admitted + h0->bytes <= budget_) return S.queue.begin();
                if (now() - h0->result.t_submit >= kReserveAfter) return S.queue.end();
                for (auto it = S.queue.begin() + 1; it != S.queue.end(); ++it)
                    if (S.admitted + (*it)->bytes <= budget_) return it;
                return S.queue.end();
            };
            auto it = S.queue.end();
            for (;;) {
                if (S.stop && S.queue.empty()) return;  // stopping and drained
                it = pick();
                if (it != S.queue.end()) break;
                // aging changes the answer without a notification: look again after a while
                S.work.wait_for(lk, std::chrono::milliseconds(20));
            }
            // queued jobs of the same kind and shape join the picked one
            Job *head = *it;
            S.queue.erase(it);
            batch.push_back(head);
            S.admitted += head->bytes;
            if (head->kind != JobKind::Matmul)
                for (auto it = S.queue.begin(); it != S.queue.end() && batch.size() < max_merge_;) {
                    Job *j = *it;
                    const bool same = j->kind == head->kind && mergeable(j->input, head->input) &&
                                      (head->kind == JobKind::Rotate ? j->step == head->step
                                                                     : j->members == head->members);
                    if (same && S.admitted + j->bytes <= budget_) {
                        S.admitted += j->bytes;
                        batch.push_back(j);
                        it = S.queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            S.inflight++;
            S.stats.max_inflight = std::max(S.stats.max_inflight, S.inflight);
            S.stats.peak_admitted = std::max(S.stats.peak_admitted, S.admitted);
            S.stats.batches++;
        }
        run(S.slots[slot], batch);
        {
            std::lock_guard<std::mutex> g(S.mu);
            for (Job *j : batch) {
                S.admitted -= j->bytes;
                j->done = true;
                S.stats.jobs++;
            }
            S.inflight--;
        }
        S.done.notify_all();
        S.work.notify_all();
    }
}

void Server::run(Slot &s, std::vector<Job *> &batch) {
    const double t0 = now();
    for (Job *j : batch) {
        j->result.t_start = t0;
        j->result.batched_with = (uint32_t)batch.size();
    }
    const Evaluator &ev = *s.ev;
    try {
        Job &h = *batch[0];
        Ciphertext in;
        if (batch.size() == 1) {
            in = std::move(h.input);
        } else {
            in = ev.concat(batch[0]->input, batch[1]->input);
            for (size_t i = 2; i < batch.size(); i++) in = ev.concat(in, batch[i]->input);
        }
        Ciphertext out;
        switch (h.kind) {
            case JobKind::Rotate:
                out = ev.rotate_vector(in, h.step);
                break;
            case JobKind::Matmul:
                out = ev.ctpt_matmul(in, h.W, h.n_out, h.w_scale);
                break;
            case JobKind::Bootstrap:
                if (h.members) {
                    s.ev->shared_keys = &shared_->at(h.members);
                    out = boot_->bootstrap_shared_a_s2c_first(in, h.members, &ev);
                } else {
                    out = boot_->bootstrap_ordinary_s2c_first(in, &ev);
                }
                break;
        }
        // hand each job its rows; outputs outlive the slot's stream work, so they are
        // freed through the base context once this slot has synchronised
        uint32_t first = 0;
        std::vector<Ciphertext> parts;
        for (Job *j : batch) {
            const uint32_t rows = j->kind == JobKind::Matmul ? j->n_out : j->input.count ? j->input.count : in.count;
            parts.push_back(batch.size() == 1 ? std::move(out) : ev.slice(out, first, rows));
            first += rows;
        }
        s.view->synchronize();
        for (size_t i = 0; i < batch.size(); i++) {
            parts[i].data.rebind(base_.context());
            batch[i]->result.output = std::move(parts[i]);
            batch[i]->input = Ciphertext();  // inputs were read by the synchronised stream
        }
    } catch (const std::exception &e) {
        s.view->synchronize();
        for (Job *j : batch) {
            j->result.error = e.what();
            j->input = Ciphertext();
        }
    }
    const double t1 = now();
    for (Job *j : batch) j->result.t_end = t1;
}

ServeResult Server::wait(uint64_t id) {
    std::unique_lock<std::mutex> lk(st_->mu);
    auto it = st_->jobs.find(id);
    if (it == st_->jobs.end()) throw Error("unknown job id");
    Job *j = it->second.get();
    st_->done.wait(lk, [&] { return j->done; });
    ServeResult r = std::move(j->result);
    st_->jobs.erase(it);
    return r;
}

void Server::set_paused(bool paused) {
    {
        std::lock_guard<std::mutex> g(st_->mu);
        st_->paused = paused;
    }
    st_->work.notify_all();
}

ServeStats Server::stats() const {
    std::lock_guard<std::mutex> g(st_->mu);
    return st_->stats;
}

}  // namespace shmoai
