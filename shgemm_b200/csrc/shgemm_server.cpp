// Sketch server: continuous batching of sketch requests Y = A [Omega_1 .. Omega_d]
// onto grouped SHGEMM launches, with first-come first-served admission under an HBM
// budget. No counterpart in the reference, whose callers loop over shgemm() one
// problem at a time (src/shgemm.cu:517-686 per call).
//
// One server thread owns every CUDA call: it moves submitted requests into the FIFO,
// admits the head while its A + Omega + Y bytes fit the budget (Omega and Y are
// carved from one device arena allocated at creation; A stays in the caller's
// memory and is only counted), and, whenever one of its streams is free, generates
// the Omega draws of every admitted request and runs them as one grouped launch on
// that stream. A batch therefore starts while earlier batches are still on the GPU.
// Completions are found by polling each stream's event; a request's latency is the
// host time from submit to the poll that saw its batch finish.
#include "shgemm_b200.h"
#include "server_host.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

using shgemm_b200_server_host::OffsetAllocator;
using shgemm_b200_server_host::round_up;

// The server's device memory: one allocation, carved by the first-fit offset allocator.
class Arena {
   public:
    bool init(size_t bytes) {
        bytes = round_up(bytes);
        if (cudaMalloc(&base_, bytes) != cudaSuccess) {
            cudaGetLastError();
            base_ = nullptr;
            return false;
        }
        offs_.reset(bytes);
        return true;
    }
    void destroy() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
    }
    static constexpr size_t kNone = OffsetAllocator::kNone;
    size_t alloc(size_t bytes) { return offs_.alloc(bytes); }
    void release(size_t off, size_t bytes) { offs_.release(off, bytes); }
    uint8_t* ptr(size_t off) const { return base_ + off; }
    size_t size() const { return offs_.size(); }

   private:
    uint8_t* base_ = nullptr;
    OffsetAllocator offs_;
};

struct Request {
    unsigned long long ticket = 0;
    shgemm_b200_sketch_request r{};
    int state = SHGEMM_REQ_QUEUED;
    Clock::time_point t_submit, t_done;
    size_t a_bytes = 0, om_bytes = 0, y_bytes = 0;
    size_t om_off = Arena::kNone, y_off = Arena::kNone;
    size_t ldb = 0;  // Omega leading dimension (elements)
    bool y_held = false;
    // Large requests run as row chunks, one per launch, so that requests arriving behind them
    // share the next launch instead of waiting for all of them. Omega is generated with the
    // first chunk; a later chunk launched on another stream while that batch runs waits for
    // it on the device (cudaStreamWaitEvent), so several chunks may be in flight.
    size_t row_next = 0;   // rows handed to launches
    size_t rows_done = 0;  // rows whose launches completed
    int chunks_in_flight = 0;
    bool omega_made = false;
    int omega_slot = -1;        // slot whose batch generates Omega
    bool omega_ready = false;   // that batch completed
    bool failed = false;
};

// One launch's share of a request: rows [row0, row0 + rows) of its Y.
struct Piece {
    std::shared_ptr<Request> q;
    size_t row0 = 0, rows = 0;
};

struct Slot {
    shgemm_b200_handle_t h = nullptr;
    cudaStream_t stream = nullptr;
    // batch start, Omega generated (grouped launch starts), batch done: timing events
    cudaEvent_t start = nullptr, mid = nullptr, done = nullptr;
    bool busy = false;
    std::vector<Piece> pieces;
};

}  // namespace

struct shgemm_b200_server {
    int device = 0;
    shgemm_b200_server_config cfg{};
    Arena arena;
    std::vector<Slot> slots;

    std::mutex mu;
    std::condition_variable cv_done;  // a request finished
    std::condition_variable cv_work;  // a request was submitted
    std::unordered_map<unsigned long long, std::shared_ptr<Request>> reqs;
    std::deque<std::shared_ptr<Request>> inbox;    // submitted, not yet seen by the server thread
    std::deque<std::shared_ptr<Request>> waiting;  // FIFO awaiting admission
    std::deque<std::shared_ptr<Request>> ready;    // admitted, not yet launched
    unsigned long long next_ticket = 1;
    size_t resident = 0, peak_resident = 0;
    unsigned long long n_submitted = 0, n_completed = 0, n_failed = 0, n_batches = 0, n_unfinished = 0;
    std::vector<double> latencies_ms;
    double flops_done = 0;
    // device timing of completed batches, in ms after `ref` (recorded on an idle stream)
    cudaStream_t ref_stream = nullptr;
    cudaEvent_t ref = nullptr;
    std::vector<std::pair<float, float>> kernel_iv;  // grouped launch intervals
    double omega_ms = 0;
    unsigned long long n_launches = 0;
    bool have_first = false;
    Clock::time_point first_submit, last_done;

    std::atomic<bool> stop{false};
    std::thread worker;

    void run();
    bool admit_locked();
    bool launch_locked(Slot& s);
    bool complete_locked(Slot& s, bool ok);
    void release_y_locked(Request& q) {
        if (q.y_held) {
            arena.release(q.y_off, q.y_bytes);
            resident -= round_up(q.y_bytes);
            q.y_held = false;
        }
    }
};

namespace {

size_t omega_elem(const shgemm_b200_server& s) { return s.cfg.compute_type == SHGEMM_TC_TF32 ? 4 : 2; }

void fill_sizes(const shgemm_b200_server& s, Request& q) {
    const size_t cols = q.r.n * static_cast<size_t>(q.r.draws);
    const size_t e = omega_elem(s);
    q.ldb = (q.r.k + (16 / e) - 1) / (16 / e) * (16 / e);  // 16-byte leading dimension for TMA
    q.a_bytes = q.r.lda * q.r.k * sizeof(float);
    q.om_bytes = std::max<size_t>(1, q.ldb * cols * e);
    q.y_bytes = std::max<size_t>(1, q.r.m * cols * sizeof(float));
}

using shgemm_b200_server_host::kMaxUnitsPerLaunch;

// Rows of the next chunk of q (server_host.hpp).
size_t chunk_rows(const Request& q) {
    return shgemm_b200_server_host::chunk_rows(q.r.m, q.row_next, q.r.n, q.r.draws, q.r.k);
}

// Tiles a launch makes of `rows` rows of q.
int piece_units(const Request& q, size_t rows) {
    return shgemm_b200_server_host::piece_units(rows, q.r.n * static_cast<size_t>(q.r.draws));
}

}  // namespace

bool shgemm_b200_server::admit_locked() {
    bool any = false;
    while (!waiting.empty()) {
        Request& q = *waiting.front();
        const size_t need = q.a_bytes + round_up(q.om_bytes) + round_up(q.y_bytes);
        if (resident + need > cfg.hbm_budget_bytes) break;
        const size_t om = arena.alloc(q.om_bytes);
        if (om == Arena::kNone) break;
        const size_t y = arena.alloc(q.y_bytes);
        if (y == Arena::kNone) {
            arena.release(om, q.om_bytes);
            break;
        }
        q.om_off = om;
        q.y_off = y;
        q.y_held = true;
        resident += need;
        peak_resident = std::max(peak_resident, resident);
        q.state = SHGEMM_REQ_ADMITTED;
        ready.push_back(waiting.front());
        waiting.pop_front();
        any = true;
    }
    return any;
}

bool shgemm_b200_server::launch_locked(Slot& s) {
    const int tc = cfg.compute_type;
    const int fp32 = tc == SHGEMM_TC_TF32 ? 1 : 0;
    std::vector<shgemm_b200_problem> probs;
    std::vector<shgemm_b200_omega_job> jobs;
    s.pieces.clear();
    int units = 0;
    const int me = static_cast<int>(&s - slots.data());
    std::vector<char> wait_on(slots.size(), 0);  // other slots whose Omega batch this one needs
    // first come first served, one chunk per request and launch
    for (auto it = ready.begin(); it != ready.end() && static_cast<int>(s.pieces.size()) < cfg.max_batch;) {
        Request& q = **it;
        const size_t rows = chunk_rows(q);
        const int pu = piece_units(q, rows);
        if (!s.pieces.empty() && units + pu > kMaxUnitsPerLaunch) break;
        units += pu;
        s.pieces.push_back({*it, q.row_next, rows});
        ++q.chunks_in_flight;
        q.state = SHGEMM_REQ_RUNNING;
        const size_t cols = q.r.n * static_cast<size_t>(q.r.draws);
        if (q.omega_made && !q.omega_ready && q.omega_slot != me) wait_on[q.omega_slot] = 1;
        if (!q.omega_made) {
            q.omega_slot = me;
            // draw j of Omega from (seed, j): column block j of the k x (draws n) operand
            for (int j = 0; j < q.r.draws; ++j) {
                uint8_t* dst = arena.ptr(q.om_off) + static_cast<size_t>(j) * q.r.n * q.ldb * omega_elem(*this);
                jobs.push_back({dst, q.ldb, q.r.k, q.r.n,
                                q.r.omega_seed * 0x100000001B3ull + static_cast<unsigned long long>(j),
                                q.r.omega_scale, q.r.omega_dist});
            }
            q.omega_made = true;
        }
        shgemm_b200_problem p{};
        p.m = rows;
        p.n = cols;
        p.k = q.r.k;
        p.a = q.r.a + q.row_next;  // rows row_next .. of the column-major A (128-row aligned)
        p.lda = q.r.lda;
        p.b = arena.ptr(q.om_off);
        p.ldb = q.ldb;
        p.c = reinterpret_cast<float*>(arena.ptr(q.y_off)) + q.row_next;
        p.ldc = std::max<size_t>(1, q.r.m);
        p.alpha = 1.0f;
        p.beta = 0.0f;
        probs.push_back(p);
        q.row_next += rows;
        if (q.row_next >= q.r.m)
            it = ready.erase(it);  // every row handed out
        else
            ++it;
    }
    if (s.pieces.empty()) return false;
    bool ok = true;
    for (size_t o = 0; o < slots.size() && ok; ++o)
        if (wait_on[o]) ok = cudaStreamWaitEvent(s.stream, slots[o].done, 0) == cudaSuccess;
    ok = ok && cudaEventRecord(s.start, s.stream) == cudaSuccess;
    // every draw of the batch in one launch (per 64 draws)
    ok = ok && shgemm_b200_generate_omega_batch(s.stream, jobs.data(), static_cast<int>(jobs.size()), fp32) ==
                   SHGEMM_STATUS_OK;
    n_launches += (jobs.size() + 63) / 64;
    ok = ok && cudaEventRecord(s.mid, s.stream) == cudaSuccess;
    ok = ok && shgemm_b200_shgemm_grouped(s.h, SHGEMM_OP_N, SHGEMM_OP_N, tc, SHGEMM_OP_N, probs.data(),
                                          static_cast<int>(probs.size())) == SHGEMM_STATUS_OK;
    if (ok) ++n_launches;
    ok = ok && cudaEventRecord(s.done, s.stream) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        // whatever was enqueued before the failure finishes before its memory is reused
        cudaStreamSynchronize(s.stream);
        cudaGetLastError();
        complete_locked(s, false);
        return true;
    }
    s.busy = true;
    ++n_batches;
    return true;
}

bool shgemm_b200_server::complete_locked(Slot& s, bool ok) {
    const auto now = Clock::now();
    if (ok && s.busy) {
        float t0 = 0, t1 = 0, t2 = 0;
        if (cudaEventElapsedTime(&t0, ref, s.start) == cudaSuccess &&
            cudaEventElapsedTime(&t1, ref, s.mid) == cudaSuccess && cudaEventElapsedTime(&t2, ref, s.done) == cudaSuccess) {
            omega_ms += t1 - t0;
            kernel_iv.emplace_back(t1, t2);
        } else {
            cudaGetLastError();
        }
    }
    const int me = static_cast<int>(&s - slots.data());
    for (auto& pc : s.pieces) {
        Request& q = *pc.q;
        --q.chunks_in_flight;
        if (q.omega_slot == me) q.omega_ready = true;
        if (ok) q.rows_done += pc.rows;
        if (!ok && !q.failed) {  // drop its remaining chunks
            q.failed = true;
            auto it = std::find(ready.begin(), ready.end(), pc.q);
            if (it != ready.end()) ready.erase(it);
        }
        // finished: every row done, or failed with no chunk left reading its Omega
        if (q.failed ? q.chunks_in_flight > 0 : q.rows_done < q.r.m) continue;
        if (q.state != SHGEMM_REQ_RUNNING) continue;
        const bool good = !q.failed;
        arena.release(q.om_off, q.om_bytes);
        resident -= q.a_bytes + round_up(q.om_bytes);
        q.t_done = now;
        if (good) {
            q.state = SHGEMM_REQ_DONE;
            ++n_completed;
            latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - q.t_submit).count());
            flops_done += 2.0 * q.r.m * q.r.n * q.r.draws * q.r.k;
            last_done = now;
        } else {
            q.state = SHGEMM_REQ_FAILED;
            ++n_failed;
        }
        if (cfg.auto_release || !good) release_y_locked(q);  // else Y stays resident until released
        --n_unfinished;
    }
    s.pieces.clear();
    s.busy = false;
    cv_done.notify_all();
    return true;
}

void shgemm_b200_server::run() {
    cudaSetDevice(device);
    while (!stop.load()) {
        bool work = false;
        std::unique_lock<std::mutex> lk(mu);
        for (auto& s : slots) {
            if (!s.busy) continue;
            const cudaError_t e = cudaEventQuery(s.done);
            if (e == cudaErrorNotReady) continue;
            int code = 0;
            bool ok = e == cudaSuccess;
            if (ok && shgemm_b200_check_error(s.h, &code) != SHGEMM_STATUS_OK) ok = false;
            if (!ok) cudaGetLastError();
            complete_locked(s, ok);
            work = true;
        }
        while (!inbox.empty()) {
            waiting.push_back(inbox.front());
            inbox.pop_front();
            work = true;
        }
        work |= admit_locked();
        for (auto& s : slots)
            if (!s.busy && !ready.empty()) work |= launch_locked(s);
        const bool idle = inbox.empty() && waiting.empty() && ready.empty() &&
                          std::none_of(slots.begin(), slots.end(), [](const Slot& s) { return s.busy; });
        if (idle) {
            cv_work.wait_for(lk, std::chrono::milliseconds(5));
        } else if (!work) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
}

extern "C" {

int shgemm_b200_server_create(shgemm_b200_server_t* out, int device, const shgemm_b200_server_config* config) {
    if (!out || !config) return SHGEMM_STATUS_INVALID_VALUE;
    *out = nullptr;
    shgemm_b200_server_config c = *config;
    if (c.max_batch == 0) c.max_batch = 512;
    if (c.streams == 0) c.streams = 3;
    if ((c.compute_type != SHGEMM_TC_FP16 && c.compute_type != SHGEMM_TC_TF32) || c.max_batch < 1 ||
        c.max_batch > 8192 || c.streams < 1 || c.streams > 8 || c.hbm_budget_bytes == 0)
        return SHGEMM_STATUS_INVALID_VALUE;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return SHGEMM_STATUS_INVALID_VALUE;
    }
    auto* s = new shgemm_b200_server();
    s->device = device;
    s->cfg = c;
    if (!s->arena.init(c.hbm_budget_bytes)) {
        delete s;
        return SHGEMM_STATUS_ALLOC_FAILED;
    }
    s->slots.resize(c.streams);
    for (auto& sl : s->slots) {
        int st = shgemm_b200_create(&sl.h, device);
        if (st == SHGEMM_STATUS_OK && (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
                                       cudaEventCreate(&sl.start) != cudaSuccess ||
                                       cudaEventCreate(&sl.mid) != cudaSuccess ||
                                       cudaEventCreate(&sl.done) != cudaSuccess))
            st = SHGEMM_STATUS_CUDA_ERROR;
        if (st == SHGEMM_STATUS_OK) st = shgemm_b200_set_stream(sl.h, sl.stream);
        if (st == SHGEMM_STATUS_OK && c.compute_type == SHGEMM_TC_TF32)
            st = shgemm_b200_set_config(sl.h, SHGEMM_CFG_GROUPED_B_FP32, 1);
        if (st != SHGEMM_STATUS_OK) {
            cudaGetLastError();
            for (auto& t : s->slots) {
                if (t.h) shgemm_b200_destroy(t.h);
                if (t.start) cudaEventDestroy(t.start);
                if (t.mid) cudaEventDestroy(t.mid);
                if (t.done) cudaEventDestroy(t.done);
                if (t.stream) cudaStreamDestroy(t.stream);
            }
            s->arena.destroy();
            delete s;
            return st;
        }
    }
    if (cudaStreamCreateWithFlags(&s->ref_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s->ref) != cudaSuccess || cudaEventRecord(s->ref, s->ref_stream) != cudaSuccess ||
        cudaEventSynchronize(s->ref) != cudaSuccess) {
        cudaGetLastError();
        for (auto& t : s->slots) {
            shgemm_b200_destroy(t.h);
            cudaEventDestroy(t.start);
            cudaEventDestroy(t.mid);
            cudaEventDestroy(t.done);
            cudaStreamDestroy(t.stream);
        }
        if (s->ref) cudaEventDestroy(s->ref);
        if (s->ref_stream) cudaStreamDestroy(s->ref_stream);
        s->arena.destroy();
        delete s;
        return SHGEMM_STATUS_CUDA_ERROR;
    }
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_server_destroy(shgemm_b200_server_t s) {
    if (!s) return SHGEMM_STATUS_INVALID_VALUE;
    s->stop.store(true);
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    for (auto& t : s->slots) {
        if (t.stream) cudaStreamSynchronize(t.stream);
        if (t.h) shgemm_b200_destroy(t.h);
        if (t.start) cudaEventDestroy(t.start);
        if (t.mid) cudaEventDestroy(t.mid);
        if (t.done) cudaEventDestroy(t.done);
        if (t.stream) cudaStreamDestroy(t.stream);
    }
    if (s->ref) cudaEventDestroy(s->ref);
    if (s->ref_stream) cudaStreamDestroy(s->ref_stream);
    s->arena.destroy();
    delete s;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_server_submit(shgemm_b200_server_t s, const shgemm_b200_sketch_request* r, unsigned long long* ticket) {
    if (!s || !r || !ticket) return SHGEMM_STATUS_INVALID_VALUE;
    if (r->draws < 1 || r->m == 0 || r->n == 0 || r->k == 0 || !r->a || r->lda < r->m ||
        (r->omega_dist != SHGEMM_OMEGA_GAUSSIAN && r->omega_dist != SHGEMM_OMEGA_RADEMACHER))
        return SHGEMM_STATUS_INVALID_VALUE;
    // grouped launches address A with TMA: 16-byte aligned base and leading dimension
    if ((reinterpret_cast<uintptr_t>(r->a) & 15) || (r->lda % 4) || r->m >= (size_t(1) << 31) ||
        r->k >= (size_t(1) << 31) || r->n * static_cast<size_t>(r->draws) >= (size_t(1) << 22))
        return SHGEMM_STATUS_NOT_SUPPORTED;
    auto q = std::make_shared<Request>();
    q->r = *r;
    fill_sizes(*s, *q);
    if (piece_units(*q, chunk_rows(*q)) > kMaxUnitsPerLaunch) return SHGEMM_STATUS_NOT_SUPPORTED;
    const size_t need = q->a_bytes + round_up(q->om_bytes) + round_up(q->y_bytes);
    if (need > s->cfg.hbm_budget_bytes || round_up(q->om_bytes) + round_up(q->y_bytes) > s->arena.size())
        return SHGEMM_STATUS_NOT_SUPPORTED;
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        q->ticket = s->next_ticket++;
        if (!s->have_first) {
            s->have_first = true;
            s->first_submit = q->t_submit;
        }
        s->reqs[q->ticket] = q;
        s->inbox.push_back(q);
        ++s->n_submitted;
        ++s->n_unfinished;
    }
    s->cv_work.notify_one();
    *ticket = q->ticket;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_server_poll(shgemm_b200_server_t s, unsigned long long ticket, int* state, float** y, size_t* ldy,
                            double* latency_ms) {
    if (!s) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) {
        if (state) *state = SHGEMM_REQ_UNKNOWN;
        return SHGEMM_STATUS_INVALID_VALUE;
    }
    const Request& q = *it->second;
    if (state) *state = q.state;
    if (y) *y = (q.state == SHGEMM_REQ_DONE && q.y_held) ? reinterpret_cast<float*>(s->arena.ptr(q.y_off)) : nullptr;
    if (ldy) *ldy = q.r.m;
    if (latency_ms)
        *latency_ms = q.state == SHGEMM_REQ_DONE
                          ? std::chrono::duration<double, std::milli>(q.t_done - q.t_submit).count()
                          : -1.0;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_server_wait(shgemm_b200_server_t s, unsigned long long ticket, double timeout_ms, int* state) {
    if (!s) return SHGEMM_STATUS_INVALID_VALUE;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return SHGEMM_STATUS_INVALID_VALUE;
    auto q = it->second;
    const bool fin = s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), [&] {
        return q->state == SHGEMM_REQ_DONE || q->state == SHGEMM_REQ_FAILED;
    });
    if (state) *state = q->state;
    return fin ? SHGEMM_STATUS_OK : SHGEMM_STATUS_TIMEOUT;
}

int shgemm_b200_server_drain(shgemm_b200_server_t s, double timeout_ms) {
    if (!s) return SHGEMM_STATUS_INVALID_VALUE;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool fin = s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                         [&] { return s->n_unfinished == 0; });
    return fin ? SHGEMM_STATUS_OK : SHGEMM_STATUS_TIMEOUT;
}

int shgemm_b200_server_release(shgemm_b200_server_t s, unsigned long long ticket) {
    if (!s) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return SHGEMM_STATUS_INVALID_VALUE;
    Request& q = *it->second;
    if (q.state != SHGEMM_REQ_DONE && q.state != SHGEMM_REQ_FAILED) return SHGEMM_STATUS_INVALID_VALUE;
    s->release_y_locked(q);
    s->reqs.erase(it);
    s->cv_work.notify_one();
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_server_get_stats(shgemm_b200_server_t s, shgemm_b200_server_stats* out) {
    if (!s || !out) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->n_submitted;
    out->completed = s->n_completed;
    out->failed = s->n_failed;
    out->batches = s->n_batches;
    out->flops_completed = s->flops_done;
    out->peak_resident_bytes = s->peak_resident;
    out->resident_bytes = s->resident;
    out->queued = s->inbox.size() + s->waiting.size();
    out->in_flight = s->n_unfinished - out->queued;
    if (!s->latencies_ms.empty()) {
        std::vector<double> v = s->latencies_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const size_t i = static_cast<size_t>(p * static_cast<double>(v.size() - 1) + 0.5);
            return v[std::min(i, v.size() - 1)];
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        double sum = 0;
        for (double x : v) sum += x;
        out->mean_ms = sum / static_cast<double>(v.size());
        out->max_ms = v.back();
        out->span_s = std::chrono::duration<double>(s->last_done - s->first_submit).count();
    }
    // union of the grouped launches' intervals
    std::vector<std::pair<float, float>> iv = s->kernel_iv;
    std::sort(iv.begin(), iv.end());
    double busy_ms = 0;
    float cur0 = 0, cur1 = 0;
    bool open = false;
    for (const auto& x : iv) {
        if (open && x.first <= cur1) {
            cur1 = std::max(cur1, x.second);
            continue;
        }
        if (open) busy_ms += cur1 - cur0;
        cur0 = x.first;
        cur1 = x.second;
        open = true;
    }
    if (open) busy_ms += cur1 - cur0;
    out->kernel_busy_s = busy_ms * 1e-3;
    out->omega_s = s->omega_ms * 1e-3;
    out->launches = s->n_launches;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_server_reset_stats(shgemm_b200_server_t s) {
    if (!s) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies_ms.clear();
    s->n_submitted = 0;
    s->n_completed = s->n_failed = s->n_batches = 0;
    s->flops_done = 0;
    s->kernel_iv.clear();
    s->omega_ms = 0;
    s->n_launches = 0;
    s->have_first = false;
    s->peak_resident = s->resident;
    return SHGEMM_STATUS_OK;
}

}  // extern "C"
