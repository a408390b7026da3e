// Serving loop: continuous batching of proof and recovery requests.
//
// The reference has no serving layer (its API is one blocking batch call per
// caller, serialised per prover: src/vkzg.cpp:1183-1218).  Here requests of any
// blob count are submitted asynchronously and tracked by ticket.  A dispatcher
// thread cuts the pending queue into batches (one kind per batch, FIFO, at most
// max_blobs_per_batch blobs, larger requests split into parts) and hands each
// batch to a free lane.  A lane is a prover with its own CUDA stream, device
// buffers and worker thread, so batches on different lanes overlap on the GPU,
// and requests that arrive while lanes are busy join the next batch a lane
// takes.  Admission is capped by an HBM working-set budget.  Every blob is
// computed independently, so a request's output does not depend on what it was
// batched with.
#include "../../include/vkzg.h"
#include "../../include/vkzg_b200.h"
#include "kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string.h>
#include <thread>
#include <vector>

namespace {

constexpr size_t kBlob = VKZG_BYTES_PER_BLOB;
constexpr size_t kExt = (size_t)VKZG_NUM_CELL_PROOFS * VKZG_BYTES_PER_CELL;
constexpr size_t kProofs = (size_t)VKZG_NUM_CELL_PROOFS * VKZG_BYTES_PER_PROOF;
// lane I/O buffers per blob of capacity: cells (or blob) in, cells (or proofs) out, presence, error word
constexpr uint64_t kLaneBytesPerBlob = 2 * kExt + VKZG_NUM_CELL_PROOFS + sizeof(uint32_t);

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    int kind = 0; // 0 proofs, 1 recovery
    size_t n = 0;
    const uint8_t *in = nullptr, *present = nullptr;
    uint8_t *out = nullptr;
    vkzg_result status = VKZG_OK;
    size_t parts_left = 0;
    bool done = false;
    Clock::time_point t_submit, t_done;
};

struct Part {
    std::shared_ptr<Request> req;
    size_t first = 0, count = 0;
};

struct Batch {
    int kind = 0;
    size_t blobs = 0;
    uint64_t bytes = 0;
    std::vector<Part> parts;
};

struct Lane {
    vkzg_prover *p = nullptr;
    cudaStream_t stream = nullptr;
    uint8_t *d_in = nullptr, *d_out = nullptr, *d_present = nullptr;
    uint32_t *d_err = nullptr, *h_err = nullptr;
    std::thread worker;
    bool busy = false;
    Batch batch;
    std::condition_variable cv;
};

} // namespace

struct vkzg_server {
    vkzg_server_options opts{};
    std::vector<std::unique_ptr<Lane>> lanes;
    std::mutex mu;
    std::condition_variable cv_dispatch, cv_done;
    std::deque<Part> pending;
    std::map<uint64_t, std::shared_ptr<Request>> requests;
    uint64_t next_id = 1;
    uint64_t bytes_in_flight = 0, peak_in_flight = 0, deferrals = 0;
    // admission charges: device working set per blob of a batch in flight
    // (measured from the lanes' allocations), and the resident tables
    uint64_t proof_bytes_per_blob = 0, recover_bytes_per_blob = kLaneBytesPerBlob, resident_bytes = 0;
    // the head request does not fit the HBM budget beside the batches in
    // flight: the dispatcher sleeps until one of them completes
    bool over_budget = false;
    bool stopping = false;
    std::thread dispatcher;
    // completed-request statistics since the last reset
    std::vector<double> lat_ms;
    uint64_t done_requests = 0, done_blobs = 0;
    Clock::time_point stats_since = Clock::now();

    void dispatch_loop();
    void lane_loop(Lane *lane);
    void run_batch(Lane *lane);
};

void vkzg_server::dispatch_loop() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_dispatch.wait(lk, [&] {
            if (stopping) return true;
            if (pending.empty() || over_budget) return false;
            for (auto &l : lanes)
                if (!l->busy) return true;
            return false;
        });
        if (stopping) return;
        for (auto &l : lanes) {
            if (l->busy || pending.empty()) continue;
            Batch b;
            b.kind = pending.front().req->kind;
            const uint64_t per_blob = b.kind == 0 ? proof_bytes_per_blob : recover_bytes_per_blob;
            for (auto it = pending.begin(); it != pending.end();) {
                if (it->req->kind != b.kind) {
                    ++it;
                    continue;
                }
                if (b.blobs + it->count > opts.max_blobs_per_batch) break;
                const uint64_t bytes = per_blob * it->count;
                // admission: the HBM budget caps the working set of all batches in flight
                if (bytes_in_flight + b.bytes + bytes > opts.hbm_budget_bytes && (bytes_in_flight + b.bytes) > 0) break;
                b.blobs += it->count;
                b.bytes += bytes;
                b.parts.push_back(*it);
                it = pending.erase(it);
            }
            if (b.parts.empty()) { // budget exhausted until something completes
                over_budget = true;
                deferrals++;
                break;
            }
            bytes_in_flight += b.bytes;
            peak_in_flight = std::max(peak_in_flight, bytes_in_flight);
            l->batch = std::move(b);
            l->busy = true;
            l->cv.notify_one();
        }
    }
}

void vkzg_server::run_batch(Lane *lane) {
    Batch &b = lane->batch;
    cudaStream_t s = lane->stream;
    vkzg_result rc = VKZG_OK;
    const size_t in_b = b.kind == 0 ? kBlob : kExt, out_b = b.kind == 0 ? kProofs : kExt;
    size_t off = 0;
    for (auto &part : b.parts) {
        if (cudaMemcpyAsync(lane->d_in + off * in_b, part.req->in + part.first * in_b, part.count * in_b,
                            cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = VKZG_ERR_GPU;
        if (b.kind == 1 &&
            cudaMemcpyAsync(lane->d_present + off * VKZG_NUM_CELL_PROOFS,
                            part.req->present + part.first * VKZG_NUM_CELL_PROOFS, part.count * VKZG_NUM_CELL_PROOFS,
                            cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = VKZG_ERR_GPU;
        off += part.count;
    }
    if (rc == VKZG_OK) {
        rc = b.kind == 0 ? vkzg_b200_compute_proofs_device(lane->p, lane->d_out, lane->d_in, lane->d_err, b.blobs, s)
                         : vkzg_b200_recover_cells_device(lane->p, lane->d_out, lane->d_in, lane->d_present,
                                                          lane->d_err, b.blobs, s);
    }
    if (rc == VKZG_OK &&
        cudaMemcpyAsync(lane->h_err, lane->d_err, b.blobs * sizeof(uint32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = VKZG_ERR_GPU;
    if (rc == VKZG_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = VKZG_ERR_GPU;
    // outputs of a part are copied only when every blob of its request part is valid
    off = 0;
    std::vector<vkzg_result> part_rc(b.parts.size(), rc);
    for (size_t k = 0; k < b.parts.size(); k++) {
        const Part &part = b.parts[k];
        if (part_rc[k] == VKZG_OK) {
            for (size_t i = 0; i < part.count; i++)
                if (lane->h_err[off + i] & VKZG_B200_DEVICE_FAILED) part_rc[k] = VKZG_ERR_GPU;
                else if (lane->h_err[off + i]) part_rc[k] = b.kind == 0 ? VKZG_ERR_INVALID_BLOB : VKZG_ERR_BADARGS;
        }
        if (part_rc[k] == VKZG_OK &&
            cudaMemcpyAsync(part.req->out + part.first * out_b, lane->d_out + off * out_b, part.count * out_b,
                            cudaMemcpyDeviceToHost, s) != cudaSuccess)
            part_rc[k] = VKZG_ERR_GPU;
        off += part.count;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess)
        for (auto &r : part_rc) r = r == VKZG_OK ? VKZG_ERR_GPU : r;
    const auto now = Clock::now();
    std::lock_guard<std::mutex> lk(mu);
    for (size_t k = 0; k < b.parts.size(); k++) {
        Request &r = *b.parts[k].req;
        if (part_rc[k] != VKZG_OK && r.status == VKZG_OK) r.status = part_rc[k];
        if (--r.parts_left == 0) {
            r.done = true;
            r.t_done = now;
            lat_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count());
            done_requests++;
            done_blobs += r.n;
        }
    }
    bytes_in_flight -= b.bytes;
    over_budget = false;
    lane->busy = false;
    b.parts.clear();
    cv_done.notify_all();
    cv_dispatch.notify_one();
}

void vkzg_server::lane_loop(Lane *lane) {
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            lane->cv.wait(lk, [&] { return stopping || (lane->busy && !lane->batch.parts.empty()); });
            if (stopping) return;
        }
        run_batch(lane);
    }
}

extern "C" {

void vkzg_b200_server_options_default(vkzg_server_options *o) {
    if (!o) return;
    o->max_blobs_per_batch = 0;
    o->lanes = 0;
    o->hbm_budget_bytes = 0;
    o->table_budget_bytes = 0;
}

vkzg_result vkzg_b200_server_new(vkzg_server **out, const vkzg_server_options *opts) {
    if (!out) return VKZG_ERR_BADARGS;
    *out = nullptr;
    auto *s = new (std::nothrow) vkzg_server();
    if (!s) return VKZG_ERR_MALLOC;
    vkzg_b200_server_options_default(&s->opts);
    if (opts) s->opts = *opts;
    if (!s->opts.max_blobs_per_batch) s->opts.max_blobs_per_batch = 128;
    if (!s->opts.lanes) s->opts.lanes = 3;
    if (!s->opts.hbm_budget_bytes) s->opts.hbm_budget_bytes = 8ull << 30;
    const uint32_t cap = s->opts.max_blobs_per_batch;
    if (!s->opts.table_budget_bytes) s->opts.table_budget_bytes = 20ull << 30;
    vkzg_result rc = VKZG_OK;
    for (uint32_t k = 0; k < s->opts.lanes && rc == VKZG_OK; k++) {
        auto lane = std::make_unique<Lane>();
        vkzg_options po;
        vkzg_options_default(&po);
        po.max_batch_size = cap;
        rc = vkzg_prover_new(&lane->p, &po);
        if (rc != VKZG_OK) break;
        vkzg::set_comb_budget(lane->p, s->opts.table_budget_bytes);
        vkzg::disable_coop(lane->p);
        if (cudaStreamCreateWithFlags(&lane->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaMalloc(&lane->d_in, cap * kExt) != cudaSuccess || cudaMalloc(&lane->d_out, cap * kExt) != cudaSuccess ||
            cudaMalloc(&lane->d_present, cap * VKZG_NUM_CELL_PROOFS) != cudaSuccess ||
            cudaMalloc(&lane->d_err, cap * sizeof(uint32_t)) != cudaSuccess ||
            cudaMallocHost(&lane->h_err, cap * sizeof(uint32_t)) != cudaSuccess) {
            rc = VKZG_ERR_MALLOC;
        }
        s->lanes.push_back(std::move(lane));
    }
    if (rc != VKZG_OK) {
        vkzg_b200_server_free(s);
        return rc;
    }
    // tune every batch size class once, before any request, and share the
    // decisions (and with plan 3 the digit table) with every lane: no request
    // waits for a tuning run
    if (vkzg_b200_autotune(s->lanes[0]->p, cap) != VKZG_OK) {
        vkzg_b200_server_free(s);
        return VKZG_ERR_GPU;
    }
    for (auto &l : s->lanes) vkzg::adopt_tuning(l->p, s->lanes[0]->p);
    // then each lane keeps only its tuned plans' buffers (its per-blob charge below)
    for (auto &l : s->lanes) vkzg::trim_working_set(l->p);
    // and capture every batch size's proof pipeline on every lane: a capture on
    // first use would hold up the request that meets it
    for (auto &l : s->lanes) vkzg::precapture_graphs(l->p, cap);
    // admission charges from what the lanes hold: a proof blob in flight uses
    // its share of a lane prover's working set and of the lane's I/O buffers
    uint64_t working = 0, tables = 0, digit = 0;
    vkzg_b200_prover_device_bytes(s->lanes[0]->p, &working, &tables, &digit);
    s->proof_bytes_per_blob = working / cap + kLaneBytesPerBlob;
    for (auto &l : s->lanes) {
        vkzg_b200_prover_device_bytes(l->p, &working, &tables, nullptr);
        s->resident_bytes += tables;
    }
    s->resident_bytes += digit; // shared by the lanes
    for (auto &l : s->lanes) {
        Lane *lp = l.get();
        l->worker = std::thread([s, lp] { s->lane_loop(lp); });
    }
    s->dispatcher = std::thread([s] { s->dispatch_loop(); });
    *out = s;
    return VKZG_OK;
}

void vkzg_b200_server_free(vkzg_server *s) {
    if (!s) return;
    {
        // let queued work finish
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] {
            if (!s->pending.empty()) return false;
            for (auto &l : s->lanes)
                if (l->busy) return false;
            return true;
        });
        s->stopping = true;
    }
    s->cv_dispatch.notify_all();
    for (auto &l : s->lanes) l->cv.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    for (auto &l : s->lanes) {
        if (l->worker.joinable()) l->worker.join();
        if (l->stream) cudaStreamSynchronize(l->stream);
        cudaFree(l->d_in);
        cudaFree(l->d_out);
        cudaFree(l->d_present);
        cudaFree(l->d_err);
        if (l->h_err) cudaFreeHost(l->h_err);
        if (l->stream) cudaStreamDestroy(l->stream);
        vkzg_prover_free(l->p);
    }
    delete s;
}

static vkzg_result submit(vkzg_server *s, int kind, uint8_t *out, const uint8_t *in, const uint8_t *present, size_t n,
                          uint64_t *ticket) {
    if (!s || !out || !in || !ticket || (kind == 1 && !present)) return VKZG_ERR_BADARGS;
    auto r = std::make_shared<Request>();
    r->kind = kind;
    r->n = n;
    r->in = in;
    r->present = present;
    r->out = out;
    r->t_submit = Clock::now();
    const size_t cap = s->opts.max_blobs_per_batch;
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    *ticket = r->id;
    s->requests[r->id] = r;
    if (n == 0) {
        r->done = true;
        r->t_done = r->t_submit;
        s->cv_done.notify_all();
        return VKZG_OK;
    }
    for (size_t first = 0; first < n; first += cap) {
        Part p;
        p.req = r;
        p.first = first;
        p.count = std::min(cap, n - first);
        r->parts_left++;
        s->pending.push_back(p);
    }
    s->cv_dispatch.notify_one();
    return VKZG_OK;
}

vkzg_result vkzg_b200_server_submit_proofs(vkzg_server *s, uint8_t *proofs, const uint8_t *blobs, size_t num_blobs,
                                           uint64_t *ticket) {
    return submit(s, 0, proofs, blobs, nullptr, num_blobs, ticket);
}

vkzg_result vkzg_b200_server_submit_recovery(vkzg_server *s, uint8_t *cells_out, const uint8_t *cells,
                                             const uint8_t *cell_present, size_t num_blobs, uint64_t *ticket) {
    return submit(s, 1, cells_out, cells, cell_present, num_blobs, ticket);
}

vkzg_result vkzg_b200_server_wait(vkzg_server *s, uint64_t ticket, int64_t timeout_ms) {
    if (!s) return VKZG_ERR_BADARGS;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return VKZG_ERR_BADARGS;
    std::shared_ptr<Request> r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        return VKZG_B200_PENDING; // still running: the ticket stays valid
    }
    s->requests.erase(ticket);
    return r->status;
}

vkzg_result vkzg_b200_server_stats(vkzg_server *s, vkzg_server_stats *out, int reset) {
    if (!s || !out) return VKZG_ERR_BADARGS;
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
    memset(out, 0, sizeof *out);
    out->requests = s->done_requests;
    out->blobs = s->done_blobs;
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->p999_ms = pct(0.999);
    out->max_ms = v.empty() ? 0.0 : v.back();
    double sum = 0;
    for (double x : v) sum += x;
    out->mean_ms = v.empty() ? 0.0 : sum / v.size();
    out->seconds = std::chrono::duration<double>(Clock::now() - s->stats_since).count();
    out->deferrals = s->deferrals;
    out->peak_in_flight_bytes = s->peak_in_flight;
    out->resident_bytes = s->resident_bytes;
    out->proof_bytes_per_blob = s->proof_bytes_per_blob;
    out->recover_bytes_per_blob = s->recover_bytes_per_blob;
    if (reset) {
        s->lat_ms.clear();
        s->deferrals = 0;
        s->peak_in_flight = s->bytes_in_flight;
        s->done_requests = s->done_blobs = 0;
        s->stats_since = Clock::now();
    }
    return VKZG_OK;
}

} // extern "C"
