// Multi-slot execution engine on one GPU: continuous batching of partition
// requests and packed multi-graph batches.
//
// The reference partitions one graph per process run on the default stream
// (app/partition_main.cu:20-142) and has no batching or serving layer.  Here a
// server owns `slots` contexts, each with its own CUDA stream, caching device
// allocator and host worker thread.  Requests wait in one FIFO queue and are
// admitted, in arrival order, as soon as a slot is idle and the projected
// device footprint of the running requests plus the new one stays within the
// memory budget; requests that arrive while others run are admitted the
// moment a slot and memory free up, and their kernels overlap with the running
// ones on the device.  Every request runs the same pipeline as gp_partition
// on its own context, so its result does not depend on what else is running
// (bit-identical in deterministic mode).
#include "gpart_b200.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    gp_graph graph{};
    bool packed = false;
    int64_t vertex_begin = 0, vertex_end = 0;
    gp_options options{};
    int32_t* labels = nullptr;
    uint64_t footprint = 0;
    Clock::time_point submitted, started, finished;
    gp_status status = GP_OK;
    std::string message;
    gp_report report{};
    int slot = -1;
    bool done = false;
};

}  // namespace

struct gp_server {
    int device = 0;
    uint64_t budget = 0;
    uint64_t in_use = 0;         // projected bytes of the running requests
    std::vector<gp_ctx*> slots;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> requests;
    uint64_t next_ticket = 1;
    uint64_t completed = 0;
    bool stopping = false;
    std::string error;
};

namespace {

// Device bytes a partition of an (n, m) graph is projected to hold at its
// peak: the level-0 copy of the input (and its int64 staging buffer), the
// coarser levels (each at most 0.9x the previous one), the contraction
// scatter buffers, the SCLP and hub-table scratch, and the n x k refinement
// cache.  Calibrated as an upper bound of the caching allocator's measured
// peak on grid, RGG and RMAT inputs.
uint64_t footprint(int64_t n, int64_t m, int parts, int width, int index64_host) {
    const double o = width == GP_WIDTH_BIG ? 8.0 : 4.0;
    const double w = width == GP_WIDTH_BIG ? 8.0 : 4.0;
    const double c = width == GP_WIDTH_BIG ? 8.0 : 4.0;
    const double nn = static_cast<double>(n), mm = static_cast<double>(m);
    double bytes = 0.0;
    bytes += (nn + 1) * o + mm * 4.0;                          // level 0
    if (index64_host) bytes += std::max(nn + 1, mm) * 8.0;     // staging
    bytes += 2.0 * ((nn + 1) * o + mm * (4.0 + w) + nn * (w + 4.0));  // coarser levels + maps
    bytes += 2.0 * mm * (4.0 + w);                              // contraction scatter + segment scratch
    bytes += mm * 16.0;                                         // hub tables and chunk lists
    bytes += nn * (160.0 + parts * c);                          // SCLP / refinement state, n x k cache
    bytes += 64.0 * 1024 * 1024;                                // fixed scratch
    return static_cast<uint64_t>(bytes);
}

void worker(gp_server* s, int slot) {
    gp_ctx* ctx = s->slots[static_cast<size_t>(slot)];
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                return (s->stopping && s->queue.empty()) ||
                       (!s->queue.empty() && s->in_use + s->queue.front()->footprint <= s->budget);
            });
            if (s->queue.empty()) return;   // stopping and drained
            r = s->queue.front();
            s->queue.pop_front();
            s->in_use += r->footprint;
            r->slot = slot;
            r->started = Clock::now();
            // a slot left idle may admit the next request as well
            s->cv_work.notify_all();
        }
        gp_report rep{};
        const gp_status st = r->packed
            ? gp_partition_range(ctx, &r->graph, r->vertex_begin, r->vertex_end, &r->options, r->labels, &rep)
            : gp_partition(ctx, &r->graph, &r->options, r->labels, &rep);
        std::string msg = st == GP_OK ? std::string() : std::string(gp_ctx_error(ctx));
        // a slot keeps at most its share of the budget cached between requests
        uint64_t live = 0, cached = 0;
        gp_ctx_memory(ctx, &live, &cached, nullptr, 0);
        if (cached + live > s->budget / std::max<size_t>(1, s->slots.size())) gp_ctx_trim(ctx);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->report = rep;
            r->status = st;
            r->message = std::move(msg);
            r->finished = Clock::now();
            r->done = true;
            s->in_use -= r->footprint;
            ++s->completed;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

gp_status submit(gp_server* s, const gp_graph* g, bool packed, int64_t vb, int64_t ve, const gp_options* o,
                 int32_t* labels, uint64_t* ticket) {
    if (!s || !g || !ticket) return GP_EINVAL;
    auto r = std::make_shared<Request>();
    r->graph = *g;
    r->packed = packed;
    r->vertex_begin = vb;
    r->vertex_end = ve;
    if (o) r->options = *o; else gp_options_default(&r->options);
    r->labels = labels;
    const int64_t n = packed ? ve - vb : g->n;
    int64_t m = g->m;
    if (packed) {
        // host offsets give the instance's edge count; for device offsets its
        // share of the packed edges by vertices stands in for the projection
        if (g->memory == GP_MEMORY_HOST && g->offsets) {
            if (g->index64 || g->width == GP_WIDTH_BIG) {
                const auto* off = static_cast<const int64_t*>(g->offsets);
                m = off[ve] - off[vb];
            } else {
                const auto* off = static_cast<const int32_t*>(g->offsets);
                m = static_cast<int64_t>(off[ve]) - off[vb];
            }
        } else {
            m = g->n ? static_cast<int64_t>(static_cast<double>(g->m) * static_cast<double>(n) / g->n) : 0;
        }
    }
    r->footprint = footprint(n, m, r->options.parts, g->width, g->index64 && g->memory == GP_MEMORY_HOST);
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->footprint > s->budget) {
        s->error = "request's projected device footprint exceeds the server's memory budget";
        return GP_ENOMEM;
    }
    r->ticket = s->next_ticket++;
    r->submitted = Clock::now();
    s->requests.emplace(r->ticket, r);
    s->queue.push_back(r);
    *ticket = r->ticket;
    s->cv_work.notify_one();
    return GP_OK;
}

double seconds(Clock::duration d) { return std::chrono::duration<double>(d).count(); }

}  // namespace

extern "C" {

uint64_t gp_footprint_bytes(int64_t n, int64_t m, int32_t parts, int32_t width, int32_t index64_host) {
    return footprint(n, m, parts, width, index64_host);
}

gp_status gp_server_create(int device, int32_t slots, uint64_t memory_budget, gp_server** out) {
    if (!out || slots < 1 || slots > 64 || memory_budget == 0) return GP_EINVAL;
    auto s = std::make_unique<gp_server>();
    s->device = device;
    s->budget = memory_budget;
    for (int i = 0; i < slots; ++i) {
        gp_ctx* c = nullptr;
        const gp_status st = gp_ctx_create(device, &c);
        if (st != GP_OK) {
            for (auto* x : s->slots) gp_ctx_destroy(x);
            *out = nullptr;
            return st;
        }
        gp_ctx_set_device_share(c, slots);
        s->slots.push_back(c);
    }
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker, s.get(), i);
    *out = s.release();
    return GP_OK;
}

void gp_server_destroy(gp_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto* c : s->slots) gp_ctx_destroy(c);
    delete s;
}

const char* gp_server_error(const gp_server* s) { return s ? s->error.c_str() : "null server"; }

gp_status gp_server_submit(gp_server* s, const gp_graph* graph, const gp_options* options, int32_t* labels,
                           uint64_t* ticket) {
    return submit(s, graph, false, 0, 0, options, labels, ticket);
}

gp_status gp_server_submit_range(gp_server* s, const gp_graph* packed, int64_t vertex_begin, int64_t vertex_end,
                                 const gp_options* options, int32_t* labels, uint64_t* ticket) {
    if (!packed || vertex_begin < 0 || vertex_end < vertex_begin || vertex_end > packed->n) return GP_EINVAL;
    return submit(s, packed, true, vertex_begin, vertex_end, options, labels, ticket);
}

gp_status gp_server_poll(gp_server* s, uint64_t ticket, int32_t* done) {
    if (!s || !done) return GP_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return GP_EINVAL;
    *done = it->second->done ? 1 : 0;
    return GP_OK;
}

gp_status gp_server_wait(gp_server* s, uint64_t ticket, gp_report* report, gp_request_info* info) {
    if (!s) return GP_EINVAL;
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->requests.find(ticket);
        if (it == s->requests.end()) return GP_EINVAL;
        r = it->second;
        s->cv_done.wait(lk, [&] { return r->done; });
        s->requests.erase(it);
    }
    if (report) *report = r->report;
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->status = r->status;
        info->slot = r->slot;
        info->queued_seconds = seconds(r->started - r->submitted);
        info->service_seconds = seconds(r->finished - r->started);
        info->latency_seconds = seconds(r->finished - r->submitted);
        info->footprint_bytes = r->footprint;
        std::strncpy(info->message, r->message.c_str(), sizeof(info->message) - 1);
    }
    return r->status;
}

gp_status gp_partition_batch(gp_server* s, const gp_graph* packed, int32_t count, const int64_t* vertex_offsets,
                             const gp_options* options, int32_t* labels, gp_report* reports, int32_t* statuses) {
    if (!s || !packed || count < 0 || (count > 0 && !vertex_offsets)) return GP_EINVAL;
    if (vertex_offsets && (vertex_offsets[0] != 0 || vertex_offsets[count] != packed->n)) return GP_EINVAL;
    for (int32_t i = 0; i < count; ++i)
        if (vertex_offsets[i + 1] < vertex_offsets[i]) return GP_EINVAL;
    // largest instances first, so the small ones fill the tail
    std::vector<int32_t> order(static_cast<size_t>(count));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return vertex_offsets[a + 1] - vertex_offsets[a] > vertex_offsets[b + 1] - vertex_offsets[b];
    });

    std::vector<uint64_t> tickets(static_cast<size_t>(count), 0);
    gp_status first = GP_OK;
    for (int32_t i : order) {
        const gp_status st = gp_server_submit_range(s, packed, vertex_offsets[i], vertex_offsets[i + 1],
                                                    options ? &options[i] : nullptr,
                                                    labels ? labels + vertex_offsets[i] : nullptr,
                                                    &tickets[static_cast<size_t>(i)]);
        if (st != GP_OK) {
            if (statuses) statuses[i] = st;
            if (first == GP_OK) first = st;
        }
    }
    for (int32_t i = 0; i < count; ++i) {
        if (!tickets[static_cast<size_t>(i)]) continue;
        gp_request_info info;
        const gp_status st = gp_server_wait(s, tickets[static_cast<size_t>(i)], reports ? &reports[i] : nullptr, &info);
        if (statuses) statuses[i] = st;
        if (st != GP_OK && first == GP_OK) {
            first = st;
            std::lock_guard<std::mutex> lk(s->mu);
            s->error = "instance " + std::to_string(i) + ": " + info.message;
        }
    }
    return first;
}

}  // extern "C"
