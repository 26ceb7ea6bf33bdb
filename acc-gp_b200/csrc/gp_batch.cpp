// Many graphs on one GPU: gp_partition_batch and the partition server.
//
// One graph's V-cycle is a chain of short kernels separated by host
// decisions, so a small or medium graph leaves most of the GPU idle.  Both
// forms therefore keep several graphs in flight at once, each on its own
// worker context (stream + device arenas) driven by its own host thread; the
// GPU interleaves their kernels.  A graph's result does not depend on what
// else runs: every worker executes the same deterministic single-graph path
// (METIS calls are serialised, see gp_metis.cpp).
#include "gp_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

namespace gp {

namespace {

double seconds_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

// Device bytes a partition of (n, m, k) may hold at once, before any request
// of that graph has been measured: the input and the hierarchy (about three
// CSR copies), the coarsening and contraction temporaries (about 24 bytes per
// entry) and the dense k-wide affinity cache of the refinement.
uint64_t footprint(int64_t n, int64_t m, int k) {
    return static_cast<uint64_t>(m) * 40 + static_cast<uint64_t>(n) * (static_cast<uint64_t>(k) * 4 + 64) + (64ULL << 20);
}

// The k-dependent part of a footprint: the dense n x k affinity cache of the
// input level (4-byte counters) and the k-wide scratch beside it.
uint64_t cache_bytes(int64_t n, int k) { return static_cast<uint64_t>(n) * static_cast<uint64_t>(k) * 4; }

// Work estimate of one partition for placement: one CSR sweep with its
// neighbour gathers, in bytes (proportional to the V-cycle's compulsory
// traffic, which is dominated by the input level).
uint64_t work_of(const gp_csr& g) {
    return 4ULL * static_cast<uint64_t>(g.n + 1) + 8ULL * static_cast<uint64_t>(g.m) +
           (g.edge_weights ? 4ULL * static_cast<uint64_t>(g.m) : 0ULL);
}

// Longest-processing-time placement: items in decreasing work (ties: lower
// index first), each to the device with the least work so far (ties: lower
// device).  Deterministic, so every process computes the same plan.
void plan(const uint64_t* work, int32_t count, int32_t devices, int32_t* device_of, uint64_t* device_work) {
    std::vector<int32_t> order(static_cast<size_t>(count));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return work[a] > work[b]; });
    std::vector<uint64_t> load(static_cast<size_t>(devices), 0);
    for (int32_t i : order) {
        const auto d = static_cast<int32_t>(std::min_element(load.begin(), load.end()) - load.begin());
        device_of[i] = d;
        load[static_cast<size_t>(d)] += work[i];
    }
    if (device_work) std::copy(load.begin(), load.end(), device_work);
}

}  // namespace

// Worker contexts of the batched form, per device, kept by the calling
// context for later batches.
struct WorkerPool {
    std::map<int, std::vector<gp_context*>> contexts;
};

void destroy_worker_pool(WorkerPool* pool) {
    if (!pool) return;
    for (auto& entry : pool->contexts)
        for (gp_context* c : entry.second) gp_context_destroy(c);
    delete pool;
}

}  // namespace gp

using namespace gp;

extern "C" gp_status gp_plan_placement(const uint64_t* work, int32_t count, int32_t devices, int32_t* device_of,
                                       uint64_t* device_work) {
    if (count < 0 || devices < 1 || (count > 0 && (!work || !device_of))) {
        set_error("count must be >= 0, devices >= 1, work and device_of non-NULL");
        return GP_INVALID_ARGUMENT;
    }
    plan(work, count, devices, device_of, device_work);
    return GP_OK;
}

extern "C" gp_status gp_partition_batch_devices(gp_context* ctx, const int32_t* devices, int32_t device_count,
                                                gp_request* requests, int32_t count, int32_t concurrency) {
    if (!ctx || (count > 0 && !requests) || !devices) { set_error("context, devices or requests is NULL"); return GP_INVALID_ARGUMENT; }
    if (count < 0 || concurrency < 1 || concurrency > 64 || device_count < 1 || device_count > 64) {
        set_error("count must be >= 0, concurrency in 1..64 and device_count in 1..64");
        return GP_INVALID_ARGUMENT;
    }
    int available = 0;
    if (cudaGetDeviceCount(&available) != cudaSuccess) {
        cudaGetLastError();
        available = 0;
    }
    for (int32_t d = 0; d < device_count; ++d)
        if (devices[d] < 0 || devices[d] >= available) { set_error("device ordinal out of range"); return GP_INVALID_ARGUMENT; }
    if (count == 0) return GP_OK;
    // Graphs to devices, longest processing time first; on each device the
    // largest graphs start first, so that the last ones to start are short.
    std::vector<uint64_t> work(static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i) work[static_cast<size_t>(i)] = work_of(requests[i].graph);
    std::vector<int32_t> device_of(static_cast<size_t>(count));
    plan(work.data(), count, device_count, device_of.data(), nullptr);
    std::vector<std::vector<int32_t>> lists(static_cast<size_t>(device_count));
    for (int32_t i = 0; i < count; ++i) lists[static_cast<size_t>(device_of[static_cast<size_t>(i)])].push_back(i);
    WorkerPool*& pool = worker_pool(ctx);
    if (!pool) pool = new WorkerPool;
    struct Lane { gp_context* context; int32_t list; };
    std::vector<Lane> lanes;
    std::map<int, size_t> taken;  // contexts of a device already given a lane (a device may be listed twice)
    for (int32_t d = 0; d < device_count; ++d) {
        auto& list = lists[static_cast<size_t>(d)];
        std::stable_sort(list.begin(), list.end(), [&](int32_t a, int32_t b) {
            return work[static_cast<size_t>(a)] > work[static_cast<size_t>(b)];
        });
        const size_t workers = std::min<size_t>(static_cast<size_t>(concurrency), list.size());
        auto& contexts = pool->contexts[devices[d]];
        size_t& first = taken[devices[d]];
        while (contexts.size() < first + workers) {
            gp_context* c = nullptr;
            if (gp_status st = gp_context_create(devices[d], &c); st != GP_OK) return st;
            contexts.push_back(c);
        }
        for (size_t w = first; w < first + workers; ++w) {
            copy_options(ctx, contexts[w]);
            lanes.push_back({contexts[w], d});
        }
        first += workers;
    }
    std::vector<std::atomic<int32_t>> next(static_cast<size_t>(device_count));
    for (auto& x : next) x.store(0);
    std::vector<std::string> messages(static_cast<size_t>(count));
    auto work_loop = [&](Lane lane) {
        const auto& list = lists[static_cast<size_t>(lane.list)];
        auto& cursor = next[static_cast<size_t>(lane.list)];
        for (int32_t i = cursor.fetch_add(1); i < static_cast<int32_t>(list.size()); i = cursor.fetch_add(1)) {
            gp_request& r = requests[list[static_cast<size_t>(i)]];
            const auto start = std::chrono::steady_clock::now();
            r.status = gp_partition(lane.context, &r.graph, r.k, r.epsilon, r.seed, r.flags, r.labels_out, &r.stats);
            r.queue_seconds = 0;
            r.run_seconds = seconds_since(start);
            if (r.status != GP_OK) messages[static_cast<size_t>(list[static_cast<size_t>(i)])] = last_error();
        }
    };
    std::vector<std::thread> threads;
    for (size_t w = 1; w < lanes.size(); ++w) threads.emplace_back(work_loop, lanes[w]);
    work_loop(lanes[0]);
    for (auto& t : threads) t.join();
    for (int32_t i = 0; i < count; ++i)
        if (requests[i].status != GP_OK) {
            set_error("request " + std::to_string(i) + ": " + messages[static_cast<size_t>(i)]);
            return requests[i].status;
        }
    return GP_OK;
}

extern "C" gp_status gp_partition_batch(gp_context* ctx, gp_request* requests, int32_t count, int32_t concurrency) {
    if (!ctx) { set_error("context or requests is NULL"); return GP_INVALID_ARGUMENT; }
    const int32_t device = context_device(ctx);
    return gp_partition_batch_devices(ctx, &device, 1, requests, count, concurrency);
}

// ---------------------------------------------------------------- server

struct gp_server {
    // A resident graph: one copy of its arrays on every device of the server.
    struct Graph {
        int64_t n = 0, m = 0;
        struct Arrays { int32_t* off = nullptr; int32_t* nbr = nullptr; uint32_t* vw = nullptr; uint32_t* ew = nullptr; };
        std::vector<Arrays> on;  // per device index
        // Measured footprint without the k-dependent cache: the largest
        // (device peak - n k 4) over this graph's completed requests; 0 until
        // one has run.
        uint64_t measured_base = 0;
    };
    struct Job {
        gp_request* request = nullptr;
        int32_t graph = -1;
        uint64_t bytes = 0;
        int device = -1;  // device index the job runs on, once admitted
        std::chrono::steady_clock::time_point submitted;
        bool done = false;
    };
    std::vector<int> devices;
    std::vector<HierarchyCache*> caches;  // per device index; empty until gp_server_keep_hierarchies
    uint64_t budget = 0;            // per device
    std::vector<uint64_t> in_use;   // per device index
    bool stopping = false;
    std::vector<gp_context*> contexts;
    std::vector<int> context_device;  // device index of each worker
    std::vector<std::thread> threads;
    std::vector<Graph> graphs;
    std::mutex mu;
    std::condition_variable work_cv, done_cv;
    std::deque<uint64_t> queue;
    std::map<uint64_t, Job> jobs;
    uint64_t next_ticket = 1;

    // Admission estimate of a request: for a resident graph that has run
    // before, its measured base plus the cache of this k and a 1/8 margin;
    // otherwise the static estimate.
    uint64_t estimate(int32_t graph, int64_t n, int64_t m, int k) const {
        if (graph >= 0) {
            const Graph& g = graphs[static_cast<size_t>(graph)];
            if (g.measured_base) {
                const uint64_t b = g.measured_base + cache_bytes(n, k) + 4ULL * static_cast<uint64_t>(n);
                return b + b / 8;
            }
        }
        return footprint(n, m, k);
    }

    // Index in `queue` of the first job that fits the budget of device index
    // d, or -1.  An idle device always admits (oversize requests run alone).
    long admissible(int d) const {
        for (size_t i = 0; i < queue.size(); ++i) {
            const uint64_t b = jobs.at(queue[i]).bytes;
            if (!budget || in_use[static_cast<size_t>(d)] == 0 || in_use[static_cast<size_t>(d)] + b <= budget)
                return static_cast<long>(i);
        }
        return -1;
    }

    void worker(gp_context* c, int d) {
        const int device = devices[static_cast<size_t>(d)];
        int32_t* labels_dev = nullptr;
        size_t labels_cap = 0;
        while (true) {
            uint64_t ticket = 0;
            Job job;
            Graph::Arrays arrays;  // copied under the lock: gp_server_add_graph may grow `graphs` meanwhile
            int64_t gn = 0, gm = 0;
            {
                std::unique_lock<std::mutex> lock(mu);
                work_cv.wait(lock, [&] { return (stopping && queue.empty()) || admissible(d) >= 0; });
                const long at = admissible(d);
                if (at < 0) break;  // stopping with an empty queue
                ticket = queue[static_cast<size_t>(at)];
                queue.erase(queue.begin() + at);
                Job& stored = jobs.at(ticket);
                stored.device = d;
                job = stored;
                if (job.graph >= 0) {
                    const Graph& g = graphs[static_cast<size_t>(job.graph)];
                    arrays = g.on[static_cast<size_t>(d)];
                    gn = g.n;
                    gm = g.m;
                }
                in_use[static_cast<size_t>(d)] += job.bytes;
            }
            gp_request& r = *job.request;
            const auto start = std::chrono::steady_clock::now();
            r.queue_seconds = std::chrono::duration<double>(start - job.submitted).count();
            if (job.graph < 0) {
                r.status = gp_partition(c, &r.graph, r.k, r.epsilon, r.seed, r.flags, r.labels_out, &r.stats);
            } else {
                r.status = GP_OK;
                if (labels_cap < static_cast<size_t>(gn)) {
                    cudaSetDevice(device);
                    if (labels_dev) cudaFree(labels_dev);
                    labels_dev = nullptr;
                    if (cudaMalloc(&labels_dev, sizeof(int32_t) * static_cast<size_t>(gn)) != cudaSuccess) {
                        cudaGetLastError();  // handled: this request reports GP_OUT_OF_MEMORY
                        labels_dev = nullptr;
                        labels_cap = 0;
                        r.status = GP_OUT_OF_MEMORY;
                    } else {
                        labels_cap = static_cast<size_t>(gn);
                    }
                }
                if (r.status == GP_OK) {
                    const gp_csr dg{gn, gm, arrays.off, arrays.nbr, arrays.vw, arrays.ew};
                    HierarchyCache* cache = caches.empty() ? nullptr : caches[static_cast<size_t>(d)];
                    r.status = cache ? partition_resident(c, cache, static_cast<uint64_t>(job.graph), &dg, r.k, r.epsilon,
                                                          r.seed, r.flags, labels_dev, &r.stats)
                                     : gp_partition_device(c, &dg, r.k, r.epsilon, r.seed, r.flags, labels_dev, nullptr,
                                                           &r.stats);
                }
                if (r.status == GP_OK &&
                    cudaMemcpy(r.labels_out, labels_dev, sizeof(int32_t) * static_cast<size_t>(gn),
                               cudaMemcpyDeviceToHost) != cudaSuccess) {
                    cudaGetLastError();
                    r.status = GP_CUDA_ERROR;
                }
            }
            r.run_seconds = seconds_since(start);
            // Arenas only grow, so an idle worker would keep the memory of the
            // largest request it ran: with a budget, a worker holding more than
            // its share of it gives the memory back.
            const size_t per_device = contexts.size() / devices.size();
            if (budget && context_reserved(c) > budget / std::max<size_t>(1, per_device)) context_trim(c);
            {
                std::lock_guard<std::mutex> lock(mu);
                in_use[static_cast<size_t>(d)] -= job.bytes;
                if (job.graph >= 0 && r.status == GP_OK) {
                    Graph& g = graphs[static_cast<size_t>(job.graph)];
                    const uint64_t measured = r.stats.device_peak_bytes + 4ULL * static_cast<uint64_t>(gn);
                    const uint64_t cache = cache_bytes(gn, r.k);
                    g.measured_base = std::max(g.measured_base, measured > cache ? measured - cache : measured);
                }
                jobs.at(ticket).done = true;
            }
            done_cv.notify_all();
            work_cv.notify_all();
        }
        if (labels_dev) {
            cudaSetDevice(device);
            cudaFree(labels_dev);
        }
    }
};

extern "C" gp_status gp_server_create_devices(const int32_t* devices, int32_t device_count, int32_t workers_per_device,
                                              uint64_t hbm_budget_bytes, gp_server** out) {
    if (!out || !devices || device_count < 1 || device_count > 64 || workers_per_device < 1 || workers_per_device > 64) {
        set_error("out or devices is NULL, device_count outside 1..64 or workers outside 1..64");
        return GP_INVALID_ARGUMENT;
    }
    auto server = std::make_unique<gp_server>();
    server->budget = hbm_budget_bytes;
    for (int32_t d = 0; d < device_count; ++d) {
        server->devices.push_back(devices[d]);
        for (int w = 0; w < workers_per_device; ++w) {
            gp_context* c = nullptr;
            if (gp_status st = gp_context_create(devices[d], &c); st != GP_OK) {
                for (gp_context* x : server->contexts) gp_context_destroy(x);
                return st;
            }
            server->contexts.push_back(c);
            server->context_device.push_back(d);
        }
    }
    server->in_use.assign(server->devices.size(), 0);
    gp_server* s = server.release();
    for (size_t i = 0; i < s->contexts.size(); ++i) s->threads.emplace_back(&gp_server::worker, s, s->contexts[i], s->context_device[i]);
    *out = s;
    return GP_OK;
}

extern "C" gp_status gp_server_create(int device, int32_t workers, uint64_t hbm_budget_bytes, gp_server** out) {
    const int32_t d = device;
    return gp_server_create_devices(&d, 1, workers, hbm_budget_bytes, out);
}

extern "C" gp_status gp_server_add_graph(gp_server* server, const gp_csr* graph, int32_t* graph_id) {
    if (!server || !graph || !graph_id) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    if (gp_status st = validate_host_csr(graph, true); st != GP_OK) return st;
    gp_server::Graph g;
    g.n = graph->n;
    g.m = graph->m;
    auto upload = [&](void** dst, const void* src, size_t bytes) -> bool {
        if (!src) return true;
        if (cudaMalloc(dst, bytes ? bytes : 4) != cudaSuccess) {
            cudaGetLastError();  // handled: gp_server_add_graph reports it
            *dst = nullptr;
            return false;
        }
        if (bytes && cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return true;
    };
    bool ok = true;
    for (int device : server->devices) {
        gp_server::Graph::Arrays a;
        ok = ok && cudaSetDevice(device) == cudaSuccess &&
             upload(reinterpret_cast<void**>(&a.off), graph->offsets, sizeof(int32_t) * (g.n + 1)) &&
             upload(reinterpret_cast<void**>(&a.nbr), graph->neighbors, sizeof(int32_t) * g.m) &&
             upload(reinterpret_cast<void**>(&a.vw), graph->vertex_weights, sizeof(uint32_t) * g.n) &&
             upload(reinterpret_cast<void**>(&a.ew), graph->edge_weights, sizeof(uint32_t) * g.m);
        g.on.push_back(a);
        if (!ok) break;
    }
    if (!ok) {
        for (size_t d = 0; d < g.on.size(); ++d) {
            cudaSetDevice(server->devices[d]);
            cudaFree(g.on[d].off); cudaFree(g.on[d].nbr); cudaFree(g.on[d].vw); cudaFree(g.on[d].ew);
        }
        set_error("cannot place the graph on the device");
        return GP_OUT_OF_MEMORY;
    }
    std::lock_guard<std::mutex> lock(server->mu);
    server->graphs.push_back(g);
    *graph_id = static_cast<int32_t>(server->graphs.size() - 1);
    return GP_OK;
}

extern "C" gp_status gp_server_keep_hierarchies(gp_server* server, uint64_t bytes_per_device) {
    if (!server) { set_error("server is NULL"); return GP_INVALID_ARGUMENT; }
    std::lock_guard<std::mutex> lock(server->mu);
    if (!server->caches.empty() || !server->jobs.empty()) {
        set_error("set the hierarchy budget once, before the first request");
        return GP_INVALID_ARGUMENT;
    }
    if (!bytes_per_device) return GP_OK;
    for (int device : server->devices) server->caches.push_back(hierarchy_cache_create(device, bytes_per_device));
    return GP_OK;
}

extern "C" gp_status gp_server_kept_bytes(gp_server* server, uint64_t* bytes) {
    if (!server || !bytes) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    uint64_t total = 0;
    for (HierarchyCache* c : server->caches) total += hierarchy_cache_bytes(c);
    *bytes = total;
    return GP_OK;
}

extern "C" gp_status gp_server_footprint(gp_server* server, int32_t graph_id, int32_t k, uint64_t* bytes) {
    if (!server || !bytes) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    std::lock_guard<std::mutex> lock(server->mu);
    if (graph_id < 0 || graph_id >= static_cast<int32_t>(server->graphs.size())) { set_error("no such resident graph"); return GP_INVALID_ARGUMENT; }
    const auto& g = server->graphs[static_cast<size_t>(graph_id)];
    *bytes = server->estimate(graph_id, g.n, g.m, k);
    return GP_OK;
}

extern "C" gp_status gp_server_submit(gp_server* server, gp_request* request, int32_t graph_id, uint64_t* ticket) {
    if (!server || !request || !ticket || !request->labels_out) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    gp_server::Job job;
    job.request = request;
    job.graph = graph_id;
    job.submitted = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lock(server->mu);
        int64_t n = request->graph.n, m = request->graph.m;
        if (graph_id >= 0) {
            if (graph_id >= static_cast<int32_t>(server->graphs.size())) { set_error("no such resident graph"); return GP_INVALID_ARGUMENT; }
            n = server->graphs[static_cast<size_t>(graph_id)].n;
            m = server->graphs[static_cast<size_t>(graph_id)].m;
        }
        if (server->stopping) { set_error("server is stopping"); return GP_INVALID_ARGUMENT; }
        job.bytes = server->estimate(graph_id, n, m, request->k);
        *ticket = server->next_ticket++;
        request->status = GP_OK;
        server->jobs.emplace(*ticket, job);
        server->queue.push_back(*ticket);
    }
    server->work_cv.notify_all();
    return GP_OK;
}

extern "C" gp_status gp_server_wait(gp_server* server, uint64_t ticket, double timeout_seconds) {
    if (!server) { set_error("server is NULL"); return GP_INVALID_ARGUMENT; }
    std::unique_lock<std::mutex> lock(server->mu);
    auto it = server->jobs.find(ticket);
    if (it == server->jobs.end()) { set_error("unknown ticket"); return GP_INVALID_ARGUMENT; }
    // Another thread waiting on the same ticket may erase it first.
    auto finished = [&] {
        auto j = server->jobs.find(ticket);
        return j == server->jobs.end() || j->second.done;
    };
    if (timeout_seconds < 0) {
        server->done_cv.wait(lock, finished);
    } else if (!server->done_cv.wait_for(lock, std::chrono::duration<double>(timeout_seconds), finished)) {
        set_error("request still running");
        return GP_DEVICE_TIMEOUT;
    }
    if (server->jobs.erase(ticket) == 0) {
        set_error("unknown ticket (another wait already collected it)");
        return GP_INVALID_ARGUMENT;
    }
    return GP_OK;
}

extern "C" void gp_server_destroy(gp_server* server) {
    if (!server) return;
    {
        std::lock_guard<std::mutex> lock(server->mu);
        server->stopping = true;
    }
    server->work_cv.notify_all();
    for (auto& t : server->threads) t.join();
    for (gp_context* c : server->contexts) gp_context_destroy(c);
    for (HierarchyCache* c : server->caches) hierarchy_cache_destroy(c);
    for (auto& g : server->graphs)
        for (size_t d = 0; d < g.on.size(); ++d) {
            cudaSetDevice(server->devices[d]);
            cudaFree(g.on[d].off); cudaFree(g.on[d].nbr); cudaFree(g.on[d].vw); cudaFree(g.on[d].ew);
        }
    delete server;
}
