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

// Device bytes a partition of (n, m, k) may hold at once: the input and the
// hierarchy (about three CSR copies), the coarsening and contraction
// temporaries (about 24 bytes per entry) and the dense k-wide affinity cache
// of the refinement.  An estimate for admission, not an exact bound.
uint64_t footprint(int64_t n, int64_t m, int k) {
    return static_cast<uint64_t>(m) * 40 + static_cast<uint64_t>(n) * (static_cast<uint64_t>(k) * 4 + 64) + (64ULL << 20);
}

}  // namespace

struct WorkerPool {
    std::vector<gp_context*> contexts;
};

void destroy_worker_pool(WorkerPool* pool) {
    if (!pool) return;
    for (gp_context* c : pool->contexts) gp_context_destroy(c);
    delete pool;
}

}  // namespace gp

using namespace gp;

extern "C" gp_status gp_partition_batch(gp_context* ctx, gp_request* requests, int32_t count, int32_t concurrency) {
    if (!ctx || (count > 0 && !requests)) { set_error("context or requests is NULL"); return GP_INVALID_ARGUMENT; }
    if (count < 0 || concurrency < 1 || concurrency > 64) {
        set_error("count must be >= 0 and concurrency in 1..64");
        return GP_INVALID_ARGUMENT;
    }
    if (count == 0) return GP_OK;
    const int workers = std::min<int>(concurrency, count);
    WorkerPool*& pool = worker_pool(ctx);
    if (!pool) pool = new WorkerPool;
    while (static_cast<int>(pool->contexts.size()) < workers) {
        gp_context* c = nullptr;
        if (gp_status st = gp_context_create(context_device(ctx), &c); st != GP_OK) return st;
        pool->contexts.push_back(c);
    }
    for (int w = 0; w < workers; ++w) copy_options(ctx, pool->contexts[w]);
    // Largest first, so that the last graphs to start are short.
    std::vector<int32_t> order(static_cast<size_t>(count));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return requests[a].graph.n + requests[a].graph.m > requests[b].graph.n + requests[b].graph.m;
    });
    std::atomic<int32_t> next{0};
    std::vector<std::string> messages(static_cast<size_t>(count));
    auto work = [&](gp_context* c) {
        for (int32_t i = next.fetch_add(1); i < count; i = next.fetch_add(1)) {
            gp_request& r = requests[order[i]];
            const auto start = std::chrono::steady_clock::now();
            r.status = gp_partition(c, &r.graph, r.k, r.epsilon, r.seed, r.flags, r.labels_out, &r.stats);
            r.queue_seconds = 0;
            r.run_seconds = seconds_since(start);
            if (r.status != GP_OK) messages[order[i]] = last_error();
        }
    };
    std::vector<std::thread> threads;
    for (int w = 1; w < workers; ++w) threads.emplace_back(work, pool->contexts[w]);
    work(pool->contexts[0]);
    for (auto& t : threads) t.join();
    for (int32_t i = 0; i < count; ++i)
        if (requests[i].status != GP_OK) {
            set_error("request " + std::to_string(i) + ": " + messages[i]);
            return requests[i].status;
        }
    return GP_OK;
}

// ---------------------------------------------------------------- server

struct gp_server {
    struct Graph {
        int64_t n = 0, m = 0;
        int32_t* off = nullptr;
        int32_t* nbr = nullptr;
        uint32_t* vw = nullptr;
        uint32_t* ew = nullptr;
    };
    struct Job {
        gp_request* request = nullptr;
        int32_t graph = -1;
        uint64_t bytes = 0;
        std::chrono::steady_clock::time_point submitted;
        bool done = false;
    };
    int device = 0;
    uint64_t budget = 0, in_use = 0;
    bool stopping = false;
    std::vector<gp_context*> contexts;
    std::vector<std::thread> threads;
    std::vector<Graph> graphs;
    std::mutex mu;
    std::condition_variable work_cv, done_cv;
    std::deque<uint64_t> queue;
    std::map<uint64_t, Job> jobs;
    uint64_t next_ticket = 1;

    // Index in `queue` of the first job that fits the budget, or -1.
    long admissible() const {
        for (size_t i = 0; i < queue.size(); ++i) {
            const uint64_t b = jobs.at(queue[i]).bytes;
            if (!budget || in_use == 0 || in_use + b <= budget) return static_cast<long>(i);
        }
        return -1;
    }

    void worker(gp_context* c) {
        int32_t* labels_dev = nullptr;
        size_t labels_cap = 0;
        while (true) {
            uint64_t ticket = 0;
            Job job;
            Graph g;  // copied under the lock: gp_server_add_graph may grow `graphs` meanwhile
            {
                std::unique_lock<std::mutex> lock(mu);
                work_cv.wait(lock, [&] { return (stopping && queue.empty()) || admissible() >= 0; });
                const long at = admissible();
                if (at < 0) break;  // stopping with an empty queue
                ticket = queue[static_cast<size_t>(at)];
                queue.erase(queue.begin() + at);
                job = jobs.at(ticket);
                if (job.graph >= 0) g = graphs[static_cast<size_t>(job.graph)];
                in_use += job.bytes;
            }
            gp_request& r = *job.request;
            const auto start = std::chrono::steady_clock::now();
            r.queue_seconds = std::chrono::duration<double>(start - job.submitted).count();
            if (job.graph < 0) {
                r.status = gp_partition(c, &r.graph, r.k, r.epsilon, r.seed, r.flags, r.labels_out, &r.stats);
            } else {
                r.status = GP_OK;
                if (labels_cap < static_cast<size_t>(g.n)) {
                    cudaSetDevice(device);
                    if (labels_dev) cudaFree(labels_dev);
                    labels_dev = nullptr;
                    if (cudaMalloc(&labels_dev, sizeof(int32_t) * static_cast<size_t>(g.n)) != cudaSuccess) {
                        cudaGetLastError();  // handled: this request reports GP_OUT_OF_MEMORY
                        labels_dev = nullptr;
                        labels_cap = 0;
                        r.status = GP_OUT_OF_MEMORY;
                    } else {
                        labels_cap = static_cast<size_t>(g.n);
                    }
                }
                if (r.status == GP_OK) {
                    const gp_csr dg{g.n, g.m, g.off, g.nbr, g.vw, g.ew};
                    r.status = gp_partition_device(c, &dg, r.k, r.epsilon, r.seed, r.flags, labels_dev, nullptr, &r.stats);
                }
                if (r.status == GP_OK &&
                    cudaMemcpy(r.labels_out, labels_dev, sizeof(int32_t) * static_cast<size_t>(g.n),
                               cudaMemcpyDeviceToHost) != cudaSuccess)
                    r.status = GP_CUDA_ERROR;
            }
            r.run_seconds = seconds_since(start);
            // Arenas only grow, so an idle worker would keep the memory of the
            // largest request it ran: with a budget, a worker holding more than
            // its share of it gives the memory back.
            if (budget && context_reserved(c) > budget / contexts.size()) context_trim(c);
            {
                std::lock_guard<std::mutex> lock(mu);
                in_use -= job.bytes;
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

extern "C" gp_status gp_server_create(int device, int32_t workers, uint64_t hbm_budget_bytes, gp_server** out) {
    if (!out || workers < 1 || workers > 64) { set_error("out is NULL or workers outside 1..64"); return GP_INVALID_ARGUMENT; }
    auto server = std::make_unique<gp_server>();
    server->device = device;
    server->budget = hbm_budget_bytes;
    for (int w = 0; w < workers; ++w) {
        gp_context* c = nullptr;
        if (gp_status st = gp_context_create(device, &c); st != GP_OK) {
            for (gp_context* d : server->contexts) gp_context_destroy(d);
            return st;
        }
        server->contexts.push_back(c);
    }
    gp_server* s = server.release();
    for (gp_context* c : s->contexts) s->threads.emplace_back(&gp_server::worker, s, c);
    *out = s;
    return GP_OK;
}

extern "C" gp_status gp_server_add_graph(gp_server* server, const gp_csr* graph, int32_t* graph_id) {
    if (!server || !graph || !graph_id) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    if (gp_status st = validate_host_csr(graph, true); st != GP_OK) return st;
    gp_server::Graph g;
    g.n = graph->n;
    g.m = graph->m;
    cudaSetDevice(server->device);
    auto upload = [&](void** dst, const void* src, size_t bytes) -> bool {
        if (!src) return true;
        if (cudaMalloc(dst, bytes ? bytes : 4) != cudaSuccess) {
            cudaGetLastError();  // handled: gp_server_add_graph reports it
            *dst = nullptr;
            return false;
        }
        return !bytes || cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    const bool ok = upload(reinterpret_cast<void**>(&g.off), graph->offsets, sizeof(int32_t) * (g.n + 1)) &&
                    upload(reinterpret_cast<void**>(&g.nbr), graph->neighbors, sizeof(int32_t) * g.m) &&
                    upload(reinterpret_cast<void**>(&g.vw), graph->vertex_weights, sizeof(uint32_t) * g.n) &&
                    upload(reinterpret_cast<void**>(&g.ew), graph->edge_weights, sizeof(uint32_t) * g.m);
    if (!ok) {
        cudaFree(g.off); cudaFree(g.nbr); cudaFree(g.vw); cudaFree(g.ew);
        set_error("cannot place the graph on the device");
        return GP_OUT_OF_MEMORY;
    }
    std::lock_guard<std::mutex> lock(server->mu);
    server->graphs.push_back(g);
    *graph_id = static_cast<int32_t>(server->graphs.size() - 1);
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
        job.bytes = footprint(n, m, request->k);
        *ticket = server->next_ticket++;
        request->status = GP_OK;
        server->jobs.emplace(*ticket, job);
        server->queue.push_back(*ticket);
    }
    server->work_cv.notify_one();
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
    cudaSetDevice(server->device);
    for (auto& g : server->graphs) {
        cudaFree(g.off); cudaFree(g.nbr); cudaFree(g.vw); cudaFree(g.ew);
    }
    delete server;
}
