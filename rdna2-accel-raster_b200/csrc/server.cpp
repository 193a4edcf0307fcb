// server.cpp — the serving loop of include/rq_serve.h.
//
// One worker thread per server owns every device call.  Its loop:
//   1. take newly submitted requests into the FIFO of pending requests;
//   2. poll the in-flight launches: a request is complete when its
//      host-mapped flag holds its launch's sequence number (the kernel sets it
//      when the request's last ray finishes, while the launch may still run);
//      a launch slot frees when its event has completed;
//   3. if a slot is free, admit pending requests in arrival order into one
//      launch (a "wave") until the wave's ray or request cap is reached or
//      the next request's mesh cannot be made resident: a resident mesh is
//      pinned, a missing one is uploaded from its pinned host copy and built
//      on the build stream after least-recently-used unpinned meshes are
//      evicted to fit the budget (a mesh larger than the whole budget fails
//      its requests with RQ_ERR_BUDGET); the wave's requests are ordered
//      smallest first, so small requests finish early inside the launch;
//   4. enqueue the job table copy and one k_serve launch on the slot's stream
//      (after the build stream's work), and record the slot's event.
// Several slots keep several launches in flight on separate streams, so a
// new wave fills the SMs that the tail of the previous one leaves idle.
// Plain mode is the same loop with one request per launch and one slot.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "rq_internal.h"
#include "rq_serve_internal.h"

size_t rq_bvh_alloc_bytes(uint32_t n, uint32_t node2_cap, uint32_t node4_cap);

namespace {

constexpr uint32_t kMaxSlots = 8;

struct MeshRec {
    float* h_pos = nullptr;  // pinned copies
    uint32_t* h_idx = nullptr;
    uint32_t nv = 0, nt = 0;
    uint64_t bytes = 0;
    bool resident = false;
    float* d_pos = nullptr;
    uint32_t* d_idx = nullptr;
    rq_bvh* bvh = nullptr;
    uint32_t depth4 = 0;
    int pins = 0;
    uint64_t last_use = 0;
};

struct Pending {
    rq_request req;
    uint64_t ticket;
    double t_submit;
};

struct Job {
    Pending p;
    double t_admit;
    bool built;
    bool done;
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    uint32_t seq = 0;
    void* d_buf = nullptr;   // ServeJob[RQ_SERVE_MAX_JOBS] | begins[RQ_SERVE_MAX_JOBS + 1] | done[...] | ctr
    void* h_buf = nullptr;   // pinned mirror of the table part
    uint32_t* h_flags = nullptr;  // host-mapped completion words
    uint32_t* d_flags = nullptr;
    std::vector<Job> jobs;
    uint32_t remaining = 0;
};

constexpr size_t kJobsBytes = sizeof(ServeJob) * RQ_SERVE_MAX_JOBS;
constexpr size_t kBeginsOff = kJobsBytes;
constexpr size_t kBeginsBytes = sizeof(uint32_t) * (RQ_SERVE_MAX_JOBS + 4);
constexpr size_t kDoneOff = kBeginsOff + kBeginsBytes;
constexpr size_t kDoneBytes = sizeof(uint32_t) * RQ_SERVE_MAX_JOBS;
constexpr size_t kCtrOff = kDoneOff + kDoneBytes;
constexpr size_t kSlotBytes = kCtrOff + 256;

uint64_t align256(uint64_t b) { return (b + 255) & ~uint64_t(255); }

}  // namespace

struct rq_server {
    rq_server_config cfg{};
    int device = 0;
    rq_ctx* ctx = nullptr;
    cudaStream_t build_st = nullptr;
    cudaEvent_t build_ev = nullptr;
    std::chrono::steady_clock::time_point t0;
    std::string last_error;

    std::mutex mesh_mu;
    std::vector<std::unique_ptr<MeshRec>> meshes;
    std::atomic<uint32_t> max_mesh_tris{0};

    std::mutex in_mu;
    std::condition_variable in_cv;
    std::deque<Pending> incoming;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::unordered_set<uint64_t> cancel_in;  // tickets to cancel, handed to the worker

    // host-side fault injection (rq_server_inject_fault)
    std::atomic<uint32_t> fault_alloc{0}, fault_launch{0};

    std::mutex out_mu;
    std::condition_variable out_cv;
    std::deque<rq_completion> done;

    // worker-owned
    std::deque<Pending> pending;
    std::unordered_set<uint64_t> cancelled;
    Slot slots[kMaxSlots];
    uint32_t seq = 0;
    uint64_t tick = 0;
    uint64_t resident_bytes = 0;
    rq_server_stats st{};
    std::mutex stats_mu;
    std::thread worker;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    void complete(const Pending& p, int status, double t_admit, bool built) {
        rq_completion c{};
        c.ticket = p.ticket;
        c.user = p.req.user;
        c.status = status;
        c.built = built ? 1u : 0u;
        c.t_submit = p.t_submit;
        c.t_admit = t_admit;
        c.t_done = now();
        {
            std::lock_guard<std::mutex> g(stats_mu);
            if (status == RQ_OK) {
                ++st.completed;
                st.rays += p.req.num_rays;
            } else {
                ++st.failed;
            }
        }
        {
            std::lock_guard<std::mutex> g(out_mu);
            done.push_back(c);
        }
        out_cv.notify_all();
    }

    MeshRec* mesh(uint32_t id) {
        std::lock_guard<std::mutex> g(mesh_mu);
        return id < meshes.size() ? meshes[id].get() : nullptr;
    }

    void evict(MeshRec* m) {
        rq_bvh_destroy(m->bvh);  // frees device memory (synchronises the device)
        cudaFree(m->d_pos);
        cudaFree(m->d_idx);
        m->bvh = nullptr;
        m->d_pos = nullptr;
        m->d_idx = nullptr;
        m->resident = false;
        resident_bytes -= m->bytes;
        std::lock_guard<std::mutex> g(stats_mu);
        ++st.evictions;
        st.resident_bytes = resident_bytes;
    }

    // 0 resident (built: uploaded and built now), 1 wait for memory, else a
    // status that fails the request.
    int make_resident(MeshRec* m, bool& built) {
        built = false;
        if (m->resident) return 0;
        if (m->bytes > cfg.hbm_budget_bytes) return RQ_ERR_BUDGET;
        while (resident_bytes + m->bytes > cfg.hbm_budget_bytes) {
            MeshRec* lru = nullptr;
            {
                std::lock_guard<std::mutex> g(mesh_mu);
                for (auto& r : meshes)
                    if (r->resident && r->pins == 0 && (!lru || r->last_use < lru->last_use)) lru = r.get();
            }
            if (!lru) return 1;
            evict(lru);
        }
        if (fault_alloc.load() > 0) {  // injected: as if the allocation failed
            --fault_alloc;
            return RQ_ERR_OOM;
        }
        // scratch for the largest mesh registered so far, so it rarely regrows
        BuildScratch probe;
        int rc = rq_ensure_scratch(ctx, rq_build_scratch_carve(nullptr, max_mesh_tris.load(), probe), build_st);
        if (rc) return rc;
        cudaError_t e = cudaMalloc(&m->d_pos, align256(12ull * m->nv));
        if (e == cudaSuccess) e = cudaMalloc(&m->d_idx, align256(12ull * m->nt));
        if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_pos, m->h_pos, 12ull * m->nv, cudaMemcpyHostToDevice, build_st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_idx, m->h_idx, 12ull * m->nt, cudaMemcpyHostToDevice, build_st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cudaFree(m->d_pos);
            cudaFree(m->d_idx);
            m->d_pos = nullptr;
            m->d_idx = nullptr;
            return e == cudaErrorMemoryAllocation ? RQ_ERR_OOM : RQ_ERR_CUDA;
        }
        rq_bvh* b = nullptr;
        rc = rq_build(ctx, m->d_pos, 12, m->nv, m->d_idx, m->nt, cfg.max_leaf, RQ_BUILD_BVH4, &b, build_st);
        if (rc) {
            cudaFree(m->d_pos);
            cudaFree(m->d_idx);
            m->d_pos = nullptr;
            m->d_idx = nullptr;
            return rc;
        }
        rq_bvh_info inf{};
        rq_bvh_info_get(b, &inf);
        m->bvh = b;
        m->depth4 = inf.depth4;
        m->resident = true;
        built = true;
        resident_bytes += m->bytes;
        std::lock_guard<std::mutex> g(stats_mu);
        ++st.builds;
        st.resident_bytes = resident_bytes;
        st.peak_resident_bytes = std::max<uint64_t>(st.peak_resident_bytes, resident_bytes);
        return 0;
    }

    void unpin(uint32_t mesh_id) {
        MeshRec* m = mesh(mesh_id);
        if (m) --m->pins;
    }

    // Step 2: completions and free slots.  Returns true if anything changed.
    bool poll() {
        bool changed = false;
        for (uint32_t s = 0; s < cfg.slots; ++s) {
            Slot& sl = slots[s];
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.ev);
            const bool ended = q != cudaErrorNotReady;
            if (q != cudaSuccess && q != cudaErrorNotReady) cudaGetLastError();
            for (size_t j = 0; j < sl.jobs.size(); ++j) {
                Job& jb = sl.jobs[j];
                if (jb.done) continue;
                const bool flagged = reinterpret_cast<volatile uint32_t*>(sl.h_flags)[j] == sl.seq;
                if (!flagged && !ended) continue;
                jb.done = true;
                --sl.remaining;
                unpin(jb.p.req.mesh);
                // flagged: the request's last ray finished (the launch may run on);
                // otherwise the launch ended without finishing it
                const int status = flagged ? RQ_OK : (q == cudaSuccess ? RQ_ERR_DEVICE_TIMEOUT : RQ_ERR_CUDA);
                complete(jb.p, status, jb.t_admit, jb.built);
                cancelled.erase(jb.p.ticket);  // a cancel that came too late
                changed = true;
            }
            if (ended && sl.remaining == 0) {
                sl.busy = false;
                sl.jobs.clear();
                changed = true;
            }
        }
        return changed;
    }

    uint32_t busy_slots() const {
        uint32_t n = 0;
        for (uint32_t s = 0; s < cfg.slots; ++s) n += slots[s].busy ? 1u : 0u;
        return n;
    }

    // Steps 3 and 4.  Returns true if a launch was made or a request failed.
    bool launch_wave() {
        if (pending.empty()) return false;
        Slot* sl = nullptr;
        for (uint32_t s = 0; s < cfg.slots && !sl; ++s)
            if (!slots[s].busy) sl = &slots[s];
        if (!sl) return false;
        std::vector<Job> sel;
        uint64_t rays = 0;
        bool any_built = false, failed = false;
        while (!pending.empty() && sel.size() < cfg.max_wave_requests) {
            Pending& p = pending.front();
            if (cancelled.erase(p.ticket)) {
                complete(p, RQ_ERR_CANCELLED, now(), false);
                pending.pop_front();
                failed = true;
                continue;
            }
            if (!sel.empty() && rays + p.req.num_rays > cfg.max_wave_rays) break;
            MeshRec* m = mesh(p.req.mesh);
            bool built = false;
            int rc = m ? make_resident(m, built) : RQ_ERR_INVALID_ARG;
            if (rc == 1) break;  // wait for in-flight requests to unpin memory
            if (rc == 0 && !built && cfg.rebuild) {
                // plain per-request build: in place on the build stream (one
                // launch in flight in plain mode, so nothing else reads it)
                rc = rq_build(ctx, m->d_pos, 12, m->nv, m->d_idx, m->nt, cfg.max_leaf, RQ_BUILD_BVH4, &m->bvh,
                              build_st);
                built = rc == 0;
                if (built) {
                    std::lock_guard<std::mutex> g(stats_mu);
                    ++st.builds;
                }
            }
            if (rc == 0 && 3u * (m->depth4 + 2u) + 1u > 128u) rc = RQ_ERR_UNSUPPORTED;
            if (rc != 0) {
                complete(p, rc, now(), false);
                pending.pop_front();
                failed = true;
                continue;
            }
            ++m->pins;
            m->last_use = ++tick;
            any_built |= built;
            sel.push_back(Job{p, 0.0, built, false});
            rays += p.req.num_rays;
            pending.pop_front();
        }
        if (sel.empty()) return failed;
        std::stable_sort(sel.begin(), sel.end(),
                         [](const Job& a, const Job& b) { return a.p.req.num_rays < b.p.req.num_rays; });
        ServeJob* hj = static_cast<ServeJob*>(sl->h_buf);
        uint32_t* hb = reinterpret_cast<uint32_t*>(static_cast<char*>(sl->h_buf) + kBeginsOff);
        const uint32_t seqno = ++seq;
        uint32_t begin = 0, depth = 0;
        for (size_t j = 0; j < sel.size(); ++j) {
            const rq_request& r = sel[j].p.req;
            MeshRec* m = mesh(r.mesh);
            ServeJob& J = hj[j];
            J.nodes4 = m->bvh->nodes4;
            J.tris = m->bvh->tris;
            J.perm = m->bvh->perm;
            J.pos = m->d_pos;
            J.idx = m->d_idx;
            J.rays = r.rays;
            J.hits = r.hits;
            J.flag = sl->d_flags + j;
            J.begin = begin;
            J.count = r.num_rays;
            J.kind = r.kind;
            J.seed = r.seed;
            J.ntri = m->nt;
            J.flags = r.flags;
            J.pad0 = J.pad1 = 0;
            hb[j] = begin;
            begin += (r.num_rays + 31u) & ~31u;
            depth = std::max(depth, m->depth4);
        }
        const uint32_t nj = uint32_t(sel.size());
        hb[nj] = begin;
        char* d = static_cast<char*>(sl->d_buf);
        cudaError_t e = cudaSuccess;
        if (any_built) {
            e = cudaEventRecord(build_ev, build_st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(sl->st, build_ev, 0);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(d, hj, sizeof(ServeJob) * nj, cudaMemcpyHostToDevice, sl->st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d + kBeginsOff, hb, sizeof(uint32_t) * (nj + 1), cudaMemcpyHostToDevice, sl->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(d + kDoneOff, 0, kDoneBytes + 256, sl->st);
        int rc = e == cudaSuccess ? RQ_OK : rq_cuda_status(ctx, e, "serve table upload");
        if (rc == RQ_OK && fault_launch.load() > 0) {  // injected: as if the launch had failed
            --fault_launch;
            rc = rq_set_error(ctx, RQ_ERR_CUDA, "injected launch failure");
        }
        if (rc == RQ_OK)
            rc = rq_launch_serve(ctx, reinterpret_cast<const ServeJob*>(d), reinterpret_cast<const uint32_t*>(d + kBeginsOff),
                                 nj, begin, depth, cfg.trace_flags, seqno, reinterpret_cast<uint32_t*>(d + kDoneOff),
                                 reinterpret_cast<uint32_t*>(d + kCtrOff), sl->st);
        if (rc == RQ_OK) rc = rq_cuda_status(ctx, cudaEventRecord(sl->ev, sl->st), "serve event");
        const double t = now();
        if (rc != RQ_OK) {
            last_error = rq_ctx_last_error(ctx);
            cudaStreamSynchronize(sl->st);  // the table copies read the slot's pinned buffer
            cudaGetLastError();
            for (Job& j : sel) {
                unpin(j.p.req.mesh);
                complete(j.p, rc, t, j.built);
            }
            return true;
        }
        for (Job& j : sel) j.t_admit = t;
        sl->seq = seqno;
        sl->jobs = std::move(sel);
        sl->remaining = nj;
        sl->busy = true;
        std::lock_guard<std::mutex> g(stats_mu);
        ++st.launches;
        st.max_requests_per_launch = std::max<uint64_t>(st.max_requests_per_launch, nj);
        st.max_launches_in_flight = std::max<uint64_t>(st.max_launches_in_flight, busy_slots());
        return true;
    }

    void run() {
        cudaSetDevice(device);
        for (;;) {
            bool stopping;
            {
                std::unique_lock<std::mutex> g(in_mu);
                if (incoming.empty() && pending.empty() && busy_slots() == 0 && !stop)
                    in_cv.wait_for(g, std::chrono::milliseconds(20));
                while (!incoming.empty()) {
                    pending.push_back(incoming.front());
                    incoming.pop_front();
                }
                cancelled.insert(cancel_in.begin(), cancel_in.end());
                cancel_in.clear();
                stopping = stop;
            }
            bool changed = poll();
            changed |= launch_wave();
            if (stopping && pending.empty() && busy_slots() == 0) break;
            if (!changed && busy_slots() > 0) std::this_thread::yield();
        }
    }
};

namespace {

int make_slots(rq_server* s) {
    for (uint32_t k = 0; k < s->cfg.slots; ++k) {
        Slot& sl = s->slots[k];
        cudaError_t e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_buf, kSlotBytes);
        if (e == cudaSuccess) e = cudaHostAlloc(&sl.h_buf, kDoneOff, cudaHostAllocDefault);
        if (e == cudaSuccess)
            e = cudaHostAlloc(reinterpret_cast<void**>(&sl.h_flags), sizeof(uint32_t) * RQ_SERVE_MAX_JOBS,
                              cudaHostAllocMapped);
        if (e == cudaSuccess) {
            std::memset(sl.h_flags, 0, sizeof(uint32_t) * RQ_SERVE_MAX_JOBS);
            e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&sl.d_flags), sl.h_flags, 0);
        }
        if (e != cudaSuccess) return rq_cuda_status(s->ctx, e, "serve slot setup");
    }
    return RQ_OK;
}

void free_server(rq_server* s) {
    for (uint32_t k = 0; k < kMaxSlots; ++k) {
        Slot& sl = s->slots[k];
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.d_buf) cudaFree(sl.d_buf);
        if (sl.h_buf) cudaFreeHost(sl.h_buf);
        if (sl.h_flags) cudaFreeHost(sl.h_flags);
    }
    for (auto& m : s->meshes) {
        if (m->bvh) rq_bvh_destroy(m->bvh);
        if (m->d_pos) cudaFree(m->d_pos);
        if (m->d_idx) cudaFree(m->d_idx);
        if (m->h_pos) cudaFreeHost(m->h_pos);
        if (m->h_idx) cudaFreeHost(m->h_idx);
    }
    if (s->build_ev) cudaEventDestroy(s->build_ev);
    if (s->build_st) cudaStreamDestroy(s->build_st);
    if (s->ctx) rq_ctx_destroy(s->ctx);
    delete s;
}

}  // namespace

extern "C" {

uint64_t rq_server_mesh_bytes(uint32_t num_vertices, uint32_t num_triangles) {
    return align256(12ull * num_vertices) + align256(12ull * num_triangles) +
           rq_bvh_alloc_bytes(num_triangles, 2 * num_triangles, std::max(1u, num_triangles));
}

int rq_server_create(int device, const rq_server_config* cfg, rq_server** out) {
    if (!cfg || !out) return RQ_ERR_INVALID_ARG;
    rq_server_config c = *cfg;
    if (c.mode > RQ_SERVE_PLAIN || c.max_leaf < 1 || c.max_leaf > 16 || (c.trace_flags & ~RQ_TRI_MT) ||
        c.rebuild > 1 || (c.rebuild && c.mode != RQ_SERVE_PLAIN))
        return RQ_ERR_INVALID_ARG;
    if (c.mode == RQ_SERVE_PLAIN) {
        c.slots = 1;
        c.max_wave_requests = 1;
    }
    if (c.slots < 1 || c.slots > kMaxSlots || c.max_wave_requests < 1 || c.max_wave_requests > RQ_SERVE_MAX_JOBS ||
        c.max_wave_rays < 1 || c.max_wave_rays > (1u << 30))
        return RQ_ERR_INVALID_ARG;
    rq_server* s = new (std::nothrow) rq_server();
    if (!s) return RQ_ERR_OOM;
    s->cfg = c;
    s->device = device;
    s->t0 = std::chrono::steady_clock::now();
    int rc = rq_ctx_create(device, &s->ctx);
    if (rc) {
        s->ctx = nullptr;
        free_server(s);
        return rc;
    }
    cudaSetDevice(device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->build_st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->build_ev, cudaEventDisableTiming);
    rc = e == cudaSuccess ? make_slots(s) : rq_cuda_status(s->ctx, e, "serve stream setup");
    if (rc) {
        free_server(s);
        return rc;
    }
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return RQ_OK;
}

int rq_server_destroy(rq_server* s) {
    if (!s) return RQ_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> g(s->in_mu);
        s->stop = true;
    }
    s->in_cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    free_server(s);
    return RQ_OK;
}

int rq_server_add_mesh(rq_server* s, const float* pos, uint32_t num_vertices, const uint32_t* idx,
                       uint32_t num_triangles, uint32_t* mesh_id) {
    if (!s || !pos || !idx || !mesh_id || num_vertices == 0 || num_triangles == 0) return RQ_ERR_INVALID_ARG;
    if (num_triangles >= RQ_MAX_TRIANGLES) return RQ_ERR_UNSUPPORTED;
    for (uint64_t k = 0; k < 3ull * num_triangles; ++k)
        if (idx[k] >= num_vertices) return RQ_ERR_INVALID_ARG;
    cudaSetDevice(s->device);
    auto m = std::make_unique<MeshRec>();
    m->nv = num_vertices;
    m->nt = num_triangles;
    m->bytes = rq_server_mesh_bytes(num_vertices, num_triangles);
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&m->h_pos), 12ull * num_vertices, cudaHostAllocDefault);
    if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void**>(&m->h_idx), 12ull * num_triangles, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (m->h_pos) cudaFreeHost(m->h_pos);
        return RQ_ERR_OOM;
    }
    std::memcpy(m->h_pos, pos, 12ull * num_vertices);
    std::memcpy(m->h_idx, idx, 12ull * num_triangles);
    uint32_t cur = s->max_mesh_tris.load();
    while (cur < num_triangles && !s->max_mesh_tris.compare_exchange_weak(cur, num_triangles)) {
    }
    std::lock_guard<std::mutex> g(s->mesh_mu);
    *mesh_id = uint32_t(s->meshes.size());
    s->meshes.push_back(std::move(m));
    return RQ_OK;
}

int rq_server_submit(rq_server* s, const rq_request* req, uint64_t* ticket) {
    if (!s || !req) return RQ_ERR_INVALID_ARG;
    const rq_request& r = *req;
    if (r.num_rays == 0 || r.num_rays > (1u << 30) || !r.hits || (reinterpret_cast<uintptr_t>(r.hits) & 15u) || r.kind > RQ_RAYS_CLOSEST)
        return RQ_ERR_INVALID_ARG;
    if (r.kind == RQ_RAYS_BUFFER && (!r.rays || (reinterpret_cast<uintptr_t>(r.rays) & 15u) || (r.flags & ~1u)))
        return RQ_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> g(s->mesh_mu);
        if (r.mesh >= s->meshes.size()) return RQ_ERR_INVALID_ARG;
    }
    uint64_t t;
    {
        std::lock_guard<std::mutex> g(s->in_mu);
        t = s->next_ticket++;
        s->incoming.push_back(Pending{r, t, s->now()});
    }
    {
        std::lock_guard<std::mutex> g(s->stats_mu);
        ++s->st.submitted;
    }
    s->in_cv.notify_one();
    if (ticket) *ticket = t;
    return RQ_OK;
}

int rq_server_replay(rq_server* s, const rq_request* reqs, const double* arrival, uint32_t n, uint64_t* tickets) {
    if (!s || (n && (!reqs || !arrival))) return RQ_ERR_INVALID_ARG;
    const double t0 = s->now();
    for (uint32_t i = 0; i < n; ++i) {
        const double target = t0 + arrival[i];
        for (;;) {
            const double left = target - s->now();
            if (left <= 0.0) break;
            if (left > 5e-4)
                std::this_thread::sleep_for(std::chrono::microseconds(200));
            else
                std::this_thread::yield();
        }
        int rc = rq_server_submit(s, reqs + i, tickets ? tickets + i : nullptr);
        if (rc) return rc;
    }
    return RQ_OK;
}

int rq_server_poll(rq_server* s, rq_completion* out, uint32_t capacity, uint32_t* count) {
    if (!s || !count || (capacity && !out)) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(s->out_mu);
    uint32_t k = 0;
    while (k < capacity && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *count = k;
    return RQ_OK;
}

int rq_server_drain(rq_server* s, uint32_t timeout_ms) {
    if (!s) return RQ_ERR_INVALID_ARG;
    const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
    for (;;) {
        {
            std::lock_guard<std::mutex> g(s->stats_mu);
            if (s->st.completed + s->st.failed >= s->st.submitted) return RQ_OK;
        }
        std::unique_lock<std::mutex> g(s->out_mu);
        if (s->out_cv.wait_until(g, std::min(until, std::chrono::steady_clock::now() + std::chrono::milliseconds(5))) ==
                std::cv_status::timeout &&
            std::chrono::steady_clock::now() >= until)
            return RQ_ERR_DEVICE_TIMEOUT;
    }
}

double rq_server_now(const rq_server* s) { return s ? s->now() : 0.0; }

int rq_server_stats_get(rq_server* s, rq_server_stats* out) {
    if (!s || !out) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(s->stats_mu);
    *out = s->st;
    return RQ_OK;
}

const char* rq_server_last_error(const rq_server* s) { return s ? s->last_error.c_str() : ""; }

int rq_server_cancel(rq_server* s, uint64_t ticket) {
    if (!s) return RQ_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> g(s->in_mu);
        if (ticket == 0 || ticket >= s->next_ticket) return RQ_ERR_INVALID_ARG;
        s->cancel_in.insert(ticket);
    }
    s->in_cv.notify_one();
    return RQ_OK;
}

int rq_server_inject_fault(rq_server* s, uint32_t kind, uint32_t count) {
    if (!s) return RQ_ERR_INVALID_ARG;
    if (kind == RQ_FAULT_ALLOC)
        s->fault_alloc += count;
    else if (kind == RQ_FAULT_LAUNCH)
        s->fault_launch += count;
    else
        return RQ_ERR_INVALID_ARG;
    return RQ_OK;
}

int rq_gen_mesh_rays(rq_ctx* ctx, const float* pos, const uint32_t* idx, uint32_t num_triangles, uint32_t kind,
                     uint32_t seed, uint32_t num_rays, rq_ray* rays, uint32_t* any_flags, rq_stream stream) {
    if (!ctx || (num_rays && !rays) || kind < RQ_RAYS_SHADOW || kind > RQ_RAYS_CLOSEST) return RQ_ERR_INVALID_ARG;
    if (kind != RQ_RAYS_CLOSEST && (!pos || !idx || num_triangles == 0)) return RQ_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(rays) & 15u) return RQ_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    return rq_launch_gen_mesh_rays(ctx, pos, idx, num_triangles, kind, seed, num_rays, rays, any_flags,
                                   static_cast<cudaStream_t>(stream));
}

}  // extern "C"
