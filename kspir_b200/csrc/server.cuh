// Serving loop: continuous batching of online answers on one context.
//
// Requests (client id, query) arrive from any host thread.  A worker thread
// owns `lanes` lanes; a lane is a range of lane_size workspace slots, a CUDA
// stream, pinned staging for queries and responses and a completion event.
// Whenever a lane is free and requests are waiting, the worker admits up to
// lane_size of them into one batch on that lane -- while the other lanes'
// batches are still running on the device -- so arrivals join the next batch
// as slots free up (continuous batching, not a queue in front of one launch).
//
// Client key-switching keys are held on the host by the caller and cached in
// the context's device key slots: a request is admitted only when its client's
// keys are resident or can be made resident, evicting the least recently used
// client that has no queued or running request.  The number of key slots the
// server may use follows from its HBM budget (key_budget_bytes / key slot
// size, at most the context's max_clients).  Keys are checked canonical and
// page-locked once, at registration; admission then copies the raw words
// asynchronously on the lane's stream into a per-lane staging buffer and a
// kernel converts them into the slot, so the copy overlaps the other lanes'
// batches; a per-slot event orders every later use of the slot after it.
//
// Each response equals kspir_answer on the same client and query: a batch
// runs the same kernels on disjoint workspace slots, and no kernel reads
// another slot.  Latency = host wall time from submit to the response being in
// the caller's buffer.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

struct kspir_server {
    struct Req {
        uint64_t ticket;
        int64_t client;
        const uint64_t* query;
        uint64_t* out;
        std::chrono::steady_clock::time_point t0;
        int state = 0;   // 0 waiting, 1 running, 2 done
        int rc = KSPIR_OK;
    };
    struct Lane {
        int slot0 = 0;
        cudaStream_t st = nullptr;
        cudaEvent_t done = nullptr;
        uint64_t* hq = nullptr;   // pinned [lane_size][4][N]
        uint64_t* hr = nullptr;   // pinned [lane_size][2][N]
        uint64_t* kstage = nullptr;   // device staging of one client's key words
        std::vector<Req*> reqs;
        bool busy = false;
    };
    struct Client {
        const uint64_t *baby = nullptr, *giant = nullptr, *packing = nullptr, *rgsw = nullptr;
        std::vector<const void*> pinned;   // caller ranges page-locked at registration
        int slot = -1;
        bool fresh = false;       // slot assigned, words not yet copied
        int active = 0;           // requests queued or running
        uint64_t last_use = 0;
    };

    kspir_ctx* c = nullptr;
    kspir_server_params p{};
    int key_slots = 0;
    std::vector<Lane> lanes;
    std::unordered_map<int64_t, Client> clients;
    std::vector<int64_t> slot_owner;   // key slot -> client id, -1 free
    std::vector<cudaEvent_t> slot_ready;   // recorded after each upload into the slot
    size_t kw_baby = 0, kw_giant = 0, kw_pack = 0, kw_rgsw = 0;   // raw key words per client
    std::deque<Req*> pending;
    std::unordered_map<uint64_t, Req*> reqs;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    uint64_t next_ticket = 1, use_clock = 0;
    std::string err;
    // statistics since the last reset
    std::vector<double> lat_us;
    long batches = 0, served = 0, key_uploads = 0, evictions = 0, batched_queries = 0;
    int max_running_lanes = 0;
    std::chrono::steady_clock::time_point t_stats;
};

namespace {

using Srv = kspir_server;

// a key slot for `id` (caller holds s.mu); false when every slot is held by a
// client with requests in flight.  A newly assigned slot is marked fresh: its
// words are copied by the batch that admitted the client (srv_upload).
bool srv_make_resident(Srv& s, int64_t id) {
    Srv::Client& cl = s.clients[id];
    if (cl.slot >= 0) return true;
    int slot = -1;
    for (int k = 0; k < s.key_slots; k++)
        if (s.slot_owner[k] < 0) { slot = k; break; }
    if (slot < 0) {
        uint64_t best = ~0ull;
        for (int k = 0; k < s.key_slots; k++) {
            const Srv::Client& o = s.clients[s.slot_owner[k]];
            if (o.active == 0 && o.last_use < best) { best = o.last_use; slot = k; }
        }
        if (slot < 0) return false;
        s.clients[s.slot_owner[slot]].slot = -1;
        s.evictions++;
    }
    s.slot_owner[slot] = id;
    cl.slot = slot;
    cl.fresh = true;
    s.key_uploads++;
    return true;
}

// enqueues the copy of a fresh client's key words into its slot on lane L
int srv_upload(Srv& s, Srv::Lane& L, Srv::Client& cl) {
    kspir_ctx* c = s.c;
    uint64_t* b = L.kstage;
    uint64_t* g = b + s.kw_baby;
    uint64_t* pk = g + s.kw_giant;
    uint64_t* rg = pk + s.kw_pack;
    if (cudaMemcpyAsync(b, cl.baby, s.kw_baby * 8, cudaMemcpyHostToDevice, L.st) != cudaSuccess) return KSPIR_ERR_CUDA;
    if (s.kw_giant && cudaMemcpyAsync(g, cl.giant, s.kw_giant * 8, cudaMemcpyHostToDevice, L.st) != cudaSuccess)
        return KSPIR_ERR_CUDA;
    if (s.kw_pack && cudaMemcpyAsync(pk, cl.packing, s.kw_pack * 8, cudaMemcpyHostToDevice, L.st) != cudaSuccess)
        return KSPIR_ERR_CUDA;
    if (cudaMemcpyAsync(rg, cl.rgsw, s.kw_rgsw * 8, cudaMemcpyHostToDevice, L.st) != cudaSuccess) return KSPIR_ERR_CUDA;
    const ClientKeysDev d = keys_host(c, cl.slot);
    const long polys = (long)(s.kw_baby + s.kw_giant + s.kw_pack + s.kw_rgsw) / kN;
    k_keys_from_words<<<blocks_for(polys * kN, 256), 256, 0, L.st>>>(
        b, g, pk, rg, const_cast<uint32_t*>(d.baby_crt), const_cast<uint32_t*>(d.baby_bs),
        const_cast<uint32_t*>(d.giant), const_cast<uint32_t*>(d.packing), const_cast<uint32_t*>(d.rgsw), c->N1h,
        (int)(s.kw_giant / kN), (int)(s.kw_pack / kN));
    if (cudaGetLastError() != cudaSuccess) return KSPIR_ERR_CUDA;
    if (cudaEventRecord(s.slot_ready[cl.slot], L.st) != cudaSuccess) return KSPIR_ERR_CUDA;
    cl.fresh = false;
    return KSPIR_OK;
}

void srv_finish_lane(Srv& s, Srv::Lane& L) {
    // error words of the lane's slots
    std::vector<int> e((size_t)L.reqs.size() * kErrStride);
    int rc = KSPIR_OK;
    if (cudaMemcpyAsync(e.data(), s.c->errs + (size_t)L.slot0 * kErrStride, e.size() * 4, cudaMemcpyDeviceToHost,
                        L.st) != cudaSuccess ||
        cudaStreamSynchronize(L.st) != cudaSuccess)
        rc = KSPIR_ERR_CUDA;
    for (size_t i = 0; i < L.reqs.size() && !rc; i++)
        if (e[i * kErrStride]) rc = KSPIR_ERR_TIMEOUT;
    if (rc == KSPIR_ERR_TIMEOUT) {
        cudaMemsetAsync(s.c->errs + (size_t)L.slot0 * kErrStride, 0, e.size() * 4, L.st);
        cudaStreamSynchronize(L.st);
    }
    const auto now = std::chrono::steady_clock::now();
    for (size_t i = 0; i < L.reqs.size(); i++) {
        Srv::Req* r = L.reqs[i];
        if (!rc) memcpy(r->out, L.hr + i * 2 * kN, 2 * kN * 8);
        r->rc = rc;
        r->state = 2;
        s.clients[r->client].active--;
        s.lat_us.push_back(std::chrono::duration<double, std::micro>(now - r->t0).count());
        s.served++;
    }
    L.reqs.clear();
    L.busy = false;
}

// launches one batch of up to lane_size waiting requests on lane L
void srv_launch(Srv& s, Srv::Lane& L) {
    std::vector<int> slots;
    std::deque<Srv::Req*> keep;
    while (!s.pending.empty() && (int)L.reqs.size() < s.p.lane_size) {
        Srv::Req* r = s.pending.front();
        s.pending.pop_front();
        if (!srv_make_resident(s, r->client)) {
            keep.push_back(r);   // no free key slot now: stays queued, in order
            continue;
        }
        Srv::Client& cl = s.clients[r->client];
        cl.last_use = ++s.use_clock;
        memcpy(L.hq + L.reqs.size() * 4 * kN, r->query, 4 * kN * 8);
        slots.push_back(cl.slot);
        r->state = 1;
        L.reqs.push_back(r);
    }
    while (!keep.empty()) { s.pending.push_front(keep.back()); keep.pop_back(); }
    if (L.reqs.empty()) return;
    const int n = (int)L.reqs.size();
    kspir_ctx* c = s.c;
    int rc = KSPIR_OK;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        // keys: copy the fresh ones on this lane, wait for the others' last upload
        for (Srv::Req* r : L.reqs) {
            Srv::Client& cl = s.clients[r->client];
            if (cl.fresh && !rc) rc = srv_upload(s, L, cl);
        }
        for (int k : slots)
            if (!rc && cudaStreamWaitEvent(L.st, s.slot_ready[k], 0) != cudaSuccess) rc = KSPIR_ERR_CUDA;
        if (!rc && cudaMemcpyAsync(c->bq64 + (size_t)L.slot0 * 4 * kN, L.hq, (size_t)n * 4 * kN * 8,
                                   cudaMemcpyHostToDevice, L.st) != cudaSuccess)
            rc = KSPIR_ERR_CUDA;
        // a lane whose slots include the single-answer slots is ordered
        // against direct kspir_answer / kspir_answer_device calls
        const bool shares = L.slot0 < c->single_slots;
        if (!rc && shares) rc = wait_singles(c, L.st);
        // a single query beside another lane's batch takes the scan ring
        // shape that leaves room for that batch's key-switch CTAs
        bool others = false;
        for (const auto& O : s.lanes) others = others || (&O != &L && O.busy);
        if (!rc) rc = enqueue_answer(c, L.slot0, n, slots.data(), L.st, false, others);
        if (!rc && cudaMemcpyAsync(L.hr, c->bresp + (size_t)L.slot0 * 2 * kN, (size_t)n * 2 * kN * 8,
                                   cudaMemcpyDeviceToHost, L.st) != cudaSuccess)
            rc = KSPIR_ERR_CUDA;
        if (!rc && shares) rc = mark_singles(c, L.st);
        if (!rc && cudaEventRecord(L.done, L.st) != cudaSuccess) rc = KSPIR_ERR_CUDA;
    }
    if (rc) {
        for (Srv::Req* r : L.reqs) {
            r->rc = rc;
            r->state = 2;
            Srv::Client& cl = s.clients[r->client];
            cl.active--;
            if (cl.slot >= 0) {   // the slot's contents are unknown after a failure
                s.slot_owner[cl.slot] = -1;
                cl.slot = -1;
            }
        }
        L.reqs.clear();
        s.cv_done.notify_all();
        return;
    }
    L.busy = true;
    s.batches++;
    s.batched_queries += n;
}

void srv_loop(Srv* sp) {
    Srv& s = *sp;
    cudaSetDevice(s.c->device);
    std::unique_lock<std::mutex> lk(s.mu);
    while (true) {
        bool progressed = false;
        int running = 0;
        for (auto& L : s.lanes) {
            if (L.busy && cudaEventQuery(L.done) != cudaErrorNotReady) {
                srv_finish_lane(s, L);
                progressed = true;
            }
        }
        if (progressed) s.cv_done.notify_all();
        for (auto& L : s.lanes) {
            if (!L.busy && !s.pending.empty()) {
                srv_launch(s, L);
                progressed = progressed || L.busy;
            }
            running += L.busy;
        }
        s.max_running_lanes = std::max(s.max_running_lanes, running);
        if (s.stop && s.pending.empty() && running == 0) break;
        if (!progressed) {
            if (running) s.cv_work.wait_for(lk, std::chrono::microseconds(20));
            else s.cv_work.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

double pct(std::vector<double> v, double q) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    const size_t i = std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5));
    return v[i];
}

}  // namespace

extern "C" {

size_t kspir_client_key_bytes(const kspir_ctx* c) { return c ? c->key_bytes : 0; }

int kspir_server_create(kspir_ctx* c, const kspir_server_params* params, kspir_server** out) {
    if (!c || !params || !out) return KSPIR_ERR_INVALID_ARG;
    kspir_server_params p = *params;
    if (p.lanes < 1 || p.lane_size < 1 || p.lane_size > kMaxBatch)
        return set_err(c, KSPIR_ERR_INVALID_ARG, "lanes and lane_size must be >= 1, lane_size <= 256");
    const int stride = c->mma ? (int)align_up((size_t)p.lane_size, 32) : p.lane_size;   // disjoint operand regions
    if ((long)stride * (p.lanes - 1) + p.lane_size > c->p.max_inflight)
        return set_err(c, KSPIR_ERR_INVALID_ARG, "lanes x lane_size exceed the context's workspaces");
    if (!c->db_loaded || !c->perms_loaded) return set_err(c, KSPIR_ERR_NOT_READY, "database or permutations missing");
    std::unique_ptr<kspir_server> s(new kspir_server());
    s->c = c;
    s->p = p;
    long budget_slots = p.key_budget_bytes > 0 ? (long)(p.key_budget_bytes / (long)c->key_bytes) : c->p.max_clients;
    s->key_slots = (int)std::min<long>(budget_slots, c->p.max_clients);
    if (s->key_slots < 1) return set_err(c, KSPIR_ERR_INVALID_ARG, "key budget below one client's keys");
    s->slot_owner.assign(s->key_slots, -1);
    s->kw_baby = (size_t)c->N1h * 6 * 2 * kN;
    s->kw_giant = (size_t)(c->N2 - 1) * 2 * 2 * kN;
    s->kw_pack = (size_t)c->levels * 4 * 2 * kN;
    s->kw_rgsw = (size_t)4 * 2 * kN;
    const size_t kwords = s->kw_baby + s->kw_giant + s->kw_pack + s->kw_rgsw;
    KS_CUDA(c, cudaSetDevice(c->device));
    s->slot_ready.assign(s->key_slots, nullptr);
    for (auto& e : s->slot_ready) KS_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    s->lanes.resize(p.lanes);
    for (int l = 0; l < p.lanes; l++) {
        auto& L = s->lanes[l];
        L.slot0 = l * stride;
        KS_CUDA(c, cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking));
        KS_CUDA(c, cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
        KS_CUDA(c, cudaMallocHost(&L.hq, (size_t)p.lane_size * 4 * kN * 8));
        KS_CUDA(c, cudaMallocHost(&L.hr, (size_t)p.lane_size * 2 * kN * 8));
        KS_CUDA(c, cudaMalloc(&L.kstage, kwords * 8));
    }
    s->t_stats = std::chrono::steady_clock::now();
    s->worker = std::thread(srv_loop, s.get());
    *out = s.release();
    return KSPIR_OK;
}

int kspir_server_destroy(kspir_server* s) {
    if (!s) return KSPIR_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->worker.join();
    cudaSetDevice(s->c->device);
    for (auto& L : s->lanes) {
        cudaStreamSynchronize(L.st);
        cudaStreamDestroy(L.st);
        cudaEventDestroy(L.done);
        cudaFreeHost(L.hq);
        cudaFreeHost(L.hr);
        cudaFree(L.kstage);
    }
    for (auto& e : s->slot_ready) cudaEventDestroy(e);
    for (auto& kv : s->clients)
        for (const void* ptr : kv.second.pinned) cudaHostUnregister(const_cast<void*>(ptr));
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
    return KSPIR_OK;
}

int kspir_server_register_client(kspir_server* s, int64_t client, const uint64_t* baby, const uint64_t* giant,
                                 const uint64_t* packing, const uint64_t* rgsw) {
    if (!s || !baby || !rgsw) return KSPIR_ERR_INVALID_ARG;
    kspir_ctx* c = s->c;
    if ((s->kw_giant && !giant) || (s->kw_pack && !packing)) return KSPIR_ERR_INVALID_ARG;
    // canonical words, checked once: rows 0-2 of each baby key mod crtMod, 3-5 mod bsMod
    for (size_t p = 0; p < s->kw_baby / kN; p++)
        if (!canonical(baby + p * kN, kN, ((p / 2) % 6) < 3 ? kCrtMod : (uint64_t)kBsMod))
            return set_err(c, KSPIR_ERR_INVALID_ARG, "key word not canonical");
    if ((giant && !canonical(giant, s->kw_giant, kCrtMod)) || (packing && !canonical(packing, s->kw_pack, kCrtMod)) ||
        !canonical(rgsw, s->kw_rgsw, kCrtMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "key word not canonical");
    std::lock_guard<std::mutex> lk(s->mu);
    Srv::Client& cl = s->clients[client];
    if (cl.active) return set_err(c, KSPIR_ERR_BUSY, "client has requests in flight");
    KS_CUDA(c, cudaSetDevice(c->device));
    for (const void* ptr : cl.pinned) cudaHostUnregister(const_cast<void*>(ptr));
    cl.pinned.clear();
    cl.baby = baby;
    cl.giant = giant;
    cl.packing = packing;
    cl.rgsw = rgsw;
    // page-lock the caller's words so admission copies are asynchronous; if
    // that is refused the copies still work, through pageable staging
    const std::pair<const uint64_t*, size_t> ranges[4] = {
        {baby, s->kw_baby}, {giant, s->kw_giant}, {packing, s->kw_pack}, {rgsw, s->kw_rgsw}};
    for (const auto& rg : ranges)
        if (rg.first && rg.second &&
            cudaHostRegister(const_cast<uint64_t*>(rg.first), rg.second * 8, cudaHostRegisterDefault) == cudaSuccess)
            cl.pinned.push_back(rg.first);
    cudaGetLastError();   // a refused registration leaves no error behind
    if (cl.slot >= 0) {   // new keys: drop the resident copy
        s->slot_owner[cl.slot] = -1;
        cl.slot = -1;
    }
    return KSPIR_OK;
}

int kspir_server_submit(kspir_server* s, int64_t client, const uint64_t* query, uint64_t* response,
                        uint64_t* ticket) {
    if (!s || !query || !response || !ticket) return KSPIR_ERR_INVALID_ARG;
    if (!canonical(query, 2 * kN, kCrtMod) || !canonical(query + 2 * kN, 2 * kN, kBsMod))
        return set_err(s->c, KSPIR_ERR_INVALID_ARG, "query word not canonical");
    Srv::Req* r = new Srv::Req();
    r->client = client;
    r->query = query;
    r->out = response;
    r->t0 = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->clients.find(client);
        if (it == s->clients.end() || !it->second.baby) {
            delete r;
            return set_err(s->c, KSPIR_ERR_NOT_READY, "client not registered");
        }
        it->second.active++;
        r->ticket = s->next_ticket++;
        s->reqs[r->ticket] = r;
        s->pending.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return KSPIR_OK;
}

// 1 = done (and released), 0 = not yet, < 0 = the request's error (released)
int kspir_server_poll(kspir_server* s, uint64_t ticket) {
    if (!s) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return KSPIR_ERR_INVALID_ARG;
    if (it->second->state != 2) return 0;
    const int rc = it->second->rc;
    delete it->second;
    s->reqs.erase(it);
    return rc ? rc : 1;
}

int kspir_server_wait(kspir_server* s, uint64_t ticket, int timeout_ms) {
    if (!s) return KSPIR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return KSPIR_ERR_INVALID_ARG;
    Srv::Req* r = it->second;
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->state == 2; })) return 0;
    const int rc = r->rc;
    delete r;
    s->reqs.erase(ticket);
    return rc ? rc : 1;
}

int kspir_server_get_stats(kspir_server* s, kspir_server_stats* out) {
    if (!s || !out) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t_stats).count();
    out->served = s->served;
    out->batches = s->batches;
    out->mean_batch = s->batches ? (double)s->batched_queries / s->batches : 0;
    out->p50_us = pct(s->lat_us, 0.50);
    out->p95_us = pct(s->lat_us, 0.95);
    out->p99_us = pct(s->lat_us, 0.99);
    out->max_us = pct(s->lat_us, 1.0);
    out->queries_per_s = secs > 0 ? s->served / secs : 0;
    out->key_uploads = s->key_uploads;
    out->evictions = s->evictions;
    out->key_slots = s->key_slots;
    out->max_running_lanes = s->max_running_lanes;
    return KSPIR_OK;
}

int kspir_server_latencies(kspir_server* s, double* out, size_t capacity, size_t* count) {
    if (!s || !count) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *count = s->lat_us.size();
    if (out) memcpy(out, s->lat_us.data(), std::min(capacity, s->lat_us.size()) * sizeof(double));
    return KSPIR_OK;
}

int kspir_server_reset_stats(kspir_server* s) {
    if (!s) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat_us.clear();
    s->batches = s->served = s->key_uploads = s->evictions = s->batched_queries = 0;
    s->max_running_lanes = 0;
    s->t_stats = std::chrono::steady_clock::now();
    return KSPIR_OK;
}

}  // extern "C"
