// Continuous-batching server of scene-simulation requests (avbd_server_* in
// include/avbd.h).  No counterpart in the reference, whose caller steps one
// Solver per frame (GameManager.cpp:68-83).
//
// Every admitted scene stays resident in one AvbdBatch and all resident
// scenes advance one step per tick through the batch's CUDA graph (one
// persistent-kernel launch).  A tick is pipelined with the step in flight:
//
//   1. newcomers whose arrival time has passed are placed in the pools (first
//      fit, in arrival order; a scene that does not fit waits) and staged
//      into a page-locked arena, while the previous step still runs;
//   2. the host waits for that step, which also brought back the poses of
//      the scenes it finished (and of sampled scenes after their first step);
//      those scenes retire: their results are kept, their pool space is
//      freed for the next admissions;
//   3. the newcomers' copies, the live-scene order and the next step are
//      issued on the stream, followed by the readback of the scenes that step
//      will finish; the call returns while the GPU steps.
//
// A scene's arithmetic does not depend on what else is resident, so a served
// result is the one the scene gets alone (tested).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <new>
#include <vector>

#include "avbd_pools.h"

using namespace avbd;
using namespace avbd::host;

namespace {

struct ServedRequest {
    int id = -1;
    int slot = -1;
    int steps = 0;          // steps asked for
    int taken = 0;          // steps issued so far
    int flags = 0;          // AVBD_SERVE_KEEP_*
    int status = AVBD_STATUS_OK;
    int nbody = 0;
    int64_t dynamic = 0;
    double arrival = 0.0, admitted = -1.0, finished = -1.0;
    HostScene scene;        // the staged scene until it is admitted
    std::vector<float4> first_pos, first_rot, pos, rot;   // kept results (x y z / x y z w)
};

// One pose readback enqueued after a step: `n` float4 of pos and of rot into
// the readback arena at `off`, plus the scene's state word.
struct Readback {
    int req;
    bool final;             // the request's last step (else its first-step sample)
    size_t off;
    int n;
    int state_off;
};

}  // namespace

struct AvbdServer {
    AvbdBatch* b = nullptr;
    std::vector<ServedRequest> reqs;    // by request id
    std::deque<int> pending;            // request ids waiting for admission, arrival order
    std::vector<int> slot_req;          // request id of each batch slot (-1 free)
    std::vector<int> live;              // resident slots, largest scene first (ties by slot)
    // per slot, what a tick needs of its request (compact: the tick loop
    // touches every resident scene)
    struct SlotRun {
        int rid = -1, taken = 0, steps = 0, flags = 0, nbody = 0;
    };
    std::vector<SlotRun> run;
    int64_t live_weight = 1;            // queue weight the live order was made with
    std::vector<int> free_slots;        // retired slots, reused before new ones
    std::deque<int> finished;           // request ids ready for avbd_server_poll
    ArenaSink arena[2];                 // upload staging, alternating per tick
    int arena_cur = 0;
    char* d_stage = nullptr;            // device copy of the upload arena, scattered by k_scatter
    size_t d_stage_cap = 0;
    float4* rb = nullptr;               // page-locked readback arena
    std::vector<void*> free_after_step; // page-locked buffers replaced while a step was in flight
    size_t rb_cap = 0;
    SceneState* rb_state = nullptr;     // page-locked scene states of the readbacks
    int rb_state_cap = 0;
    std::vector<Readback> rb_list;      // readbacks of the step in flight
    int* order_host = nullptr;          // page-locked live-slot order
    int order_cap = 0;
    cudaEvent_t step_done = nullptr;
    cudaEvent_t step_begin = nullptr, step_end = nullptr;   // device time of each step
    bool in_flight = false;
    int64_t resident_dynamic = 0;
    int64_t pool_bodies = 0;            // pool capacity, reserved at the first tick
    int max_scenes = 0;
    AvbdServerStats stats{};
};

namespace {

// Replaces a page-locked buffer by a larger one.  The old one may still be
// the target of a readback in flight; it is freed after the next wait (a
// free of page-locked memory would wait for the device).
int grow_pinned(AvbdServer* s, void** p, size_t bytes) {
    if (*p) s->free_after_step.push_back(*p);
    *p = nullptr;
    if (cudaHostAlloc(p, bytes, cudaHostAllocDefault) != cudaSuccess) return AVBD_ERR_NOMEM;
    return 0;
}

// The upload arena's copies and memsets, one block per op: bytes from the
// device copy of the arena (or zeros) to their pool addresses.  Ops are
// whole 4-byte words (every pool element is 4, 8 or 16 bytes); 16-byte
// vectors where source, destination and length allow.
__global__ void k_scatter(const char* stage, const ArenaSink::ScatterOp* ops) {
    const ArenaSink::ScatterOp o = ops[blockIdx.x];
    const bool zero = (o.bytes >> 63) != 0;
    const size_t bytes = (size_t)(o.bytes & ~(1ull << 63));
    char* dst = reinterpret_cast<char*>(o.dst);
    const char* src = stage + o.src;
    const bool v16 = ((o.dst | (zero ? 0ull : reinterpret_cast<unsigned long long>(src)) | bytes) & 15ull) == 0;
    if (v16) {
        const size_t n = bytes / 16;
        float4* d = reinterpret_cast<float4*>(dst);
        const float4* s = reinterpret_cast<const float4*>(src);
        for (size_t i = threadIdx.x; i < n; i += blockDim.x) d[i] = zero ? make_float4(0.f, 0.f, 0.f, 0.f) : s[i];
    } else {
        const size_t n = bytes / 4;
        int* d = reinterpret_cast<int*>(dst);
        const int* s = reinterpret_cast<const int*>(src);
        for (size_t i = threadIdx.x; i < n; i += blockDim.x) d[i] = zero ? 0 : s[i];
    }
}

// Issues the arena on the stream as one copy plus one scatter launch.
int issue_arena(AvbdServer* s, ArenaSink& a, cudaStream_t st) {
    if (a.ops.empty()) return 0;
    const int64_t table = a.append_table();
    if (table < 0) return AVBD_ERR_NOMEM;
    if (a.used > s->d_stage_cap) {
        if (s->d_stage) cudaFree(s->d_stage);   // the previous scatter finished: the step after it was waited for
        s->d_stage = nullptr;
        const size_t cap = std::max(a.used, 2 * s->d_stage_cap);
        if (cudaMalloc(&s->d_stage, cap) != cudaSuccess) { s->d_stage_cap = 0; return AVBD_ERR_NOMEM; }
        s->d_stage_cap = cap;
    }
    cudaMemcpyAsync(s->d_stage, a.arena, a.used, a.pinned ? cudaMemcpyHostToDevice : cudaMemcpyDefault, st);
    k_scatter<<<(unsigned)a.ops.size(), 256, 0, st>>>(
        s->d_stage, reinterpret_cast<const ArenaSink::ScatterOp*>(s->d_stage + table));
    int64_t bytes = 0;
    for (const auto& o : a.ops) bytes += o.memset ? 0 : (int64_t)o.bytes;
    s->stats.uploaded_bytes += bytes;
    return cudaGetLastError() == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

// Order of the resident scenes in the queue: largest queue_key first, ties by slot.
bool live_before(const AvbdBatch* b, int x, int y) {
    const int64_t wa = queue_key(b, b->descs[x]), wc = queue_key(b, b->descs[y]);
    return wa != wc ? wa > wc : x < y;
}

// Places a newcomer in the pools and stages its upload; false if it does not fit.
bool server_admit(AvbdServer* s, int rid, double now) {
    AvbdBatch* b = s->b;
    ServedRequest& r = s->reqs[rid];
    if (s->free_slots.empty()) {
        // a new slot joins the free list (and stays there if the scene does not fit)
        if ((int)b->state.size() >= b->P.ns) return false;
        s->free_slots.push_back((int)b->state.size());
        b->scenes.emplace_back();
        b->state.push_back(0);
        b->regions.emplace_back();
        b->descs.emplace_back();
        b->bodies.push_back(0);
        b->dynamic.push_back(0);
        s->slot_req.push_back(-1);
    }
    const int slot = s->free_slots.back();
    const HostScene& h = r.scene;
    int cc, kc, nsinc, nsp;
    scene_caps(h, cc, kc);
    static_counts(h, nsinc, nsp);
    Region reg;
    if (!place_scene(b->A, h, cc, kc, nsinc, nsp, reg)) return false;
    s->free_slots.pop_back();
    b->regions[slot] = reg;
    upload_scene(b->P, h, static_incidence(h, reg), reg, scene_group(h, b->group_rigid, b->group_fem), slot,
                 b->descs[slot], s->arena[s->arena_cur]);
    b->state[slot] = 1;
    b->bodies[slot] = h.nbody();
    b->dynamic[slot] = h.ndynamic();
    if ((int)b->steps_due.size() <= slot) b->steps_due.resize(slot + 1, 0);
    b->steps_due[slot] = 0;
    b->order_dirty = true;
    s->slot_req[slot] = rid;
    if ((int)s->run.size() <= slot) s->run.resize(slot + 1);
    s->run[slot] = AvbdServer::SlotRun{rid, 0, r.steps, r.flags, r.nbody};
    {
        const auto pos = std::lower_bound(s->live.begin(), s->live.end(), slot,
                                          [&](int x, int y) { return live_before(b, x, y); });
        s->live.insert(pos, slot);
    }
    r.slot = slot;
    r.admitted = now;
    r.scene = HostScene();   // the device holds it now
    s->resident_dynamic += r.dynamic;
    s->stats.admitted += 1;
    return true;
}

// Completes the step in flight: waits for it, files the readbacks it
// brought, retires the scenes it finished.
int server_complete(AvbdServer* s, double now) {
    if (!s->in_flight) return 0;
    AvbdBatch* b = s->b;
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    if (cudaEventSynchronize(s->step_done) != cudaSuccess) return AVBD_ERR_CUDA;
    const auto t_wait = clock::now();
    s->stats.wait_us += std::chrono::duration_cast<std::chrono::microseconds>(t_wait - t0).count();
    for (void* p : s->free_after_step) cudaFreeHost(p);
    s->free_after_step.clear();
    s->in_flight = false;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s->step_begin, s->step_end) == cudaSuccess) s->stats.device_us += (int64_t)(ms * 1e3f);
    // scenes a full table stopped grow and catch up before anything reads them
    const auto t1 = clock::now();
    if (int r = batch_fix_capacity(b, &s->stats.regrown)) return r;
    s->stats.catchup_us += std::chrono::duration_cast<std::chrono::microseconds>(clock::now() - t1).count();
    bool refetch = false;
    for (const Readback& rb : s->rb_list)
        if (s->rb_state[rb.state_off].status == kStatusCapacity) refetch = true;
    if (refetch) {
        // a scene the catch-up re-ran: read its poses again now
        for (const Readback& rb : s->rb_list) {
            const ServedRequest& r = s->reqs[rb.req];
            const SceneDesc& d = b->descs[r.slot];
            cudaMemcpyAsync(s->rb + rb.off, b->P.W.pos + d.body0, rb.n * sizeof(float4), cudaMemcpyDeviceToHost,
                            b->stream);
            cudaMemcpyAsync(s->rb + rb.off + rb.n, b->P.W.rot + d.body0, rb.n * sizeof(float4),
                            cudaMemcpyDeviceToHost, b->stream);
            cudaMemcpyAsync(s->rb_state + rb.state_off, b->P.d_sstate + r.slot, sizeof(SceneState),
                            cudaMemcpyDeviceToHost, b->stream);
        }
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    }
    for (const Readback& rb : s->rb_list) {
        ServedRequest& r = s->reqs[rb.req];
        const float4* p = s->rb + rb.off;
        if (!rb.final) {
            r.first_pos.assign(p, p + rb.n);
            r.first_rot.assign(p + rb.n, p + 2 * rb.n);
            continue;
        }
        r.status = s->rb_state[rb.state_off].status;
        if (r.flags & AVBD_SERVE_KEEP_RESULT) {
            r.pos.assign(p, p + rb.n);
            r.rot.assign(p + rb.n, p + 2 * rb.n);
        }
        // retire: the slot and its pool ranges go back to the allocator
        b->A.release(b->regions[r.slot]);
        b->state[r.slot] = 0;
        b->bodies[r.slot] = 0;
        b->dynamic[r.slot] = 0;
        b->order_dirty = true;
        {
            const auto pos = std::lower_bound(s->live.begin(), s->live.end(), r.slot,
                                              [&](int x, int y) { return live_before(b, x, y); });
            if (pos != s->live.end() && *pos == r.slot) s->live.erase(pos);
        }
        s->free_slots.push_back(r.slot);
        s->slot_req[r.slot] = -1;
        s->resident_dynamic -= r.dynamic;
        r.finished = now;
        s->finished.push_back(r.id);
        s->stats.completed += 1;
    }
    s->rb_list.clear();
    s->stats.retire_us += std::chrono::duration_cast<std::chrono::microseconds>(clock::now() - t_wait).count();
    return 0;
}

// Issues the order list (page-locked copy) when the live set changed.
int server_sync_order(AvbdServer* s) {
    AvbdBatch* b = s->b;
    if (!b->order_dirty) return 0;
    const std::vector<int>& order = s->live;
    const int n = (int)order.size();
    if (n + 2 > s->order_cap) {
        const int cap = std::max(n + 2 + 1024, s->max_scenes + 2);
        if (grow_pinned(s, reinterpret_cast<void**>(&s->order_host), (size_t)cap * sizeof(int))) return AVBD_ERR_NOMEM;
        s->order_cap = cap;
    }
    std::copy(order.begin(), order.end(), s->order_host + 2);
    s->order_host[0] = n;
    s->order_host[1] = cluster_scenes(b, order);
    b->nlive = n;
    if (n) cudaMemcpyAsync(b->d_order, s->order_host + 2, n * sizeof(int), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->d_nlive, s->order_host, 2 * sizeof(int), cudaMemcpyHostToDevice, b->stream);
    b->order_dirty = false;
    return 0;
}

}  // namespace

extern "C" {

int32_t avbd_server_create(const AvbdParams* params, int32_t device, int64_t bodies, int32_t max_scenes,
                           AvbdServer** out) {
    if (!out || bodies < 1 || max_scenes < 1) return AVBD_ERR_INVALID;
    AvbdBatch* b = nullptr;
    int r = avbd_batch_create(params, device, &b);
    if (r) return r;
    AvbdServer* s = new (std::nothrow) AvbdServer();
    if (!s) {
        avbd_batch_destroy(b);
        return AVBD_ERR_NOMEM;
    }
    s->b = b;
    s->pool_bodies = bodies;
    s->max_scenes = max_scenes;
    if (cudaEventCreateWithFlags(&s->step_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&s->step_begin) != cudaSuccess || cudaEventCreate(&s->step_end) != cudaSuccess)
        r = AVBD_ERR_CUDA;
    if (r) {
        avbd_server_destroy(s);
        return r;
    }
    *out = s;
    return 0;
}

int32_t avbd_server_destroy(AvbdServer* s) {
    if (!s) return AVBD_ERR_INVALID;
    if (s->b) {
        cudaSetDevice(s->b->device);
        if (s->b->stream) cudaStreamSynchronize(s->b->stream);
    }
    if (s->step_done) cudaEventDestroy(s->step_done);
    if (s->step_begin) cudaEventDestroy(s->step_begin);
    if (s->step_end) cudaEventDestroy(s->step_end);
    for (void* p : s->free_after_step) cudaFreeHost(p);
    if (s->d_stage) cudaFree(s->d_stage);
    if (s->rb) cudaFreeHost(s->rb);
    if (s->rb_state) cudaFreeHost(s->rb_state);
    if (s->order_host) cudaFreeHost(s->order_host);
    s->arena[0].release();
    s->arena[1].release();
    if (s->b) avbd_batch_destroy(s->b);
    delete s;
    return 0;
}

AvbdBatch* avbd_server_batch(AvbdServer* s) { return s ? s->b : nullptr; }

int32_t avbd_server_submit(AvbdServer* s, const AvbdWorld* scene, int32_t steps, double arrival_s, int32_t flags) {
    if (!s || !scene || steps < 1) return AVBD_ERR_INVALID;
    ServedRequest r;
    r.id = (int)s->reqs.size();
    r.steps = steps;
    r.flags = flags;
    r.arrival = arrival_s;
    r.scene = scene->h;
    r.nbody = r.scene.nbody();
    r.dynamic = r.scene.ndynamic();
    s->reqs.push_back(std::move(r));
    // arrival order: requests are usually submitted in order; keep the queue sorted
    auto it = s->pending.end();
    while (it != s->pending.begin() && s->reqs[*(it - 1)].arrival > arrival_s) --it;
    s->pending.insert(it, s->reqs.back().id);
    s->stats.submitted += 1;
    return s->reqs.back().id;
}

int32_t avbd_server_tick(AvbdServer* s, double now_s) {
    if (!s) return AVBD_ERR_INVALID;
    const Range range("avbd_server_tick");
    {
        // a queue weight set since the live order was made: order again
        const int64_t w = s->b->cluster > 1 ? 1 : s->b->queue_body_weight;
        if (w != s->live_weight) {
            s->live_weight = w;
            AvbdBatch* b = s->b;
            std::sort(s->live.begin(), s->live.end(), [&](int x, int y) { return live_before(b, x, y); });
            b->order_dirty = true;
        }
    }
    AvbdBatch* b = s->b;
    if (cudaSetDevice(b->device) != cudaSuccess) return AVBD_ERR_CUDA;
    if (!b->reserved) {
        // pools: the body budget, a quarter as many forces and triangles, two tets per body
        const int64_t nb = s->pool_bodies;
        if (int r = avbd_batch_reserve(b, nb, nb / 4, 2 * nb, nb / 4, s->max_scenes)) return r;
    }
    if (!b->grid && batch_launch_shape(b)) return AVBD_ERR_CUDA;
    using clock = std::chrono::steady_clock;
    auto us_since = [](clock::time_point t) {
        return (int64_t)std::chrono::duration_cast<std::chrono::microseconds>(clock::now() - t).count();
    };
    const auto t_stage = clock::now();
    // 1. admissions staged while the previous step runs
    s->arena_cur ^= 1;
    ArenaSink& arena = s->arena[s->arena_cur];
    arena.clear();
    int admitted = 0;
    while (!s->pending.empty() && s->reqs[s->pending.front()].arrival <= now_s) {
        if (!server_admit(s, s->pending.front(), now_s)) break;   // no room: wait in arrival order
        s->pending.pop_front();
        ++admitted;
    }
    if (arena.overflow) return AVBD_ERR_NOMEM;
    s->stats.stage_us += us_since(t_stage);
    // 2. the step in flight and its readbacks
    if (int r = server_complete(s, now_s)) return r;
    const auto t_issue = clock::now();
    // 3. uploads, order, next step, readbacks of the scenes it finishes
    if (int r = issue_arena(s, arena, b->stream)) return r;
    if (int r = server_sync_order(s)) return r;
    if (b->nlive == 0) return 0;
    b->P.W.P = to_params(b->params);
    if (!b->graph && batch_build_graph(b)) return AVBD_ERR_CUDA;
    cudaMemsetAsync(b->d_fail, 0, sizeof(int), b->stream);
    cudaEventRecord(s->step_begin, b->stream);
    if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaEventRecord(s->step_end, b->stream);
    s->stats.ticks += 1;
    s->stats.body_iterations += s->resident_dynamic * b->params.num_iterations;
    size_t need = 0;
    int nstate = 0;
    for (const int slot : s->live) {
        AvbdServer::SlotRun& q = s->run[slot];
        q.taken += 1;
        b->steps_due[slot] += 1;
        const bool final = q.taken >= q.steps;
        const bool first = q.taken == 1 && (q.flags & AVBD_SERVE_KEEP_FIRST);
        if (final || first) {
            s->reqs[q.rid].taken = q.taken;
            s->rb_list.push_back({q.rid, final, need, q.nbody, nstate});
            need += 2 * (size_t)q.nbody;
            ++nstate;
            if (final && first) {   // a one-step request: the same poses serve both
                s->rb_list.push_back({q.rid, false, need - 2 * (size_t)q.nbody, q.nbody, nstate - 1});
            }
        }
    }
    if (need > s->rb_cap) {
        const size_t cap = std::max(need + need / 2, 2 * s->rb_cap);
        if (grow_pinned(s, reinterpret_cast<void**>(&s->rb), cap * sizeof(float4))) return AVBD_ERR_NOMEM;
        s->rb_cap = cap;
    }
    if (nstate > s->rb_state_cap) {
        const int cap = std::max(nstate + 256, 2 * s->rb_state_cap);
        if (grow_pinned(s, reinterpret_cast<void**>(&s->rb_state), (size_t)cap * sizeof(SceneState)))
            return AVBD_ERR_NOMEM;
        s->rb_state_cap = cap;
    }
    for (const Readback& rb : s->rb_list) {
        const ServedRequest& r = s->reqs[rb.req];
        const SceneDesc& d = b->descs[r.slot];
        if (!rb.final && r.taken >= r.steps) continue;   // shares the final readback
        cudaMemcpyAsync(s->rb + rb.off, b->P.W.pos + d.body0, rb.n * sizeof(float4), cudaMemcpyDeviceToHost,
                        b->stream);
        cudaMemcpyAsync(s->rb + rb.off + rb.n, b->P.W.rot + d.body0, rb.n * sizeof(float4), cudaMemcpyDeviceToHost,
                        b->stream);
        cudaMemcpyAsync(s->rb_state + rb.state_off, b->P.d_sstate + r.slot, sizeof(SceneState),
                        cudaMemcpyDeviceToHost, b->stream);
    }
    if (cudaEventRecord(s->step_done, b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    s->in_flight = true;
    s->stats.issue_us += us_since(t_issue);
    return b->nlive;
}

int32_t avbd_server_drain(AvbdServer* s, double now_s) {
    if (!s) return AVBD_ERR_INVALID;
    if (cudaSetDevice(s->b->device) != cudaSuccess) return AVBD_ERR_CUDA;
    return server_complete(s, now_s);
}

int32_t avbd_server_poll(AvbdServer* s, AvbdServedRequest* out) {
    if (!s || !out) return AVBD_ERR_INVALID;
    if (s->finished.empty()) return 0;
    const ServedRequest& r = s->reqs[s->finished.front()];
    s->finished.pop_front();
    out->request = r.id;
    out->status = r.status;
    out->steps = r.steps;
    out->bodies = r.nbody;
    out->arrival_s = r.arrival;
    out->admitted_s = r.admitted;
    out->finished_s = r.finished;
    return 1;
}

int32_t avbd_server_result(AvbdServer* s, int32_t request, float* pos, float* quat_wxyz, float* first_pos,
                           float* first_quat_wxyz) {
    if (!s || request < 0 || request >= (int)s->reqs.size()) return AVBD_ERR_INVALID;
    const ServedRequest& r = s->reqs[request];
    if (r.finished < 0.0) return AVBD_ERR_STATE;
    auto put = [](const std::vector<float4>& p, const std::vector<float4>& q, float* pd, float* qd) {
        for (size_t i = 0; i < p.size(); ++i) {
            if (pd) { pd[3 * i] = p[i].x; pd[3 * i + 1] = p[i].y; pd[3 * i + 2] = p[i].z; }
            if (qd) { qd[4 * i] = q[i].w; qd[4 * i + 1] = q[i].x; qd[4 * i + 2] = q[i].y; qd[4 * i + 3] = q[i].z; }
        }
    };
    if ((pos || quat_wxyz) && r.pos.empty()) return AVBD_ERR_STATE;
    if ((first_pos || first_quat_wxyz) && r.first_pos.empty()) return AVBD_ERR_STATE;
    put(r.pos, r.rot, pos, quat_wxyz);
    put(r.first_pos, r.first_rot, first_pos, first_quat_wxyz);
    return r.nbody;
}

int32_t avbd_server_release(AvbdServer* s, int32_t request) {
    if (!s || request < 0 || request >= (int)s->reqs.size()) return AVBD_ERR_INVALID;
    ServedRequest& r = s->reqs[request];
    std::vector<float4>().swap(r.pos);
    std::vector<float4>().swap(r.rot);
    std::vector<float4>().swap(r.first_pos);
    std::vector<float4>().swap(r.first_rot);
    return 0;
}

int32_t avbd_server_stats(const AvbdServer* s, AvbdServerStats* out) {
    if (!s || !out) return AVBD_ERR_INVALID;
    *out = s->stats;
    out->pending = (int64_t)s->pending.size();
    int64_t active = 0;
    for (int rid : s->slot_req) active += rid >= 0 ? 1 : 0;
    out->active = active;
    out->resident_dynamic = s->resident_dynamic;
    return 0;
}

}  // extern "C"
