// Batched path, host side: scene slots, pool ranges, staged upload, the CUDA
// graph of the persistent kernel, table growth with catch-up steps, and the
// avbd_batch_* entry points of include/avbd.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

#include "avbd_batch.h"
#include "avbd_pools.h"

using namespace avbd;
using namespace avbd::host;

namespace avbd {
namespace host {

// ===========================================================================
// Batched path: the persistent kernel builds live in their own translation
// units (avbd_batch_v.cu, compiled once per build); this table indexes them.
// ===========================================================================
struct BatchVariant {
    BatchKernel fn;
    int max_threads;
};
// Index = register variant of avbd_batch_set_kernel.
const BatchVariant kBatchVariants[] = {
    {nullptr, 0},
    {batch_kernel_v1(), 256}, {batch_kernel_v2(), 256}, {batch_kernel_v3(), 256},
    {batch_kernel_v4(), 256}, {batch_kernel_v5(), 512}, {batch_kernel_v6(), 512},
    {batch_kernel_v7(), 1024},
};
constexpr int kNumBatchVariants = 7;



void batch_drop_graph(AvbdBatch* b) {
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
}

int batch_stream(AvbdBatch* b) {
    int r = device_ready(b->device);
    if (r) return r;
    if (!b->stream) {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return AVBD_ERR_CUDA;
        cudaEventCreate(&b->e0);
        cudaEventCreate(&b->e1);
    }
    return 0;
}

// Allocates the pools with the given capacities (empty of scenes).
int batch_reserve(AvbdBatch* b, int64_t bodies, int64_t forces, int64_t tets, int64_t tris, int64_t nscenes,
                  int64_t nsinc, int64_t nsp) {
    int r = batch_stream(b);
    if (r) return r;
    const int64_t ncand = 16 * bodies + 64 * nscenes, nk = 8 * bodies + 128 * nscenes;
    const int64_t ninc = nsinc + 2 * ncand;
    const int64_t lim = 0x07FFFFFF;   // incidence entries index 27 bits
    if (bodies > lim || forces > lim || tets > lim || tris > lim || ncand > lim || nk > INT32_MAX || ninc > INT32_MAX ||
        nsinc > INT32_MAX || nscenes > (1 << 20))
        return AVBD_ERR_INVALID;
    Pools& P = b->P;
    P.release();
    P.ns = (int)nscenes; P.nb = (int)bodies; P.nf = (int)forces; P.nt = (int)tets; P.nr = (int)tris;
    P.ncand = (int)ncand; P.nk = (int)nk; P.nsinc = (int)nsinc; P.nsp = (int)nsp; P.ninc = (int)ninc;
    if (P.allocate_all() != cudaSuccess) {
        P.release();
        return AVBD_ERR_NOMEM;
    }
    P.W.P = to_params(b->params);
    b->A.reset(P);
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_nlive) cudaFree(b->d_nlive);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_fail) cudaFree(b->d_fail);
    if (b->d_fix_order) cudaFree(b->d_fix_order);
    if (b->d_fix_n) cudaFree(b->d_fix_n);
    if (b->d_scene_ns) {   // timing stays on, sized for the new slot count
        cudaFree(b->d_scene_ns);
        b->d_scene_ns = nullptr;
        const size_t n = (size_t)kSceneStamps * std::max<int64_t>(nscenes, 1);
        if (cudaMalloc(&b->d_scene_ns, n * sizeof(unsigned long long)) != cudaSuccess) return AVBD_ERR_NOMEM;
        cudaMemset(b->d_scene_ns, 0, n * sizeof(unsigned long long));
    }
    if (cudaMalloc(&b->d_order, std::max<int64_t>(nscenes, 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_nlive, 2 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_queue, 2 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_fail, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_fix_order, std::max<int64_t>(nscenes, 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_fix_n, 2 * sizeof(int)) != cudaSuccess)
        return AVBD_ERR_NOMEM;
    cudaMemset(b->d_fail, 0, sizeof(int));
    cudaMemset(b->d_nlive, 0, 2 * sizeof(int));
    b->reserved = true;
    b->order_dirty = true;
    batch_drop_graph(b);
    return 0;
}

// Takes pool ranges for the staged scene of `slot`; AVBD_ERR_NOMEM if the pools are full.
int batch_place(AvbdBatch* b, int slot) {
    if (slot >= b->P.ns) return AVBD_ERR_NOMEM;
    const HostScene& h = b->scenes[slot];
    int cc, kc, nsinc, nsp;
    scene_caps(h, cc, kc);
    static_counts(h, nsinc, nsp);
    Region reg;
    if (!place_scene(b->A, h, cc, kc, nsinc, nsp, reg)) return AVBD_ERR_NOMEM;
    b->regions[slot] = reg;
    return 0;
}

// Writes a placed scene through `sink` and marks it live.
template <typename Sink>
void batch_upload(AvbdBatch* b, int slot, Sink& sink) {
    const HostScene& h = b->scenes[slot];
    const Region& reg = b->regions[slot];
    upload_scene(b->P, h, static_incidence(h, reg), reg, scene_group(h, b->group_rigid, b->group_fem), slot,
                 b->descs[slot], sink);
}

// Places and uploads the staged scene of `slot` (live admission).
int batch_admit(AvbdBatch* b, int slot) {
    int r = batch_place(b, slot);
    if (r) return r;
    DirectSink sink{b->stream};
    batch_upload(b, slot, sink);
    b->state[slot] = 1;
    if ((int)b->steps_due.size() <= slot) b->steps_due.resize(slot + 1, 0);
    b->steps_due[slot] = 0;
    b->order_dirty = true;
    return 0;
}

// Uploads the live queue (largest scenes first) when it changed.
void batch_sync_order(AvbdBatch* b) {
    if (!b->order_dirty) return;
    std::vector<int> order;
    for (size_t i = 0; i < b->state.size(); ++i)
        if (b->state[i] == 1) order.push_back((int)i);
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return queue_key(b, b->descs[x]) > queue_key(b, b->descs[y]); });
    b->nlive = (int)order.size();
    const int counts[2] = {b->nlive, cluster_scenes(b, order)};
    if (!order.empty())
        cudaMemcpyAsync(b->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->d_nlive, counts, sizeof(counts), cudaMemcpyHostToDevice, b->stream);
    cudaStreamSynchronize(b->stream);
    b->order_dirty = false;
}

int cluster_scenes(const AvbdBatch* b, const std::vector<int>& order) {
    if (b->cluster < 2) return 0;
    int n = 0;
    for (int slot : order) {
        const SceneDesc& d = b->descs[slot];
        if (d.nbody + d.ntet < b->cluster_min) break;   // the order is by size, largest first
        ++n;
    }
    return n;
}

cudaError_t launch_batch_kernel(AvbdBatch* b, const World& W, const int* order, const int* nlive, int* queue) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(b->grid);
    cfg.blockDim = dim3(b->threads);
    cfg.dynamicSmemBytes = (size_t)b->stage * sizeof(float4);
    cfg.stream = b->stream;
    cudaLaunchAttribute attr[1];
    if (b->cluster > 1) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)b->cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    World w = W;
    void* args[] = {&w, &order, &nlive, &queue};
    return cudaLaunchKernelExC(&cfg, (const void*)kBatchVariants[b->variant].fn, args);
}

// First step without an explicit reservation: pools sized to the staged scenes.
// Reserves fresh pools for every staged scene, places them, and stages them
// into page-locked host buffers from all host threads (their ranges are
// disjoint); the copy waits for batch_flush.
int batch_stage(AvbdBatch* b, bool pin) {
    int64_t nb = 0, nf = 0, nt = 0, nr = 0, nsinc = 0, nsp = 0;
    for (size_t i = 0; i < b->scenes.size(); ++i) {
        if (b->state[i] != 2) continue;
        const HostScene& h = b->scenes[i];
        int a, c;
        static_counts(h, a, c);
        nb += h.nbody(); nf += h.nforce(); nt += h.ntet(); nr += h.ntri(); nsinc += a; nsp += c;
    }
    int r = batch_reserve(b, nb, nf, nt, nr, (int64_t)b->scenes.size(), nsinc, nsp);
    if (r) return r;
    std::vector<int> slots;
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (b->state[i] == 2) {
            if ((r = batch_place(b, (int)i))) return r;
            slots.push_back((int)i);
        }
    if (b->upload) b->upload->release();
    b->upload.reset(new StagedSink());
    StagedSink& staged = *b->upload;
    staged.st = b->stream;
    staged.P = &b->P;
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k = next++; k < slots.size(); k = next++) batch_upload(b, slots[k], staged);
    };
    const unsigned nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nthreads && slots.size() > 64; ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    if (staged.overflow) return AVBD_ERR_STATE;
    if (pin) staged.lock();
    b->upload_pinned = pin;
    for (int i : slots) {
        b->state[i] = 1;
        if ((int)b->steps_due.size() <= i) b->steps_due.resize(i + 1, 0);
        b->steps_due[i] = 0;
        b->scenes[i] = HostScene();   // the staged copy is what is uploaded
    }
    b->upload_pending = true;
    b->order_dirty = true;
    return cudaGetLastError() == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

// Copies the staged scenes into the pools (one copy per device array).
int batch_flush(AvbdBatch* b) {
    if (!b->upload_pending) return 0;
    b->upload_pending = false;
    if (!b->upload->flush()) return AVBD_ERR_STATE;
    b->uploaded_bytes = b->upload->copied;
    // pageable staging is not kept; page-locked staging (avbd_batch_prepare)
    // is held until the batch is destroyed, since unpinning it costs about as
    // much as the copy
    if (!b->upload_pinned) b->upload.reset();
    return cudaGetLastError() == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int batch_launch_shape(AvbdBatch* b) {
    const BatchVariant& kv = kBatchVariants[b->variant];
    int threads = b->threads > 0 ? std::min(b->threads, kv.max_threads) : kv.max_threads;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    int per_sm = 0;
    const int stage = std::max(256, kStagedBodies * threads / 256);
    const size_t smem = stage * sizeof(float4);
    cudaFuncSetAttribute(kv.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kv.fn, threads, smem);
    if (per_sm < 1) per_sm = 1;
    if (b->ctas_per_sm > 0) per_sm = std::min(per_sm, b->ctas_per_sm);
    b->threads = threads;
    b->stage = stage;
    b->ctas_per_sm = per_sm;
    b->grid = sms * per_sm;
    if (b->cluster > 1) {
        // as many whole clusters as can be resident at once; a cluster team has at most 1024 threads
        if (b->cluster * threads > 1024) b->cluster = std::max(1, 1024 / threads);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(b->grid);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)b->cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (b->cluster > 1 && cudaOccupancyMaxActiveClusters(&nclusters, kv.fn, &cfg) == cudaSuccess &&
            nclusters > 0) {
            b->grid = std::min(b->grid / b->cluster, nclusters) * b->cluster;
        } else {
            cudaGetLastError();
            b->cluster = 1;
        }
    }
    return 0;
}

int batch_build_graph(AvbdBatch* b);

// Shifts the contact bases and live-slot entries of a relocated manifold table.
__global__ void k_rebase_table(const __grid_constant__ World W, int t, int cand0, int nslot, int nlive, int dk, int dc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nslot; i += gridDim.x * blockDim.x) {
        W.kbase[t][cand0 + i] += dk;
        if (i < nlive) W.live[t][cand0 + i] += dc;
    }
}

// Extends a pool's free ranges after the pool grew from old_cap to new_cap.
void ranges_extend(Ranges& rg, int old_cap, int new_cap) {
    if (new_cap <= old_cap) return;
    rg.cap = new_cap;
    rg.release(old_cap, new_cap - old_cap);
}

template <typename T>
void copy_range(T* base, int to, int from, int n, cudaStream_t st) {
    if (n > 0) cudaMemcpyAsync(base + to, base + from, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st);
}

// Gives a scene stopped by a full candidate, contact or incidence table larger
// ranges (growing a pool when it has no room), moves its last completed
// manifold table and that table's contacts there, and clears the status so
// its step can run again.  The moved table is the one the next step warm
// starts from; the other table only held the interrupted attempt.
int batch_grow_scene(AvbdBatch* b, int slot, const SceneState& st) {
    Pools& P = b->P;
    Allocs& A = b->A;
    Region& r = b->regions[slot];
    SceneDesc& d = b->descs[slot];
    const int t = st.cur;
    const int nc = std::max(2 * r.ncand, st.need_cand + st.need_cand / 2 + 64);
    const int nk = std::max(2 * r.nk, st.need_k + st.need_k / 2 + 128);
    const int ni = r.nsinc + 2 * nc;
    int c0 = A.cand.alloc(nc), k0 = A.k.alloc(nk), i0 = A.inc.alloc(ni);
    if (c0 < 0 || k0 < 0 || i0 < 0) {
        if (c0 >= 0) A.cand.release(c0, nc);
        if (k0 >= 0) A.k.release(k0, nk);
        if (i0 >= 0) A.inc.release(i0, ni);
        // grow the pools, keeping every scene's contents
        cudaStreamSynchronize(b->stream);
        const int oc = P.ncand, ok = P.nk, oi = P.ninc;
        const int gc = std::max(oc + nc, oc + oc / 2), gk = std::max(ok + nk, ok + ok / 2);
        const int gi = std::max(oi + ni, oi + oi / 2);
        if (P.grow_tables(gc, gk, oc, oc, ok, ok) != cudaSuccess) return AVBD_ERR_NOMEM;
        if (P.grow(P.W.inc, (size_t)oi, (size_t)gi, (size_t)oi) != cudaSuccess) return AVBD_ERR_NOMEM;
        P.ninc = gi;
        ranges_extend(A.cand, oc, gc);
        ranges_extend(A.k, ok, gk);
        ranges_extend(A.inc, oi, gi);
        batch_drop_graph(b);   // the graph holds the old pool pointers
        c0 = A.cand.alloc(nc); k0 = A.k.alloc(nk); i0 = A.inc.alloc(ni);
        if (c0 < 0 || k0 < 0 || i0 < 0) return AVBD_ERR_NOMEM;
    }
    World& W = P.W;
    cudaStream_t s = b->stream;
    const int nslot = st.ncand[t], ncont = st.kused[t];
    copy_range(W.cpair[t], c0, r.cand0, nslot, s);
    copy_range(W.cn[t], c0, r.cand0, nslot, s);
    copy_range(W.cfric[t], c0, r.cand0, nslot, s);
    copy_range(W.kbase[t], c0, r.cand0, nslot, s);
    copy_range(W.cbirth[t], c0, r.cand0, nslot, s);
    copy_range(W.live[t], c0, r.cand0, nslot, s);
    copy_range(W.kid[t], k0, r.k0, ncont, s);
    copy_range(W.krA[t], k0, r.k0, ncont, s);
    copy_range(W.krB[t], k0, r.k0, ncont, s);
    copy_range(W.kn[t], k0, r.k0, ncont, s);
    copy_range(W.kt1[t], k0, r.k0, ncont, s);
    copy_range(W.kt2[t], k0, r.k0, ncont, s);
    copy_range(W.krAw[t], k0, r.k0, ncont, s);
    copy_range(W.krBw[t], k0, r.k0, ncont, s);
    copy_range(W.kpen[t], k0, r.k0, ncont, s);
    copy_range(W.klam[t], k0, r.k0, ncont, s);
    if (nslot > 0)
        k_rebase_table<<<blocks_for(nslot), kThreads, 0, s>>>(W, t, c0, nslot, st.nlive[t], k0 - r.k0, c0 - r.cand0);
    A.cand.release(r.cand0, r.ncand);
    A.k.release(r.k0, r.nk);
    A.inc.release(r.inc0, r.ninc);
    r.cand0 = c0; r.ncand = nc; r.k0 = k0; r.nk = nk; r.inc0 = i0; r.ninc = ni;
    d.cand0 = c0; d.candcap = nc; d.k0 = k0; d.kcap = nk; d.inc0 = i0; d.inccap = ni;
    SceneState fixed = st;
    fixed.status = kStatusOk;
    fixed.need_cand = fixed.need_k = fixed.need_inc = 0;
    cudaMemcpyAsync(P.d_scenes + slot, &d, sizeof(SceneDesc), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(P.d_sstate + slot, &fixed, sizeof(SceneState), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    return 0;
}

// Runs one step of the listed scenes only (same kernel build and launch shape).
int batch_step_listed(AvbdBatch* b, const std::vector<int>& slots) {
    const int n = (int)slots.size();
    cudaStream_t s = b->stream;
    cudaMemcpyAsync(b->d_fix_order, slots.data(), n * sizeof(int), cudaMemcpyHostToDevice, s);
    const int counts[2] = {n, 0};   // catch-up steps: no cluster phase
    cudaMemcpyAsync(b->d_fix_n, counts, sizeof(counts), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(int), s);
    World W = b->P.W;
    W.stage_bodies = b->stage;
    W.team_work = b->team_work;
    W.fem_team_work = b->fem_team_work;
    W.grid_min = b->grid_min;
    W.fail_count = b->d_fail;
    W.scene_ns = b->d_scene_ns;
    if (launch_batch_kernel(b, W, b->d_fix_order, b->d_fix_n, b->d_queue) != cudaSuccess) return AVBD_ERR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

// After a batched step: scenes a full table stopped get larger tables and
// take the steps they missed (a few rounds, in case one growth is not enough).
int batch_fix_capacity(AvbdBatch* b, int64_t* grown_count) {
    const int nslots = (int)b->state.size();
    std::vector<SceneState> hs(nslots);
    for (int round = 0; round < 4; ++round) {
        int fails = 0;
        cudaMemcpy(&fails, b->d_fail, sizeof(int), cudaMemcpyDeviceToHost);
        if (fails == 0) return 0;
        cudaMemset(b->d_fail, 0, sizeof(int));
        if (cudaMemcpy(hs.data(), b->P.d_sstate, nslots * sizeof(SceneState), cudaMemcpyDeviceToHost) != cudaSuccess)
            return AVBD_ERR_CUDA;
        std::vector<int> grown;
        for (int i = 0; i < nslots; ++i) {
            if (b->state[i] != 1 || hs[i].status != kStatusCapacity) continue;
            if (!(hs[i].need_cand || hs[i].need_k || hs[i].need_inc)) continue;   // colour slots: not growable
            if (batch_grow_scene(b, i, hs[i]) == 0) grown.push_back(i);
        }
        if (grown.empty()) return 0;
        if (grown_count) *grown_count += (int64_t)grown.size();
        if (!b->graph) batch_build_graph(b);
        // catch up: every grown scene takes the steps it missed
        for (;;) {
            std::vector<int> due;
            if (cudaMemcpy(hs.data(), b->P.d_sstate, nslots * sizeof(SceneState), cudaMemcpyDeviceToHost) !=
                cudaSuccess)
                return AVBD_ERR_CUDA;
            for (int i : grown)
                if (hs[i].status == kStatusOk && hs[i].step < b->steps_due[i]) due.push_back(i);
            if (due.empty()) break;
            int r = batch_step_listed(b, due);
            if (r) return r;
        }
    }
    return 0;
}

int batch_build_graph(AvbdBatch* b) {
    batch_drop_graph(b);
    cudaGraph_t g;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(int), b->stream);
    b->P.W.stage_bodies = b->stage;
    b->P.W.team_work = b->team_work;
    b->P.W.fem_team_work = b->fem_team_work;
    b->P.W.grid_min = b->grid_min;
    b->P.W.fail_count = b->d_fail;
    b->P.W.scene_ns = b->d_scene_ns;
    const cudaError_t launched = launch_batch_kernel(b, b->P.W, b->d_order, b->d_nlive, b->d_queue);
    if (cudaStreamEndCapture(b->stream, &g) != cudaSuccess || launched != cudaSuccess) return AVBD_ERR_CUDA;
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    return e == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}


// Scenes staged by avbd_batch_prepare reach the device with the first step;
// every entry point that reads device state or hands out pool space first
// completes that copy, so it never acts on unwritten memory and a later copy
// never overwrites a range given to another scene.
int batch_settle(AvbdBatch* b) {
    if (!b->upload_pending) return 0;
    if (cudaSetDevice(b->device) != cudaSuccess) return AVBD_ERR_CUDA;
    return batch_flush(b);
}

}  // namespace host
}  // namespace avbd

extern "C" {

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------
int32_t avbd_batch_create(const AvbdParams* params, int32_t device, AvbdBatch** out) {
    if (!out) return AVBD_ERR_INVALID;
    AvbdParams p;
    avbd_default_params(&p);
    if (params) {
        if (!valid_params(params)) return AVBD_ERR_INVALID;
        p = *params;
    }
    int r = device_ready(device);
    if (r) return r;
    AvbdBatch* b = new (std::nothrow) AvbdBatch();
    if (!b) return AVBD_ERR_NOMEM;
    b->params = p;
    b->device = device;
    *out = b;
    return 0;
}

int32_t avbd_batch_destroy(AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->copy_stream) {
        cudaStreamSynchronize(b->copy_stream);
        cudaStreamDestroy(b->copy_stream);
    }
    for (int k = 0; k < 2; ++k) {
        if (b->d_pose_snap[k]) cudaFree(b->d_pose_snap[k]);
        if (b->snap_ev[k]) cudaEventDestroy(b->snap_ev[k]);
        if (b->read_ev[k]) cudaEventDestroy(b->read_ev[k]);
    }
    batch_drop_graph(b);
    if (b->upload) b->upload->release();
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_nlive) cudaFree(b->d_nlive);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_fail) cudaFree(b->d_fail);
    if (b->d_fix_order) cudaFree(b->d_fix_order);
    if (b->d_fix_n) cudaFree(b->d_fix_n);
    if (b->d_scene_ns) cudaFree(b->d_scene_ns);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return 0;
}

int32_t avbd_batch_reserve(AvbdBatch* b, int64_t bodies, int64_t forces, int64_t tets, int64_t tris, int32_t scenes) {
    if (!b || bodies < 0 || forces < 0 || tets < 0 || tris < 0 || scenes < 1) return AVBD_ERR_INVALID;
    if (b->reserved) return AVBD_ERR_STATE;
    int r = batch_reserve(b, bodies, forces, tets, tris, scenes, 2 * forces + 4 * tets + 3 * tris, 2 * forces);
    if (r) return r;
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (b->state[i] == 2 && (r = batch_admit(b, (int)i))) return r;
    return 0;
}

int32_t avbd_batch_add_scene(AvbdBatch* b, const AvbdWorld* w) {
    if (!b || !w) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    int slot = -1;
    for (size_t i = 0; i < b->state.size(); ++i)
        if (b->state[i] == 0) { slot = (int)i; break; }
    if (slot < 0) {
        if (b->reserved && (int)b->state.size() >= b->P.ns) return AVBD_ERR_NOMEM;
        slot = (int)b->state.size();
        b->scenes.emplace_back();
        b->state.push_back(0);
        b->regions.emplace_back();
        b->descs.emplace_back();
        b->bodies.push_back(0);
        b->dynamic.push_back(0);
    }
    b->scenes[slot] = w->h;
    b->bodies[slot] = w->h.nbody();
    b->dynamic[slot] = w->h.ndynamic();
    b->state[slot] = 2;
    if (b->reserved) {
        cudaSetDevice(b->device);
        int r = batch_admit(b, slot);
        if (r) {   // no room in the pools: nothing was placed
            b->scenes[slot] = HostScene();
            b->state[slot] = 0;
            return r;
        }
        b->scenes[slot] = HostScene();   // the device holds it now
    }
    return slot;
}

int32_t avbd_batch_remove_scene(AvbdBatch* b, int32_t scene) {
    if (!b || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    if (b->state[scene] == 1) {
        b->A.release(b->regions[scene]);
        b->order_dirty = true;
    }
    b->state[scene] = 0;
    b->scenes[scene] = HostScene();
    b->bodies[scene] = 0;
    b->dynamic[scene] = 0;
    return 0;
}

int32_t avbd_batch_prepare(AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    if (b->reserved) return 0;
    int r = batch_stage(b, true);
    if (r) return r;
    cudaSetDevice(b->device);
    if (!b->grid) batch_launch_shape(b);
    return cudaGetLastError() == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int32_t avbd_batch_step(AvbdBatch* b, int32_t steps) {
    if (!b || steps < 0) return AVBD_ERR_INVALID;
    const Range range("avbd_batch_step");
    int r;
    if (!b->reserved && (r = batch_stage(b, false))) return r;
    cudaSetDevice(b->device);
    if ((r = batch_flush(b))) return r;
    batch_sync_order(b);
    if (!b->grid) batch_launch_shape(b);
    b->P.W.P = to_params(b->params);
    if (!b->graph && (r = batch_build_graph(b))) return r;
    cudaMemsetAsync(b->d_fail, 0, sizeof(int), b->stream);
    cudaEventRecord(b->e0, b->stream);
    for (int i = 0; i < steps; ++i)
        if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaEventRecord(b->e1, b->stream);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaEventElapsedTime(&b->last_ms, b->e0, b->e1);
    if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_CUDA;
    for (size_t i = 0; i < b->state.size() && i < b->steps_due.size(); ++i)
        if (b->state[i] == 1) b->steps_due[i] += steps;
    {
        const Range grow("grow and catch up");
        if ((r = batch_fix_capacity(b))) return r;
    }
    return AVBD_STATUS_OK;
}

int32_t avbd_batch_num_scenes(const AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    int n = 0;
    for (int s : b->state) n += s != 0;
    return n;
}

static bool live_slot(const AvbdBatch* b, int scene) {
    return b && scene >= 0 && scene < (int)b->state.size() && b->state[scene] == 1;
}

int32_t avbd_batch_scene_status(AvbdBatch* b, int32_t scene) {
    if (!b || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    if (b->state[scene] == 2) return AVBD_STATUS_OK;
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    SceneState st;
    if (cudaMemcpy(&st, b->P.d_sstate + scene, sizeof(SceneState), cudaMemcpyDeviceToHost) != cudaSuccess)
        return AVBD_ERR_CUDA;
    return st.status;
}

int32_t avbd_batch_scene_info(AvbdBatch* b, int32_t scene, int32_t out[6]) {
    if (!b || !out || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    if (b->state[scene] == 2) { for (int i = 0; i < 6; ++i) out[i] = 0; return 0; }
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    SceneState st;
    if (cudaMemcpy(&st, b->P.d_sstate + scene, sizeof(SceneState), cudaMemcpyDeviceToHost) != cudaSuccess)
        return AVBD_ERR_CUDA;
    out[0] = st.status; out[1] = st.ncolours; out[2] = st.ncand[st.cur]; out[3] = st.kused[st.cur];
    out[4] = st.ninc; out[5] = st.step;
    return 0;
}

int32_t avbd_batch_scene_bodies(const AvbdBatch* b, int32_t scene) {
    if (!b || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    return b->bodies[scene];
}

int64_t avbd_batch_dynamic_bodies(const AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    int64_t n = 0;
    for (size_t i = 0; i < b->state.size(); ++i)
        if (b->state[i] != 0) n += b->dynamic[i];
    return n;
}

int32_t avbd_batch_get_state(AvbdBatch* b, int32_t scene, float* pos, float* quat, float* vel, float* omega) {
    if (!live_slot(b, scene)) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    const int n = b->bodies[scene];
    cudaSetDevice(b->device);
    const int b0 = b->descs[scene].body0;
    std::vector<float4> buf(n);
    const World& W = b->P.W;
    auto fetch = [&](const float4* src, float* dst, bool q) {
        if (!dst || n == 0) return;
        cudaMemcpy(buf.data(), src + b0, n * sizeof(float4), cudaMemcpyDeviceToHost);
        for (int i = 0; i < n; ++i) {
            const float4 x = buf[i];
            if (q) { dst[4 * i] = x.w; dst[4 * i + 1] = x.x; dst[4 * i + 2] = x.y; dst[4 * i + 3] = x.z; }
            else { dst[3 * i] = x.x; dst[3 * i + 1] = x.y; dst[3 * i + 2] = x.z; }
        }
    };
    fetch(W.pos, pos, false);
    fetch(W.rot, quat, true);
    fetch(W.vel, vel, false);
    fetch(W.omega, omega, false);
    return n;
}

int32_t avbd_batch_get_all_poses(AvbdBatch* b, float* pos, float* quat, int64_t max_bodies) {
    if (!b || !b->reserved) return AVBD_ERR_STATE;
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    const int n = b->P.nb;
    if (n > max_bodies) return AVBD_ERR_INVALID;
    const World& W = b->P.W;
    if (pos && cudaMemcpyAsync(pos, W.pos, n * sizeof(float4), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (quat && cudaMemcpyAsync(quat, W.rot, n * sizeof(float4), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    return n;
}

// Pose readback overlapped with the next step: the poses are copied to a
// device snapshot on the batch stream (so the next step may change them at
// once) and from there to the caller's (page-locked) buffers on a copy
// stream.  Two snapshots alternate; a third read waits for the first's copy.
int32_t avbd_batch_read_poses(AvbdBatch* b, float* pos, float* quat, int64_t max_bodies) {
    if (!b || !b->reserved) return AVBD_ERR_STATE;
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    const int64_t n = b->P.nb;
    if (n > max_bodies) return AVBD_ERR_INVALID;
    if (!b->copy_stream) {
        if (cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking) != cudaSuccess) return AVBD_ERR_CUDA;
        for (int k = 0; k < 2; ++k)
            if (cudaEventCreateWithFlags(&b->snap_ev[k], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&b->read_ev[k], cudaEventDisableTiming) != cudaSuccess)
                return AVBD_ERR_CUDA;
    }
    if (b->pose_snap_n < n) {
        cudaStreamSynchronize(b->copy_stream);
        for (int k = 0; k < 2; ++k) {
            if (b->d_pose_snap[k]) cudaFree(b->d_pose_snap[k]);
            b->d_pose_snap[k] = nullptr;
            if (cudaMalloc(&b->d_pose_snap[k], 2 * (size_t)n * sizeof(float4)) != cudaSuccess) {
                b->pose_snap_n = 0;
                return AVBD_ERR_NOMEM;
            }
        }
        b->pose_snap_n = n;
    }
    const int k = b->pose_snap_cur;
    b->pose_snap_cur ^= 1;
    if (cudaEventSynchronize(b->read_ev[k]) != cudaSuccess) return AVBD_ERR_CUDA;   // this snapshot's last read
    const World& W = b->P.W;
    float4* snap = b->d_pose_snap[k];
    cudaMemcpyAsync(snap, W.pos, n * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(snap + n, W.rot, n * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream);
    cudaEventRecord(b->snap_ev[k], b->stream);
    cudaStreamWaitEvent(b->copy_stream, b->snap_ev[k], 0);
    if (pos) cudaMemcpyAsync(pos, snap, n * sizeof(float4), cudaMemcpyDeviceToHost, b->copy_stream);
    if (quat) cudaMemcpyAsync(quat, snap + n, n * sizeof(float4), cudaMemcpyDeviceToHost, b->copy_stream);
    if (cudaEventRecord(b->read_ev[k], b->copy_stream) != cudaSuccess) return AVBD_ERR_CUDA;
    return (int32_t)n;
}

int32_t avbd_host_alloc_pinned(int32_t device, int64_t bytes, void** out) {
    if (!out || bytes < 0) return AVBD_ERR_INVALID;
    *out = nullptr;
    if (int r = device_ready(device)) return r;
    if (cudaHostAlloc(out, std::max<int64_t>(bytes, 1), cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return AVBD_ERR_NOMEM;
    }
    return 0;
}

int32_t avbd_host_free_pinned(void* p) {
    if (!p) return AVBD_ERR_INVALID;
    return cudaFreeHost(p) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int32_t avbd_batch_read_poses_wait(AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    if (!b->copy_stream) return 0;
    cudaSetDevice(b->device);
    return cudaStreamSynchronize(b->copy_stream) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int32_t avbd_batch_export_instances(AvbdBatch* b, int32_t scene, AvbdInstance* dst, int32_t capacity,
                                    int32_t first_per_model[3], int32_t count_per_model[3]) {
    if (!live_slot(b, scene)) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    if (cudaSetDevice(b->device) != cudaSuccess) return AVBD_ERR_CUDA;
    return export_instances(b->P.W, b->descs[scene].body0, b->bodies[scene], dst, capacity, first_per_model,
                            count_per_model, b->stream);
}

int32_t avbd_batch_scene_body_offset(const AvbdBatch* b, int32_t scene) {
    if (!live_slot(b, scene)) return AVBD_ERR_INVALID;
    return b->descs[scene].body0;
}

// Device bytes per unit of each pool (allocate_all / alloc_tables).
constexpr int64_t kBytesPerBody = 16 * 16 + 18 * 4;        // float4 state + per-body ints
constexpr int64_t kBytesPerCand = 2 * (8 + 4 + 4 + 4 + 4 + 4);  // two manifold tables
constexpr int64_t kBytesPerContact = 2 * (4 + 9 * 16);      // two contact pools
constexpr int64_t kBytesPerForce = 4 + 8 + 6 * 16 + 6 * 6 * 4;
constexpr int64_t kBytesPerTet = 16 + 36 + 48 + 16 + 16 + 4;
constexpr int64_t kBytesPerTri = 16 + 16 + 24 + 16;

int64_t avbd_scene_footprint_bytes(const AvbdWorld* w) {
    if (!w) return AVBD_ERR_INVALID;
    int cc, kc, nsinc, nsp;
    scene_caps(w->h, cc, kc);
    static_counts(w->h, nsinc, nsp);
    int64_t bytes = (int64_t)w->h.nbody() * kBytesPerBody + (int64_t)w->h.nforce() * kBytesPerForce +
                    (int64_t)w->h.ntet() * kBytesPerTet + (int64_t)w->h.ntri() * kBytesPerTri;
    bytes += (int64_t)cc * kBytesPerCand + (int64_t)kc * kBytesPerContact;
    bytes += 4 * ((int64_t)nsinc + 2 * cc) + 4 * (int64_t)nsinc + 8 * (int64_t)nsp;
    bytes += sizeof(SceneDesc) + sizeof(SceneState) + 4 * (kMaxColours + 1);
    return bytes;
}

int64_t avbd_batch_uploaded_bytes(const AvbdBatch* b) { return b ? b->uploaded_bytes : AVBD_ERR_INVALID; }

int32_t avbd_batch_set_launch(AvbdBatch* b, int32_t threads, int32_t ctas_per_sm) {
    if (!b || threads < 0 || ctas_per_sm < 0 || (threads && (threads % 32 || threads > 1024))) return AVBD_ERR_INVALID;
    b->threads = threads;
    b->ctas_per_sm = ctas_per_sm;
    b->grid = 0;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_kernel(AvbdBatch* b, int32_t register_variant) {
    if (!b || register_variant < 1 || register_variant > kNumBatchVariants) return AVBD_ERR_INVALID;
    b->variant = register_variant;
    b->grid = 0;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_team_work(AvbdBatch* b, int32_t units_per_lane) {
    if (!b || units_per_lane < 0) return AVBD_ERR_INVALID;
    b->team_work = units_per_lane;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_fem_team_work(AvbdBatch* b, int32_t units_per_lane) {
    if (!b || units_per_lane < 0) return AVBD_ERR_INVALID;
    b->fem_team_work = units_per_lane;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_cluster(AvbdBatch* b, int32_t cluster_size, int32_t min_units) {
    if (!b || !(cluster_size == 1 || cluster_size == 2 || cluster_size == 4 || cluster_size == 8) || min_units < 0)
        return AVBD_ERR_INVALID;
    if (b->graph || b->grid) return AVBD_ERR_STATE;   // before the launch shape is fixed
    b->cluster = cluster_size;
    b->cluster_min = min_units;
    b->order_dirty = true;
    return 0;
}

int32_t avbd_batch_set_scene_timing(AvbdBatch* b, int32_t on) {
    if (!b) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (!on) {
        if (b->d_scene_ns) cudaFree(b->d_scene_ns);
        b->d_scene_ns = nullptr;
    } else if (!b->d_scene_ns) {
        const size_t n = (size_t)kSceneStamps * (std::max(b->P.ns, (int)b->state.size()) + 1);
        if (cudaMalloc(&b->d_scene_ns, n * sizeof(unsigned long long)) != cudaSuccess) return AVBD_ERR_NOMEM;
        cudaMemset(b->d_scene_ns, 0, n * sizeof(unsigned long long));
    }
    b->P.W.scene_ns = b->d_scene_ns;
    batch_drop_graph(b);
    return 0;
}

static_assert(kSceneStamps == AVBD_SCENE_STAMPS, "stamps per scene");

int32_t avbd_batch_check_word(AvbdBatch* b, int32_t out[4]) {
    if (!b || !out) return AVBD_ERR_INVALID;
#ifdef AVBD_CHECKS
    if (int r = batch_settle(b)) return r;
    for (int i = 0; i < 4; ++i) out[i] = 0;
    if (!b->P.W.check) return 1;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    return cudaMemcpy(out, b->P.W.check, 4 * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess ? 1 : AVBD_ERR_CUDA;
#else
    return 0;
#endif
}

int32_t avbd_batch_scene_times(AvbdBatch* b, int64_t* stamps_ns, int32_t max_slots) {
    if (!b || max_slots < 0) return AVBD_ERR_INVALID;
    if (!stamps_ns) return (int32_t)b->state.size();
    if (!b->d_scene_ns) return AVBD_ERR_STATE;
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    const int n = std::min(max_slots, (int)b->state.size());
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (n > 0 && cudaMemcpy(stamps_ns, b->d_scene_ns, (size_t)kSceneStamps * n * sizeof(int64_t),
                            cudaMemcpyDeviceToHost) != cudaSuccess)
        return AVBD_ERR_CUDA;
    return n;
}

int32_t avbd_batch_set_queue_weight(AvbdBatch* b, int32_t body_weight) {
    if (!b || body_weight < 1 || body_weight > 64) return AVBD_ERR_INVALID;
    b->queue_body_weight = body_weight;
    b->order_dirty = true;
    return 0;
}

int32_t avbd_batch_set_grid_broadphase(AvbdBatch* b, int32_t min_bodies) {
    if (!b || min_bodies < 0) return AVBD_ERR_INVALID;
    b->grid_min = min_bodies;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_get_launch(const AvbdBatch* b, int32_t* threads, int32_t* ctas_per_sm) {
    if (!b) return AVBD_ERR_INVALID;
    if (threads) *threads = b->threads;
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    return 0;
}

float avbd_batch_last_ms(const AvbdBatch* b) { return b ? b->last_ms : -1.f; }

static_assert(kGroupFlat == AVBD_GROUP_FLAT, "flat sweep selector");

int32_t avbd_batch_set_groups(AvbdBatch* b, int32_t rigid_group, int32_t fem_group) {
    if (!b || !valid_group(rigid_group) || !(valid_group(fem_group) || fem_group == kGroupFlat))
        return AVBD_ERR_INVALID;
    if (b->reserved) return AVBD_ERR_STATE;
    b->group_rigid = rigid_group;
    b->group_fem = fem_group;
    return 0;
}


}  // extern "C"
