// batch.cu — census stereo (both directions + cross-check) for many pairs of
// mixed sizes and disparity ranges in one persistent, work-queue-scheduled
// matching launch, replayable as a CUDA graph.
//
// Per process call, on one stream:
//   1. a copy of the per-call pair table (caller image tensor maps, output
//      pointers) from pinned host memory, and a memset of the queue counter;
//   2. one census launch: every CTA is one 64 x 32 census tile of one image of
//      one pair (census_tile.cuh), found by a scan of per-pair prefix counts;
//   3. one persistent matching launch, one CTA per SM: each CTA takes work
//      items (pair, strip, column tile, disparity block) from a global atomic
//      counter, largest pairs first, and runs the fused census match tile
//      (census_match.cuh, left-to-right with the right view's winners bid
//      into the pair's right-view key plane) on the pair's pair-planar
//      descriptors. The last CTA of a (strip, column tile) group merges the
//      disparity blocks; the last group of a strip (all column tiles) runs
//      the cross-check of that strip into the caller's map from the left map
//      and the right-view keys, then resets the strip's keys. Counters reset
//      themselves, so nothing waits on anything.
// Results are bit-identical to processing each pair alone: every tile's
// arithmetic is the same and the winner-take-all keys are order-free.
#include "ct_internal.h"
#include "ct_device.cuh"
#include "census_match.cuh"
#include "census_tile.cuh"

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

namespace ct {
namespace batch {

constexpr int kMaxPairs = 256;

// Device-side description of one pair (fixed at configure, except the
// per-call fields at the end, rewritten by every process call).
struct PairDev {
    int W, H, D, th, tiles_x, strips, zc, tol;
    int census_tx, census_ty, census_item0;  // census tiles per image, prefix over census CTAs
    int match_item0, match_items;            // prefix over matching items
    uint64_t* desc[2];                       // pair-planar descriptors: left, right
    uint32_t* keys;                          // zc left-to-right key planes
    uint32_t* counters;                      // strips x tiles_x group counters
    uint32_t* strip_counter;                 // strips
    uint16_t* map;                           // U16 left-to-right disparity map
    size_t map_pitch;                        // bytes
    uint32_t* rl_keys;                       // right-view keys (tag 0), 0xFFFFFFFF between calls
    size_t rl_pitch;                         // words
    // per call
    void* out;
    size_t out_pitch;
    int out_type;
    int pad;
};

// Per-call tensor maps of the caller's images, 64-byte aligned in device memory.
struct alignas(64) CallMaps {
    CUtensorMap img[2];  // left, right
};

__device__ __forceinline__ void tmap_acquire(const CUtensorMap* m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(m))
                 : "memory");
}

__device__ __forceinline__ int find_pair(const PairDev* pairs, int n, int item, bool census) {
    int lo = 0, hi = n - 1;  // last pair whose first item <= item
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int first = census ? pairs[mid].census_item0 : pairs[mid].match_item0;
        if (first <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(census::kNT) census_batch_kernel(const PairDev* pairs, int n,
                                                                    const CallMaps* maps, int32_t* status) {
    __shared__ __align__(128) census::TileSmem sm;
    const int item = blockIdx.x;
    const int p = find_pair(pairs, n, item, true);
    const PairDev& P = pairs[p];
    const int local = item - P.census_item0;
    const int per_img = P.census_tx * P.census_ty;
    if (local < 0 || local >= 2 * per_img) {  // table inconsistent with the grid
        if (threadIdx.x == 0) dev::report(status, CT_EINTERNAL);
        return;
    }
    const int img = local / per_img, t = local % per_img;
    const CUtensorMap* tm = &maps[p].img[img];
    if (threadIdx.x == 0) tmap_acquire(tm);
    __syncthreads();
    census::census_tile(tm, P.W, P.H, (t % P.census_tx) * census::kTX, (t / P.census_tx) * census::kTY,
                        P.desc[img], 0, 1, status, sm);
}

// Cross-check of rows [y0, y1) of a pair from its U16 left map and the
// right-view keys into the caller's map (CrossCheckDisparityMaps.cu:63-110
// rule, left-to-right: the right view's code at x - d, as its map would hold
// it, within tol of the left code); then the rows' keys are reset.
__device__ void crosscheck_rows(const PairDev& P, int y0, int y1, int nt) {
    const int W = P.W;
    for (int idx = threadIdx.x; idx < (y1 - y0) * W; idx += nt) {
        const int y = y0 + idx / W, x = idx % W;
        const uint16_t v = __ldcg(reinterpret_cast<const uint16_t*>(
                                      reinterpret_cast<const char*>(P.map) + (size_t)y * P.map_pitch) + x);
        const bool disp = v >= CT_DISP_FIRST && v <= CT_DISP_LAST;
        bool keep = false;
        if (disp) {
            const int d = int(v) - 1, xo = x - d;
            if (xo >= 0 && xo < W) {
                const bool inside = y >= cm::kAR && y < P.H - cm::kAR && xo >= cm::kAR && xo < W - cm::kAR;
                const uint16_t vo = cm::rl_code<uint16_t>(__ldcg(P.rl_keys + (size_t)y * P.rl_pitch + xo), 0u, inside);
                keep = abs(int(vo) - int(v)) <= P.tol;  // raw codes, CrossCheckDisparityMaps.cu:94
            }
        }
        char* row = static_cast<char*>(P.out) + (size_t)y * P.out_pitch;
        if (P.out_type == CT_PIX_U8) {
            reinterpret_cast<uint8_t*>(row)[x] = keep ? uint8_t(v - 1) : uint8_t(0xFF);
        } else {
            reinterpret_cast<uint16_t*>(row)[x] = keep ? v : (disp ? uint16_t(CT_DISP_INCONSISTENT) : v);
        }
    }
    __syncthreads();  // every read of the rows' keys done
    for (int idx = threadIdx.x; idx < (y1 - y0) * W; idx += nt)
        P.rl_keys[(size_t)(y0 + idx / W) * P.rl_pitch + idx % W] = 0xFFFFFFFFu;
}

__global__ void __launch_bounds__(cm::Var<4>::kNT, 1)
    match_batch_kernel(const PairDev* pairs, int n, int total_items, const CUtensorMap* match_maps,
                       unsigned* queue, int32_t* status) {
    using namespace cm;
    constexpr int NT = Var<4>::kNT;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const Smem sm(smem_raw);
    __shared__ int s_item, s_last;
    init_barriers(sm);
    uint32_t par[2] = {0, 0};
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = int(atomicAdd(queue, 1u));
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total_items) break;
        const int p = find_pair(pairs, n, item, false);
        const PairDev& P = pairs[p];
        int local = item - P.match_item0;
        if (local < 0 || local >= P.match_items || P.match_items != P.strips * P.tiles_x * P.zc) {
            if (tid == 0) dev::report(status, CT_EINTERNAL);  // table inconsistent
            break;
        }
        // disparity blocks of one group are consecutive items, so the group's
        // CTAs run close together and the merging one finds its inputs in L2
        const Tile t{(local / P.zc) % P.tiles_x, local / (P.zc * P.tiles_x), local % P.zc, P.tiles_x, P.zc};
        MatchArgs a{};
        a.W = P.W; a.H = P.H; a.D = P.D; a.th = P.th;
        a.keys = P.keys;
        a.counters = P.counters;
        a.merge_last = 1;
        a.out = P.map; a.out_pitch = P.map_pitch; a.out_type = CT_PIX_U16;
        a.status = status;
        a.rl_keys = P.rl_keys;  // tag 0: the strip's cross-check resets the keys it read
        a.rl_pitch = P.rl_pitch;
        a.rl_tag = 0u;
        const CUtensorMap* tb = &match_maps[p * 2 + 0];
        const CUtensorMap* tm = &match_maps[p * 2 + 1];
        if (tid == 0) {  // maps written by a host copy: make them visible to the TMA unit
            tmap_acquire(tb);
            tmap_acquire(tm);
        }
        const TileResult res = run_tile<0, 4, false, true>(tb, tm, a, t, sm, par);
        if (res.aborted) break;  // status already set; the CTA stops taking work
        if (res.group_done) {
            // one more finished column tile group of this strip
            if (tid == 0) {
                __threadfence();
                unsigned* sc = reinterpret_cast<unsigned*>(&P.strip_counter[t.by]);
                const unsigned prev = atomicAdd(sc, 1u);
                s_last = prev == unsigned(P.tiles_x) - 1;
                if (s_last) *sc = 0u;
            }
            __syncthreads();
            if (s_last) {
                __threadfence();
                const int y0 = t.by * P.th;
                crosscheck_rows(P, y0, min(P.H, y0 + P.th), NT);
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
// Pinned host staging of one call's pair table and image tensor maps. The
// host rewrites a slot only after the copies that read it have run (event
// `copied`, recorded behind them): cuTensorMapEncodeTiled does not write a
// descriptor in one store, so a copy racing a rewrite could deliver a torn
// tensor map even when the new bytes equal the old ones.
struct Staging {
    PairDev* pairs = nullptr;
    CallMaps* maps = nullptr;
    cudaEvent_t copied = nullptr;
    bool pending = false;  // `copied` recorded and not yet waited for
    int wait() {
        if (pending) CT_CUDA_TRY(cudaEventSynchronize(copied));
        pending = false;
        return CT_OK;
    }
    int alloc(int n) {
        if (!copied) CT_CUDA_TRY(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
        release_host();
        CT_CUDA_TRY(cudaMallocHost(&pairs, sizeof(PairDev) * n));
        CT_CUDA_TRY(cudaMallocHost(&maps, sizeof(CallMaps) * n));
        return CT_OK;
    }
    void release_host() {
        wait();
        cudaFreeHost(pairs);
        cudaFreeHost(maps);
        pairs = nullptr;
        maps = nullptr;
    }
    void release() {
        release_host();
        if (copied) cudaEventDestroy(copied);
        copied = nullptr;
    }
};

// Staging slots used in turn by process calls, so the host fills call k + 1
// while the copies of call k are still queued behind earlier work.
constexpr int kSlots = 3;

struct BatchHandle : ct_handle {
    BatchHandle() : ct_handle(Kind::Batch) {}
    ~BatchHandle() override {
        if (device >= 0) cudaSetDevice(device);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        for (Staging& st : stage) st.release();
        graph_stage.release();
        cudaFree(arena);
    }
    int n = 0;
    int tol = 1;
    std::vector<ct_batch_shape> shapes;
    std::vector<PairDev> pairs;          // host copy (per-call fields filled per call)
    std::vector<int> order;              // pair index -> position in the device table
    int total_census = 0, total_match = 0;
    unsigned char* arena = nullptr;      // one device allocation for all scratch
    PairDev* d_pairs = nullptr;
    CallMaps* d_maps = nullptr;
    CUtensorMap* d_match_maps = nullptr;
    unsigned* d_queue = nullptr;
    Staging stage[kSlots];               // process calls
    int next_slot = 0;
    Staging graph_stage;                 // snapshot read by every graph launch; `copied`
                                         // is recorded behind each launch
    cudaGraphExec_t graph_exec = nullptr;
    int sms = 148;
};

int fill_call(BatchHandle* h, const ct_batch_item* items, int n, PairDev* pd, CallMaps* cm_) {
    if (n != h->n) return fail(CT_EFORMAT, "item count %d differs from the configured %d", n, h->n);
    for (int i = 0; i < n; ++i) {
        const ct_batch_item& it = items[i];
        const ct_batch_shape& s = h->shapes[i];
        if (int rc = check_image(&it.left, "left", 1u << CT_PIX_U8)) return rc;
        if (int rc = check_image(&it.right, "right", 1u << CT_PIX_U8)) return rc;
        if (int rc = check_image(&it.disp, "disp", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
        if (it.left.width != s.width || it.left.height != s.height || it.right.width != s.width ||
            it.right.height != s.height || it.disp.width != s.width || it.disp.height != s.height)
            return fail(CT_EFORMAT, "pair %d: image sizes differ from the configured shape", i);
        if (it.disp.type == CT_PIX_U8 && s.disp_count > 255)
            return fail(CT_ETYPE, "pair %d: U8 maps need disp_count <= 255", i);
        const int slot = h->order[i];
        PairDev& P = pd[slot];
        P = h->pairs[slot];
        P.out = it.disp.ptr;
        P.out_pitch = it.disp.pitch_bytes;
        P.out_type = it.disp.type;
        const ct_image* im[2] = {&it.left, &it.right};
        for (int k = 0; k < 2; ++k)
            if (int rc = make_tmap_2d(&cm_[slot].img[k], im[k]->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, s.width,
                                      s.height, im[k]->pitch_bytes, census::kBoxW, census::kBoxH))
                return rc;
    }
    return CT_OK;
}

// Enqueues one call: table copies from `st` (its event recorded behind them
// unless `record` is false, as inside a stream capture), queue reset, census
// launch, matching launch.
int enqueue(BatchHandle* h, Staging& st, bool record, cudaStream_t s) {
    CT_CUDA_TRY(cudaMemcpyAsync(h->d_pairs, st.pairs, sizeof(PairDev) * h->n, cudaMemcpyHostToDevice, s));
    CT_CUDA_TRY(cudaMemcpyAsync(h->d_maps, st.maps, sizeof(CallMaps) * h->n, cudaMemcpyHostToDevice, s));
    if (record) {
        CT_CUDA_TRY(cudaEventRecord(st.copied, s));
        st.pending = true;
    }
    CT_CUDA_TRY(cudaMemsetAsync(h->d_queue, 0, sizeof(unsigned), s));
    census_batch_kernel<<<h->total_census, census::kNT, 0, s>>>(h->d_pairs, h->n, h->d_maps, h->d_status);
    CT_LAUNCH_CHECK();
    match_batch_kernel<<<h->sms, cm::Var<4>::kNT, cm::smem_bytes_rl(), s>>>(h->d_pairs, h->n, h->total_match,
                                                                        h->d_match_maps, h->d_queue, h->d_status);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

// Lays out the table (largest pairs first), item prefixes and scratch for the
// current shapes and strip heights; (re)creates the fixed tensor maps.
int layout(BatchHandle* h, const std::vector<int>& th) {
    const int n = h->n;
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    auto cost = [&](int i) {
        const ct_batch_shape& s = h->shapes[i];
        return double(s.width) * s.height * ((s.disp_count + cm::kDPC - 1) / cm::kDPC);
    };
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost(a) > cost(b); });
    h->order.assign(n, 0);
    for (int k = 0; k < n; ++k) h->order[idx[k]] = k;
    // sizes
    size_t bytes = 0;
    auto take = [&](size_t b) { const size_t o = bytes; bytes += (b + 255) / 256 * 256; return o; };
    struct Off { size_t desc[2], keys, cnt, strip, map, rl; };
    std::vector<Off> off(n);
    h->pairs.assign(n, PairDev{});
    int census0 = 0, match0 = 0;
    for (int k = 0; k < n; ++k) {
        const int i = idx[k];
        const ct_batch_shape& s = h->shapes[i];
        PairDev& P = h->pairs[k];
        P.W = s.width; P.H = s.height; P.D = s.disp_count; P.th = th[i];
        P.tiles_x = (P.W + cm::kTWO - 1) / cm::kTWO;
        P.strips = (P.H + P.th - 1) / P.th;
        P.zc = (P.D + cm::kDPC - 1) / cm::kDPC;
        P.tol = h->tol;
        P.census_tx = (P.W + census::kTX - 1) / census::kTX;
        P.census_ty = (P.H + census::kTY - 1) / census::kTY;
        P.census_item0 = census0;
        census0 += 2 * P.census_tx * P.census_ty;
        P.match_item0 = match0;
        P.match_items = P.strips * P.tiles_x * P.zc;
        match0 += P.match_items;
        P.map_pitch = ((size_t)P.W * 2 + 255) / 256 * 256;
        Off& o = off[k];
        for (int v = 0; v < 2; ++v) o.desc[v] = take(cm::planar_pitch(P.W) * P.H * 8);
        o.keys = take((size_t)P.zc * P.W * P.H * 4);
        o.cnt = take((size_t)P.strips * P.tiles_x * 4);
        o.map = take(P.map_pitch * P.H);
        P.rl_pitch = cm::rl_pitch_words(P.W);
        o.rl = take(P.rl_pitch * P.H * 4);
        o.strip = take((size_t)P.strips * 4);
    }
    const size_t o_pairs = take(sizeof(PairDev) * n), o_maps = take(sizeof(CallMaps) * n);
    const size_t o_mmaps = take(sizeof(CUtensorMap) * 2 * n), o_queue = take(256);
    cudaFree(h->arena);
    h->arena = nullptr;
    if (cudaMalloc(&h->arena, bytes) != cudaSuccess) return fail(CT_ENOMEM, "batch scratch (%zu bytes)", bytes);
    CT_CUDA_TRY(cudaMemset(h->arena, 0, bytes));  // counters start at 0
    unsigned char* A = h->arena;
    for (int k = 0; k < n; ++k) {
        PairDev& P = h->pairs[k];
        for (int v = 0; v < 2; ++v) P.desc[v] = reinterpret_cast<uint64_t*>(A + off[k].desc[v]);
        P.keys = reinterpret_cast<uint32_t*>(A + off[k].keys);
        P.counters = reinterpret_cast<uint32_t*>(A + off[k].cnt);
        P.map = reinterpret_cast<uint16_t*>(A + off[k].map);
        P.rl_keys = reinterpret_cast<uint32_t*>(A + off[k].rl);
        CT_CUDA_TRY(cudaMemset(P.rl_keys, 0xFF, P.rl_pitch * P.H * 4));
        P.strip_counter = reinterpret_cast<uint32_t*>(A + off[k].strip);
    }
    h->d_pairs = reinterpret_cast<PairDev*>(A + o_pairs);
    h->d_maps = reinterpret_cast<CallMaps*>(A + o_maps);
    h->d_match_maps = reinterpret_cast<CUtensorMap*>(A + o_mmaps);
    h->d_queue = reinterpret_cast<unsigned*>(A + o_queue);
    h->total_census = census0;
    h->total_match = match0;
    std::vector<CUtensorMap> mm(2 * n);  // left as base, right as match
    for (int k = 0; k < n; ++k) {
        const PairDev& P = h->pairs[k];
        if (int rc = cm::make_planar_maps(&mm[2 * k + 0], &mm[2 * k + 1], P.desc[0], P.desc[1], P.W, P.H)) return rc;
    }
    CT_CUDA_TRY(cudaMemcpy(h->d_match_maps, mm.data(), sizeof(CUtensorMap) * 2 * n, cudaMemcpyHostToDevice));
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    return CT_OK;
}

BatchHandle* as_batch(ct_handle* h) { return (h && h->kind == Kind::Batch) ? static_cast<BatchHandle*>(h) : nullptr; }

}  // namespace batch
}  // namespace ct

using namespace ct;
using namespace ct::batch;

extern "C" {

int ct_batch_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new BatchHandle();
    return CT_OK;
}

int ct_batch_configure(ct_handle* hh, int32_t device, const ct_batch_shape* shapes, int32_t n, int32_t tol) {
    clear_error();
    auto* h = as_batch(hh);
    if (!h) return fail(CT_ESTATE, "not a batch handle");
    if (!shapes || n < 1 || n > kMaxPairs) return fail(CT_EINVAL, "need 1..%d pair shapes", kMaxPairs);
    if (tol < 0) return fail(CT_EINVAL, "tol must be >= 0");
    for (int i = 0; i < n; ++i) {
        const ct_batch_shape& s = shapes[i];
        if (s.width < 8 || s.height < 8 || s.width > 32768 || s.height > 32768)
            return fail(CT_EINVAL, "pair %d: size %dx%d out of range", i, s.width, s.height);
        if (s.disp_count < 1 || s.disp_count > 256) return fail(CT_EINVAL, "pair %d: disp_count must be 1..256", i);
    }
    if (int rc = use_device(device)) return rc;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    CT_CUDA_TRY(cm::prepare_census_match());
    CT_CUDA_TRY(cudaFuncSetAttribute(match_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(cm::smem_bytes_rl())));
    h->sms = sm_count(device);
    h->n = n;
    h->tol = tol;
    h->shapes.assign(shapes, shapes + n);
    std::vector<int> th(n);
    for (int i = 0; i < n; ++i)
        th[i] = cm::pick_strip_height(shapes[i].width, shapes[i].height, shapes[i].disp_count, h->sms);
    if (int rc = layout(h, th)) return rc;
    for (Staging& st : h->stage)
        if (int rc = st.alloc(n)) return rc;
    h->configured = true;
    return CT_OK;
}

int ct_batch_process(ct_handle* hh, const ct_batch_item* items, int32_t n, ct_stream stream) {
    clear_error();
    auto* h = as_batch(hh);
    if (!h) return fail(CT_ESTATE, "not a batch handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (!items) return fail(CT_EINVAL, "null items");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    Staging& st = h->stage[h->next_slot];
    if (int rc = st.wait()) return rc;  // the slot may still feed a copy of an earlier call
    if (int rc = fill_call(h, items, n, st.pairs, st.maps)) return rc;
    h->next_slot = (h->next_slot + 1) % kSlots;
    return enqueue(h, st, true, s);
}

int ct_batch_autotune(ct_handle* hh, const ct_batch_item* items, int32_t n, ct_stream stream) {
    clear_error();
    auto* h = as_batch(hh);
    if (!h) return fail(CT_ESTATE, "not a batch handle");
    if (!h->configured) return fail(CT_ESTATE, "autotune before configure");
    if (!items) return fail(CT_EINVAL, "null items");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // current strip heights by original pair index
    std::vector<int> th(h->n);
    for (int i = 0; i < h->n; ++i) th[i] = h->pairs[h->order[i]].th;
    // distinct (W, H, D) shapes
    std::map<std::tuple<int, int, int>, std::vector<int>> groups;
    for (int i = 0; i < h->n; ++i)
        groups[{h->shapes[i].width, h->shapes[i].height, h->shapes[i].disp_count}].push_back(i);
    cudaEvent_t e0, e1;
    CT_CUDA_TRY(cudaEventCreate(&e0));
    CT_CUDA_TRY(cudaEventCreate(&e1));
    auto time_batch = [&](float* ms_out) -> int {
        float best = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            if (int rc = ct_batch_process(hh, items, n, stream)) return rc;
            cudaEventRecord(e0, s);
            if (int rc = ct_batch_process(hh, items, n, stream)) return rc;
            cudaEventRecord(e1, s);
            const cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) return fail(CT_ECUDA, "autotune timing failed: %s", cudaGetErrorString(e));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            best = std::min(best, ms);
        }
        *ms_out = best;
        return CT_OK;
    };
    int rc = CT_OK;
    float cur = 0.f;
    if ((rc = time_batch(&cur))) goto done;
    // one pass of coordinate descent over the shapes' strip heights
    for (auto& g : groups) {
        const int base = th[g.second[0]];
        int best_th = base;
        for (int cand : {base / 2 - (base / 2 + 4) % 10, base - 40, base + 40, 26, 66}) {
            if (cand < 16 || cand > 506 || cand == best_th || (cand + 4) % 5 != 0) continue;
            for (int i : g.second) th[i] = cand;
            if ((rc = layout(h, th))) goto done;
            float t = 0.f;
            if ((rc = time_batch(&t))) goto done;
            if (t < cur) { cur = t; best_th = cand; }
        }
        for (int i : g.second) th[i] = best_th;
        if ((rc = layout(h, th))) goto done;
    }
done:
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int ct_batch_strip_height(ct_handle* hh, int32_t pair, int32_t* strip_height) {
    clear_error();
    auto* h = as_batch(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured batch handle");
    if (pair < 0 || pair >= h->n || !strip_height) return fail(CT_EINVAL, "bad pair index");
    *strip_height = h->pairs[h->order[pair]].th;
    return CT_OK;
}

int ct_batch_graph_create(ct_handle* hh, const ct_batch_item* items, int32_t n) {
    clear_error();
    auto* h = as_batch(hh);
    if (!h) return fail(CT_ESTATE, "not a batch handle");
    if (!h->configured) return fail(CT_ESTATE, "graph before configure");
    if (!items) return fail(CT_EINVAL, "null items");
    if (int rc = use_device(h->device)) return rc;
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    if (!h->graph_stage.pairs) {
        if (int rc = h->graph_stage.alloc(kMaxPairs)) return rc;
    }
    if (int rc = h->graph_stage.wait()) return rc;  // earlier launches read the snapshot
    if (int rc = fill_call(h, items, n, h->graph_stage.pairs, h->graph_stage.maps)) return rc;
    cudaStream_t cs;
    CT_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    int rc = CT_OK;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = fail(CT_ECUDA, "stream capture failed to begin");
    } else {
        rc = enqueue(h, h->graph_stage, false, cs);
        const cudaError_t e = cudaStreamEndCapture(cs, &g);
        if (!rc && e != cudaSuccess) rc = fail(CT_ECUDA, "stream capture failed: %s", cudaGetErrorString(e));
    }
    if (!rc && cudaGraphInstantiate(&h->graph_exec, g, 0) != cudaSuccess) rc = fail(CT_ECUDA, "graph instantiate failed");
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    return rc;
}

int ct_batch_graph_launch(ct_handle* hh, ct_stream stream) {
    clear_error();
    auto* h = as_batch(hh);
    if (!h || !h->graph_exec) return fail(CT_ESTATE, "no graph: call ct_batch_graph_create first");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    CT_CUDA_TRY(cudaGraphLaunch(h->graph_exec, s));
    CT_CUDA_TRY(cudaEventRecord(h->graph_stage.copied, s));
    h->graph_stage.pending = true;
    return CT_OK;
}

}  // extern "C"
