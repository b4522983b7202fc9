// weftk_pipeline.cu — the refined fit of a whole image as one native call
// (include/weftk_pipeline.h): the host side of the per-image pipeline, driving the device entry
// points of the other translation units over a workspace that is kept between calls.
//
// Per call: image -> device, quadtree (weftk_quadtree.h), tile count and tile list back in one
// copy, the tile layout built here (pixel and slot offsets, the tile lists per side for the pool
// generator, the scoring work items per size class, the refine order and loss weights) and sent
// in one copy, then extraction, pool generation, the init round, the Adam steps and the wire
// snap, and the results back.  The layout rules are the ones the package's Python front end
// uses (the fit's static work items, the stack set's order and weights), so both give the same
// bits.
#include <cuda_runtime.h>

#include <map>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/weftk_fit.h"
#include "../../include/weftk_pipeline.h"
#include "../../include/weftk_pool.h"
#include "../../include/weftk_quadtree.h"
#include "../../include/weftk_refine.h"
#include "../../include/weftk_wire.h"
#include "weftk_common.cuh"

static_assert(sizeof(WeftRefineParams) == 96, "WeftRefineParams layout is part of the C ABI");

namespace {

constexpr int STRIDE = WEFTK_POOL_MAX_CONST_LINEAR;  // candidate slots per tile

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

// grow a device buffer to at least `bytes` (contents are not kept)
int grow(DevBuf& b, size_t bytes) {
    if (bytes <= b.cap) return WEFTK_OK;
    if (b.p) WEFTK_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
    const size_t want = std::max<size_t>(bytes + bytes / 8, 256);
    WEFTK_CUDA(cudaMalloc(&b.p, want));
    b.cap = want;
    return WEFTK_OK;
}

struct HostBuf {
    void* p = nullptr;
    size_t cap = 0;
};

int grow_host(HostBuf& b, size_t bytes) {
    if (bytes <= b.cap) return WEFTK_OK;
    if (b.p) WEFTK_CUDA(cudaFreeHost(b.p));
    b.p = nullptr;
    b.cap = 0;
    const size_t want = std::max<size_t>(bytes + bytes / 8, 256);
    WEFTK_CUDA(cudaMallocHost(&b.p, want));
    b.cap = want;
    return WEFTK_OK;
}

// slot order of a uniform-stride pool: each tile's slots in their own order
__global__ void local_slot_kernel(int32_t* perm, long long n, int stride) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = (int32_t)(i % stride);
}

template <class T>
T* at(const DevBuf& b, size_t byte_off) {
    return reinterpret_cast<T*>(static_cast<char*>(b.p) + byte_off);
}

}  // namespace

struct WeftRefiner {
    WeftRefineParams prm;
    int device = 0;
    // image-sized
    DevBuf img, qwork, qtiles;
    // tile-sized (capacity ncap tiles): int32 state, doubles, selections, rows
    DevBuf tint, tdbl, tsel, trows;
    // slot-sized (ncap * STRIDE): records, prepared terms, flags, partial sums, slot order
    DevBuf cand, prep, alive, kind, partial, perm;
    // pixel-sized: tile pixels and the composite
    DevBuf src4, bg;
    // per-image layout upload and the scoring queue
    DevBuf layout, queue, misc;
    HostBuf h_qt, h_layout;
    long long ncap = 0, pxcap = 0, perm_ready = 0, items_cap = 0;
};

using namespace weftk;

extern "C" int weftk_refiner_create(const WeftRefineParams* params, WeftRefiner** out) {
    WEFTK_REQUIRE(params && out, "refiner_create: null argument");
    const WeftRefineParams& p = *params;
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    WEFTK_REQUIRE(p.cap >= 1 && p.steps >= 0, "refiner_create: cap >= 1 and steps >= 0");
    WEFTK_REQUIRE(pow2(p.min_tile) && pow2(p.max_tile) && p.min_tile >= 8 && p.min_tile <= p.max_tile &&
                      p.max_tile <= 64,
                  "refiner_create: tile sides must be powers of two with 8 <= min <= max <= 64");
    for (int i = 0; i < 3; ++i) {
        WEFTK_REQUIRE(p.chunk[i] >= 1, "refiner_create: chunk must be positive");
        WEFTK_REQUIRE(p.variant[i] >= 0 && p.variant[i] < WEFTK_FIT_VARIANTS, "refiner_create: bad scoring variant");
    }
    WEFTK_REQUIRE(p.tables && p.srgb_lut, "refiner_create: tables and sRGB table are required");
    WEFTK_REQUIRE(p.tables->side_bits, "refiner_create: the tables' side bits are not filled");
    auto* r = new WeftRefiner();
    r->prm = p;
    cudaError_t e = cudaGetDevice(&r->device);
    if (e != cudaSuccess) {
        delete r;
        return cuda_fail(e, "cudaGetDevice");
    }
    *out = r;
    return WEFTK_OK;
}

extern "C" int weftk_refiner_destroy(WeftRefiner* r) {
    if (!r) return WEFTK_OK;
    for (DevBuf* b : {&r->img, &r->qwork, &r->qtiles, &r->tint, &r->tdbl, &r->tsel, &r->trows, &r->cand, &r->prep,
                      &r->alive, &r->kind, &r->partial, &r->perm, &r->src4, &r->bg, &r->layout, &r->queue, &r->misc})
        if (b->p) cudaFree(b->p);
    for (HostBuf* b : {&r->h_qt, &r->h_layout})
        if (b->p) cudaFreeHost(b->p);
    delete r;
    return WEFTK_OK;
}

namespace {

// the tile layout of one image, in the order it is uploaded (int32 words)
struct Layout {
    int n = 0;
    long long n_px = 0;
    std::vector<int32_t> words;
    // word offsets of each section
    size_t px_off, size, cap, pool_off, pool_cap, order, rows, prim_off, lists[4], items[3], weights;
    int n_list[4] = {0, 0, 0, 0}, n_items[3] = {0, 0, 0};
    int n_big = 0, n_mid = 0, n_s16 = 0;
};

void build_layout(const int32_t* tiles, int n, const WeftRefineParams& p, Layout& L) {
    L.n = n;
    std::vector<int32_t> side(n);
    for (int t = 0; t < n; ++t) side[t] = tiles[3 * t + 2];
    auto& w = L.words;
    w.clear();
    auto section = [&](size_t count) {
        const size_t off = w.size();
        w.resize(off + count);
        return off;
    };
    // pixel offsets (tile-major float4 pixels), sides, caps, slot offsets and capacities
    L.px_off = section(n);
    long long px = 0;
    for (int t = 0; t < n; ++t) {
        w[L.px_off + t] = (int32_t)px;
        px += (long long)side[t] * side[t];
    }
    L.n_px = px;
    L.size = section(n);
    L.cap = section(n);
    L.pool_off = section(n);
    L.pool_cap = section(n);
    for (int t = 0; t < n; ++t) {
        w[L.size + t] = side[t];
        w[L.cap + t] = p.cap;
        w[L.pool_off + t] = t * STRIDE;
        w[L.pool_cap + t] = STRIDE;
    }
    // refine order: sides > 32, then 17..32, then 9..16, then the rest, each in tile order
    L.order = section(n);
    size_t k = L.order;
    int cls_n[4] = {0, 0, 0, 0};
    for (int c = 0; c < 4; ++c)
        for (int t = 0; t < n; ++t) {
            const int s = side[t];
            const int cc = s > 32 ? 0 : s > 16 ? 1 : s > 8 ? 2 : 3;
            if (cc == c) {
                w[k++] = t;
                ++cls_n[c];
            }
        }
    L.n_big = cls_n[0];
    L.n_mid = cls_n[1];
    L.n_s16 = cls_n[2];
    // one parameter row per tile
    L.rows = section(n);
    L.prim_off = section(n + 1);
    for (int t = 0; t < n; ++t) w[L.rows + t] = t;
    for (int t = 0; t <= n; ++t) w[L.prim_off + t] = t;
    // tiles of each side for the pool generator
    for (int si = 0; si < 4; ++si) {
        const int s = 8 << si;
        int cnt = 0;
        for (int t = 0; t < n; ++t) cnt += side[t] == s;
        L.lists[si] = section(cnt);
        L.n_list[si] = cnt;
        size_t q = L.lists[si];
        for (int t = 0; t < n; ++t)
            if (side[t] == s) w[q++] = t;
    }
    // scoring work items per size class (8, 16, 32 + 64 px): each tile's slot range in runs of
    // `chunk` candidates x 1024-pixel blocks, the class's largest tiles first
    for (int ci = 0; ci < 3; ++ci) {
        const int chunk = p.chunk[ci];
        std::vector<int> ts;
        for (int want : (ci == 0 ? std::vector<int>{8} : ci == 1 ? std::vector<int>{16} : std::vector<int>{64, 32}))
            for (int t = 0; t < n; ++t)
                if (side[t] == want) ts.push_back(t);
        const int nch = (STRIDE + chunk - 1) / chunk;
        size_t count = 0;
        for (int t : ts) count += (size_t)nch * std::max(1, side[t] * side[t] / 1024);
        L.items[ci] = section(4 * count);
        L.n_items[ci] = (int)count;
        size_t q = L.items[ci];
        for (int t : ts) {
            const int blocks = std::max(1, side[t] * side[t] / 1024);
            for (int j = 0; j < nch * blocks; ++j) {
                const int first = (j / blocks) * chunk;
                w[q++] = t;
                w[q++] = j % blocks;
                w[q++] = first;
                w[q++] = std::min(chunk, STRIDE - first);
            }
        }
    }
    // loss weights: each tile's share of the pixels, float32(side^2) / float32(total)
    L.weights = section(n);
    const float total = (float)px;
    for (int t = 0; t < n; ++t) {
        const float v = (float)((long long)side[t] * side[t]) / total;
        std::memcpy(&w[L.weights + t], &v, sizeof(float));
    }
}

}  // namespace

extern "C" int weftk_refine_image(WeftRefiner* r, const uint8_t* h_img, int h, int w, int32_t* h_tiles,
                                  float* h_rows, int32_t* h_kinds, int max_tiles, int* n_tiles, void* stream) {
    WEFTK_REQUIRE(r && h_img && n_tiles && h > 0 && w > 0, "refine_image: bad argument");
    WEFTK_REQUIRE(max_tiles >= 0 && (max_tiles == 0 || (h_tiles && h_rows && h_kinds)),
                  "refine_image: null output");
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    WEFTK_REQUIRE(dev == r->device, "refine_image: the refiner belongs to another device");
    const WeftRefineParams& p = r->prm;
    cudaStream_t s = (cudaStream_t)stream;
    int rc;

    // 1. image to the device, quadtree, tile count and list back in one copy
    const size_t img_bytes = (size_t)h * w * 3;
    if ((rc = grow(r->img, img_bytes))) return rc;
    WEFTK_CUDA(cudaMemcpyAsync(r->img.p, h_img, img_bytes, cudaMemcpyHostToDevice, s));
    int64_t qbytes = 0;
    if ((rc = weftk_quadtree_work_bytes(h, w, p.max_tile, p.min_tile, &qbytes))) return rc;
    if ((rc = grow(r->qwork, (size_t)qbytes))) return rc;
    const long long macro = (long long)((h + p.max_tile - 1) / p.max_tile) * ((w + p.max_tile - 1) / p.max_tile);
    const long long per = (long long)(p.max_tile / p.min_tile) * (p.max_tile / p.min_tile);
    WEFTK_REQUIRE(macro * per < (1ll << 28), "refine_image: image too large");
    const int tcap = (int)(macro * per);
    // int32 count first, then (x, y, side) per tile
    if ((rc = grow(r->qtiles, ((size_t)tcap * 3 + 4) * sizeof(int32_t)))) return rc;
    int32_t* d_n = at<int32_t>(r->qtiles, 0);
    int32_t* d_qt = at<int32_t>(r->qtiles, 4 * sizeof(int32_t));
    if ((rc = weftk_quadtree_variance(static_cast<const uint8_t*>(r->img.p), h, w, p.threshold, p.max_tile,
                                      p.min_tile, d_qt, tcap, d_n, r->qwork.p, stream)))
        return rc;
    if ((rc = grow_host(r->h_qt, ((size_t)tcap * 3 + 4) * sizeof(int32_t)))) return rc;
    WEFTK_CUDA(cudaMemcpyAsync(r->h_qt.p, r->qtiles.p, ((size_t)tcap * 3 + 4) * sizeof(int32_t),
                               cudaMemcpyDeviceToHost, s));
    WEFTK_CUDA(cudaStreamSynchronize(s));
    const int32_t* hq = static_cast<const int32_t*>(r->h_qt.p);
    const int n = hq[0];
    *n_tiles = n;
    WEFTK_REQUIRE(n >= 0 && n <= tcap, "refine_image: quadtree tile count out of range");
    if (n > max_tiles) return fail(WEFTK_E_RANGE, "refine_image: more tiles than max_tiles");
    std::memcpy(h_tiles, hq + 4, (size_t)n * 3 * sizeof(int32_t));
    if (n == 0) return WEFTK_OK;

    // 2. the tile layout, one upload
    Layout L;
    build_layout(hq + 4, n, p, L);
    const size_t lay_bytes = L.words.size() * sizeof(int32_t);
    if ((rc = grow_host(r->h_layout, lay_bytes))) return rc;
    if ((rc = grow(r->layout, lay_bytes))) return rc;
    std::memcpy(r->h_layout.p, L.words.data(), lay_bytes);
    WEFTK_CUDA(cudaMemcpyAsync(r->layout.p, r->h_layout.p, lay_bytes, cudaMemcpyHostToDevice, s));
    auto lay = [&](size_t word) { return at<int32_t>(r->layout, word * sizeof(int32_t)); };

    // 3. workspace for n tiles, n * STRIDE slots, n_px pixels
    const long long slots = (long long)n * STRIDE;
    if (n > r->ncap) {
        const long long nc = n;
        // int32 per tile: pool_cnt, gen counts, n_alive, n_sel, sel_bits, flags, zero_first, kinds
        if ((rc = grow(r->tint, (size_t)nc * 8 * sizeof(int32_t)))) return rc;
        if ((rc = grow(r->tdbl, (size_t)nc * 7 * sizeof(double)))) return rc;  // cur_obj, moments x6
        if ((rc = grow(r->trows, (size_t)nc * (4 * 16 + 1) * sizeof(float)))) return rc;  // p, m, v, q, loss
        if ((rc = grow(r->cand, (size_t)nc * STRIDE * sizeof(WeftPrim)))) return rc;
        if ((rc = grow(r->prep, (size_t)nc * STRIDE * 16 * sizeof(float)))) return rc;
        if ((rc = grow(r->alive, (size_t)nc * STRIDE))) return rc;
        if ((rc = grow(r->kind, (size_t)nc * STRIDE))) return rc;
        if ((rc = grow(r->partial, (size_t)nc * STRIDE * 4 * sizeof(float)))) return rc;
        r->ncap = nc;
    }
    if ((rc = grow(r->tsel, (size_t)n * p.cap * sizeof(int32_t)))) return rc;
    if (slots > r->perm_ready) {
        if ((rc = grow(r->perm, (size_t)slots * sizeof(int32_t)))) return rc;
        const long long cover = (long long)(r->perm.cap / sizeof(int32_t));
        local_slot_kernel<<<ceil_div(cover, 256), 256, 0, s>>>(static_cast<int32_t*>(r->perm.p), cover, STRIDE);
        WEFTK_CUDA(cudaGetLastError());
        r->perm_ready = cover;
    }
    if (L.n_px > r->pxcap) {
        if ((rc = grow(r->src4, (size_t)L.n_px * 4 * sizeof(float)))) return rc;
        if ((rc = grow(r->bg, (size_t)L.n_px * 4 * sizeof(float)))) return rc;
        r->pxcap = L.n_px;
    }
    const long long items = (long long)L.n_items[0] + L.n_items[1] + L.n_items[2];
    if ((rc = grow(r->queue, (size_t)std::max<long long>(items, 1) * sizeof(int32_t)))) return rc;
    // round status [4], queue control [8], work counters [2] (u64)
    if ((rc = grow(r->misc, 16 * sizeof(int32_t) + 2 * sizeof(unsigned long long)))) return rc;

    const size_t nc = (size_t)r->ncap;
    int32_t* pool_cnt = at<int32_t>(r->tint, 0);
    int32_t* gen_cnt = at<int32_t>(r->tint, nc * 4);
    int32_t* n_alive = at<int32_t>(r->tint, nc * 8);
    int32_t* n_sel = at<int32_t>(r->tint, nc * 12);
    int32_t* sel_bits = at<int32_t>(r->tint, nc * 16);
    int32_t* flags = at<int32_t>(r->tint, nc * 20);
    int32_t* zero_first = at<int32_t>(r->tint, nc * 24);
    int32_t* kinds = at<int32_t>(r->tint, nc * 28);
    double* cur_obj = at<double>(r->tdbl, 0);
    double* moments = at<double>(r->tdbl, nc * 8);
    float* prm_p = at<float>(r->trows, 0);
    float* prm_m = at<float>(r->trows, nc * 64);
    float* prm_v = at<float>(r->trows, nc * 128);
    float* q_rows = at<float>(r->trows, nc * 192);
    float* loss = at<float>(r->trows, nc * 256);
    int32_t* status = at<int32_t>(r->misc, 0);
    int32_t* queue_ctl = at<int32_t>(r->misc, 4 * sizeof(int32_t));
    unsigned long long* work = at<unsigned long long>(r->misc, 16 * sizeof(int32_t));
    WEFTK_CUDA(cudaMemsetAsync(zero_first, 0, (size_t)n * sizeof(int32_t), s));
    WEFTK_CUDA(cudaMemsetAsync(r->misc.p, 0, r->misc.cap, s));

    // 4. tile pixels, pools
    const int32_t* d_px_off = lay(L.px_off);
    if ((rc = weftk_extract_tiles(static_cast<const uint8_t*>(r->img.p), h, w, p.srgb_lut, d_qt, n, d_px_off,
                                  static_cast<float*>(r->src4.p), stream)))
        return rc;
    WeftPoolJob job{};
    job.src = static_cast<const float*>(r->src4.p);
    job.px_off = d_px_off;
    job.pool_off = lay(L.pool_off);
    job.pool_cap = STRIDE;
    job.kinds_mask = 3;  // constant and linear patches
    job.cand = static_cast<WeftPrim*>(r->cand.p);
    job.pool_cnt = gen_cnt;
    for (int si = 0; si < 4; ++si) {
        job.tiles[si] = L.n_list[si] ? lay(L.lists[si]) : nullptr;
        job.n_tiles[si] = L.n_list[si];
    }
    if ((rc = weftk_gen_pools(p.tables, &job, stream))) return rc;

    // 5. the init round over the pools (constants in closed form from the tile moments)
    WeftFitState st{};
    st.n_tiles = n;
    st.cap_max = p.cap;
    st.n_slots = slots;
    st.src = static_cast<const float*>(r->src4.p);
    st.bg = nullptr;  // only the init round runs: nothing reads a composite
    st.px_off = d_px_off;
    st.size = lay(L.size);
    st.cap = lay(L.cap);
    st.pool_off = lay(L.pool_off);
    st.pool_cnt = pool_cnt;
    st.pool_cap = lay(L.pool_cap);
    st.n_alive = n_alive;
    st.n_sel = n_sel;
    st.sel_bits = sel_bits;
    st.flags = flags;
    st.cur_obj = cur_obj;
    st.sel = static_cast<int32_t*>(r->tsel.p);
    st.cand = static_cast<const WeftPrim*>(r->cand.p);
    st.prep = static_cast<float*>(r->prep.p);
    st.alive = static_cast<uint8_t*>(r->alive.p);
    st.kind = static_cast<uint8_t*>(r->kind.p);
    st.partial = static_cast<float*>(r->partial.p);
    st.status = status;
    st.work = work;
    for (int i = 0; i < 3; ++i) st.variant[i] = p.variant[i];
    st.moments = moments;
    st.queue = static_cast<int32_t*>(r->queue.p);
    st.queue_ctl = queue_ctl;
    // the tiles' pixel moments beside the reset and the preparation (a side stream of this host
    // thread, joined before the round)
    {
        thread_local std::map<int, std::pair<cudaStream_t, cudaEvent_t[2]>> side_of;
        auto& sd = side_of[r->device];
        if (sd.first == nullptr) {
            WEFTK_CUDA(cudaStreamCreateWithFlags(&sd.first, cudaStreamNonBlocking));
            for (int i = 0; i < 2; ++i) WEFTK_CUDA(cudaEventCreateWithFlags(&sd.second[i], cudaEventDisableTiming));
        }
        WEFTK_CUDA(cudaEventRecord(sd.second[0], (cudaStream_t)stream));
        WEFTK_CUDA(cudaStreamWaitEvent(sd.first, sd.second[0], 0));
        if ((rc = weftk_fit_moments(&st, moments, sd.first))) return rc;
        WEFTK_CUDA(cudaEventRecord(sd.second[1], sd.first));
        if ((rc = weftk_fit_reset(&st, gen_cnt, stream))) return rc;
        if ((rc = weftk_fit_prepare(&st, zero_first, stream))) return rc;
        WEFTK_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, sd.second[1], 0));
    }
    const WeftFitItem* it[3];
    for (int ci = 0; ci < 3; ++ci)
        it[ci] = L.n_items[ci] ? reinterpret_cast<const WeftFitItem*>(lay(L.items[ci])) : nullptr;
    if ((rc = weftk_fit_round(&st, WEFTK_FIT_INIT, p.lambda, p.complex_threshold, static_cast<int32_t*>(r->perm.p),
                              it[0], L.n_items[0], it[1], L.n_items[1], it[2], L.n_items[2], stream)))
        return rc;

    // 6. Adam steps on each tile's pick, the snap to the wire grid
    const int32_t* rows = lay(L.rows);
    if ((rc = weftk_refine_start(&st, rows, n, prm_p, prm_m, prm_v, kinds, stream))) return rc;
    WeftStackSet ss{};
    ss.n_tiles = n;
    ss.max_prims = 1;
    ss.src = static_cast<const float*>(r->src4.p);
    ss.px_off = d_px_off;
    ss.size = lay(L.size);
    ss.prim_off = lay(L.prim_off);
    ss.kind = kinds;
    ss.order = lay(L.order);
    ss.n_big = L.n_big;
    ss.n_mid = L.n_mid;
    ss.n_s16 = L.n_s16;
    ss.kinds_mask = 3;
    ss.moments = moments;
    if (p.steps > 0 &&
        (rc = weftk_refine_steps(&ss, p.steps, prm_p, prm_m, prm_v, reinterpret_cast<const float*>(lay(L.weights)),
                                 loss, nullptr, p.lr, p.beta1, p.beta2, p.eps, 0, stream)))
        return rc;
    if ((rc = weftk_quantize_rows(prm_p, kinds, n, q_rows, stream))) return rc;

    // 7. results
    WEFTK_CUDA(cudaMemcpyAsync(h_rows, q_rows, (size_t)n * 16 * sizeof(float), cudaMemcpyDeviceToHost, s));
    WEFTK_CUDA(cudaMemcpyAsync(h_kinds, kinds, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    WEFTK_CUDA(cudaStreamSynchronize(s));
    return WEFTK_OK;
}
