// weftk_api.cu — C ABI entry points of libweftk.so, error state and the device arena
// used by the synchronous host-buffer entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "weftk_common.cuh"

static_assert(sizeof(WeftPrim) == 60, "WeftPrim must match the reference's 60-byte PrimData");
static_assert(sizeof(WeftEval) == 16, "WeftEval must match the reference's EvalDesc");
static_assert(sizeof(WeftTileDecodeDesc) == 48, "WeftTileDecodeDesc must match TileDecodeDesc");

namespace weftk {

int launch_score_evals(const WeftEval*, int, const WeftPrim*, const float*, float*, int, cudaStream_t);
int launch_render_tiles(const WeftTileDecodeDesc*, int, const int2*, int, const WeftPrim*, const float*, int,
                        const float*, int, float*, int, int, cudaStream_t);
int read_device_status(int* status, bool clear);

static thread_local std::string t_last_error;

void set_error(const std::string& msg) { t_last_error = msg; }

int fail(int code, const std::string& msg) {
    t_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    t_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return WEFTK_E_CUDA;
}

// Growable device buffers for the host-buffer entry points: one set per device,
// reused across calls (no allocation once warm), guarded by a mutex because the
// host-buffer calls are synchronous and may come from several threads.
struct Arena {
    std::vector<void*> ptr;
    std::vector<size_t> cap;
    cudaStream_t stream = nullptr;
};
static std::mutex g_arena_mu;
static std::vector<Arena> g_arenas;

static int arena_get(int slot, size_t bytes, void** out, Arena& a) {
    if ((int)a.ptr.size() <= slot) {
        a.ptr.resize(slot + 1, nullptr);
        a.cap.resize(slot + 1, 0);
    }
    bytes = bytes < 256 ? 256 : bytes;
    if (a.cap[slot] < bytes) {
        if (a.ptr[slot]) WEFTK_CUDA(cudaFree(a.ptr[slot]));
        a.ptr[slot] = nullptr;
        a.cap[slot] = 0;
        size_t want = bytes + bytes / 4;
        WEFTK_CUDA(cudaMalloc(&a.ptr[slot], want));
        a.cap[slot] = want;
    }
    *out = a.ptr[slot];
    return WEFTK_OK;
}

static int arena_for_current(Arena** out) {
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    if ((int)g_arenas.size() <= dev) g_arenas.resize(dev + 1);
    Arena& a = g_arenas[dev];
    if (!a.stream) WEFTK_CUDA(cudaStreamCreateWithFlags(&a.stream, cudaStreamNonBlocking));
    *out = &a;
    return WEFTK_OK;
}

static int check_status_after_sync() {
    int st = 0;
    int rc = read_device_status(&st, true);
    if (rc) return rc;
    if (st) return fail(WEFTK_E_DEVICE, "a kernel rejected its input (bad descriptor or size)");
    return WEFTK_OK;
}

}  // namespace weftk

using namespace weftk;

extern "C" {

int weftk_version(void) { return 1 * 10000 + 0 * 100 + 0; }

int weftk_last_error(char* buf, size_t n) {
    const std::string& s = t_last_error;
    if (buf && n) {
        size_t k = s.size() < n - 1 ? s.size() : n - 1;
        std::memcpy(buf, s.data(), k);
        buf[k] = '\0';
    }
    return (int)s.size();
}

int weftk_init(int device) {
    int count = 0;
    WEFTK_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(WEFTK_E_ARG, "weftk_init: no such device");
    WEFTK_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    WEFTK_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(WEFTK_E_DEVICE, std::string("weftk_init: built for sm_100a, device is ") + prop.name);
    return WEFTK_OK;
}

int weftk_device_status(int* status) {
    WEFTK_REQUIRE(status, "device_status: null pointer");
    return read_device_status(status, true);
}

int weftk_score_evals(const WeftEval* d_evals, int n_evals, const WeftPrim* d_prims, const float* d_tiles,
                      float* d_mse, int flags, void* stream) {
    return launch_score_evals(d_evals, n_evals, d_prims, d_tiles, d_mse, flags, (cudaStream_t)stream);
}

int weftk_score_evals_host(const WeftEval* h_evals, int n_evals, const WeftPrim* h_prims, int n_prims,
                           const float* h_tiles, int64_t n_tile_floats, float* h_mse, int flags) {
    if (n_evals == 0) return WEFTK_OK;
    WEFTK_REQUIRE(n_evals > 0 && h_evals && h_mse && n_prims >= 0 && n_tile_floats >= 0, "score_evals_host: bad arguments");
    for (int i = 0; i < n_evals; ++i) {
        const WeftEval& e = h_evals[i];
        if (e.tile_size <= 0 || e.tile_size > 64 || e.prim_count < 0 || e.prim_offset < 0 ||
            (int64_t)e.prim_offset + e.prim_count > n_prims || e.tile_offset < 0 ||
            (int64_t)e.tile_offset + 3LL * e.tile_size * e.tile_size > n_tile_floats)
            return fail(WEFTK_E_ARG, "score_evals_host: eval " + std::to_string(i) + " is out of range");
    }
    std::lock_guard<std::mutex> lock(g_arena_mu);
    Arena* a = nullptr;
    int rc = arena_for_current(&a);
    if (rc) return rc;
    void *de, *dp, *dt, *dm;
    if ((rc = arena_get(0, sizeof(WeftEval) * (size_t)n_evals, &de, *a))) return rc;
    if ((rc = arena_get(1, sizeof(WeftPrim) * (size_t)(n_prims > 0 ? n_prims : 1), &dp, *a))) return rc;
    if ((rc = arena_get(2, sizeof(float) * (size_t)(n_tile_floats > 0 ? n_tile_floats : 1), &dt, *a))) return rc;
    if ((rc = arena_get(3, sizeof(float) * (size_t)n_evals, &dm, *a))) return rc;
    cudaStream_t s = a->stream;
    WEFTK_CUDA(cudaMemcpyAsync(de, h_evals, sizeof(WeftEval) * (size_t)n_evals, cudaMemcpyHostToDevice, s));
    if (n_prims > 0) WEFTK_CUDA(cudaMemcpyAsync(dp, h_prims, sizeof(WeftPrim) * (size_t)n_prims, cudaMemcpyHostToDevice, s));
    if (n_tile_floats > 0)
        WEFTK_CUDA(cudaMemcpyAsync(dt, h_tiles, sizeof(float) * (size_t)n_tile_floats, cudaMemcpyHostToDevice, s));
    if ((rc = launch_score_evals((const WeftEval*)de, n_evals, (const WeftPrim*)dp, (const float*)dt, (float*)dm, flags, s)))
        return rc;
    WEFTK_CUDA(cudaMemcpyAsync(h_mse, dm, sizeof(float) * (size_t)n_evals, cudaMemcpyDeviceToHost, s));
    WEFTK_CUDA(cudaStreamSynchronize(s));
    return check_status_after_sync();
}

int weftk_render_tiles(const WeftTileDecodeDesc* d_descs, int n_tiles, const int32_t* d_items, int n_items,
                       const WeftPrim* d_prims, const float* d_cp48, int n_cp48, const float* d_res1, int n_res1,
                       float* d_out, int out_h, int out_w, int flags, void* stream) {
    (void)flags;
    return launch_render_tiles(d_descs, n_tiles, reinterpret_cast<const int2*>(d_items), n_items, d_prims, d_cp48,
                               n_cp48, d_res1, n_res1, d_out, out_h, out_w, (cudaStream_t)stream);
}

int weftk_render_tiles_host(const WeftTileDecodeDesc* h_descs, int n_tiles, const WeftPrim* h_prims, int n_prims,
                            const float* h_cp48, int n_cp48, const float* h_res1, int n_res1, float* h_out,
                            int out_h, int out_w, int flags) {
    (void)flags;
    WEFTK_REQUIRE(n_tiles >= 0 && out_h > 0 && out_w > 0 && h_out && n_prims >= 0 && n_cp48 >= 0 && n_res1 >= 0,
                  "render_tiles_host: bad arguments");
    // work items (tile, first row) in descending cost order (pixels, times 4 for a tile
    // evaluated per pixel: anything but a lone constant layer without a RES1 grid)
    std::vector<std::pair<long long, int2>> costed;
    for (int i = 0; i < n_tiles; ++i) {
        const WeftTileDecodeDesc& d = h_descs[i];
        if (d.target_w > 0 && d.target_h > 0 && d.target_w <= 8192 && d.target_h <= 8192) {
            auto fdiv4 = [](long long v) { return v >= 0 ? v / 4 : -((-v + 3) / 4); };
            const long long G = fdiv4((long long)d.target_x0 + d.target_w + 3) - fdiv4(d.target_x0);
            const long long R = std::max(1LL, WEFTK_DECODE_ITEM_GROUPS / G);
            const long long r0 = std::max(0LL, -(long long)d.target_y0);
            const long long r1 = std::min((long long)d.target_h, (long long)out_h - d.target_y0);
            const bool cols = (long long)d.target_x0 < out_w && (long long)d.target_x0 + d.target_w > 0;
            const bool fill = d.res1_index < 0 && d.prim_count == 1 && d.prim_offset >= 0 &&
                              d.prim_offset < n_prims && h_prims[d.prim_offset].kind == 0;
            if (cols)
                for (long long r = r0; r < r1; r += R)
                    costed.push_back({std::min(R, r1 - r) * d.target_w * (fill ? 1 : 4), make_int2(i, (int)r)});
        }
        if (d.prim_count < 0 || d.prim_count > 48 || d.prim_offset < 0 || (int64_t)d.prim_offset + d.prim_count > n_prims ||
            d.target_w <= 0 || d.target_h <= 0 || d.target_w > 8192 || d.target_h > 8192 || d.source_size <= 0 ||
            (n_res1 > 0 && d.res1_index >= n_res1))
            return fail(WEFTK_E_ARG, "render_tiles_host: tile " + std::to_string(i) + " is out of range");
        if (d.prim_count == 1 && h_prims[d.prim_offset].kind == 5) {
            int idx = (int)h_prims[d.prim_offset].geom[0];
            if (idx < 0 || idx >= n_cp48) return fail(WEFTK_E_ARG, "render_tiles_host: bad bicubic grid index");
        }
    }
    std::stable_sort(costed.begin(), costed.end(),
                     [](const std::pair<long long, int2>& x, const std::pair<long long, int2>& y) { return x.first > y.first; });
    std::vector<int2> items(costed.size());
    for (size_t k = 0; k < costed.size(); ++k) items[k] = costed[k].second;
    std::lock_guard<std::mutex> lock(g_arena_mu);
    Arena* a = nullptr;
    int rc = arena_for_current(&a);
    if (rc) return rc;
    size_t out_bytes = sizeof(float) * 3 * (size_t)out_h * (size_t)out_w;
    void *dd, *dp, *dc, *dr, *dout, *di;
    if ((rc = arena_get(9, sizeof(int2) * (items.empty() ? 1 : items.size()), &di, *a))) return rc;
    if ((rc = arena_get(4, sizeof(WeftTileDecodeDesc) * (size_t)(n_tiles > 0 ? n_tiles : 1), &dd, *a))) return rc;
    if ((rc = arena_get(5, sizeof(WeftPrim) * (size_t)(n_prims > 0 ? n_prims : 1), &dp, *a))) return rc;
    if ((rc = arena_get(6, sizeof(float) * 48 * (size_t)(n_cp48 > 0 ? n_cp48 : 1), &dc, *a))) return rc;
    if ((rc = arena_get(7, sizeof(float) * 48 * (size_t)(n_res1 > 0 ? n_res1 : 1), &dr, *a))) return rc;
    if ((rc = arena_get(8, out_bytes, &dout, *a))) return rc;
    cudaStream_t s = a->stream;
    if (n_tiles > 0)
        WEFTK_CUDA(cudaMemcpyAsync(dd, h_descs, sizeof(WeftTileDecodeDesc) * (size_t)n_tiles, cudaMemcpyHostToDevice, s));
    if (n_prims > 0) WEFTK_CUDA(cudaMemcpyAsync(dp, h_prims, sizeof(WeftPrim) * (size_t)n_prims, cudaMemcpyHostToDevice, s));
    if (n_cp48 > 0) WEFTK_CUDA(cudaMemcpyAsync(dc, h_cp48, sizeof(float) * 48 * (size_t)n_cp48, cudaMemcpyHostToDevice, s));
    if (n_res1 > 0) WEFTK_CUDA(cudaMemcpyAsync(dr, h_res1, sizeof(float) * 48 * (size_t)n_res1, cudaMemcpyHostToDevice, s));
    if (!items.empty())
        WEFTK_CUDA(cudaMemcpyAsync(di, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, s));
    WEFTK_CUDA(cudaMemsetAsync(dout, 0, out_bytes, s));
    if ((rc = launch_render_tiles((const WeftTileDecodeDesc*)dd, n_tiles, (const int2*)di, (int)items.size(),
                                  (const WeftPrim*)dp, n_cp48 ? (const float*)dc : nullptr, n_cp48,
                                  n_res1 ? (const float*)dr : nullptr, n_res1, (float*)dout, out_h, out_w, s)))
        return rc;
    WEFTK_CUDA(cudaMemcpyAsync(h_out, dout, out_bytes, cudaMemcpyDeviceToHost, s));
    WEFTK_CUDA(cudaStreamSynchronize(s));
    return check_status_after_sync();
}

}  // extern "C"
