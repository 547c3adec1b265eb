// The context behind ts_ctx*: one CUDA device, one stream, cached device buffers, the last error.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tomostar_cuda.h"
#include "host_geo.h"

struct ts_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // device→host copies that overlap the next solve (created on use)
    std::recursive_mutex mu;  // calls on one context are serialised (EikonalOpenCl.cs:64,165)
    std::string err;
    std::string stats;
    std::string name;
    int sm_count = 0;
    size_t total_mem = 0;
    volatile int* cancel_host = nullptr;  // host-mapped, read by kernels between rounds
    int* cancel_dev = nullptr;
    int tile_f64 = 0, tile_f32 = 0;       // engine tile shape per precision
    int scheduler = 0;                    // engine scheduler: 0 lockstep diagonals, 1 flow (per field)
    double epoch_budget_ms = 0;           // flow epochs: fields pause at the first round end after this
    // The extended domain's 1-D background for the rays' outside time (ts_set_background): node count,
    // the nodes in the "rays.background" buffer (depths, Vp, Vs).
    int bg_n = 0;
    int ray_warp_max = 2048;  // calls of at most this many rays trace one warp per ray
    // LSQR's onIteration (Numerics/Lsqr.cs:43,140): called after every iteration with its ‖r‖.
    void (*lsqr_on_iteration)(int32_t iteration, double rnorm, void* user) = nullptr;
    void* lsqr_user = nullptr;
    // CUDA-graph replay of one-shot engine solves: the last captured solve and its signature.
    bool use_graph = false;
    unsigned long long graph_sig = 0;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_replays = 0;

    // Stream-ordered allocations (rows, row staging, serving blocks) come from the context's own pool.
    // It keeps what they free, up to a quarter of the device's memory, for the next call: a pool that
    // hands freed memory back at every synchronisation maps it again on the next call, which made the
    // ray pipeline of a 1.5 M-row forward step take 1.3-2.2 s on the device instead of 0.75-0.85 s.
    cudaMemPool_t pool = nullptr;
    template <typename T>
    cudaError_t alloc_async(T** p, size_t bytes, cudaStream_t s) {
        void** q = reinterpret_cast<void**>(p);
        return pool ? cudaMallocFromPoolAsync(q, bytes, pool, s) : cudaMallocAsync(q, bytes, s);
    }

    struct Model;
    std::map<int, Model*> models;
    int next_model = 1;

    struct Buf {
        void* p = nullptr;
        size_t n = 0;
    };
    std::map<std::string, Buf> bufs;
    std::map<std::string, Buf> pinned;    // grow-only pinned host buffers

    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }
    // A grow-only named device buffer; nullptr (with err set) when the device is out of memory.
    void* buf(const std::string& key, size_t bytes) {
        Buf& b = bufs[key];
        if (b.n >= bytes && b.p) return b.p;
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.n = 0;
        size_t want = bytes < 256 ? 256 : bytes;
        if (cudaMalloc(&b.p, want) != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            err = "device buffer '" + key + "' of " + std::to_string(want) + " bytes (too large for the device?)";
            return nullptr;
        }
        b.n = want;
        return b.p;
    }
    // A grow-only named pinned host buffer.
    void* host_buf(const std::string& key, size_t bytes) {
        Buf& b = pinned[key];
        if (b.n >= bytes && b.p) return b.p;
        if (b.p) cudaFreeHost(b.p);
        b.p = nullptr;
        b.n = 0;
        size_t want = bytes < 256 ? 256 : bytes;
        if (cudaHostAlloc(&b.p, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            err = "pinned host buffer '" + key + "' of " + std::to_string(want) + " bytes";
            return nullptr;
        }
        b.n = want;
        return b.p;
    }
    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
        graph_sig = 0;
    }
    void release(const std::string& key) {
        auto it = bufs.find(key);
        if (it == bufs.end()) return;
        if (it->second.p) cudaFree(it->second.p);
        bufs.erase(it);
    }
};

#define TS_CUDA_TRY(ctx, call)                                                                        \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            char b_[512];                                                                             \
            snprintf(b_, sizeof b_, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return (ctx)->fail(e_ == cudaErrorMemoryAllocation ? TS_E_NOMEM : TS_E_CUDA, b_);        \
        }                                                                                             \
    } while (0)

#define TS_BUF(ctx, var, type, key, count)                                  \
    type* var = static_cast<type*>((ctx)->buf((key), sizeof(type) * size_t(count))); \
    if (!var) return TS_E_NOMEM

// Two timing events destroyed on every return path.
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~EventPair() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    EventPair(const EventPair&) = delete;
    EventPair& operator=(const EventPair&) = delete;
};

// The error text of calls made without a context (ts_last_error(NULL)), per host thread.
std::string& ts_thread_error();

// A resident model: grid, metric and the device slowness of its phases (ts_model_put).
struct ts_ctx::Model {
    ts_grid def{};
    std::vector<double> depth;
    ts::host::Grid* grid = nullptr;
    ts::host::Metric* metric = nullptr;
    int precision = 64;
    int n_phases = 1;
    void* slowness = nullptr;  // device, n_phases * n values of the precision
    ~Model() {
        delete metric;
        delete grid;
        if (slowness) cudaFree(slowness);
    }
};

namespace ts {
namespace eik {

// Host-side entry points of the eikonal solvers (eik_host.cu).
struct SolveIn {
    int model_id = 0;         // > 0: solve on a resident model (grid, slowness and metric from it)
    int phase = 0;
    const ts_grid* grid;
    const double* slowness;
    int n_fields;
    const int32_t* seed_offsets;
    const int32_t* seed_index;
    const double* seed_time;
    int precision;
    int mode;
    double tol;
    int max_rounds;
};

int model_put(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int n_phases, int precision, int* id);
int model_drop(ts_ctx* ctx, int id);
void models_free(ts_ctx* ctx);

// Solves and writes the fields to host `out` (dense, field-major, out_type).
int solve(ts_ctx* ctx, const SolveIn& in, void* out, int out_type, ts_eik_stats* stats);
int copy_fields_out(ts_ctx* ctx, const void* fields_dev, int precision, int64_t count, void* out, int out_type);

}  // namespace eik
}  // namespace ts
