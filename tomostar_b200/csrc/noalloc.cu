// ts_eik_solve_noalloc: the plain FP64 solve for callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc when they need a travel-time field: a process whose device
// memory is entirely held by another allocator (a framework's caching pool or a serving budget
// reserved at start-up), a plug-in host that forbids device allocation after initialisation, or a
// latency-critical path where an allocation's implicit synchronisation is not acceptable. This entry
// point takes the slowness and the output field as device pointers the caller already owns, and
// keeps all of its own working memory (fixed-node and due flags, axis weights, seeds, the round
// flag) in one file-scope __device__ array of kScratchBytes, which every GPU that loads the library
// holds until the process exits. It allocates nothing on the device.
//
// The scheme is the reference's as-is (Forward/EikonalOpenCl.cs:196-270, SphericalEikonal.Relax),
// one launch per diagonal plane, so the field equals SphericalEikonal.Relax to the bit.
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "ctx.h"
#include "eik_kernels.cuh"
#include "host_geo.h"

namespace ts {
namespace noalloc {

// Limits of one call (the scratch layout below is sized for them).
constexpr int64_t kMaxNodes = TS_NOALLOC_MAX_NODES;
constexpr int64_t kMaxRows = TS_NOALLOC_MAX_ROWS;      // ny * nz
constexpr int64_t kMaxLevels = TS_NOALLOC_MAX_LEVELS;  // nz
constexpr int64_t kMaxSeeds = TS_NOALLOC_MAX_SEEDS;

// Scratch layout (byte offsets; every block 256-byte aligned).
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffFixed = 0;
constexpr size_t kOffDue = kOffFixed + align256(kMaxNodes);
constexpr size_t kOffWx = kOffDue + align256(kMaxNodes);
constexpr size_t kOffWy = kOffWx + align256(sizeof(double) * 2 * kMaxRows);
constexpr size_t kOffSeedAt = kOffWy + align256(sizeof(double) * 2 * kMaxLevels);
constexpr size_t kOffSeedT = kOffSeedAt + align256(sizeof(int64_t) * kMaxSeeds);
constexpr size_t kOffFlags = kOffSeedT + align256(sizeof(double) * kMaxSeeds);
constexpr size_t kScratchBytes = kOffFlags + 256;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// The scratch array's device address on the current device. Looked up on every call (a host-side
// query, cheap next to a solve): an address kept from an earlier call would be stale after the
// device's primary context was reset and the library's device code loaded again.
int scratch_address(unsigned char** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ts_thread_error() = std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e);
        return TS_E_CUDA;
    }
    *out = static_cast<unsigned char*>(p);
    return TS_OK;
}

// True when p is device (or managed) memory of `device`: a kernel given a host pointer or another
// GPU's buffer would touch memory it cannot or must not address.
bool on_device(const void* p, int device) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == device;
}

__global__ void fill_f64(double* __restrict__ p, double v, int64_t n) {
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x) p[q] = v;
}

__global__ void fill_bytes(uint8_t* __restrict__ p, uint8_t v, int64_t n) {
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n; q += int64_t(gridDim.x) * blockDim.x) p[q] = v;
}

int fail(int code, const std::string& msg) {
    ts_thread_error() = msg;
    return code;
}

#define NA_TRY(call)                                                                                   \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            cudaGetLastError();                                                                        \
            return fail(TS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));                 \
        }                                                                                              \
    } while (0)

int solve(const ts_grid* grid, const double* slowness_dev, int n_seeds, const int32_t* seed_index,
          const double* seed_time, double* field_dev, double tol, int max_rounds, cudaStream_t s,
          int32_t rounds_out[2]) {
    if (!grid || !slowness_dev || !field_dev || n_seeds < 0 || (n_seeds > 0 && (!seed_index || !seed_time)))
        return fail(TS_E_ARG, "null pointer or negative seed count");
    if (const char* bad = host::Grid::validate(*grid)) return fail(TS_E_ARG, bad);
    if (grid->depth_km) return fail(TS_E_ARG, "ts_eik_solve_noalloc takes uniform grids only");
    if (!(tol >= 0)) return fail(TS_E_ARG, "tolerance must be >= 0");
    const int nx = grid->nx, ny = grid->ny, nz = grid->nz;
    const int64_t n = int64_t(nx) * ny * nz;
    if (n > kMaxNodes || int64_t(ny) * nz > kMaxRows || nz > kMaxLevels)
        return fail(TS_E_CAPACITY, "grid beyond the limits of ts_eik_solve_noalloc (nodes <= " +
                                       std::to_string(kMaxNodes) + ", ny*nz <= " + std::to_string(kMaxRows) +
                                       ", nz <= " + std::to_string(kMaxLevels) + ")");
    // Seeds as TrySolve takes them (EikonalOpenCl.cs:147-163).
    std::map<int32_t, double> merged;
    for (int q = 0; q < n_seeds; q++) {
        if (uint32_t(seed_index[q]) >= uint64_t(n)) continue;
        auto it = merged.find(seed_index[q]);
        if (it == merged.end() || seed_time[q] < it->second) merged[seed_index[q]] = seed_time[q];
    }
    if (merged.empty()) return fail(TS_E_NOSEEDS, "no seed nodes");
    if (int64_t(merged.size()) > kMaxSeeds)
        return fail(TS_E_CAPACITY, "more than " + std::to_string(kMaxSeeds) + " seed nodes");
    int device = 0;
    NA_TRY(cudaGetDevice(&device));
    if (!on_device(slowness_dev, device) || !on_device(field_dev, device))
        return fail(TS_E_ARG, "slowness_dev and field_dev must be device memory of the current device (" +
                                  std::to_string(device) + ")");
    unsigned char* base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    uint8_t* fixed = base + kOffFixed;
    uint8_t* due = base + kOffDue;
    double* wx = reinterpret_cast<double*>(base + kOffWx);
    double* wy = reinterpret_cast<double*>(base + kOffWy);
    int64_t* seed_at = reinterpret_cast<int64_t*>(base + kOffSeedAt);
    double* seed_t = reinterpret_cast<double*>(base + kOffSeedT);
    int* changed = reinterpret_cast<int*>(base + kOffFlags);
    unsigned long long* updates = reinterpret_cast<unsigned long long*>(base + kOffFlags + 16);

    host::Grid g(*grid);
    host::Metric m(g);
    std::vector<int64_t> at;
    std::vector<double> tv;
    for (auto& kv : merged) {
        at.push_back(kv.first);
        tv.push_back(kv.second);
    }
    NA_TRY(cudaMemcpyAsync(wx, m.wx.data(), sizeof(double) * m.wx.size(), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(wy, m.wy.data(), sizeof(double) * m.wy.size(), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(seed_at, at.data(), sizeof(int64_t) * at.size(), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(seed_t, tv.data(), sizeof(double) * tv.size(), cudaMemcpyHostToDevice, s));
    // The scratch keeps the previous call's contents: clear what must start cleared.
    const int blocks = int(std::min<int64_t>((n + 255) / 256, 2048));
    fill_f64<<<blocks, 256, 0, s>>>(field_dev, host::kInf, n);
    fill_bytes<<<blocks, 256, 0, s>>>(fixed, 0, n);
    NA_TRY(cudaMemsetAsync(updates, 0, sizeof(unsigned long long), s));
    const int count = int(at.size());
    eik::seed_kernel<double><<<(count + 127) / 128, 128, 0, s>>>(field_dev, fixed, seed_at, seed_t, count);
    NA_TRY(cudaGetLastError());
    const int cap = max_rounds > 0 ? max_rounds : std::max(32, (nx + ny + nz) / 4);
    const int planes = nx + ny + nz - 2;
    for (int phase = 0; phase < 2; phase++) {
        fill_bytes<<<blocks, 256, 0, s>>>(due, 1, n);
        bool settled = false;
        for (int round = 0; round < cap && !settled; round++) {
            NA_TRY(cudaMemsetAsync(changed, 0, sizeof(int), s));
            for (int dir = 0; dir < 8; dir++)
                for (int p = 0; p < planes; p++) {
                    int i0 = std::max(0, p - (ny - 1) - (nz - 1)), i1 = std::min(nx - 1, p);
                    int k0 = std::max(0, p - (nx - 1) - (ny - 1)), k1 = std::min(nz - 1, p);
                    dim3 gd((i1 - i0 + 1 + 127) / 128, k1 - k0 + 1);
                    eik::plain_sweep_kernel<double, false><<<gd, 128, 0, s>>>(
                        field_dev, slowness_dev, fixed, due, wx, wy, m.wz1, m.wz2, nullptr, nx, ny, nz, phase, changed,
                        dir, p, tol, updates);
                }
            NA_TRY(cudaGetLastError());
            int ch = 0;
            NA_TRY(cudaMemcpyAsync(&ch, changed, sizeof(int), cudaMemcpyDeviceToHost, s));
            NA_TRY(cudaStreamSynchronize(s));
            if (rounds_out) rounds_out[phase] = round + 1;
            settled = ch == 0;
        }
        if (!settled) return fail(TS_E_UNSETTLED, "sweeping not settled after " + std::to_string(cap) + " rounds");
    }
    NA_TRY(cudaStreamSynchronize(s));
    return TS_OK;
}

}  // namespace noalloc
}  // namespace ts

extern "C" int ts_eik_solve_noalloc(const ts_grid* grid, const double* slowness_dev, int32_t n_seeds,
                                    const int32_t* seed_index, const double* seed_time, double* field_dev, double tol,
                                    int32_t max_rounds, void* stream, int32_t* rounds_out) {
    return ts::noalloc::solve(grid, slowness_dev, n_seeds, seed_index, seed_time, field_dev, tol, max_rounds,
                              static_cast<cudaStream_t>(stream), rounds_out);
}
