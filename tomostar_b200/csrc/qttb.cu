// .qttb files from and to tables kept on the device (Forward/TravelTimeTable.cs:38-111): the
// writer lays out TravelTimeTable.Write's file around a device table, and the loader reads files
// that TravelTimeTable.Open accepts into a resident table set.
//
// File layout (TravelTimeTable.cs:57-80, 99-111): the 8-byte magic "QTTB" 01 00 00 00, the header's
// JSON length as a little-endian int32, the JSON (TravelTimeTableHeader serialised by the caller),
// zero bytes up to a multiple of 64, then one little-endian float32 per node in grid order with
// every non-finite value written as +inf. Written to path + ".tmp" and renamed over path.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"
#include "tables.h"

namespace ts {
namespace qttb {

const unsigned char kMagic[8] = {'Q', 'T', 'T', 'B', 1, 0, 0, 0};

// TravelTimeTable.Write's value rule: a finite float as it is, anything else +inf.
__global__ void finite_or_inf(const float* __restrict__ src, float* __restrict__ dst, int64_t n) {
    const float inf = __int_as_float(0x7f800000);
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float v = src[i];
        dst[i] = isfinite(v) ? v : inf;
    }
}

int64_t data_offset(int32_t json_len) { return 12 + int64_t(json_len) + (64 - (12 + int64_t(json_len)) % 64) % 64; }

}  // namespace qttb
}  // namespace ts

using namespace ts;

extern "C" {

int ts_tables_write_qttb(ts_tables* t, int32_t first, int32_t count, const char* const* paths,
                         const char* const* headers, const int32_t* header_len) {
    if (!t) return TS_E_ARG;
    ts_ctx* ctx = t->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (first < 0 || count < 0 || first + count > t->n_tables || (count > 0 && (!paths || !headers || !header_len)))
        return ctx->fail(TS_E_ARG, "bad table range or null arrays");
    const int64_t n = t->nodes;
    const size_t bytes = sizeof(float) * size_t(n);
    cudaStream_t s = ctx->stream;
    // Two staging slots: the copy of table k+1 runs while table k is written to its file.
    float* stage_d = static_cast<float*>(ctx->buf("qttb.stage", 2 * bytes));
    float* stage_h = static_cast<float*>(ctx->host_buf("qttb.host", 2 * bytes));
    if (!stage_d || !stage_h) return TS_E_NOMEM;
    cudaEvent_t done[2];
    cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
    auto issue = [&](int k) -> int {
        const int slot = k & 1;
        qttb::finite_or_inf<<<592, 256, 0, s>>>(t->dev + size_t(n) * (first + k), stage_d + size_t(n) * slot, n);
        TS_CUDA_TRY(ctx, cudaGetLastError());
        TS_CUDA_TRY(ctx, cudaMemcpyAsync(stage_h + size_t(n) * slot, stage_d + size_t(n) * slot, bytes,
                                         cudaMemcpyDeviceToHost, s));
        TS_CUDA_TRY(ctx, cudaEventRecord(done[slot], s));
        return TS_OK;
    };
    int rc = count > 0 ? issue(0) : TS_OK;
    for (int k = 0; k < count && rc == TS_OK; k++) {
        if (k + 1 < count) rc = issue(k + 1);
        if (rc) break;
        const int slot = k & 1;
        if (cudaEventSynchronize(done[slot]) != cudaSuccess) {
            rc = ctx->fail(TS_E_CUDA, "table copy failed");
            break;
        }
        if (!paths[k] || !headers[k] || header_len[k] < 0) {
            rc = ctx->fail(TS_E_ARG, "null path or header");
            break;
        }
        const std::string path = paths[k], tmp = path + ".tmp";
        FILE* f = std::fopen(tmp.c_str(), "wb");
        if (!f) {
            rc = ctx->fail(TS_E_ARG, "cannot create " + tmp + ": " + std::strerror(errno));
            break;
        }
        unsigned char len[4];
        const uint32_t L = uint32_t(header_len[k]);
        for (int b = 0; b < 4; b++) len[b] = (unsigned char)((L >> (8 * b)) & 0xff);
        const int64_t pad = qttb::data_offset(header_len[k]) - 12 - header_len[k];
        static const unsigned char zeros[64] = {0};
        bool ok = std::fwrite(qttb::kMagic, 1, 8, f) == 8 && std::fwrite(len, 1, 4, f) == 4 &&
                  std::fwrite(headers[k], 1, size_t(L), f) == size_t(L) &&
                  std::fwrite(zeros, 1, size_t(pad), f) == size_t(pad) &&
                  std::fwrite(stage_h + size_t(n) * slot, 1, bytes, f) == bytes;  // little-endian host
        ok = (std::fclose(f) == 0) && ok;
        if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
            std::remove(tmp.c_str());
            rc = ctx->fail(TS_E_ARG, "cannot write " + path + ": " + std::strerror(errno));
            break;
        }
    }
    cudaStreamSynchronize(s);
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
    return rc;
}

int ts_tables_load_qttb(ts_ctx* ctx, const ts_grid* grid, int32_t count, const char* const* paths, ts_tables** out) {
    if (!ctx || !out) return TS_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    if (!grid || count <= 0 || !paths) return ctx->fail(TS_E_ARG, "bad arguments");
    if (const char* bad = host::Grid::validate(*grid)) return ctx->fail(TS_E_ARG, bad);
    if (grid->depth_km) return ctx->fail(TS_E_ARG, "tables need a uniform grid");
    const int64_t n = int64_t(grid->nx) * grid->ny * grid->nz;
    const size_t bytes = sizeof(float) * size_t(n);
    auto* t = new ts_tables();
    t->ctx = ctx;
    t->def = *grid;
    t->n_tables = count;
    t->nodes = n;
    if (cudaMalloc(&t->dev, bytes * size_t(count)) != cudaSuccess) {
        cudaGetLastError();
        delete t;
        return ctx->fail(TS_E_NOMEM, "no device memory for the tables");
    }
    float* stage_h = static_cast<float*>(ctx->host_buf("qttb.host", 2 * bytes));
    cudaEvent_t done[2];
    cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
    bool used[2] = {false, false};
    int rc = stage_h ? TS_OK : TS_E_NOMEM;
    for (int k = 0; k < count && rc == TS_OK; k++) {
        const int slot = k & 1;
        if (used[slot]) cudaEventSynchronize(done[slot]);  // the slot's previous upload is done
        // TravelTimeTable.Open (:99-111): the magic, the header length, the data after the padding.
        FILE* f = paths[k] ? std::fopen(paths[k], "rb") : nullptr;
        if (!f) {
            rc = ctx->fail(TS_E_ARG, std::string("cannot open ") + (paths[k] ? paths[k] : "(null)"));
            break;
        }
        unsigned char head[12];
        const bool head_ok = std::fread(head, 1, 12, f) == 12 && std::memcmp(head, qttb::kMagic, 8) == 0;
        int32_t L = 0;
        if (head_ok) L = int32_t(uint32_t(head[8]) | uint32_t(head[9]) << 8 | uint32_t(head[10]) << 16 | uint32_t(head[11]) << 24);
        const bool data_ok = head_ok && L >= 0 && std::fseek(f, long(qttb::data_offset(L)), SEEK_SET) == 0 &&
                             std::fread(stage_h + size_t(n) * slot, 1, bytes, f) == bytes;
        std::fclose(f);
        if (!head_ok) {
            rc = ctx->fail(TS_E_ARG, std::string("not a travel-time table: ") + paths[k]);
            break;
        }
        if (!data_ok) {
            rc = ctx->fail(TS_E_ARG, std::string("table shorter than the grid: ") + paths[k]);
            break;
        }
        if (cudaMemcpyAsync(t->dev + size_t(n) * k, stage_h + size_t(n) * slot, bytes, cudaMemcpyHostToDevice,
                            ctx->stream) != cudaSuccess ||
            cudaEventRecord(done[slot], ctx->stream) != cudaSuccess) {
            rc = ctx->fail(TS_E_CUDA, "table upload failed");
            break;
        }
        used[slot] = true;
    }
    cudaStreamSynchronize(ctx->stream);
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
    if (rc) {
        cudaFree(t->dev);
        delete t;
        return rc;
    }
    *out = t;
    return TS_OK;
}

}  // extern "C"
