// The tiled engine's host interface: a job of fields over one or more grids, solved by one
// cooperative persistent launch (or several, for continuous batching).
#pragma once

#include <vector>

#include "ctx.h"
#include "host_geo.h"

namespace ts {
namespace eik {

struct EngineField {
    int grid = 0;                              // index into EngineJob::grids
    const void* slowness = nullptr;            // device, Real[n] of its grid (dense grid order)
    void* T = nullptr;                         // set by engine_run: the field, padded rows
    const std::vector<int32_t>* seed_idx = nullptr;  // merged seeds (ascending nodes)
    const std::vector<double>* seed_t = nullptr;
    int cap = 32;                              // round cap per phase
    // results
    int status = 0;                            // 1 settled, 2 refused at the cap, 0 unfinished
    int rounds[2] = {0, 0};
};

struct EngineJob {
    std::vector<const host::Grid*> grids;
    std::vector<const host::Metric*> metrics;
    std::vector<EngineField> fields;
    double tol = 1e-7;
    double wake_rel = 0;     // 0: the reference's dirty rule (bitwise); TS_WAKE_REL for TS_MODE_FAST
    int tile = 0;            // tile shape id (0 = default for the precision)
    int warps = 0;           // warps per block (0 = default)
    // Set by engine_run: the padded field layout. Node (i, j, k) of a field on grid g sits at
    // T[(k * ny + j) * pitch[g] + xoff + i]; the pads hold +inf.
    std::vector<int> pitch;
    int xoff = 0;
};

// Copies padded engine fields to dense grid order (one cudaMemcpy2D per field block), converting
// to out_type (TS_OUT_F64 / TS_OUT_F32) on the device when it differs from the field precision.
int fields_to_dense_host(ts_ctx* ctx, const EngineJob& job, int precision, void* out, int out_type);
int fields_to_dense_f32_device(ts_ctx* ctx, const EngineJob& job, int precision, float* out);

// Tile shapes compiled into the library (id → BX×BY×BZ).
struct TileShapeInfo {
    int id, bx, by, bz;
};
const std::vector<TileShapeInfo>& tile_shapes();

template <typename Real>
int engine_run(ts_ctx* ctx, EngineJob& job, ts_eik_stats* stats);

}  // namespace eik
}  // namespace ts
