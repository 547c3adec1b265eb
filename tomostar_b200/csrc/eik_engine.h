// The tiled engine's host interface.
//
// A field of the engine owns persistent device buffers (its padded time array, per-tile due flags
// and due masks, its solve state), so a field's solve can span several launches ("epochs"): one-shot
// solves run a single epoch to completion; the serving loop runs short epochs over the fields in
// flight and admits new fields between them (continuous batching).
#pragma once

#include <vector>

#include "ctx.h"
#include "host_geo.h"
#include "ts_common.cuh"

namespace ts {
namespace eik {

struct EngineField {
    int grid = 0;                       // index into the job's grids
    const void* slowness = nullptr;     // device, Real[n] of its grid (dense grid order)
    std::vector<int32_t> seed_idx;      // merged seeds (ascending nodes)
    std::vector<double> seed_t;
    int cap = 32;                       // round cap per phase
    // Device buffers, set by engine_run (one-shot, from the context's pool) or engine_field_alloc.
    void* T = nullptr;                  // the field, padded rows (node (i,j,k) at (k*ny+j)*pitch + xoff + i)
    uint8_t* dirty = nullptr;           // one "some node due" flag per tile
    uint32_t* dmask = nullptr;          // per tile, one due bit per node
    void* state = nullptr;              // its FieldState
    void* block = nullptr;              // its own allocation (serving), freed by engine_field_free
    bool initialized = false;           // +inf, all due and seeds written
    // Its seed tiles (ascending tile id) with their fixed-node masks, for the tile shape `seed_shape`
    // (BX | BY << 8 | BZ << 16); kept between epochs.
    int seed_shape = -1;
    std::vector<int> seed_tiles;
    std::vector<uint32_t> seed_masks;
    // results
    int status = 0;                     // 1 settled, 2 refused at the cap, 0 running
    int rounds[2] = {0, 0};
};

struct EngineJob {
    std::vector<const host::Grid*> grids;
    std::vector<const host::Metric*> metrics;
    std::vector<EngineField> fields;
    double tol = 1e-7;
    double wake_rel = 0;     // 0: the reference's dirty rule (bitwise); TS_WAKE_REL for TS_MODE_FAST
    int tile = 0;            // tile shape id
    // Set by the engine: the padded layout of each grid's fields.
    std::vector<int> pitch;
    int xoff = 0;
};

// Tile shapes compiled into the library (id → BX×BY×BZ).
struct TileShapeInfo {
    int id, bx, by, bz;
};
const std::vector<TileShapeInfo>& tile_shapes();

// Layout of a field on a grid for a tile shape and precision: elements per padded row, x offset,
// tiles, due-mask words per tile.
struct FieldLayout {
    int pitch, xoff, tiles, mask_words;
    int64_t rows_;  // ny * nz
    int64_t elems() const;
    int64_t bytes(int precision) const;  // the whole allocation: time array, flags, masks, state
};
FieldLayout field_layout(const host::Grid& g, int tile, int precision);

// One-shot: allocates every field's buffers from the context's pool and runs to completion.
template <typename Real>
int engine_run(ts_ctx* ctx, EngineJob& job, ts_eik_stats* stats);

// One epoch over the given fields (whose buffers are set): new fields are initialised, then at
// most max_rounds rounds run (<= 0: until every field is done). Statuses and rounds are read back.
template <typename Real>
int engine_epoch(ts_ctx* ctx, const std::vector<const host::Grid*>& grids,
                 const std::vector<const host::Metric*>& metrics, const std::vector<EngineField*>& fields,
                 double tol, double wake_rel, int tile, int max_rounds, ts_eik_stats* stats, cudaStream_t s);

// Points a field's buffers into one device block of field_layout(...).bytes(precision) bytes.
void engine_field_place(EngineField& f, const FieldLayout& L, int precision, void* block);

// One-shot with the results to page-locked host memory: the fields are solved in two halves and the
// first half's fields are converted and copied to the host (on a second stream) while the second
// half is solved. out: the fields one after another in dense grid order, of out_type.
template <typename Real>
int engine_run_to_host(ts_ctx* ctx, EngineJob& job, void* out, int out_type, ts_eik_stats* stats);

// Copies padded engine fields to dense grid order (converting to out_type, TS_OUT_F64 / TS_OUT_F32).
int fields_to_dense_host(ts_ctx* ctx, const EngineJob& job, int precision, void* out, int out_type);
int fields_to_dense_f32_device(ts_ctx* ctx, const EngineJob& job, int precision, float* out);
// One field, padded → dense float32 on the device (on stream s).
int field_to_dense_f32_device(ts_ctx* ctx, const host::Grid& g, const FieldLayout& L, const void* T, int precision,
                              float* out, cudaStream_t s);

}  // namespace eik
}  // namespace ts
