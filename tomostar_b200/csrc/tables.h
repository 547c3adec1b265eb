// Travel-time tables kept on the device (TravelTimeTableSet, Forward/TravelTimeTable.cs:247-412):
// float32 fields of (source, phase) pairs on one uniform grid, node-major per table as a .qttb
// file holds them (:57-80), in one device allocation owned by the handle.
#pragma once

#include <utility>
#include <vector>

#include "ctx.h"
#include "host_geo.h"

struct ts_tables {
    ts_ctx* ctx = nullptr;
    ts_grid def{};            // the grid (uniform: def.depth_km is null)
    int n_tables = 0;
    int64_t nodes = 0;        // nodes per table
    float* dev = nullptr;     // n_tables * nodes floats
};

namespace ts {
namespace fwd {

// The tables of `tables` ((phase, source) pairs; sources: lon, lat, depth) solved by the engine into
// tab (nodes floats per table) with the .qttb float32 rounding (TravelTimeTable.cs:264-308, :373).
template <typename Real>
int solve_tables(ts_ctx* ctx, const host::Grid& g, const double* slowness, int n_phases, int mode,
                 const std::vector<std::pair<int, int>>& tables, const double* sources, float* tab,
                 ts_eik_stats* stats);

}  // namespace fwd
}  // namespace ts
