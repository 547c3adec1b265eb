// Host interface of the ray pipeline (rays.cu).
#pragma once

#include "ctx.h"
#include "host_geo.h"

#include <vector>

namespace ts {
namespace rays {

struct RayStats {
    double device_ms = 0;   // from the first kernel to the row offsets on the stream (events)
    double setup_ms = 0;    // host: per-ray record rooms and the table order
    double wall_ms = 0;     // the whole call on the host
    int chunks = 0;
    int retraced_chunks = 0;
    unsigned long long steps = 0;  // back-tracing steps taken (rays traced again count again)
};

// Traces n_rays rays on device-resident float32 tables (n_tables fields on fwd) and builds their
// CSR rows on the inversion grid; host arrays: table_station (3 per table), table_of and events.
// With a background set on the context (ts_set_background) pieces outside the inversion grid give
// time outside instead of row entries, at the Vp (table phase 0) or Vs (1) of the background.
int trace_on_device(ts_ctx* ctx, const host::Grid& fwd, const float* tables_dev, int n_tables,
                    const double* table_station_host, const host::Grid& inv, int n_rays, const int32_t* table_of_host,
                    const double* events_host, double step_km, ts_rows** out, RayStats* st,
                    const int32_t* table_phase_host = nullptr);

// The same with each table in a buffer of its own (tables[t] on the device).
int trace_on_device(ts_ctx* ctx, const host::Grid& fwd, const std::vector<const float*>& tables,
                    const double* table_station_host, const host::Grid& inv, int n_rays, const int32_t* table_of_host,
                    const double* events_host, double step_km, ts_rows** out, RayStats* st,
                    const int32_t* table_phase_host = nullptr);

// Cuts a result into consecutive row ranges [row_begin[k], row_begin[k+1]), each a result of its
// own (stream-ordered copies on the context's stream).
int split_rows(ts_ctx* ctx, const ts_rows* all, const std::vector<int>& row_begin, std::vector<ts_rows*>& parts);
void free_rows(ts_rows* rows);
// The device arrays of a result (row_ptr[n_rows + 1], col[nnz], len[nnz]).
void rows_view(const ts_rows* rows, int* n_rows, int64_t* nnz, const int** row_ptr, const int** col, const float** len);

}  // namespace rays
}  // namespace ts
