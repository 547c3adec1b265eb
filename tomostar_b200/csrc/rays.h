// Host interface of the ray pipeline (rays.cu).
#pragma once

#include "ctx.h"
#include "host_geo.h"

namespace ts {
namespace rays {

struct RayStats {
    double device_ms = 0;
    int retraced_chunks = 0;
};

// Traces n_rays rays on device-resident float32 tables (n_tables fields on fwd) and builds their
// CSR rows on the inversion grid; host arrays: table_station (3 per table), table_of and events.
int trace_on_device(ts_ctx* ctx, const host::Grid& fwd, const float* tables_dev, int n_tables,
                    const double* table_station_host, const host::Grid& inv, int n_rays, const int32_t* table_of_host,
                    const double* events_host, double step_km, ts_rows** out, RayStats* st);

}  // namespace rays
}  // namespace ts
