// sort_resample.cu -- cell-key radix sort and per-cell resampling (placeholder entry points).
#include "host_util.h"

extern "C" {
MCS_API int mcs_sort_cells(mcs_pop* p, mcs_grid*) {
    return mcs::set_err(p ? p->ctx : nullptr, MCS_ERR_UNSUPPORTED, "sort not built yet");
}
MCS_API int mcs_resample_cells(mcs_pop* p, mcs_grid*, int, int) {
    return mcs::set_err(p ? p->ctx : nullptr, MCS_ERR_UNSUPPORTED, "resample not built yet");
}
}
