// diag.cu -- a self-test of the library's failure detection that faults nothing.
//
// Every wait in the kernels (the decoupled look-back of ordered appends) is bounded: when
// the iteration limit runs out the kernel raises ST_TIMEOUT, abandons the wait and returns,
// and the next synchronising call reports MCS_ERR_TIMEOUT while the context stays usable.
// mcs_diag_wait_timeout makes such waits run out on purpose, in both forms: one thread's
// (tile 1 waits for tile 0) and a warp's (tile 3 waits for tiles 0-2); nothing ever sets the
// status words waited on.
#include "host_util.h"
#include "pop_ops.h"

namespace mcs {
namespace {

__global__ void k_diag_wait(unsigned long long* tile_status, unsigned long long* tile_status_w, uint32_t* st_word,
                            uint32_t max_spins, uint32_t* prefix_out) {
    // epoch 1; the tiles waited on never publish, so each wait gives up after max_spins checks
    bool ok = true;
    uint32_t excl = 0;
    if (threadIdx.x == 0) excl = tile_lookback_from(tile_status, 0u, 1u, 1u, 5u, st_word, &ok, max_spins);
    if (threadIdx.x == 0) prefix_out[0] = ok ? excl : 0xffffffffu;
    bool okw = true;
    const uint32_t exw = tile_lookback_wait_warp(tile_status_w, 0u, 3u, 1u, 5u, st_word, &okw, max_spins);
    if (threadIdx.x == 0) prefix_out[1] = okw ? exw : 0xffffffffu;
}

}  // namespace
}  // namespace mcs

using namespace mcs;

extern "C" {

MCS_API int mcs_diag_wait_timeout(mcs_ctx* c, uint32_t max_spins) {
    if (!c || max_spins < 1 || max_spins > (1u << 20)) return MCS_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    if (int st = sync_status(c)) return st;
    unsigned long long* tiles = nullptr;   // [0..1] the one-thread wait, [2..5] the warp's
    uint32_t* out = nullptr;
    if (cudaMalloc(&tiles, 6 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&out, 2 * sizeof(uint32_t)) != cudaSuccess) {
        cudaFree(tiles);
        return set_err(c, MCS_ERR_NOMEM, "diagnostic buffers");
    }
    cudaMemsetAsync(tiles, 0, 6 * sizeof(unsigned long long), c->stream);
    k_diag_wait<<<1, 32, 0, c->stream>>>(tiles, tiles + 2, c->d_status, max_spins, out);
    cudaError_t e = cudaGetLastError();
    uint32_t prefix[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(prefix, out, sizeof(prefix), cudaMemcpyDeviceToHost, c->stream);
    const int st = sync_status(c);
    cudaFree(tiles);
    cudaFree(out);
    if (e != cudaSuccess) return set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    // both waits must have given up (flagged invalid) and reported through the status word
    if (st == MCS_ERR_TIMEOUT && prefix[0] == 0xffffffffu && prefix[1] == 0xffffffffu) return MCS_ERR_TIMEOUT;
    return st ? st : set_err(c, MCS_ERR_CUDA, "the bounded wait did not time out");
}

}  // extern "C"
