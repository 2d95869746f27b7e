// lpk_internal.h — context layout shared by the ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/lipika_cuda.h"
#include "lpk_device.cuh"

struct lpk_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    std::string err;
    // scene arena: every table of the uploaded transmitters
    std::vector<void *> scene_allocs;
    std::vector<lpk::DevTx> h_tx;
    lpk::DevTx *d_tx = nullptr;
    int32_t n_tx = 0;
    // growable device scratch for the host-buffer entry points
    void *d_scratch = nullptr;
    size_t scratch_bytes = 0;
    // pinned host staging
    void *h_pinned = nullptr;
    size_t pinned_bytes = 0;
    // last kernel time (ms) of the fan-out, for profiling hooks
    float last_kernel_ms = 0.0f;
};

namespace lpk {

lpk_status fail(lpk_ctx *ctx, lpk_status code, const std::string &msg);
lpk_status cuda_fail(lpk_ctx *ctx, cudaError_t e, const char *what);
lpk_status ensure_scratch(lpk_ctx *ctx, size_t bytes);
lpk_status ensure_pinned(lpk_ctx *ctx, size_t bytes);
lpk_status build_dev_band(lpk_ctx *ctx, const lpk_band_desc *b, int64_t i0, int64_t n, DevBand &out);
lpk_status check_active(lpk_ctx *ctx, const int32_t *active, int32_t n_active);

// launchers (lpk_kernels.cu)
cudaError_t launch_band_reference(const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                                  int32_t n_active, float2 *d_out, uint32_t *d_unocc, cudaStream_t s);
cudaError_t launch_tx_contribution(const DevBand &b, const DevTx *d_tx, int32_t tx, float2 *d_out,
                                   double *d_phase, double *d_temit, double *d_range, cudaStream_t s);
cudaError_t launch_rx_chain(const DevBand &b, float2 *d_iq, cudaStream_t s);
cudaError_t launch_solve(const DevTx *d_tx, int32_t tx, const double *d_obs, const double *d_t, int64_t n,
                         double epoch, int32_t iterations, double inv_c, double *d_temit, double *d_range,
                         cudaStream_t s);

}  // namespace lpk
