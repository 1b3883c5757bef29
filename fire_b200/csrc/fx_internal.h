// fx_internal.h — host-side declarations shared by the engine and the kernel files.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "fx_device.cuh"

// Batched step passes (fx_kernels.cu). `bricks` is the batch's brick total for the
// pass's shape; grids are persistent (full residency) capped at that total.
void fx_launch_step_begin(cudaStream_t s, FxBatchDev* B);
void fx_launch_step_end(cudaStream_t s, FxBatchDev* B);
void fx_launch_step_tables(cudaStream_t s, const FxBatchDev* B, int bricks);
// The source pass with bricks of 32 x by x (8 / by) cells (by = 2, 4 or 8).
// early: the neighbour terms before the advection (fx_simulate_cell<EARLY>; same results;
// FP32 storage only, mixed storage always takes the reference order).
void fx_launch_simulate(cudaStream_t s, int storage, int by, bool early, const FxBatchDev* B, int bricks);
void fx_launch_divergence(cudaStream_t s, const FxBatchDev* B, int bricks, int phase);
void fx_launch_jacobi(cudaStream_t s, bool half, const FxBatchDev* B, int bricks, int phase, int launch, int sweep);
// One sweep by z-marching tiles of zc planes (fx_jacobi_zm.cuh).
void fx_launch_jacobi_zm(cudaStream_t s, bool half, const FxBatchDev* B, int bricks, int phase, int launch, int sweep,
                         int zc);
// K fused sweeps per launch; pmode selects the pressure storage and rounding.
enum { FX_TB_F32 = 0, FX_TB_F16_ROUND = 1, FX_TB_F16 = 2 };
// Two sweeps per launch (k = 2); with tma (FP32 pressure only) the planes are staged by TMA.
bool fx_launch_jacobi_tb(cudaStream_t s, int pmode, int k, const FxBatchDev* B, int bricks, int phase, int launch, int zc,
                         bool tma);
// Tensor maps of a simulation's pressure pair, correction pair and divergence for the
// TMA-staged two-sweep pass; false when the driver refuses one (the pass then uses cp.async).
bool fx_make_tensor_maps(FxSimDev* h);
void fx_launch_project(cudaStream_t s, bool half, const FxBatchDev* B, int bricks, int phase);
// The primary projection (phase 0) and the divergence of its result (the residual solve's
// right-hand side) in one pass.
void fx_launch_project_div(cudaStream_t s, bool half, const FxBatchDev* B, int bricks);
// Every sweep of a phase in one cooperative launch of `ctas` CTAs with `smem` bytes of
// dynamic shared memory (fx_jacobi_res.cuh; variant 0 column, 1 faces-first, 2 faces-first
// for small boxes, 3 faces-first with interior columns, 4 variant 3 with a copy warp);
// fx_res_capacity: the most CTAs of that variant one such launch can hold resident on this
// device (0 when unavailable). epi (variant 4, residual phase): the launch also projects the
// flow with the final correction (fx_res_project_epi), replacing fx_launch_project's phase 1.
cudaError_t fx_launch_jacobi_res(cudaStream_t s, bool half, int variant, const FxBatchDev* B, int ctas, int phase,
                                 int smem, bool epi);
int fx_res_capacity(bool half, int variant);

// Single-simulation utilities.
void fx_launch_init(cudaStream_t s, int storage, const FxSimDev* S, float tAmbient, float oxygen, float noise);
void fx_launch_emitter_mask(cudaStream_t s, const FxSimDev* S, uint8_t* mask);
void fx_launch_final_divergence(cudaStream_t s, const FxSimDev* S, float* out);
// The particle passes of every member whose water runs (liquid clear, density,
// integration, deposition), before simulate (fx_sph.cuh).
void fx_launch_sph(cudaStream_t s, const FxBatchDev* B, int rowBricks, int partBricks);
// Render volumes: one simulation (a read), or every packing member of a batch (step end).
void fx_launch_pack_sim(cudaStream_t s, const FxSimDev* S);
void fx_launch_pack_batch(cudaStream_t s, const FxBatchDev* B, int bricks);
int fx_norm_partial_blocks(long long cells);
void fx_launch_divergence_norm(cudaStream_t s, const FxSimDev* S, long long cells, double* partial, double* out);
void fx_launch_upload_desc(cudaStream_t s, const FxSimDev& host, FxSimDev* dev);
void fx_launch_upload_batch(cudaStream_t s, const FxBatchDev& host, FxBatchDev* dev);

// Exhaustive check of fx_div_by_const against IEEE division for one denominator.
void fx_launch_check_div(cudaStream_t s, float d, float rcp, float lo, float hi, unsigned long long* mismatches);

// Sets the text that firex_last_error(NULL) returns on the calling thread (fx_engine.cu).
void fx_set_thread_error(const std::string& msg);
