// fx_internal.h — host-side declarations shared by the engine and the kernel files.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fx_device.cuh"

// ---- plain FP32 passes (fx_kernels_f32.cu) -------------------------------------------------
void fx_launch_simulate_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flowIn, const float4* speciesIn,
                            const uint32_t* liquid, float4* flowOut, float4* speciesOut, float* reaction);
void fx_launch_divergence_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flow, float* div);
void fx_launch_jacobi_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float* pin, const float* div, float* pout);
void fx_launch_project_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flowIn, const float* p,
                           float4* flowOut);
void fx_launch_init(cudaStream_t s, FxGrid g, float4* flow, float4* species, uint64_t seed, float noise, float tAmbient,
                    float oxygen);
void fx_launch_emitter_mask(cudaStream_t s, const FxParams* prm, FxGrid g, uint8_t* mask);
int fx_norm_partial_blocks(FxGrid g);
void fx_launch_divergence_norm(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flow, double* partial,
                               double* out);
void fx_launch_upload_params(cudaStream_t s, const FxParams& host, FxParams* dev);
