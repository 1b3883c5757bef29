// fx_storage.cuh — storage layouts of the step's fields.
//
// F32  : flow float4 (u v w T), species float4 — the reference's storage buffers.
// MIXED: flow float4 (u v w T: velocity and temperature share one 16-byte record, so T
//        stays FP32 at no byte cost), species 4 x FP16 (8 B), pressure and residual
//        pressure FP16; divergence, reaction and all arithmetic FP32.
// FP16 stores round to nearest even.
#pragma once

#include "fx_device.cuh"

struct StF32 {
    static constexpr int kStorage = FX_STORAGE_F32;
    FXD static float4 ld_species(const void* b, long long i) { return __ldg(reinterpret_cast<const float4*>(b) + i); }
    FXD static void st_species(void* b, long long i, float4 v) { reinterpret_cast<float4*>(b)[i] = v; }
};

struct StMixed {
    static constexpr int kStorage = FX_STORAGE_MIXED;
    FXD static float4 ld_species(const void* b, long long i) {
        uint2 r = __ldg(reinterpret_cast<const uint2*>(b) + i);
        __half2 a = *reinterpret_cast<__half2*>(&r.x);
        __half2 c = *reinterpret_cast<__half2*>(&r.y);
        float2 fa = __half22float2(a), fc = __half22float2(c);
        return make_float4(fa.x, fa.y, fc.x, fc.y);
    }
    FXD static void st_species(void* b, long long i, float4 v) {
        __half2 a = __floats2half2_rn(v.x, v.y);
        __half2 c = __floats2half2_rn(v.z, v.w);
        uint2 r;
        r.x = *reinterpret_cast<uint32_t*>(&a);
        r.y = *reinterpret_cast<uint32_t*>(&c);
        reinterpret_cast<uint2*>(b)[i] = r;
    }
};

FXD float4 fx_ld_flow(const void* b, long long i) { return __ldg(reinterpret_cast<const float4*>(b) + i); }
FXD void fx_st_flow(void* b, long long i, float4 v) { reinterpret_cast<float4*>(b)[i] = v; }

// Pressure element access: float or half storage, 1 or 4 consecutive cells (4-aligned).
template <typename PT>
struct PStore;
template <>
struct PStore<float> {
    FXD static float ld(const void* b, long long i) { return __ldg(reinterpret_cast<const float*>(b) + i); }
    FXD static float4 ld4(const void* b, long long i) { return __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const float*>(b) + i)); }
    FXD static void st4(void* b, long long i, float4 v) { *reinterpret_cast<float4*>(reinterpret_cast<float*>(b) + i) = v; }
    FXD static float round(float v) { return v; }
};
template <>
struct PStore<__half> {
    FXD static float ld(const void* b, long long i) { return __half2float(__ldg(reinterpret_cast<const __half*>(b) + i)); }
    FXD static float4 ld4(const void* b, long long i) {
        uint2 r = __ldg(reinterpret_cast<const uint2*>(reinterpret_cast<const __half*>(b) + i));
        float2 a = __half22float2(*reinterpret_cast<__half2*>(&r.x));
        float2 c = __half22float2(*reinterpret_cast<__half2*>(&r.y));
        return make_float4(a.x, a.y, c.x, c.y);
    }
    FXD static void st4(void* b, long long i, float4 v) {
        __half2 a = __floats2half2_rn(v.x, v.y), c = __floats2half2_rn(v.z, v.w);
        uint2 r;
        r.x = *reinterpret_cast<uint32_t*>(&a);
        r.y = *reinterpret_cast<uint32_t*>(&c);
        *reinterpret_cast<uint2*>(reinterpret_cast<__half*>(b) + i) = r;
    }
    FXD static float round(float v) { return __half2float(__float2half_rn(v)); }
};
