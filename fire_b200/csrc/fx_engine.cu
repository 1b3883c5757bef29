// fx_engine.cpp — the Fire-X engine behind the C ABI (include/firex.h).
//
// Host-side counterpart of FireXEngine (src/sim/firex/FireXEngine.ts): named parameters
// with the reference's clamps, the 44-float uniform block, resource allocation with
// transactional failure, reset, and the per-step dispatch graph with its ping-pong
// parity and pressure branches. All device work is queued on the handle's own stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/firex.h"
#include "fx_internal.h"

namespace {

thread_local std::string g_create_error;

// ---- named parameters -------------------------------------------------------------------
// FireXEngine.parameters defaults (FireXEngine.ts:422-451) and setParameter's rules
// (FireXEngine.ts:937-1032). Values stay doubles (JS numbers) until the uniform block.
enum ParamRule { CLAMP, FREE, ROUND_CLAMP, BOOLEAN, THRESHOLD, OPTICAL, IMPERIAL };
struct ParamSpec {
    const char* name;
    double def;
    double lo, hi;
    ParamRule rule;
};
constexpr ParamSpec kParams[] = {
    {"burnerSize", 3.1, 0.35, 3.2, CLAMP},        {"burnerDepth", 2.7, 0.35, 3.2, CLAMP},
    {"sourceThickness", 1.35, 0.35, 2.5, CLAMP},  {"firePower", 2.5, 0.1, 4, CLAMP},
    {"sourceLift", 1.6, 0, 4, CLAMP},             {"buoyancyScale", 2.15, 0, 4, CLAMP},
    {"flamePersistence", 1.45, 0.4, 3, CLAMP},    {"airEntrainment", 1.65, 0, 3, CLAMP},
    {"fuelRate", 0.30, 0, 0, FREE},               {"oxygenRate", 1, 0, 0, FREE},
    {"heatEfficiency", 0.86, 0, 0, FREE},         {"vorticity", 3.6, 0, 0, FREE},
    {"waterFlow", 0, 0, 0, FREE},                 {"sprayAngle", 10, 0, 0, FREE},
    {"waterEnabled", 0, 0, 0, BOOLEAN},           {"cameraYaw", -0.34, 0, 0, FREE},
    {"cameraPitch", 0.03, 0, 0, FREE},            {"cameraDistance", 4.9, 0, 0, FREE},
    {"viewMode", 0, 0, 7, ROUND_CLAMP},           {"aimHeight", 0.42, 0.08, 0.82, CLAMP},
    {"nozzleType", 0, 0, 0, THRESHOLD},           {"exposure", 1.25, 0.25, 3, CLAMP},
    {"frontDefinition", 1.65, 0.5, 2.5, CLAMP},   {"opticalDetailTarget", 1024, 0, 0, OPTICAL},
    {"domainWidth", 1.15, 0.5, 4, CLAMP},         {"domainHeight", 1.35, 0.5, 6, CLAMP},
    {"domainDepth", 1.15, 0.5, 4, CLAMP},         {"displayImperial", 0, 0, 0, IMPERIAL},
    {"viewZoom", 2.1, 0.5, 5, CLAMP},
};
constexpr int kNumParams = sizeof(kParams) / sizeof(kParams[0]);

int param_slot(const char* name) {
    for (int i = 0; i < kNumParams; ++i)
        if (std::strcmp(kParams[i].name, name) == 0) return i;
    return -1;
}

double apply_rule(const ParamSpec& s, double current, int kind, double v) {
    const bool number = kind == FIREX_VALUE_NUMBER;
    auto finite_or = [&](double fb) { return (number && std::isfinite(v)) ? v : fb; };
    switch (s.rule) {
        case CLAMP: return std::max(s.lo, std::min(s.hi, finite_or(current)));
        case FREE: return finite_or(current);
        case ROUND_CLAMP: return std::max(s.lo, std::min(s.hi, std::round(finite_or(current))));
        case BOOLEAN: return kind == FIREX_VALUE_BOOLEAN ? (v != 0 ? 1.0 : 0.0) : current;
        case THRESHOLD: return finite_or(current) >= 0.5 ? 1.0 : 0.0;
        case OPTICAL: {
            double t = finite_or(current);
            return t >= 768 ? 1024 : t >= 384 ? 512 : t >= 192 ? 256 : 0;
        }
        case IMPERIAL: return kind == FIREX_VALUE_BOOLEAN ? (v != 0 ? 1.0 : 0.0) : (finite_or(0) >= 0.5 ? 1.0 : 0.0);
    }
    return current;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

struct firex_sim {
    int X = 0, Y = 0, Z = 0;
    long long N = 0;
    firex_options opt{};
    int mode = FIREX_PRESSURE_WARM_F32;
    int device = 0;
    double named[kNumParams];

    double simTime = 0;
    int64_t frame = 0;
    int speciesIndex = 0, pressureIndex = 0;
    int lastCorrection = 0;
    bool lastCorrectionShared = false;

    cudaStream_t stream = nullptr;
    std::vector<void*> allocations;
    size_t bytes = 0;
    float4* flow[2] = {nullptr, nullptr};
    float4* species[2] = {nullptr, nullptr};
    float* pressure[2] = {nullptr, nullptr};
    float* correction[2] = {nullptr, nullptr};
    float* div = nullptr;
    float* reaction = nullptr;
    uint32_t* liquid = nullptr;
    FxParams* d_params = nullptr;
    double* d_partial = nullptr;
    double* d_norm = nullptr;
    float* d_tmp = nullptr;

    std::string err;
    bool poisoned = false;

    // Per-pass profiling: an event is recorded at every pass boundary; the elapsed time
    // between consecutive events is charged to the pass that ran between them.
    bool profiling = false;
    std::vector<cudaEvent_t> evPool;
    std::vector<std::pair<cudaEvent_t, int>> evMarks;  // (event, pass that ends here)
    size_t evUsed = 0;
    double passMs[FIREX_PASS_COUNT] = {0};
    int64_t passLaunches[FIREX_PASS_COUNT] = {0};
    int64_t pendingLaunches[FIREX_PASS_COUNT] = {0};

    void mark(int pass, int launches) {
        pendingLaunches[pass] += launches;
        if (!profiling) return;
        if (evUsed == evPool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            evPool.push_back(e);
        }
        cudaEvent_t e = evPool[evUsed++];
        cudaEventRecord(e, stream);
        evMarks.emplace_back(e, pass);
    }
    void begin_marks() {
        if (!profiling) return;
        if (evUsed == evPool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            evPool.push_back(e);
        }
        cudaEvent_t e = evPool[evUsed++];
        cudaEventRecord(e, stream);
        evMarks.emplace_back(e, -1);
    }
    int collect_marks() {
        cudaError_t err = cudaStreamSynchronize(stream);
        if (err != cudaSuccess) return cuda_fail(err, "pass_times");
        for (size_t i = 1; i < evMarks.size(); ++i) {
            if (evMarks[i].second < 0) continue;
            float ms = 0;
            cudaEventElapsedTime(&ms, evMarks[i - 1].first, evMarks[i].first);
            passMs[evMarks[i].second] += ms;
        }
        evMarks.clear();
        evUsed = 0;
        for (int p = 0; p < FIREX_PASS_COUNT; ++p) {
            passLaunches[p] += pendingLaunches[p];
            pendingLaunches[p] = 0;
        }
        return FIREX_OK;
    }

    FxGrid grid() const { return FxGrid{X, Y, Z}; }

    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        poisoned = true;
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return FIREX_ERR_CUDA;
    }

    template <typename T>
    T* alloc(size_t n) {
        if (n == 0) n = 1;
        void* p = nullptr;
        if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        allocations.push_back(p);
        bytes += n * sizeof(T);
        return static_cast<T*>(p);
    }

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        for (cudaEvent_t e : evPool) cudaEventDestroy(e);
        evPool.clear();
        evMarks.clear();
        for (void* p : allocations) cudaFree(p);
        allocations.clear();
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    // Bytes the resource set needs (what create allocates), for admission.
    static size_t planned_bytes(long long N, int mode) {
        size_t b = (size_t)N * (16 * 4 + 4 * 2 /*div, reaction*/ + 4 /*liquid*/ + 4 /*tmp*/);
        if (mode == FIREX_PRESSURE_WARM_F32) b += (size_t)N * 16;  // 2 pressure + 2 correction
        else b += (size_t)N * 8;                                    // 2 pressure (shared in branch C)
        return b + 64 * 1024;
    }

    // writeUniforms (FireXEngine.ts:2043-2113) plus the emitter extension.
    void build_params(FxParams& p, double dt) const {
        std::memset(&p, 0, sizeof(p));
        auto P = [&](const char* n) { return named[param_slot(n)]; };
        const double cells = (double)X * (double)Y * (double)Z;
        const double u[FIREX_UNIFORM_FLOATS] = {
            (double)X, (double)Y, (double)Z, cells,
            (double)dt, simTime, (double)frame, (double)dt,
            P("fuelRate"), P("oxygenRate"), P("heatEfficiency"), P("vorticity"),
            P("waterFlow"), (P("sprayAngle") * M_PI) / 180, P("waterEnabled") != 0 ? 1.0 : 0.0, 300,
            P("cameraYaw"), P("cameraPitch"), P("cameraDistance"), 1,  // canvas aspect (presentation only)
            1, 1, 0, 0,                                                // canvas size, rays, particles
            P("viewMode"), P("aimHeight"), P("nozzleType"), P("exposure"),
            P("burnerSize"), P("burnerDepth"), P("sourceThickness"), P("firePower"),
            P("domainWidth"), P("domainHeight"), P("domainDepth"), 0,
            P("sourceLift"), P("buoyancyScale"), P("flamePersistence"), P("viewZoom"),
            P("airEntrainment"), P("frontDefinition"), opt.cinematic ? 1.0 : 0.0, P("opticalDetailTarget")};
        for (int i = 0; i < FIREX_UNIFORM_FLOATS; ++i) p.u[i] = (float)u[i];
        p.emitter_mode = opt.emitter_mode;
        p.num_spheres = opt.emitter_mode == FIREX_EMITTER_SPHERES ? opt.num_spheres : 0;
        for (int s = 0; s < FIREX_MAX_SPHERES; ++s) p.spheres[s] = opt.spheres[s];
        p.jitter = jitter(frame);
    }

    // Seeded per-step emission factor in [1-a, 1+a] (extension): splitmix64 of the frame
    // index, 24 random bits.
    float jitter(int64_t f) const {
        auto mix = [](uint64_t z) {
            z += 0x9E3779B97F4A7C15ull;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            return z ^ (z >> 31);
        };
        uint64_t h = mix(mix(opt.seed ^ 0xBB67AE8584CAA73Bull) + (uint64_t)f);
        float u = (float)(h >> 40) * (1.0f / 16777216.0f);
        return 1.0f + opt.emission_jitter * (2.0f * u - 1.0f);
    }

    int reset() {
        simTime = 0;
        frame = 0;
        speciesIndex = 0;
        pressureIndex = 0;
        lastCorrection = 0;
        lastCorrectionShared = mode == FIREX_PRESSURE_COLD_F32;
        // clearBuffer on every field, then initializeFields (FireXEngine.ts:1948-1969)
        const size_t v4 = (size_t)N * 16, s4 = (size_t)N * 4;
        cudaMemsetAsync(flow[0], 0, v4, stream);
        cudaMemsetAsync(flow[1], 0, v4, stream);
        cudaMemsetAsync(species[0], 0, v4, stream);
        cudaMemsetAsync(species[1], 0, v4, stream);
        for (int i = 0; i < 2; ++i) {
            cudaMemsetAsync(pressure[i], 0, s4, stream);
            if (correction[i] && correction[i] != pressure[i]) cudaMemsetAsync(correction[i], 0, s4, stream);
        }
        cudaMemsetAsync(div, 0, s4, stream);
        cudaMemsetAsync(reaction, 0, s4, stream);
        cudaMemsetAsync(liquid, 0, s4, stream);
        const float oxygen = (float)named[param_slot("oxygenRate")];
        fx_launch_init(stream, grid(), flow[0], species[0], opt.seed, opt.velocity_noise, 300.0f, oxygen);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "reset");
        return FIREX_OK;
    }

    // One encodeSimulationStep (FireXEngine.ts:2115-2276) with copyFlow replaced by a
    // swap of the flow[0] / flow[1] roles.
    void enqueue_step(double dt) {
        FxParams hp;
        build_params(hp, dt);
        begin_marks();
        fx_launch_upload_params(stream, hp, d_params);
        mark(FIREX_PASS_OTHER, 1);
        const FxGrid g = grid();
        const int s = speciesIndex;
        fx_launch_simulate_f32(stream, d_params, g, flow[0], species[s], liquid, flow[1], species[1 - s], reaction);
        mark(FIREX_PASS_SIMULATE, 1);
        speciesIndex = 1 - s;
        fx_launch_divergence_f32(stream, d_params, g, flow[1], div);
        mark(FIREX_PASS_DIVERGENCE, 1);
        const int P = opt.pressure_iterations, R = opt.correction_iterations;
        const size_t s4 = (size_t)N * 4;
        if (mode == FIREX_PRESSURE_COLD_F32) {
            cudaMemsetAsync(pressure[0], 0, s4, stream);
            pressureIndex = 0;
            mark(FIREX_PASS_OTHER, 0);
        }
        for (int i = 0; i < P; ++i) {
            fx_launch_jacobi_f32(stream, d_params, g, pressure[pressureIndex], div, pressure[1 - pressureIndex]);
            pressureIndex = 1 - pressureIndex;
        }
        mark(FIREX_PASS_JACOBI, P);
        fx_launch_project_f32(stream, d_params, g, flow[1], pressure[pressureIndex], flow[0]);
        mark(FIREX_PASS_PROJECT, 1);
        fx_launch_divergence_f32(stream, d_params, g, flow[0], div);
        mark(FIREX_PASS_DIVERGENCE, 1);
        float** corr = (mode == FIREX_PRESSURE_COLD_F32) ? pressure : correction;
        cudaMemsetAsync(corr[0], 0, s4, stream);
        mark(FIREX_PASS_OTHER, 0);
        int ci = 0;
        for (int i = 0; i < R; ++i) {
            fx_launch_jacobi_f32(stream, d_params, g, corr[ci], div, corr[1 - ci]);
            ci = 1 - ci;
        }
        mark(FIREX_PASS_JACOBI, R);
        fx_launch_project_f32(stream, d_params, g, flow[0], corr[ci], flow[1]);
        mark(FIREX_PASS_PROJECT, 1);
        std::swap(flow[0], flow[1]);
        lastCorrection = ci;
        lastCorrectionShared = mode == FIREX_PRESSURE_COLD_F32;
        simTime += dt;
        frame += 1;
    }
};

// ---- C ABI ---------------------------------------------------------------------------------
extern "C" {

void firex_default_options(firex_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = FIREX_PRECISION_F32;
    o->pressure_mode = FIREX_PRESSURE_AUTO;
    o->pressure_iterations = 64;
    o->correction_iterations = 64;
    o->emitter_mode = FIREX_EMITTER_BURNER;
    o->cinematic = 1;
}

size_t firex_field_element_size(int32_t field) {
    switch (field) {
        case FIREX_FIELD_FLOW:
        case FIREX_FIELD_SPECIES: return 16;
        case FIREX_FIELD_PRESSURE:
        case FIREX_FIELD_DIVERGENCE:
        case FIREX_FIELD_REACTION:
        case FIREX_FIELD_LIQUID:
        case FIREX_FIELD_CORRECTION:
        case FIREX_FIELD_FINAL_DIVERGENCE: return 4;
        case FIREX_FIELD_EMITTER_MASK: return 1;
    }
    return 0;
}

uint64_t firex_reference_memory_estimate(const int32_t dims[3], int64_t particle_count) {
    if (!dims) return 0;
    uint64_t cells = (uint64_t)std::max(dims[0], 0) * (uint64_t)std::max(dims[1], 0) * (uint64_t)std::max(dims[2], 0);
    uint64_t per = cells >= (uint64_t)FIREX_HEAVY_GRID_CELL_THRESHOLD ? 108 : 116;
    return cells * per + (uint64_t)std::max<int64_t>(particle_count, 0) * 80 + 64ull * 64 * 64 * 4;
}

int firex_create(const int32_t dims[3], const firex_options* opt, firex_sim** out) {
    if (!out) return FIREX_ERR_BAD_ARG;
    *out = nullptr;
    if (!dims || !opt) {
        g_create_error = "dims and options are required";
        return FIREX_ERR_BAD_ARG;
    }
    for (int i = 0; i < 3; ++i)
        if (dims[i] <= 0 || dims[i] % 4 != 0 || dims[i] > 2048) {
            g_create_error = "grid axes must be positive multiples of 4 and at most 2048";
            return FIREX_ERR_BAD_ARG;
        }
    if (opt->pressure_iterations < 0 || opt->correction_iterations < 0 || opt->num_spheres < 0 ||
        opt->num_spheres > FIREX_MAX_SPHERES || (opt->emitter_mode != FIREX_EMITTER_BURNER && opt->emitter_mode != FIREX_EMITTER_SPHERES) ||
        opt->pressure_mode < FIREX_PRESSURE_AUTO || opt->pressure_mode > FIREX_PRESSURE_COLD_F32 ||
        !(opt->velocity_noise >= 0) || !(opt->emission_jitter >= 0)) {
        g_create_error = "invalid options";
        return FIREX_ERR_BAD_ARG;
    }
    const long long N = (long long)dims[0] * dims[1] * dims[2];
    if (N >= (1LL << 31)) {
        g_create_error = "grid has 2^31 cells or more";
        return FIREX_ERR_BAD_ARG;
    }
    int mode = opt->pressure_mode;
    if (mode == FIREX_PRESSURE_AUTO) mode = N >= FIREX_HEAVY_GRID_CELL_THRESHOLD ? FIREX_PRESSURE_F16 : FIREX_PRESSURE_WARM_F32;
    if (mode == FIREX_PRESSURE_F16 || opt->precision != FIREX_PRECISION_F32) {
        g_create_error = "f16 pressure storage and mixed precision are not available in this build";
        return FIREX_ERR_UNSUPPORTED;
    }
    const size_t need = firex_sim::planned_bytes(N, mode);
    if (opt->memory_budget_bytes && need > opt->memory_budget_bytes) {
        g_create_error = "grid needs " + std::to_string(need) + " device bytes, above the " +
                         std::to_string(opt->memory_budget_bytes) + "-byte budget";
        return FIREX_ERR_BUDGET;
    }
    firex_sim* s = new (std::nothrow) firex_sim();
    if (!s) return FIREX_ERR_OOM;
    s->X = dims[0];
    s->Y = dims[1];
    s->Z = dims[2];
    s->N = N;
    s->opt = *opt;
    s->mode = mode;
    for (int i = 0; i < kNumParams; ++i) s->named[i] = kParams[i].def;
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        g_create_error = std::string("CUDA unavailable: ") + cudaGetErrorString(e);
        cudaGetLastError();
        delete s;
        return FIREX_ERR_CUDA;
    }
    size_t freeB = 0, totalB = 0;
    if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess && need > freeB) {
        g_create_error = "grid needs " + std::to_string(need) + " device bytes, " + std::to_string(freeB) + " free";
        s->release();
        delete s;
        return FIREX_ERR_OOM;
    }
    bool ok = true;
    for (int i = 0; i < 2 && ok; ++i) {
        ok = (s->flow[i] = s->alloc<float4>(N)) && (s->species[i] = s->alloc<float4>(N)) &&
             (s->pressure[i] = s->alloc<float>(N));
        if (ok && mode == FIREX_PRESSURE_WARM_F32) ok = (s->correction[i] = s->alloc<float>(N)) != nullptr;
        if (ok && mode == FIREX_PRESSURE_COLD_F32) s->correction[i] = s->pressure[i];
    }
    ok = ok && (s->div = s->alloc<float>(N)) && (s->reaction = s->alloc<float>(N)) && (s->liquid = s->alloc<uint32_t>(N)) &&
         (s->d_tmp = s->alloc<float>(N)) && (s->d_params = s->alloc<FxParams>(1)) &&
         (s->d_partial = s->alloc<double>(2 * (size_t)fx_norm_partial_blocks(s->grid()))) && (s->d_norm = s->alloc<double>(2));
    if (!ok) {
        g_create_error = "device allocation failed (" + std::to_string(need) + " bytes requested)";
        s->release();
        delete s;
        return FIREX_ERR_OOM;
    }
    int rc = s->reset();
    if (rc == FIREX_OK) {
        e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = s->cuda_fail(e, "initialise");
    }
    if (rc != FIREX_OK) {
        g_create_error = s->err;
        s->release();
        delete s;
        return rc;
    }
    *out = s;
    return FIREX_OK;
}

int firex_destroy(firex_sim* s) {
    if (!s) return FIREX_ERR_BAD_ARG;
    {
        DeviceGuard dg(s->device);
        s->release();
    }
    delete s;
    return FIREX_OK;
}

const char* firex_last_error(const firex_sim* s) { return s ? s->err.c_str() : g_create_error.c_str(); }

int firex_set_parameter(firex_sim* s, const char* name, int32_t kind, double value) {
    if (!s || !name) return FIREX_ERR_BAD_ARG;
    int i = param_slot(name);
    if (i < 0) return FIREX_OK;  // unknown names are ignored (FireXEngine.ts:1029-1030)
    s->named[i] = apply_rule(kParams[i], s->named[i], kind, value);
    return FIREX_OK;
}

int firex_get_parameter(const firex_sim* s, const char* name, double* value) {
    if (!s || !name || !value) return FIREX_ERR_BAD_ARG;
    int i = param_slot(name);
    if (i < 0) return FIREX_ERR_BAD_ARG;
    *value = s->named[i];
    return FIREX_OK;
}

int firex_reset(firex_sim* s) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    DeviceGuard dg(s->device);
    return s->reset();
}

int firex_step(firex_sim* s, int32_t nsteps, double dt) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    if (nsteps < 0 || !std::isfinite(dt) || dt < 0) return s->fail(FIREX_ERR_BAD_ARG, "step count and dt must be finite and non-negative");
    DeviceGuard dg(s->device);
    for (int i = 0; i < nsteps; ++i) s->enqueue_step(dt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return s->cuda_fail(e, "step launch");
    return FIREX_OK;
}

int firex_sync(firex_sim* s) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    DeviceGuard dg(s->device);
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return s->cuda_fail(e, "sync");
    return FIREX_OK;
}

static int field_ptr(firex_sim* s, int32_t field, bool writing, void** ptr) {
    switch (field) {
        case FIREX_FIELD_FLOW: *ptr = s->flow[0]; return FIREX_OK;
        case FIREX_FIELD_SPECIES: *ptr = s->species[s->speciesIndex]; return FIREX_OK;
        case FIREX_FIELD_PRESSURE: *ptr = s->pressure[s->pressureIndex]; return FIREX_OK;
        case FIREX_FIELD_DIVERGENCE: *ptr = s->div; return FIREX_OK;
        case FIREX_FIELD_REACTION: *ptr = s->reaction; return FIREX_OK;
        case FIREX_FIELD_LIQUID: *ptr = s->liquid; return FIREX_OK;
        case FIREX_FIELD_CORRECTION:
            if (writing) return FIREX_ERR_BAD_ARG;
            *ptr = s->lastCorrectionShared ? s->pressure[s->lastCorrection] : s->correction[s->lastCorrection];
            return FIREX_OK;
        case FIREX_FIELD_EMITTER_MASK:
            if (writing) return FIREX_ERR_BAD_ARG;
            {
                FxParams hp;
                s->build_params(hp, 0.0f);
                fx_launch_upload_params(s->stream, hp, s->d_params);
                fx_launch_emitter_mask(s->stream, s->d_params, s->grid(), reinterpret_cast<uint8_t*>(s->d_tmp));
            }
            *ptr = s->d_tmp;
            return FIREX_OK;
        case FIREX_FIELD_FINAL_DIVERGENCE:
            if (writing) return FIREX_ERR_BAD_ARG;
            {
                FxParams hp;
                s->build_params(hp, 0.0f);
                fx_launch_upload_params(s->stream, hp, s->d_params);
                fx_launch_divergence_f32(s->stream, s->d_params, s->grid(), s->flow[0], s->d_tmp);
            }
            *ptr = s->d_tmp;
            return FIREX_OK;
    }
    return FIREX_ERR_BAD_ARG;
}

int firex_read_field(firex_sim* s, int32_t field, void* host, size_t bytes) {
    if (!s || !host) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    size_t es = firex_field_element_size(field);
    if (!es) return s->fail(FIREX_ERR_BAD_ARG, "unknown field id");
    if (bytes != es * (size_t)s->N) return s->fail(FIREX_ERR_BAD_ARG, "byte count does not match the field size");
    DeviceGuard dg(s->device);
    void* src = nullptr;
    if (field_ptr(s, field, false, &src) != FIREX_OK) return s->fail(FIREX_ERR_BAD_ARG, "field is not readable");
    cudaError_t e = cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return s->cuda_fail(e, "read_field");
    return FIREX_OK;
}

int firex_write_field(firex_sim* s, int32_t field, const void* host, size_t bytes) {
    if (!s || !host) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    size_t es = firex_field_element_size(field);
    if (!es) return s->fail(FIREX_ERR_BAD_ARG, "unknown field id");
    if (bytes != es * (size_t)s->N) return s->fail(FIREX_ERR_BAD_ARG, "byte count does not match the field size");
    DeviceGuard dg(s->device);
    void* dst = nullptr;
    if (field_ptr(s, field, true, &dst) != FIREX_OK) return s->fail(FIREX_ERR_BAD_ARG, "field is not writable");
    cudaError_t e = cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return s->cuda_fail(e, "write_field");
    return FIREX_OK;
}

int firex_divergence_norm(firex_sim* s, double out[3]) {
    if (!s || !out) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    DeviceGuard dg(s->device);
    FxParams hp;
    s->build_params(hp, 0.0f);
    fx_launch_upload_params(s->stream, hp, s->d_params);
    fx_launch_divergence_norm(s->stream, s->d_params, s->grid(), s->flow[0], s->d_partial, s->d_norm);
    double h[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, s->d_norm, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return s->cuda_fail(e, "divergence_norm");
    out[0] = h[0];
    out[1] = h[1];
    out[2] = (double)(s->X - 2) * (double)(s->Y - 2) * (double)(s->Z - 2);
    return FIREX_OK;
}

int firex_get_state(const firex_sim* s, firex_state* st) {
    if (!s || !st) return FIREX_ERR_BAD_ARG;
    st->simulation_time = s->simTime;
    st->frame_index = s->frame;
    st->species_index = s->speciesIndex;
    st->pressure_index = s->pressureIndex;
    return FIREX_OK;
}

int firex_set_state(firex_sim* s, const firex_state* st) {
    if (!s || !st) return FIREX_ERR_BAD_ARG;
    if ((st->species_index & ~1) || (st->pressure_index & ~1) || !std::isfinite(st->simulation_time))
        return s->fail(FIREX_ERR_BAD_ARG, "invalid state");
    s->simTime = st->simulation_time;
    s->frame = st->frame_index;
    s->speciesIndex = st->species_index;
    s->pressureIndex = st->pressure_index;
    return FIREX_OK;
}

int firex_get_uniforms(const firex_sim* s, double dt, float out[FIREX_UNIFORM_FLOATS]) {
    if (!s || !out) return FIREX_ERR_BAD_ARG;
    FxParams hp;
    s->build_params(hp, dt);
    std::memcpy(out, hp.u, sizeof(hp.u));
    return FIREX_OK;
}

int firex_get_info(const firex_sim* s, int32_t dims[3], firex_options* opt) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (dims) {
        dims[0] = s->X;
        dims[1] = s->Y;
        dims[2] = s->Z;
    }
    if (opt) {
        *opt = s->opt;
        opt->pressure_mode = s->mode;
    }
    return FIREX_OK;
}

int firex_device_bytes(const firex_sim* s, uint64_t* bytes) {
    if (!s || !bytes) return FIREX_ERR_BAD_ARG;
    *bytes = s->bytes;
    return FIREX_OK;
}

void* firex_stream(const firex_sim* s) { return s ? (void*)s->stream : nullptr; }

int firex_set_profiling(firex_sim* s, int32_t on) {
    if (!s) return FIREX_ERR_BAD_ARG;
    DeviceGuard dg(s->device);
    if (!on && s->profiling) s->collect_marks();
    s->profiling = on != 0;
    return FIREX_OK;
}

int firex_pass_times(firex_sim* s, double* ms, int64_t* launches) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    DeviceGuard dg(s->device);
    int rc = s->collect_marks();
    if (rc != FIREX_OK) return rc;
    for (int p = 0; p < FIREX_PASS_COUNT; ++p) {
        if (ms) ms[p] = s->passMs[p];
        if (launches) launches[p] = s->passLaunches[p];
        s->passMs[p] = 0;
        s->passLaunches[p] = 0;
    }
    return FIREX_OK;
}

}  // extern "C"
