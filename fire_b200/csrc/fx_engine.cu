// fx_engine.cu — the Fire-X engine behind the C ABI (include/firex.h).
//
// Host-side counterpart of FireXEngine (src/sim/firex/FireXEngine.ts): named parameters
// with the reference's clamps, the 44-float uniform block, transactional allocation,
// reset, and the per-step dispatch graph with its ping-pong parities and pressure
// branches. Each simulation owns a device descriptor (FxSimDev); a standalone simulation
// steps as a batch of one, and firex_batch_* steps many simulations through the same
// launches. A step is captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <array>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/firex.h"
#include "fx_internal.h"
#include "fx_jacobi_res.cuh"
#include "fx_jacobi_zm.cuh"
#include "fx_jacobi_zm2.cuh"

static_assert(offsetof(FxSimDev, tmap) % 64 == 0, "tensor maps must sit on 64-byte boundaries");

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

// Seeded per-step emission factor in [1-a, 1+a] (extension); same operations as the
// step prologue kernel.
float host_jitter(uint64_t seed, int64_t f, float a) {
    auto mix = [](uint64_t z) {
        z += 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    uint64_t h = mix(mix(seed ^ 0xBB67AE8584CAA73Bull) + (uint64_t)f);
    float u = (float)(h >> 40) * (1.0f / 16777216.0f);
    return 1.0f + a * (2.0f * u - 1.0f);
}

// Bricks of the source pass: 32 x by x (8 / by) cells.
long long bricks_cell(int X, int Y, int Z, int by) {
    const int bz = 256 / (FX_CELL_BX * by);
    return (long long)((X + FX_CELL_BX - 1) / FX_CELL_BX) * ((Y + by - 1) / by) * ((Z + bz - 1) / bz);
}
bool sim_by_ok(int by) { return by == 0 || by == 2 || by == 4 || by == 8; }
long long bricks_row4(int X, int Y, int Z) {
    long long groups = (long long)(X / 4) * Y * Z;
    return (groups + FX_ROW4_THREADS - 1) / FX_ROW4_THREADS;
}

// The host-side mirror of a step graph's launch sequence and its cache key.
struct StepPlan {
    int storage = 0;
    bool half = false;
    int pmode = FX_TB_F32;    // pressure storage / rounding of the fused Jacobi
    int maxP = 0, maxR = 0;
    int k = 1, zc = 16;       // fused sweeps per Jacobi launch, z planes per CTA
    int zmZc = 16;            // z planes per CTA of the single-sweep (z-marching) kernel
    bool row4 = false;        // single sweeps by the unblocked kernel instead
    bool fuseP = false, fuseR = false;
    bool pack = false;        // a member packs its render volumes at the end of every step
    bool tma = false;         // the two-sweep pass stages its planes by TMA
    int simBy = FX_CELL_BY;   // source-pass bricks: 32 x simBy x (8 / simBy) cells
    bool projDiv = true;      // the primary projection and the residual divergence in one pass
    bool res = false;         // every sweep of a phase in one resident launch
    int resVariant = 0;       // ... by this variant of the kernel
    int resSmem = 0;          // its dynamic shared memory per CTA
    bool projRes = false;     // the residual projection inside the resident launch (variant 4)
    bool simEarly = false;    // the source pass evaluates its neighbour terms before the advection
    int bricks[FX_NSHAPES] = {};
    auto key() const {
        return std::tie(storage, half, pmode, maxP, maxR, k, zc, zmZc, row4, fuseP, fuseR, pack, tma, simBy, projDiv, res,
                        resVariant, resSmem, projRes, simEarly,
                        bricks[0],
                        bricks[1], bricks[2], bricks[3], bricks[4], bricks[5], bricks[6]);
    }
    bool operator<(const StepPlan& o) const { return key() < o.key(); }
};

#ifndef FX_SIM_EARLY_CELLS
#define FX_SIM_EARLY_CELLS (12LL << 20)  // batches below this many cells: the source pass's early order
#endif
#ifndef FX_PROJ_RES
#define FX_PROJ_RES 1  // the residual projection as the resident variant 4's epilogue when it can
#endif

// A phase of n sweeps may fuse k sweeps per launch when every member runs the same n
// and the launch count (n/k fused + n%k single) has the parity of n: the result then
// lands in the buffer the reference's ping-pong leaves it in.
bool can_fuse(int k, int n) { return k > 1 && n >= k && ((k - 1) * (n / k)) % 2 == 0; }

int jacobi_phase_launches(const StepPlan& pl, int phase) {
    const int n = phase == 0 ? pl.maxP : pl.maxR;
    if (pl.res) return n > 0 ? 1 : 0;
    const bool fuse = phase == 0 ? pl.fuseP : pl.fuseR;
    return fuse ? n / pl.k + n % pl.k : n;
}

void enqueue_jacobi_phase(cudaStream_t st, const StepPlan& pl, FxBatchDev* B, int phase) {
    const int n = phase == 0 ? pl.maxP : pl.maxR;
    if (pl.res) {  // a failed launch is reported by the caller's cudaGetLastError
        if (n > 0)
            fx_launch_jacobi_res(st, pl.half, pl.resVariant, B, pl.bricks[FX_SHAPE_RES], phase, pl.resSmem,
                                 phase == 1 && pl.projRes);
        return;
    }
    const bool fuse = phase == 0 ? pl.fuseP : pl.fuseR;
    int launch = 0, sweep = 0;
    if (fuse) {
        for (; sweep + pl.k <= n; sweep += pl.k, ++launch)
            fx_launch_jacobi_tb(st, pl.pmode, pl.k, B, pl.bricks[FX_SHAPE_COL], phase, launch, pl.zc, pl.tma);
    }
    for (; sweep < n; ++sweep, ++launch) {
        if (pl.row4) fx_launch_jacobi(st, pl.half, B, pl.bricks[FX_SHAPE_ROW4], phase, launch, sweep);
        else fx_launch_jacobi_zm(st, pl.half, B, pl.bricks[FX_SHAPE_ZM], phase, launch, sweep, pl.zmZc);
    }
}

// Launches of the droplet pass (liquid clear + density, integrate + deposit) when a member sprays.
int sph_launches(const StepPlan& pl) { return pl.bricks[FX_SHAPE_PART] > 0 ? 2 : 0; }

void enqueue_step_launches(cudaStream_t st, const StepPlan& pl, FxBatchDev* B) {
    fx_launch_step_begin(st, B);
    fx_launch_step_tables(st, B, pl.bricks[FX_SHAPE_TAB]);
    if (sph_launches(pl)) fx_launch_sph(st, B, pl.bricks[FX_SHAPE_ROW4], pl.bricks[FX_SHAPE_PART]);
    fx_launch_simulate(st, pl.storage, pl.simBy, pl.simEarly, B, pl.bricks[FX_SHAPE_CELL]);
    fx_launch_divergence(st, B, pl.bricks[FX_SHAPE_ROW4], 0);
    enqueue_jacobi_phase(st, pl, B, 0);
    if (pl.projDiv) {
        fx_launch_project_div(st, pl.half, B, pl.bricks[FX_SHAPE_ROW4]);
    } else {
        fx_launch_project(st, pl.half, B, pl.bricks[FX_SHAPE_ROW4], 0);
        fx_launch_divergence(st, B, pl.bricks[FX_SHAPE_ROW4], 1);
    }
    enqueue_jacobi_phase(st, pl, B, 1);
    if (!pl.projRes) fx_launch_project(st, pl.half, B, pl.bricks[FX_SHAPE_ROW4], 1);
    fx_launch_step_end(st, B);
    if (pl.pack) fx_launch_pack_batch(st, B, pl.bricks[FX_SHAPE_ROW4]);
}

// Jacobi kernel when the caller did not choose one (measured on B200, 96+96 sweeps):
// below 8 Mi cells per batch the unblocked kernel (the pressure pair and the divergence
// stay in L2 and more CTAs hide latency; at 160x240x160 the z-marching kernel only ties
// it); from 8 Mi cells, where they outgrow L2, two sweeps per pass by z-marching tiles
// (the fused kernel with block 2) with 16-plane chunks (192x288x192: 6.29 ms per step
// against 6.48 with one sweep per pass and 7.52 unblocked), and from 16 Mi cells with
// 64-plane chunks (508^3: 45.1 ms of Jacobi per step against 56.5 ms for one sweep per
// pass). fire_b200/autotune.py refines this per workload.
void default_jacobi(long long cells, int* kernel, int* k, int* zc) {
    const bool big = cells >= (16LL << 20), mid = !big && cells >= (8LL << 20);
    *kernel = (big || mid) ? FIREX_JACOBI_FUSED : FIREX_JACOBI_UNBLOCKED;
    *k = (big || mid) ? 2 : 1;
    *zc = big ? 64 : (mid ? 16 : 32);
}

// Box decomposition of an X x Y x Z grid over at most m CTAs for the resident Jacobi
// (boxes of by x bz full x rows; G = by * bz * X / 4 groups of 4 cells per box). Cost per
// sweep: the groups a thread computes plus the halo traffic per thread (faces written and
// halo rows read, 2 (by + bz) rows of X / 4 groups, both ways).
//   variants 1, 2 (faces-first): face groups and interior groups dealt out separately,
//     within FX_RES_MAXF and FX_RES_MAXI (variant 2: FX_RES_MAXI_SMALL) per thread;
//   variant 0 (columns): thread columns of (x group, row), by * X / 4 <= T, each split into
//     parts along z; at most FX_RES_MAXG planes per column part.
// False when no box fits one CTA's shared memory and registers.
bool res_box(int X, int Y, int Z, int m, int variant, FxResBox* out) {
    const long long gx = X / 4;
    bool found = false;
    double best = 0;
    for (int by = 1; by <= Y && by <= 2047; ++by) {
        const int nby = (Y + by - 1) / by;
        if (nby > m || nby > FX_RES_MAX_CTAS) continue;
        const int maxNbz = m / nby;
        const int bz = (Z + maxNbz - 1) / maxNbz;
        if (bz > 1023) continue;
        if (fx_res_smem_bytes(X, by, bz) > FX_RES_SMEM_MAX) continue;
        const long long G = (long long)by * bz * gx;
        double work;
        if (variant == 3 || variant == 4) {
            // faces dealt out; interior columns (rows off the y faces x groups) one per
            // thread, split along z when there are fewer columns than threads (variant 4:
            // the threads but the copy warp)
            const long long T = variant == 4 ? FX_RES_COPY_TC : FX_RES_THREADS;
            if (2LL * (by + bz) * gx > (long long)FX_RES_MAXF * T) continue;
            // the most interior rows and planes a box can have: a box with a neighbour on
            // one side only keeps all but one row (plane) off its faces
            const int nbzHere = (Z + bz - 1) / bz;
            const long long rowsI = nby == 1 ? by : by - 1, planesI = nbzHere == 1 ? bz : bz - 1;
            const long long Cmax = rowsI * gx;
            if (Cmax > T) continue;
            const long long parts = std::max(1LL, T / std::max(1LL, Cmax));
            const long long zlen = (planesI + parts - 1) / parts;
            if (zlen > FX_RES_MAXZ) continue;
            if (zlen < 4) continue;  // short columns: the faces-first variants do better (measured)
            const long long F = 2LL * (by + bz) * gx;
            work = (double)zlen + (double)((F + T - 1) / T);
        } else if (variant != 0) {
            // faces (at most 2 (by + bz) rows of groups) and interior dealt out separately
            const int maxi = variant == 2 ? FX_RES_MAXI_SMALL : FX_RES_MAXI;
            if (2LL * (by + bz) * gx > (long long)FX_RES_MAXF * FX_RES_THREADS) continue;
            if (G > (long long)maxi * FX_RES_THREADS) continue;
            work = (double)((G + FX_RES_THREADS - 1) / FX_RES_THREADS);
        } else {
            if (by * gx > FX_RES_THREADS) continue;
            const int parts = (int)(FX_RES_THREADS / (by * gx));
            const int zlen = (bz + parts - 1) / parts;
            if (zlen > FX_RES_MAXG) continue;
            work = zlen;
        }
        const double cost = work + 4.0 * (by + bz) * gx / FX_RES_THREADS;
        if (!found || cost < best) {
            found = true;
            best = cost;
            *out = FxResBox{by, bz, nby, (Z + bz - 1) / bz};
        }
    }
    return found;
}

// CTAs for every simulation of a batch within `cap` (one launch of one variant): each gets
// at least the fewest CTAs its grid fits in, the rest in proportion to cells. False when
// the batch does not fit.
bool res_assign(const std::vector<std::array<int, 3>>& dims, int cap, int variant, std::vector<FxResBox>* boxes,
                int* smem) {
    const size_t n = dims.size();
    if (n == 0 || cap <= 0) return false;
    std::vector<int> mins(n), t(n);
    long long sumMin = 0;
    double cells = 0;
    FxResBox tmp;
    for (size_t i = 0; i < n; ++i) {
        const auto& d = dims[i];
        if (!res_box(d[0], d[1], d[2], cap, variant, &tmp)) return false;
        int lo = 1, hi = cap;
        while (lo < hi) {
            const int mid = (lo + hi) / 2;
            if (res_box(d[0], d[1], d[2], mid, variant, &tmp)) hi = mid;
            else lo = mid + 1;
        }
        mins[i] = lo;
        sumMin += lo;
        cells += (double)d[0] * d[1] * d[2];
    }
    if (sumMin > cap) return false;
    long long sum = 0;
    for (size_t i = 0; i < n; ++i) {
        const double share = (double)dims[i][0] * dims[i][1] * dims[i][2] / cells;
        t[i] = std::max(mins[i], (int)std::floor(share * cap));
        sum += t[i];
    }
    while (sum > cap) {  // give back CTAs from the member with the most to spare
        size_t j = 0;
        for (size_t i = 1; i < n; ++i)
            if (t[i] - mins[i] > t[j] - mins[j]) j = i;
        --t[j];
        --sum;
    }
    boxes->resize(n);
    *smem = 0;
    for (size_t i = 0; i < n; ++i) {
        res_box(dims[i][0], dims[i][1], dims[i][2], t[i], variant, &(*boxes)[i]);
        *smem = std::max(*smem, (int)fx_res_smem_bytes(dims[i][0], (*boxes)[i].by, (*boxes)[i].bz));
    }
    return true;
}

// z chunk of the z-marching kernel when not chosen: the largest of 32, 16, 8 planes that
// still yields three CTAs per SM over the batch.
int zm_chunk(long long tiles32, long long tiles16) {
    return tiles32 >= 3LL * 148 ? 32 : (tiles16 >= 3LL * 148 ? 16 : 8);
}

}  // namespace

// Sets the text that firex_last_error(NULL) returns on this thread (entry points that
// have no handle report through it).
void fx_set_thread_error(const std::string& msg) { g_create_error = msg; }

struct firex_batch;

// Whether fx_div_by_const(x, d, rcp) equals IEEE x / d for every finite float x on this
// device, checked once per (device, d) by fxk_check_div (about a millisecond). Results
// are cached for the life of the process. Any CUDA error answers "no".
static bool fast_division_ok(int device, float d, float rcp, float lo = 1.2621774483536189e-29f,
                             float hi = 3.402823466e38f) {
    static std::map<std::tuple<int, uint32_t, uint32_t, uint32_t>, bool> cache;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    uint32_t bits, lb, hb;
    std::memcpy(&bits, &d, 4);
    std::memcpy(&lb, &lo, 4);
    std::memcpy(&hb, &hi, 4);
    auto key = std::make_tuple(device, bits, lb, hb);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    bool ok = false;
    unsigned long long* dcount = nullptr;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
        cudaMalloc(&dcount, sizeof(unsigned long long)) == cudaSuccess &&
        cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), st) == cudaSuccess) {
        fx_launch_check_div(st, d, rcp, lo, hi, dcount);
        unsigned long long bad = ~0ull;
        if (cudaMemcpyAsync(&bad, dcount, sizeof(bad), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
            cudaStreamSynchronize(st) == cudaSuccess)
            ok = bad == 0;
    }
    cudaGetLastError();
    if (dcount) cudaFree(dcount);
    if (st) cudaStreamDestroy(st);
    cache[key] = ok;
    return ok;
}

// ---- one simulation ------------------------------------------------------------------------
struct firex_sim {
    int X = 0, Y = 0, Z = 0;
    long long N = 0;
    firex_options opt{};
    int mode = FIREX_PRESSURE_WARM_F32;
    int storage = FX_STORAGE_F32;
    bool half = false;  // pressure storage is FP16
    int device = 0;
    double named[kNumParams];
    int jacobiKernel = FIREX_JACOBI_AUTO, jacobiK = 1, jacobiZc = 0;
    int staging = FIREX_STAGING_AUTO;  // how the two-sweep pass stages its planes
    int simBy = 0;                     // source-pass brick height (0: FX_CELL_BY)
    int projFuse = FIREX_PROJECT_AUTO; // primary projection fused with the residual divergence?

    FxSimDev h{};           // host mirror of the device descriptor
    FxSimDev* d = nullptr;  // device descriptor
    bool dirty = true;      // host mirror has changes the device has not seen

    cudaStream_t own = nullptr;
    firex_batch* batch = nullptr;  // set while a member of a batch
    firex_batch* solo = nullptr;   // the one-member batch used for standalone steps

    std::vector<void*> allocations;
    size_t bytes = 0;
    void* d_tmp = nullptr;          // 4 B/cell scratch: emitter mask, final divergence
    double* d_partial = nullptr;    // divergence-norm partials
    double* d_norm = nullptr;
    // overlapped readback (firex_read_field_async): the field is copied on the device into
    // a staging buffer in stream order, then to the host on a copy stream while later
    // steps run; created on first use
    void* d_stage = nullptr;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evStaged = nullptr, evCopied = nullptr;
    bool copyPending = false;
    std::string err;
    bool poisoned = false;

    cudaStream_t stream() const;

    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        poisoned = true;
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return FIREX_ERR_CUDA;
    }

    // The three render volumes (8 B per cell each), allocated on first use.
    bool ensure_render_volumes() {
        if (h.render[0]) return true;
        for (int k = 0; k < 3; ++k) {
            h.render[k] = (uint2*)alloc((size_t)N * 8);
            if (!h.render[k]) return false;
        }
        dirty = true;
        return true;
    }

    // After a stream synchronisation: whether a bounded device wait of this simulation
    // expired (the resident Jacobi's group barrier). The fields are then incomplete.
    int check_device_waits() {
        unsigned word = 0;
        cudaError_t e = cudaMemcpy(&word, h.sync + 2, sizeof(word), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "error word");
        if (word != 0) {
            poisoned = true;
            err = "a bounded device wait expired (resident Jacobi barrier); the step did not complete";
            return FIREX_ERR_TIMEOUT;
        }
        return FIREX_OK;
    }

    void* alloc(size_t nbytes) {
        void* p = nullptr;
        if (cudaMalloc(&p, nbytes ? nbytes : 1) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        allocations.push_back(p);
        bytes += nbytes;
        return p;
    }

    static size_t planned_bytes(int X, int Y, int Z, int storage, int mode, int particles) {
        const long long N = (long long)X * Y * Z;
        const size_t species = storage == FX_STORAGE_MIXED ? 8 : 16;
        const size_t pbytes = mode == FIREX_PRESSURE_F16 ? 2 : 4;
        const size_t npress = mode == FIREX_PRESSURE_COLD_F32 ? 2 : 4;
        const size_t per = 16 * 2 + species * 2 + pbytes * npress + 4 /*div*/ + 4 /*reaction*/ + 4 /*liquid*/ + 4 /*tmp*/;
        return (size_t)N * per + (size_t)fx_tab_layout(X, Y, Z).total * 4 + sizeof(FxSimDev) + 64 * 1024 +
               (size_t)std::max(0, particles) * (2 * 32 + 16);  // two droplet buffers and their densities
    }
    size_t table_bytes() const { return (size_t)fx_tab_layout(X, Y, Z).total * 4;
    }

    size_t species_bytes() const { return storage == FX_STORAGE_MIXED ? 8 : 16; }
    size_t pressure_bytes() const { return half ? 2 : 4; }

    // writeUniforms (FireXEngine.ts:2043-2113); the time fields are rewritten on the
    // device at the start of every step from the counters.
    void build_params(FxParams& p, double dt) const {
        std::memset(&p, 0, sizeof(p));
        auto P = [&](const char* n) { return named[param_slot(n)]; };
        const double cells = (double)X * (double)Y * (double)Z;
        const double u[FIREX_UNIFORM_FLOATS] = {
            (double)X, (double)Y, (double)Z, cells,
            dt, h.simTime, (double)h.frame, dt,
            P("fuelRate"), P("oxygenRate"), P("heatEfficiency"), P("vorticity"),
            P("waterFlow"), (P("sprayAngle") * M_PI) / 180, P("waterEnabled") != 0 ? 1.0 : 0.0, 300,
            P("cameraYaw"), P("cameraPitch"), P("cameraDistance"), 1,  // canvas aspect (presentation only)
            1, 1, 0, (double)std::max(0, opt.particle_count),          // canvas size, rays, particles
            P("viewMode"), P("aimHeight"), P("nozzleType"), P("exposure"),
            P("burnerSize"), P("burnerDepth"), P("sourceThickness"), P("firePower"),
            P("domainWidth"), P("domainHeight"), P("domainDepth"), 0,
            P("sourceLift"), P("buoyancyScale"), P("flamePersistence"), P("viewZoom"),
            P("airEntrainment"), P("frontDefinition"), opt.cinematic ? 1.0 : 0.0, P("opticalDetailTarget")};
        for (int i = 0; i < FIREX_UNIFORM_FLOATS; ++i) p.u[i] = (float)u[i];
        p.emitter_mode = opt.emitter_mode;
        p.num_spheres = opt.emitter_mode == FIREX_EMITTER_SPHERES ? opt.num_spheres : 0;
        for (int s = 0; s < FIREX_MAX_SPHERES; ++s) p.spheres[s] = opt.spheres[s];
        p.jitter = host_jitter(opt.seed, h.frame, opt.emission_jitter);
    }

    // Stencil constants in f32, the same operations as cellMetric() and the Jacobi
    // weights of shaders.ts:39-41,386-389 (IEEE single precision on the host).
    void refresh_params() {
        build_params(h.prm, h.dt);
        const float* u = h.prm.u;
        const float ex = std::max(u[32], 0.001f), ey = std::max(u[33], 0.001f), ez = std::max(u[34], 0.001f);
        h.metric[0] = u[0] / ex;
        h.metric[1] = u[1] / ey;
        h.metric[2] = u[2] / ez;
        h.metric[3] = 0.0f;
        h.jc[0] = h.metric[0] * h.metric[0];
        h.jc[1] = h.metric[1] * h.metric[1];
        h.jc[2] = h.metric[2] * h.metric[2];
        h.jc[3] = 2.0f * (h.jc[0] + h.jc[1] + h.jc[2]);
        h.jcRcp = 1.0f / h.jc[3];
        h.jcFastDiv = fast_division_ok(device, h.jc[3], h.jcRcp) ? 1 : 0;
        // constant divisors of simulate, computed with the same f32 operations as the
        // expressions they stand for
        auto fmaxr = [](float a, float b) { return (a < b) ? b : a; };
        auto fminr = [](float a, float b) { return (b < a) ? b : a; };
        const float persistence = fminr(fmaxr(u[38], 0.4f), 3.0f);
        const float divisors[DIVC_COUNT] = {
            6.0f, 0.78f - 0.30f, 1500.0f - 400.0f, 930.0f - 690.0f, 1650.0f - 520.0f, 1040.0f - 335.0f,
            0.48f - (-0.42f), 1500.0f, fmaxr(u[9], 0.001f), fmaxr(u[4], 0.0001f), 1005.0f * persistence};
        for (int k = 0; k < DIVC_COUNT; ++k) {
            FxDivc& c = h.divc[k];
            std::memset(&c, 0, sizeof(c));
            c.d = divisors[k];
            c.rcp = 1.0f / c.d;
            c.lo = 1.2621774483536189e-29f;  // 2^-96: quotients stay normal for d < 2^30
            c.hi = (float)std::min(3.4028234663852886e38, 3.4028234663852886e38 * std::min(1.0, (double)c.d) * 0.5);
            // dt may change every call: its divisor keeps the IEEE division rather than
            // paying the device check per new value
            c.ok = (k != DIVC_DT && c.d > 0.0f && c.d < 1073741824.0f && fast_division_ok(device, c.d, c.rcp, c.lo, c.hi)) ? 1 : 0;
            // not enabled: an empty fast range sends every x to the IEEE division (fx_divc)
            if (!c.ok) c.lo = INFINITY;
        }
        dirty = true;
    }

    // Uploads the host mirror when it changed (parameters, dt, counters set by the caller).
    void flush(cudaStream_t st) {
        if (!dirty) return;
        fx_launch_upload_desc(st, h, d);
        dirty = false;
    }

    // Advances the host mirror exactly as fxk_step_end advances the device.
    void advance_mirror() {
        h.simTime = h.simTime + h.dt;
        h.frame += 1;
        h.fi ^= 1;
        h.si ^= 1;
        h.pi = (h.mode == FIREX_PRESSURE_COLD_F32) ? (h.P & 1) : (h.pi ^ (h.P & 1));
        if (h.water) h.pti ^= 1;
    }

    // ---- droplets (SPH): host-side state of FireXEngine.ts:2158-2171 ----
    bool particleFieldActive = false, liquidMayContainWater = false;
    std::vector<float> hostParticles;  // staging of the initial state (kept alive for the async copy)
    bool water_active() const { return named[param_slot("waterEnabled")] != 0 && named[param_slot("waterFlow")] > 0.001; }
    // writeParticleInitialState (FireXEngine.ts:1976-2034), into both droplet buffers
    void write_particle_initial_state(cudaStream_t st, bool active);
    // Before each step: the transitions of the reference's particle state machine.
    void prepare_particles(cudaStream_t st) {
        if (h.np <= 0) return;
        const bool on = water_active();
        if (on) {
            if (!particleFieldActive) write_particle_initial_state(st, true);
            liquidMayContainWater = true;
        } else if (liquidMayContainWater || particleFieldActive) {
            cudaMemsetAsync(h.liquid, 0, (size_t)N * 4, st);
            write_particle_initial_state(st, false);
            liquidMayContainWater = false;
        }
        if ((h.water != 0) != on) {
            h.water = on ? 1 : 0;
            dirty = true;
        }
    }

    int reset();
    void release();
};

// ---- a batch of simulations stepping together ------------------------------------------------
struct firex_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<firex_sim*> members;
    FxBatchDev* d = nullptr;
    FxBatchDev* h = nullptr;  // host copy of the table
    bool tableDirty = true;
    std::map<StepPlan, cudaGraphExec_t> graphs;
    bool useGraphs = true;
    bool profiling = false;
    bool isSolo = false;
    StepPlan last{};                 // plan of the most recent step (diagnostics)
    bool lastGraph = false;
    int jacobiKernel = FIREX_JACOBI_AUTO, jacobiK = 1, jacobiZc = 0;  // batch override (AUTO: first member's)
    int staging = FIREX_STAGING_AUTO;  // batch override of the members' staging (AUTO: first member's)
    int simBy = 0;                     // batch override of the source-pass bricks (0: first member's)
    int projFuse = FIREX_PROJECT_AUTO; // batch override of the projection fusion (AUTO: first member's)
    int tableK = -1, tableZc = -1, tableZmZc = -1;  // launch shapes the prefix sums were built for
    int tableSimBy = -1;
    int tableRes = -1;                               // whether resident boxes were requested
    std::vector<char> tableWater;                    // which members sprayed when the table was filled
    bool resOk = false;                              // ... and the batch fits one resident launch
    int resVariant = 0;                              // ... of this kernel variant
    int resSmem = 0;
    std::string err;

    // per-pass profiling (events between passes; graphs are bypassed while profiling)
    std::vector<cudaEvent_t> evPool;
    std::vector<std::pair<cudaEvent_t, int>> evMarks;
    size_t evUsed = 0;
    double passMs[FIREX_PASS_COUNT] = {0};
    int64_t passLaunches[FIREX_PASS_COUNT] = {0};
    int64_t pendingLaunches[FIREX_PASS_COUNT] = {0};

    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }

    void rebuild_table() {
        std::memset(h, 0, sizeof(FxBatchDev));
        h->nsims = (int)members.size();
        tableK = -1;
        tableDirty = true;
    }

    // Fills the brick prefix sums for the launch shape (k, zc); resident boxes when wanted,
    // of variant resForce when that is 0-4.
    void fill_table(int k, int zc, int zmZc, bool wantRes, int resForce, int simBy) {
        int acc[FX_NSHAPES] = {};
        h->nsims = (int)members.size();
        std::vector<FxResBox> boxes;
        resOk = false;
        if (wantRes && !members.empty()) {
            std::vector<std::array<int, 3>> dims;
            for (firex_sim* s : members) dims.push_back({s->X, s->Y, s->Z});
            // the first variant every member fits: faces first with interior columns and a
            // copy warp (FP32 pressure; 6.0 against 7.6 us per sweep at HD on B200), the same
            // without the copy warp (long columns only), faces first (small-box instance
            // first), then the column variant
            for (int v : {4, 3, 2, 1, 0}) {
                if (resForce >= 0 && v != resForce) continue;
                if (v == 4 && members[0]->half) continue;  // the copy warp moves FP32 rows
                const int cap = fx_res_capacity(members[0]->half, v);
                if (res_assign(dims, cap, v, &boxes, &resSmem)) {
                    resOk = true;
                    resVariant = v;
                    break;
                }
            }
        }
        for (size_t i = 0; i < members.size(); ++i) {
            firex_sim* s = members[i];
            h->sims[i] = s->d;
            h->start[FX_SHAPE_CELL][i] = acc[FX_SHAPE_CELL];
            h->start[FX_SHAPE_ROW4][i] = acc[FX_SHAPE_ROW4];
            h->start[FX_SHAPE_COL][i] = acc[FX_SHAPE_COL];
            h->start[FX_SHAPE_ZM][i] = acc[FX_SHAPE_ZM];
            h->start[FX_SHAPE_TAB][i] = acc[FX_SHAPE_TAB];
            h->start[FX_SHAPE_RES][i] = acc[FX_SHAPE_RES];
            h->start[FX_SHAPE_PART][i] = acc[FX_SHAPE_PART];
            acc[FX_SHAPE_PART] += s->h.water ? (s->h.np + FX_SPH_DROPLETS - 1) / FX_SPH_DROPLETS : 0;
            if (resOk) {
                h->res[i] = boxes[i];
                acc[FX_SHAPE_RES] += boxes[i].nby * boxes[i].nbz;
            }
            acc[FX_SHAPE_TAB] += (fx_tab_layout(s->X, s->Y, s->Z).total + 255) / 256;
            acc[FX_SHAPE_CELL] += (int)bricks_cell(s->X, s->Y, s->Z, simBy);
            acc[FX_SHAPE_ROW4] += (int)bricks_row4(s->X, s->Y, s->Z);
            acc[FX_SHAPE_COL] += k == 2 ? fx_zm2_bricks(s->X, s->Y, s->Z, zc) : 0;
            acc[FX_SHAPE_ZM] += fx_zm_bricks(s->X, s->Y, s->Z, zmZc);
        }
        for (int j = 0; j < FX_NSHAPES; ++j) {
            h->start[j][members.size()] = acc[j];
            h->total[j] = acc[j];
        }
        tableK = k;
        tableSimBy = simBy;
        tableZc = zc;
        tableZmZc = zmZc;
        tableRes = wantRes ? 2 + resForce : 0;
        tableWater = water_signature();
        tableDirty = true;
    }

    std::vector<char> water_signature() const {
        std::vector<char> w;
        for (firex_sim* s : members) w.push_back(s->h.water ? 1 : 0);
        return w;
    }

    StepPlan plan() {
        StepPlan p;
        if (members.empty()) return p;
        p.storage = members[0]->storage;
        p.half = members[0]->half;
        p.pmode = p.half ? FX_TB_F16_ROUND : FX_TB_F32;
        bool uniformP = true, uniformR = true;
        long long cells = 0;
        for (firex_sim* s : members) {
            p.maxP = std::max(p.maxP, s->h.P);
            p.maxR = std::max(p.maxR, s->h.R);
            uniformP = uniformP && s->h.P == members[0]->h.P;
            uniformR = uniformR && s->h.R == members[0]->h.R;
            cells += s->N;
            p.pack = p.pack || s->h.renderPack != 0;
        }
        const bool own = jacobiKernel != FIREX_JACOBI_AUTO;
        int kernel = own ? jacobiKernel : members[0]->jacobiKernel;
        int k = own ? jacobiK : members[0]->jacobiK;
        const int resForce = (kernel == FIREX_JACOBI_RESIDENT && k >= 1) ? k - 1 : -1;  // block = variant + 1
        int zc = own ? jacobiZc : members[0]->jacobiZc;
        // AUTO and RESIDENT try the resident launch first; the default is the fallback when
        // the batch does not fit on chip
        const bool wantRes = kernel == FIREX_JACOBI_AUTO || kernel == FIREX_JACOBI_RESIDENT;
        if (kernel == FIREX_JACOBI_AUTO || kernel == FIREX_JACOBI_RESIDENT) {
            int dk = 1, dzc = 32;
            default_jacobi(cells, &kernel, &dk, &dzc);
            k = dk;
            if (zc <= 0) zc = dzc;
        }
        if (kernel != FIREX_JACOBI_FUSED || (k != 2 && k != 3 && k != 4 && k != 6)) k = 1;
        long long zm32 = 0, zm16 = 0;
        for (firex_sim* s : members) {
            zm32 += fx_zm_bricks(s->X, s->Y, s->Z, 32);
            zm16 += fx_zm_bricks(s->X, s->Y, s->Z, 16);
        }
        p.k = k;
        p.zc = zc > 0 ? zc : 16;
        p.fuseP = uniformP && can_fuse(k, p.maxP);
        p.fuseR = uniformR && can_fuse(k, p.maxR);
        if (!p.fuseP && !p.fuseR) p.k = 1;
        p.row4 = kernel == FIREX_JACOBI_UNBLOCKED;
        p.zmZc = (kernel == FIREX_JACOBI_ZMARCH && zc > 0) ? zc : zm_chunk(zm32, zm16);
        const int by = this->simBy ? this->simBy : members[0]->simBy;
        p.simBy = by ? by : FX_CELL_BY;
        // the fused projection recomputes its backward neighbours from loads that hit L2 while
        // the batch's fields fit there; from 8 Mi cells they come from HBM and two passes are
        // faster (measured on B200, 508^3: 2.84 + 0.66 ms fused against 1.95 + 1.32 ms; HD:
        // 0.118 against 0.125 ms)
        const int pf = this->projFuse != FIREX_PROJECT_AUTO ? this->projFuse : members[0]->projFuse;
        p.projDiv = pf == FIREX_PROJECT_FUSED || (pf == FIREX_PROJECT_AUTO && cells < (8LL << 20));
        // the source pass's neighbour terms ahead of the advection below 12 Mi cells with FP32
        // storage (measured on B200, ms per pass, early against reference order: HD 0.185 /
        // 0.194, 160x240x160 0.353 / 0.361, 192x288x192 0.604 / 0.618; 256^3 1.010 / 0.964;
        // mixed storage HD 0.181 / 0.174, 160x240x160 0.344 / 0.326)
        p.simEarly = p.storage == FX_STORAGE_F32 && cells < FX_SIM_EARLY_CELLS;
        if (tableK != p.k || tableZc != p.zc || tableZmZc != p.zmZc || tableRes != (wantRes ? 2 + resForce : 0) ||
            tableWater != water_signature() || tableSimBy != p.simBy)
            fill_table(p.k, p.zc, p.zmZc, wantRes, resForce, p.simBy);
        // TMA staging of the two-sweep pass when asked for: FP32 pressure and every member's
        // tensor maps built. AUTO stages by cp.async, measured faster on B200 (508^3: 45.2 ms of
        // Jacobi per step against 49.4 with TMA; 192x288x192: 5.64 against 6.10)
        const int staging = this->staging != FIREX_STAGING_AUTO ? this->staging : members[0]->staging;
        bool maps = p.pmode == FX_TB_F32 && staging == FIREX_STAGING_TMA;
        for (firex_sim* s : members) maps = maps && s->h.tmapOk;
        p.tma = p.k == 2 && maps;
        p.res = wantRes && resOk;
        if (p.res) {
            p.resSmem = resSmem;
            p.resVariant = resVariant;
            p.k = 1;
            p.fuseP = p.fuseR = false;
            p.tma = false;
            // the residual projection as variant 4's epilogue (unless the projection passes are
            // asked to run separately): every member runs residual sweeps, and every top box has
            // two rows or more (its top row projects the row below from the box)
            bool epi = FX_PROJ_RES && resVariant == 4 && pf != FIREX_PROJECT_SEPARATE;
            for (size_t i = 0; i < members.size() && epi; ++i) {
                const FxResBox& bx = h->res[i];
                epi = members[i]->h.R >= 1 && members[i]->Y - (bx.nby - 1) * bx.by >= 2;
            }
            p.projRes = epi;
        }
        if (p.k != 2) p.tma = false;
        for (int j = 0; j < FX_NSHAPES; ++j) p.bricks[j] = h->total[j];
        return p;
    }

    cudaError_t flush_table() {
        if (!tableDirty) return cudaSuccess;
        cudaError_t e = cudaMemcpyAsync(d, h, sizeof(FxBatchDev), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // h may change right after
        tableDirty = false;
        return e;
    }

    void mark(int pass, int launches) {
        if (pass >= 0) pendingLaunches[pass] += launches;
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

    int collect_marks() {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return fail(FIREX_ERR_CUDA, std::string("pass_times: ") + cudaGetErrorString(e));
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

    // One step of every member with per-pass event marks (no graph).
    void enqueue_profiled(const StepPlan& pl) {
        mark(-1, 0);
        fx_launch_step_begin(stream, d);
        fx_launch_step_tables(stream, d, pl.bricks[FX_SHAPE_TAB]);
        mark(FIREX_PASS_OTHER, 2);
        if (sph_launches(pl)) {
            fx_launch_sph(stream, d, pl.bricks[FX_SHAPE_ROW4], pl.bricks[FX_SHAPE_PART]);
            mark(FIREX_PASS_PARTICLES, sph_launches(pl));
        }
        fx_launch_simulate(stream, pl.storage, pl.simBy, pl.simEarly, d, pl.bricks[FX_SHAPE_CELL]);
        mark(FIREX_PASS_SIMULATE, 1);
        fx_launch_divergence(stream, d, pl.bricks[FX_SHAPE_ROW4], 0);
        mark(FIREX_PASS_DIVERGENCE, 1);
        enqueue_jacobi_phase(stream, pl, d, 0);
        mark(FIREX_PASS_JACOBI, jacobi_phase_launches(pl, 0));
        if (pl.projDiv) {
            fx_launch_project_div(stream, pl.half, d, pl.bricks[FX_SHAPE_ROW4]);
            mark(FIREX_PASS_PROJECT, 1);
        } else {
            fx_launch_project(stream, pl.half, d, pl.bricks[FX_SHAPE_ROW4], 0);
            mark(FIREX_PASS_PROJECT, 1);
            fx_launch_divergence(stream, d, pl.bricks[FX_SHAPE_ROW4], 1);
            mark(FIREX_PASS_DIVERGENCE, 1);
        }
        enqueue_jacobi_phase(stream, pl, d, 1);
        mark(FIREX_PASS_JACOBI, jacobi_phase_launches(pl, 1));
        if (!pl.projRes) {
            fx_launch_project(stream, pl.half, d, pl.bricks[FX_SHAPE_ROW4], 1);
            mark(FIREX_PASS_PROJECT, 1);
        }
        fx_launch_step_end(stream, d);
        if (pl.pack) fx_launch_pack_batch(stream, d, pl.bricks[FX_SHAPE_ROW4]);
        mark(FIREX_PASS_OTHER, pl.pack ? 2 : 1);
    }

    cudaError_t graph_for(const StepPlan& pl, cudaGraphExec_t* out) {
        auto it = graphs.find(pl);
        if (it != graphs.end()) {
            *out = it->second;
            return cudaSuccess;
        }
        // a serving batch changes membership often: keep a bounded set of step graphs
        if (graphs.size() >= 16) {
            cudaError_t w = cudaStreamSynchronize(stream);  // no replay of them is still in flight
            if (w != cudaSuccess) return w;
            drop_graphs();
        }
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        enqueue_step_launches(stream, pl, d);
        e = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess) return e;
        cudaGraphExec_t ex = nullptr;
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
        graphs[pl] = ex;
        *out = ex;
        return cudaSuccess;
    }

    int step(int nsteps, double dt) {
        if (members.empty() || nsteps == 0) return FIREX_OK;
        DeviceGuard dg(device);
        for (firex_sim* s : members) {
            if (s->poisoned) return fail(FIREX_ERR_STATE, "a member simulation is poisoned");
            if (s->h.dt != dt) {
                s->h.dt = dt;
                s->refresh_params();
            }
            s->prepare_particles(stream);
            s->flush(stream);
        }
        const StepPlan pl = plan();
        cudaError_t e = flush_table();
        if (e != cudaSuccess) return poison(e, "batch table");
        cudaGraphExec_t ex = nullptr;
        if (useGraphs && !profiling) {
            e = graph_for(pl, &ex);
            if (e != cudaSuccess) {
                cudaGetLastError();
                useGraphs = false;  // direct launches remain correct
            }
        }
        last = pl;
        lastGraph = ex != nullptr;
        for (int i = 0; i < nsteps; ++i) {
            if (profiling) enqueue_profiled(pl);
            else if (ex) e = cudaGraphLaunch(ex, stream);
            else enqueue_step_launches(stream, pl, d);
            if (e != cudaSuccess) return poison(e, "step");
            for (firex_sim* s : members) s->advance_mirror();
            if (!profiling) {
                pendingLaunches[FIREX_PASS_OTHER] += pl.pack ? 4 : 3;
                pendingLaunches[FIREX_PASS_SIMULATE] += 1;
                pendingLaunches[FIREX_PASS_DIVERGENCE] += pl.projDiv ? 1 : 2;
                pendingLaunches[FIREX_PASS_JACOBI] += jacobi_phase_launches(pl, 0) + jacobi_phase_launches(pl, 1);
                pendingLaunches[FIREX_PASS_PROJECT] += pl.projRes ? 1 : 2;
                pendingLaunches[FIREX_PASS_PARTICLES] += sph_launches(pl);
            }
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return poison(e, "step launch");
        return FIREX_OK;
    }

    int poison(cudaError_t e, const char* what) {
        for (firex_sim* s : members) s->cuda_fail(e, what);
        return fail(FIREX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }

    void drop_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }

    void destroy() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graphs();
        for (cudaEvent_t e : evPool) cudaEventDestroy(e);
        evPool.clear();
        if (d) cudaFree(d);
        d = nullptr;
        delete h;
        h = nullptr;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    static firex_batch* make(int device, bool solo, std::string* err) {
        firex_batch* b = new (std::nothrow) firex_batch();
        if (!b) return nullptr;
        b->device = device;
        b->isSolo = solo;
        b->h = new (std::nothrow) FxBatchDev();
        cudaError_t e = b->h ? cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) : cudaErrorMemoryAllocation;
        if (e == cudaSuccess) e = cudaMalloc(&b->d, sizeof(FxBatchDev));
        if (e != cudaSuccess) {
            if (err) *err = std::string("batch: ") + cudaGetErrorString(e);
            cudaGetLastError();
            b->destroy();
            delete b;
            return nullptr;
        }
        b->rebuild_table();
        return b;
    }
};

cudaStream_t firex_sim::stream() const { return batch ? batch->stream : solo->stream; }

int firex_sim::reset() {
    // FireXEngine.reset (FireXEngine.ts:843-852): counters to zero, every field cleared
    // (clearBuffer, :1948-1961), then initializeFields (:1962-1969).
    cudaStream_t st = stream();
    h.simTime = 0;
    h.frame = 0;
    h.fi = h.si = h.pi = 0;
    refresh_params();
    flush(st);
    const size_t v4 = (size_t)N * 16;
    for (int i = 0; i < 2; ++i) {
        cudaMemsetAsync(h.flow[i], 0, v4, st);
        cudaMemsetAsync(h.species[i], 0, (size_t)N * species_bytes(), st);
        cudaMemsetAsync(h.p[i], 0, (size_t)N * pressure_bytes(), st);
        if (h.corr[i] != h.p[i]) cudaMemsetAsync(h.corr[i], 0, (size_t)N * pressure_bytes(), st);
    }
    cudaMemsetAsync(h.div, 0, (size_t)N * 4, st);
    cudaMemsetAsync(h.reaction, 0, (size_t)N * 4, st);
    cudaMemsetAsync(h.liquid, 0, (size_t)N * 4, st);
    fx_launch_init(st, storage, d, 300.0f, (float)named[param_slot("oxygenRate")], opt.velocity_noise);
    if (h.np > 0) {  // initializeFields (FireXEngine.ts:1972-1973)
        write_particle_initial_state(st, water_active());
        liquidMayContainWater = false;
        h.water = 0;
        dirty = true;
        flush(st);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "reset");
    return FIREX_OK;
}

void firex_sim::write_particle_initial_state(cudaStream_t st, bool active) {
    const int n = h.np;
    auto P = [&](const char* k) { return named[param_slot(k)]; };
    const double domainWidth = P("domainWidth"), domainHeight = P("domainHeight"), domainDepth = P("domainDepth");
    const double aimX = (0.52 - 0.035) * domainWidth;
    const double aimY = (P("aimHeight") - 0.5) * domainHeight;
    const double aimLength = std::hypot(aimX, aimY);
    const double base[3] = {aimX / aimLength, aimY / aimLength, 0.0};
    const double tangent[3] = {base[1], -base[0], 0.0};
    auto hash = [](double v) {
        const double x = std::sin(v * 12.9898 + 1.317) * 43758.5453;
        return x - std::floor(x);
    };
    const double nozzle = P("nozzleType"), waterFlow = P("waterFlow"), sprayAngle = P("sprayAngle");
    cudaStreamSynchronize(st);  // the staging buffer may still feed an earlier copy
    hostParticles.assign((size_t)n * 8, 0.0f);
    for (int i = 0; i < n; ++i) {
        float* o = hostParticles.data() + 8 * (size_t)i;
        const double phase = (double)i / n;
        const double angle = hash(i * 3.771 + 4.91) * M_PI * 2;
        const double radial = std::sqrt(hash(i * 3.771 + 0.17));
        const double spreadScale = nozzle >= 0.5 ? 0.72 : 0.1;
        const double cone = std::tan((sprayAngle * M_PI) / 180) * radial * spreadScale;
        const double diskX = tangent[0] * std::cos(angle), diskY = tangent[1] * std::cos(angle), diskZ = -std::sin(angle);
        double dx = base[0] + diskX * cone, dy = base[1] + diskY * cone, dz = diskZ * cone;
        const double dl = std::sqrt(dx * dx + dy * dy + dz * dz);
        dx /= dl;
        dy /= dl;
        dz /= dl;
        const double sv = nozzle >= 0.5 ? 0.24 : 0.05;
        const double speed = (0.82 + waterFlow * 0.82) * (1 - sv * 0.5 + hash(i * 3.771 + 9.37) * sv);
        const double age = phase * 0.72;
        const double originRadius = nozzle >= 0.5 ? 0.006 : 0.0028;
        o[0] = (float)(0.035 + (diskX * radial * originRadius + dx * speed * age) / domainWidth);
        o[1] = (float)std::max(0.012, 0.5 + (diskY * radial * originRadius + dy * speed * age - 0.29 * age * age) / domainHeight);
        o[2] = (float)(0.5 + (diskZ * radial * originRadius + dz * speed * age) / domainDepth);
        o[3] = (float)(active ? age : -phase * 0.72);
        o[4] = (float)(active ? dx * speed : 0.0);
        o[5] = (float)(active ? dy * speed - 0.58 * age : 0.0);
        o[6] = (float)(active ? dz * speed : 0.0);
        o[7] = (float)(active ? 0.52 + waterFlow * 0.88 : 0.0);
    }
    cudaMemcpyAsync(h.part[0], hostParticles.data(), (size_t)n * 32, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(h.part[1], hostParticles.data(), (size_t)n * 32, cudaMemcpyHostToDevice, st);
    if (h.pti != 0) {
        h.pti = 0;
        dirty = true;
    }
    particleFieldActive = active;
}

void firex_sim::release() {
    if (batch) cudaStreamSynchronize(batch->stream);  // no batch work may still use the buffers
    if (batch && batch != solo) {
        auto& m = batch->members;
        m.erase(std::remove(m.begin(), m.end(), this), m.end());
        batch->rebuild_table();
        batch->drop_graphs();
        batch = nullptr;
    }
    if (solo) {
        solo->destroy();
        delete solo;
        solo = nullptr;
    }
    if (own) cudaStreamSynchronize(own);
    if (copyStream) {
        cudaStreamSynchronize(copyStream);
        cudaStreamDestroy(copyStream);
        copyStream = nullptr;
    }
    if (evStaged) cudaEventDestroy(evStaged);
    if (evCopied) cudaEventDestroy(evCopied);
    evStaged = evCopied = nullptr;
    copyPending = false;
    d_stage = nullptr;
    for (void* p : allocations) cudaFree(p);
    allocations.clear();
    if (own) cudaStreamDestroy(own);
    own = nullptr;
}

// ---- host-side field conversion for the mixed storage -----------------------------------------
static inline float half_bits_to_float(uint16_t hb) {
    __half hv;
    std::memcpy(&hv, &hb, 2);
    return __half2float(hv);
}
static inline uint16_t float_to_half_bits(float f) {
    __half hv = __float2half_rn(f);
    uint16_t hb;
    std::memcpy(&hb, &hv, 2);
    return hb;
}

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
    o->particle_count = 640;  // the reference's balanced quality tier (FireXEngine.ts:206)
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
        case FIREX_FIELD_RENDER_FLOW:
        case FIREX_FIELD_RENDER_CHEMISTRY:
        case FIREX_FIELD_RENDER_MEDIA: return 8;
    }
    return 0;
}

uint64_t firex_reference_memory_estimate(const int32_t dims[3], int64_t particle_count) {
    if (!dims) return 0;
    uint64_t cells = (uint64_t)std::max(dims[0], 0) * (uint64_t)std::max(dims[1], 0) * (uint64_t)std::max(dims[2], 0);
    uint64_t per = cells >= (uint64_t)FIREX_HEAVY_GRID_CELL_THRESHOLD ? 108 : 116;
    return cells * per + (uint64_t)std::max<int64_t>(particle_count, 0) * 80 + 64ull * 64 * 64 * 4;
}

int firex_preflight(const int32_t dims[3], const firex_options* opt, const firex_device_limits* limits,
                    firex_preflight_result* out) {
    if (!dims || !opt || !out) return FIREX_ERR_BAD_ARG;
    std::memset(out, 0, sizeof(*out));
    firex_device_limits own = {2048, ((1ull << 31) - 1) * 16, ((1ull << 31) - 1) * 16};
    const firex_device_limits& L = limits ? *limits : own;
    const int64_t particles = std::max<int32_t>(opt->particle_count, 0);
    out->cell_count = (uint64_t)std::max(dims[0], 0) * (uint64_t)std::max(dims[1], 0) * (uint64_t)std::max(dims[2], 0);
    out->grid_bytes = out->cell_count * (out->cell_count >= (uint64_t)FIREX_HEAVY_GRID_CELL_THRESHOLD ? 108 : 116);
    out->particle_bytes = (uint64_t)particles * 80;
    out->fixed_bytes = 64ull * 64 * 64 * 4;
    out->total_bytes = out->grid_bytes + out->particle_bytes + out->fixed_bytes;
    out->largest_storage_buffer_bytes = out->cell_count * 16;
    std::string msg;
    auto issue = [&](uint32_t bit, const char* code, const std::string& text) {
        out->issues |= bit;
        out->issue_count += 1;
        msg += (msg.empty() ? "" : "; ") + std::string(code) + ": " + text;
    };
    const char* label[3] = {"X", "Y", "Z"};
    for (int i = 0; i < 3; ++i) {
        if (dims[i] <= 0)
            issue(FIREX_ISSUE_INVALID_DIMENSION, "invalid-dimension", std::string(label[i]) + " must be a positive integer.");
        else if (dims[i] % 4 != 0)
            issue(FIREX_ISSUE_UNALIGNED_DIMENSION, "unaligned-dimension", std::string(label[i]) + " must be a multiple of 4.");
        if (dims[i] > 0 && (uint64_t)dims[i] > L.max_texture_dimension_3d)
            issue(FIREX_ISSUE_TEXTURE_DIMENSION_LIMIT, "texture-dimension-limit",
                  std::string(label[i]) + "=" + std::to_string(dims[i]) + " exceeds this device's 3D-texture limit of " +
                      std::to_string(L.max_texture_dimension_3d) + ".");
    }
    if (out->largest_storage_buffer_bytes > L.max_storage_buffer_binding_size)
        issue(FIREX_ISSUE_STORAGE_BINDING_LIMIT, "storage-binding-limit",
              "A Fire-X vector field exceeds the storage-binding limit.");
    if (out->largest_storage_buffer_bytes > L.max_buffer_size)
        issue(FIREX_ISSUE_BUFFER_SIZE_LIMIT, "buffer-size-limit", "A Fire-X vector field exceeds the buffer limit.");
    if (opt->memory_budget_bytes && out->total_bytes > opt->memory_budget_bytes)
        issue(FIREX_ISSUE_MEMORY_BUDGET, "memory-budget",
              "Estimated persistent Fire-X resources require " + std::to_string(out->total_bytes) +
                  " bytes, above the configured " + std::to_string(opt->memory_budget_bytes) + " budget.");
    if (!(out->issues & (FIREX_ISSUE_INVALID_DIMENSION | FIREX_ISSUE_UNALIGNED_DIMENSION)))
        out->planned_device_bytes = firex_planned_device_bytes(dims, opt);
    std::snprintf(out->message, sizeof(out->message), "%s", msg.c_str());
    return FIREX_OK;
}

uint64_t firex_planned_device_bytes(const int32_t dims[3], const firex_options* opt) {
    if (!dims || !opt) return 0;
    const long long N = (long long)std::max(dims[0], 0) * std::max(dims[1], 0) * std::max(dims[2], 0);
    int mode = opt->pressure_mode;
    if (mode == FIREX_PRESSURE_AUTO) mode = N >= FIREX_HEAVY_GRID_CELL_THRESHOLD ? FIREX_PRESSURE_F16 : FIREX_PRESSURE_WARM_F32;
    const int storage = opt->precision == FIREX_PRECISION_MIXED ? FX_STORAGE_MIXED : FX_STORAGE_F32;
    return firex_sim::planned_bytes(dims[0], dims[1], dims[2], storage, mode, opt ? opt->particle_count : 0);
}

int firex_create(const int32_t dims[3], const firex_options* opt, firex_sim** out) {
    if (!out) return FIREX_ERR_BAD_ARG;
    *out = nullptr;
    if (!dims || !opt) {
        g_create_error = "dims and options are required";
        return FIREX_ERR_BAD_ARG;
    }
    {
        firex_preflight_result pre;
        firex_options o = *opt;
        o.memory_budget_bytes = 0;  // the budget is checked below against the planned residency
        firex_preflight(dims, &o, nullptr, &pre);
        if (pre.issues) {
            g_create_error = std::string("grid refused: ") + pre.message;
            return FIREX_ERR_BAD_ARG;
        }
    }
    if (opt->pressure_iterations < 0 || opt->correction_iterations < 0 || opt->pressure_iterations > 100000 ||
        opt->correction_iterations > 100000 || opt->num_spheres < 0 || opt->num_spheres > FIREX_MAX_SPHERES ||
        (opt->emitter_mode != FIREX_EMITTER_BURNER && opt->emitter_mode != FIREX_EMITTER_SPHERES) ||
        opt->pressure_mode < FIREX_PRESSURE_AUTO || opt->pressure_mode > FIREX_PRESSURE_COLD_F32 ||
        (opt->precision != FIREX_PRECISION_F32 && opt->precision != FIREX_PRECISION_MIXED) ||
        !(opt->velocity_noise >= 0) || !(opt->emission_jitter >= 0) || opt->jacobi_block < 0 ||
        opt->jacobi_block > 2) {
        g_create_error = "invalid options";
        return FIREX_ERR_BAD_ARG;
    }
    const long long N = (long long)dims[0] * dims[1] * dims[2];  // below 2^31: the preflight's buffer limits
    int mode = opt->pressure_mode;
    if (mode == FIREX_PRESSURE_AUTO) mode = N >= FIREX_HEAVY_GRID_CELL_THRESHOLD ? FIREX_PRESSURE_F16 : FIREX_PRESSURE_WARM_F32;
    const int storage = opt->precision == FIREX_PRECISION_MIXED ? FX_STORAGE_MIXED : FX_STORAGE_F32;
    const size_t need = firex_sim::planned_bytes(dims[0], dims[1], dims[2], storage, mode, opt->particle_count);
    if (opt->memory_budget_bytes && need > opt->memory_budget_bytes) {
        g_create_error = "memory-budget: grid needs " + std::to_string(need) + " device bytes, above the " +
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
    s->storage = storage;
    s->half = mode == FIREX_PRESSURE_F16;
    for (int i = 0; i < kNumParams; ++i) s->named[i] = kParams[i].def;
    if (opt->jacobi_block > 1) {
        s->jacobiKernel = FIREX_JACOBI_FUSED;
        s->jacobiK = opt->jacobi_block;
    }
    s->jacobiZc = std::max(0, opt->jacobi_zchunk);
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking);
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
    s->solo = firex_batch::make(s->device, true, &g_create_error);
    bool ok = s->solo != nullptr;
    FxSimDev& h = s->h;
    std::memset(&h, 0, sizeof(h));
    h.X = s->X;
    h.Y = s->Y;
    h.Z = s->Z;
    h.P = opt->pressure_iterations;
    h.R = opt->correction_iterations;
    h.mode = mode;
    h.storage = storage;
    h.active = 1;
    h.seed = opt->seed;
    h.jitterAmp = opt->emission_jitter;
    h.dt = 1.0 / 60.0;
    const size_t pb = s->pressure_bytes();
    for (int i = 0; i < 2 && ok; ++i) {
        ok = (h.flow[i] = s->alloc((size_t)N * 16)) && (h.species[i] = s->alloc((size_t)N * s->species_bytes())) &&
             (h.p[i] = s->alloc((size_t)N * pb));
        if (ok) h.corr[i] = (mode == FIREX_PRESSURE_COLD_F32) ? h.p[i] : s->alloc((size_t)N * pb);
        ok = ok && h.corr[i];
    }
    ok = ok && (h.div = (float*)s->alloc((size_t)N * 4)) && (h.reaction = (float*)s->alloc((size_t)N * 4)) &&
         (h.liquid = (uint32_t*)s->alloc((size_t)N * 4)) && (s->d_tmp = s->alloc((size_t)N * 4)) &&
         (h.tab = (float*)s->alloc(s->table_bytes())) &&
         (s->d = (FxSimDev*)s->alloc(sizeof(FxSimDev))) &&
         (s->d_partial = (double*)s->alloc(2 * sizeof(double) * (size_t)fx_norm_partial_blocks(N))) &&
         (s->d_norm = (double*)s->alloc(2 * sizeof(double))) && (h.sync = (unsigned*)s->alloc(FX_RES_SYNC_WORDS * 4)) &&
         cudaMemset(h.sync, 0, FX_RES_SYNC_WORDS * 4) == cudaSuccess;
    h.np = std::max(0, opt->particle_count);
    if (ok && h.np > 0)
        ok = (h.part[0] = (float4*)s->alloc((size_t)h.np * 32)) && (h.part[1] = (float4*)s->alloc((size_t)h.np * 32)) &&
             (h.pdens = (float4*)s->alloc((size_t)h.np * 16));
    if (!ok) {
        if (g_create_error.empty() || s->solo) g_create_error = "device allocation failed (" + std::to_string(need) + " bytes requested)";
        s->release();
        delete s;
        return FIREX_ERR_OOM;
    }
    fx_make_tensor_maps(&h);  // without them the two-sweep pass stages by cp.async
    s->solo->members.push_back(s);
    s->solo->rebuild_table();
    int rc = s->reset();
    if (rc == FIREX_OK) {
        e = cudaStreamSynchronize(s->stream());
        if (e != cudaSuccess) rc = s->cuda_fail(e, "initialise");
    }
    if (rc != FIREX_OK) {
        g_create_error = s->err;
        s->release();
        delete s;
        return rc;
    }
    g_create_error.clear();
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
    s->refresh_params();
    return FIREX_OK;
}

int firex_set_params(firex_sim* s, const float* p) {
    if (!s || !p) return FIREX_ERR_BAD_ARG;
    if (p[0] != (float)s->X || p[1] != (float)s->Y || p[2] != (float)s->Z)
        return s->fail(FIREX_ERR_BAD_ARG, "parameter block: grid slots differ from the handle's dimensions");
    // the parameter slots of the block (the layout build_params writes)
    static const struct {
        int slot;
        const char* name;
    } kSlots[] = {{8, "fuelRate"},        {9, "oxygenRate"},      {10, "heatEfficiency"},    {11, "vorticity"},
                  {12, "waterFlow"},      {13, "sprayAngle"},     {14, "waterEnabled"},      {16, "cameraYaw"},
                  {17, "cameraPitch"},    {18, "cameraDistance"}, {24, "viewMode"},          {25, "aimHeight"},
                  {26, "nozzleType"},     {27, "exposure"},       {28, "burnerSize"},        {29, "burnerDepth"},
                  {30, "sourceThickness"}, {31, "firePower"},     {32, "domainWidth"},       {33, "domainHeight"},
                  {34, "domainDepth"},    {36, "sourceLift"},     {37, "buoyancyScale"},     {38, "flamePersistence"},
                  {39, "viewZoom"},       {40, "airEntrainment"}, {41, "frontDefinition"},   {43, "opticalDetailTarget"}};
    for (const auto& e : kSlots) {
        const int i = param_slot(e.name);
        double v = p[e.slot];
        int kind = FIREX_VALUE_NUMBER;
        if (e.slot == 13) v = v * 180.0 / M_PI;  // the block holds radians, the parameter degrees
        if (e.slot == 14) kind = FIREX_VALUE_BOOLEAN;
        s->named[i] = apply_rule(kParams[i], s->named[i], kind, v);
    }
    s->refresh_params();
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
    if (s->batch) return s->fail(FIREX_ERR_STATE, "the simulation is a member of a batch; step the batch");
    if (nsteps < 0 || !std::isfinite(dt) || dt < 0) return s->fail(FIREX_ERR_BAD_ARG, "step count and dt must be finite and non-negative");
    int rc = s->solo->step(nsteps, dt);
    if (rc != FIREX_OK && s->err.empty()) s->err = s->solo->err;
    return rc;
}

int firex_sync(firex_sim* s) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    DeviceGuard dg(s->device);
    cudaError_t e = cudaStreamSynchronize(s->stream());
    if (e == cudaSuccess && s->copyStream) e = cudaStreamSynchronize(s->copyStream);
    if (e != cudaSuccess) return s->cuda_fail(e, "sync");
    s->copyPending = false;
    return s->check_device_waits();
}

// Writes sync words [first, first + n) of the simulation in stream order (the kernels read
// them at run time, so captured step graphs see the new values).
static int write_sync_words(firex_sim* s, int first, const unsigned* v, int n) {
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier error");
    DeviceGuard dg(s->device);
    cudaError_t e = cudaMemcpyAsync(s->h.sync + first, v, n * sizeof(unsigned), cudaMemcpyHostToDevice, s->stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream());
    if (e != cudaSuccess) return s->cuda_fail(e, "sync words");
    return FIREX_OK;
}

int firex_set_wait_limit(firex_sim* s, uint32_t polls) {
    if (!s) return FIREX_ERR_BAD_ARG;
    return write_sync_words(s, FX_SYNC_SPIN, &polls, 1);
}

int firex_test_hold_face(firex_sim* s, int32_t box, int32_t sweep) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (box >= FX_RES_MAX_CTAS || (box >= 0 && sweep < 0)) return s->fail(FIREX_ERR_BAD_ARG, "box or sweep out of range");
    const unsigned v[2] = {box >= 0 ? (unsigned)box + 1u : 0u, box >= 0 ? (unsigned)sweep : 0u};
    return write_sync_words(s, FX_SYNC_HOLD_BOX, v, 2);
}

// Device buffer and element size backing a field in the current parity, for direct copies.
static void* field_buffer(firex_sim* s, int32_t field) {
    const FxSimDev& h = s->h;
    switch (field) {
        case FIREX_FIELD_FLOW: return h.flow[h.fi];
        case FIREX_FIELD_SPECIES: return h.species[h.si];
        case FIREX_FIELD_PRESSURE: return h.p[h.pi];
        case FIREX_FIELD_DIVERGENCE: return h.div;
        case FIREX_FIELD_REACTION: return h.reaction;
        case FIREX_FIELD_LIQUID: return h.liquid;
        case FIREX_FIELD_CORRECTION: return h.corr[h.R & 1];
    }
    return nullptr;
}

int firex_read_field(firex_sim* s, int32_t field, void* host, size_t bytes) {
    if (!s || !host) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    const size_t es = firex_field_element_size(field);
    if (!es) return s->fail(FIREX_ERR_BAD_ARG, "unknown field id");
    if (bytes != es * (size_t)s->N) return s->fail(FIREX_ERR_BAD_ARG, "byte count does not match the field size");
    DeviceGuard dg(s->device);
    cudaStream_t st = s->stream();
    cudaError_t e = cudaSuccess;
    const size_t N = (size_t)s->N;
    if (field >= FIREX_FIELD_RENDER_FLOW && field <= FIREX_FIELD_RENDER_MEDIA) {
        if (!s->ensure_render_volumes()) return s->fail(FIREX_ERR_OOM, "render volumes: device allocation failed");
        s->flush(st);
        fx_launch_pack_sim(st, s->d);
        e = cudaMemcpyAsync(host, s->h.render[field - FIREX_FIELD_RENDER_FLOW], bytes, cudaMemcpyDeviceToHost, st);
    } else if (field == FIREX_FIELD_EMITTER_MASK || field == FIREX_FIELD_FINAL_DIVERGENCE) {
        s->flush(st);
        if (field == FIREX_FIELD_EMITTER_MASK) fx_launch_emitter_mask(st, s->d, (uint8_t*)s->d_tmp);
        else fx_launch_final_divergence(st, s->d, (float*)s->d_tmp);
        e = cudaMemcpyAsync(host, s->d_tmp, bytes, cudaMemcpyDeviceToHost, st);
    } else if ((field == FIREX_FIELD_CORRECTION && s->h.R == 0) ||
               (field == FIREX_FIELD_PRESSURE && s->mode == FIREX_PRESSURE_COLD_F32 &&
                (s->h.R == 0 || (s->h.R == 1 && s->h.pi == 0)))) {
        // Buffers the reference clears before the residual solve and no sweep rewrote
        // (FireXEngine.ts:2229-2230, :2258-2259): they read as zero.
        std::memset(host, 0, bytes);
    } else if (field == FIREX_FIELD_SPECIES && s->storage == FX_STORAGE_MIXED) {
        std::vector<uint16_t> raw(N * 4);
        e = cudaMemcpyAsync(raw.data(), field_buffer(s, field), N * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        float* o = (float*)host;
        for (size_t i = 0; i < N * 4; ++i) o[i] = half_bits_to_float(raw[i]);
    } else if ((field == FIREX_FIELD_PRESSURE || field == FIREX_FIELD_CORRECTION) && s->half) {
        std::vector<uint16_t> raw(N);
        e = cudaMemcpyAsync(raw.data(), field_buffer(s, field), N * 2, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        float* o = (float*)host;
        for (size_t i = 0; i < N; ++i) o[i] = half_bits_to_float(raw[i]);
    } else {
        e = cudaMemcpyAsync(host, field_buffer(s, field), bytes, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return s->cuda_fail(e, "read_field");
    return FIREX_OK;
}

int firex_read_field_async(firex_sim* s, int32_t field, void* host, size_t bytes) {
    if (!s || !host) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    const size_t es = firex_field_element_size(field);
    if (!es) return s->fail(FIREX_ERR_BAD_ARG, "unknown field id");
    if (bytes != es * (size_t)s->N) return s->fail(FIREX_ERR_BAD_ARG, "byte count does not match the field size");
    const bool direct = field == FIREX_FIELD_FLOW || field == FIREX_FIELD_DIVERGENCE || field == FIREX_FIELD_REACTION ||
                        field == FIREX_FIELD_LIQUID || (field == FIREX_FIELD_SPECIES && s->storage == FX_STORAGE_F32) ||
                        (field == FIREX_FIELD_PRESSURE && !s->half && s->mode != FIREX_PRESSURE_COLD_F32) ||
                        (field == FIREX_FIELD_CORRECTION && !s->half && s->h.R > 0);
    if (!direct) return s->fail(FIREX_ERR_UNSUPPORTED, "this field needs a host-side conversion: use firex_read_field");
    DeviceGuard dg(s->device);
    cudaError_t e = cudaSuccess;
    if (!s->copyStream) {
        e = cudaStreamCreateWithFlags(&s->copyStream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->evStaged, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->evCopied, cudaEventDisableTiming);
        if (e == cudaSuccess && !(s->d_stage = s->alloc((size_t)s->N * 16))) e = cudaErrorMemoryAllocation;
        if (e != cudaSuccess) return s->cuda_fail(e, "read_field_async set-up");
    }
    cudaStream_t st = s->stream();
    // the staging buffer is free once the previous host copy has finished
    if (s->copyPending) e = cudaStreamWaitEvent(st, s->evCopied, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_stage, field_buffer(s, field), bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(s->evStaged, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copyStream, s->evStaged, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, s->d_stage, bytes, cudaMemcpyDeviceToHost, s->copyStream);
    if (e == cudaSuccess) e = cudaEventRecord(s->evCopied, s->copyStream);
    if (e != cudaSuccess) return s->cuda_fail(e, "read_field_async");
    s->copyPending = true;
    return FIREX_OK;
}

int firex_write_field(firex_sim* s, int32_t field, const void* host, size_t bytes) {
    if (!s || !host) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    const size_t es = firex_field_element_size(field);
    if (!es) return s->fail(FIREX_ERR_BAD_ARG, "unknown field id");
    if (bytes != es * (size_t)s->N) return s->fail(FIREX_ERR_BAD_ARG, "byte count does not match the field size");
    if (field == FIREX_FIELD_EMITTER_MASK || field == FIREX_FIELD_FINAL_DIVERGENCE || field == FIREX_FIELD_CORRECTION ||
        field >= FIREX_FIELD_RENDER_FLOW)
        return s->fail(FIREX_ERR_BAD_ARG, "field is read only");
    DeviceGuard dg(s->device);
    cudaStream_t st = s->stream();
    const size_t N = (size_t)s->N;
    cudaError_t e;
    if (field == FIREX_FIELD_SPECIES && s->storage == FX_STORAGE_MIXED) {
        std::vector<uint16_t> raw(N * 4);
        const float* in = (const float*)host;
        for (size_t i = 0; i < N * 4; ++i) raw[i] = float_to_half_bits(in[i]);
        e = cudaMemcpyAsync(field_buffer(s, field), raw.data(), N * 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    } else if (field == FIREX_FIELD_PRESSURE && s->half) {
        std::vector<uint16_t> raw(N);
        const float* in = (const float*)host;
        for (size_t i = 0; i < N; ++i) raw[i] = float_to_half_bits(in[i]);
        e = cudaMemcpyAsync(field_buffer(s, field), raw.data(), N * 2, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    } else {
        e = cudaMemcpyAsync(field_buffer(s, field), host, bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return s->cuda_fail(e, "write_field");
    return FIREX_OK;
}

int firex_read_particles(firex_sim* s, void* host, size_t bytes) {
    if (!s || (!host && bytes)) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    if (bytes != (size_t)s->h.np * 32) return s->fail(FIREX_ERR_BAD_ARG, "byte count is not particle_count * 32");
    if (!bytes) return FIREX_OK;
    DeviceGuard dg(s->device);
    cudaStream_t st = s->stream();
    cudaError_t e = cudaMemcpyAsync(host, s->h.part[s->h.pti], bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return s->cuda_fail(e, "read_particles");
    return FIREX_OK;
}

int firex_write_particles(firex_sim* s, const void* host, size_t bytes) {
    if (!s || (!host && bytes)) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    if (bytes != (size_t)s->h.np * 32) return s->fail(FIREX_ERR_BAD_ARG, "byte count is not particle_count * 32");
    if (!bytes) return FIREX_OK;
    DeviceGuard dg(s->device);
    cudaStream_t st = s->stream();
    cudaError_t e = cudaMemcpyAsync(s->h.part[s->h.pti], host, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return s->cuda_fail(e, "write_particles");
    return FIREX_OK;
}

int firex_divergence_norm(firex_sim* s, double out[3]) {
    if (!s || !out) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    DeviceGuard dg(s->device);
    cudaStream_t st = s->stream();
    s->flush(st);
    fx_launch_divergence_norm(st, s->d, s->N, s->d_partial, s->d_norm);
    double hbuf[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(hbuf, s->d_norm, sizeof(hbuf), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return s->cuda_fail(e, "divergence_norm");
    out[0] = hbuf[0];
    out[1] = hbuf[1];
    out[2] = (double)(s->X - 2) * (double)(s->Y - 2) * (double)(s->Z - 2);
    return FIREX_OK;
}

int firex_get_state(const firex_sim* s, firex_state* st) {
    if (!s || !st) return FIREX_ERR_BAD_ARG;
    st->simulation_time = s->h.simTime;
    st->frame_index = s->h.frame;
    st->species_index = s->h.si;
    st->pressure_index = s->h.pi;
    return FIREX_OK;
}

int firex_set_state(firex_sim* s, const firex_state* st) {
    if (!s || !st) return FIREX_ERR_BAD_ARG;
    if ((st->species_index & ~1) || (st->pressure_index & ~1) || !std::isfinite(st->simulation_time))
        return s->fail(FIREX_ERR_BAD_ARG, "invalid state");
    DeviceGuard dg(s->device);
    cudaStreamSynchronize(s->stream());
    s->h.simTime = st->simulation_time;
    s->h.frame = st->frame_index;
    s->h.si = st->species_index;
    s->h.pi = st->pressure_index;
    s->refresh_params();
    s->flush(s->stream());
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

void* firex_stream(const firex_sim* s) { return s ? (void*)s->stream() : nullptr; }

int firex_set_profiling(firex_sim* s, int32_t on) {
    if (!s) return FIREX_ERR_BAD_ARG;
    firex_batch* b = s->batch ? s->batch : s->solo;
    DeviceGuard dg(s->device);
    if (!on && b->profiling) b->collect_marks();
    b->profiling = on != 0;
    return FIREX_OK;
}

int firex_pass_times(firex_sim* s, double* ms, int64_t* launches) {
    if (!s) return FIREX_ERR_BAD_ARG;
    firex_batch* b = s->batch ? s->batch : s->solo;
    DeviceGuard dg(s->device);
    int rc = b->collect_marks();
    if (rc != FIREX_OK) return s->fail(rc, b->err);
    for (int p = 0; p < FIREX_PASS_COUNT; ++p) {
        if (ms) ms[p] = b->passMs[p];
        if (launches) launches[p] = b->passLaunches[p];
        b->passMs[p] = 0;
        b->passLaunches[p] = 0;
    }
    return FIREX_OK;
}

int firex_get_diagnostics(const firex_sim* s, firex_diagnostics* out) {
    if (!s || !out) return FIREX_ERR_BAD_ARG;
    std::memset(out, 0, sizeof(*out));
    const firex_batch* b = s->batch ? s->batch : s->solo;
    const StepPlan& p = b->last;
    out->fast_division = s->h.jcFastDiv;
    out->jacobi_block = p.k;
    out->jacobi_zchunk = p.k > 1 ? p.zc : (p.row4 ? 0 : p.zmZc);
    out->graph = b->lastGraph ? 1 : 0;
    out->launches_per_step =
        (p.projDiv ? 7 : 8) - (p.projRes ? 1 : 0) + (p.pack ? 1 : 0) + sph_launches(p) + jacobi_phase_launches(p, 0) +
        jacobi_phase_launches(p, 1);
    out->jacobi_kernel = p.res ? FIREX_JACOBI_RESIDENT
                               : (p.k > 1 ? FIREX_JACOBI_FUSED : (p.row4 ? FIREX_JACOBI_UNBLOCKED : FIREX_JACOBI_ZMARCH));
    out->jacobi_variant = p.res ? p.resVariant : -1;
    out->jacobi_staging = p.tma ? FIREX_STAGING_TMA : (p.k == 2 ? FIREX_STAGING_CPASYNC : -1);
    out->simulate_by = p.simBy;
    out->project_fused = p.projDiv ? 1 : 0;
    out->project_resident = p.projRes ? 1 : 0;
    return FIREX_OK;
}

static bool jacobi_args_ok(int32_t kernel, int32_t block, int32_t zchunk) {
    if (kernel < FIREX_JACOBI_AUTO || kernel > FIREX_JACOBI_RESIDENT || zchunk < 0 || zchunk > 4096) return false;
    if (kernel == FIREX_JACOBI_RESIDENT) return block >= 0 && block <= 5;
    return kernel != FIREX_JACOBI_FUSED || block == 2;
}
// the block argument kept per kernel: sweeps per launch (FUSED), variant + 1 (RESIDENT)
static int jacobi_block_kept(int32_t kernel, int32_t block) {
    return (kernel == FIREX_JACOBI_FUSED || kernel == FIREX_JACOBI_RESIDENT) ? block : 1;
}

int firex_set_jacobi(firex_sim* s, int32_t kernel, int32_t block, int32_t zchunk) {
    if (!s || !jacobi_args_ok(kernel, block, zchunk)) return FIREX_ERR_BAD_ARG;
    s->jacobiKernel = kernel;
    s->jacobiK = jacobi_block_kept(kernel, block);
    s->jacobiZc = zchunk;
    return FIREX_OK;
}

int firex_batch_set_jacobi(firex_batch* b, int32_t kernel, int32_t block, int32_t zchunk) {
    if (!b || !jacobi_args_ok(kernel, block, zchunk)) return FIREX_ERR_BAD_ARG;
    b->jacobiKernel = kernel;
    b->jacobiK = jacobi_block_kept(kernel, block);
    b->jacobiZc = zchunk;
    return FIREX_OK;
}

int firex_set_staging(firex_sim* s, int32_t staging) {
    if (!s || staging < FIREX_STAGING_AUTO || staging > FIREX_STAGING_TMA) return FIREX_ERR_BAD_ARG;
    s->staging = staging;
    return FIREX_OK;
}

int firex_batch_set_staging(firex_batch* b, int32_t staging) {
    if (!b || staging < FIREX_STAGING_AUTO || staging > FIREX_STAGING_TMA) return FIREX_ERR_BAD_ARG;
    b->staging = staging;
    return FIREX_OK;
}

static bool proj_ok(int p) { return p >= FIREX_PROJECT_AUTO && p <= FIREX_PROJECT_SEPARATE; }

int firex_set_tiles(firex_sim* s, int32_t simulate_by, int32_t project) {
    if (!s || !sim_by_ok(simulate_by) || !proj_ok(project)) return FIREX_ERR_BAD_ARG;
    s->simBy = simulate_by;
    s->projFuse = project;
    return FIREX_OK;
}

int firex_batch_set_tiles(firex_batch* b, int32_t simulate_by, int32_t project) {
    if (!b || !sim_by_ok(simulate_by) || !proj_ok(project)) return FIREX_ERR_BAD_ARG;
    b->simBy = simulate_by;
    b->projFuse = project;
    return FIREX_OK;
}

int firex_set_render_packing(firex_sim* s, int32_t on) {
    if (!s) return FIREX_ERR_BAD_ARG;
    if (s->poisoned) return s->fail(FIREX_ERR_STATE, "handle is poisoned by an earlier CUDA error");
    DeviceGuard dg(s->device);
    if (on && !s->ensure_render_volumes()) return s->fail(FIREX_ERR_OOM, "render volumes: device allocation failed");
    s->h.renderPack = on ? 1 : 0;
    s->dirty = true;
    return FIREX_OK;
}

int firex_render_volumes(const firex_sim* s, void* out[3]) {
    if (!s || !out) return FIREX_ERR_BAD_ARG;
    for (int k = 0; k < 3; ++k) out[k] = s->h.render[k];
    return FIREX_OK;
}

int firex_set_graphs(firex_sim* s, int32_t on) {
    if (!s) return FIREX_ERR_BAD_ARG;
    s->solo->useGraphs = on != 0;
    return FIREX_OK;
}

// ---- batches -------------------------------------------------------------------------------
int firex_batch_create(firex_batch** out) {
    if (!out) return FIREX_ERR_BAD_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        g_create_error = "CUDA unavailable";
        return FIREX_ERR_CUDA;
    }
    *out = firex_batch::make(dev, false, &g_create_error);
    return *out ? FIREX_OK : FIREX_ERR_OOM;
}

int firex_batch_destroy(firex_batch* b) {
    if (!b) return FIREX_ERR_BAD_ARG;
    DeviceGuard dg(b->device);
    cudaStreamSynchronize(b->stream);
    for (firex_sim* s : b->members) {
        cudaEvent_t ev;
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        cudaEventRecord(ev, b->stream);
        cudaStreamWaitEvent(s->solo->stream, ev, 0);
        cudaEventDestroy(ev);
        s->batch = nullptr;
    }
    b->members.clear();
    b->destroy();
    delete b;
    return FIREX_OK;
}

const char* firex_batch_last_error(const firex_batch* b) { return b ? b->err.c_str() : g_create_error.c_str(); }

int firex_batch_add(firex_batch* b, firex_sim* s) {
    if (!b || !s) return FIREX_ERR_BAD_ARG;
    if (s->batch) return b->fail(FIREX_ERR_STATE, "the simulation already belongs to a batch");
    if (s->poisoned) return b->fail(FIREX_ERR_STATE, "the simulation is poisoned");
    if (s->device != b->device) return b->fail(FIREX_ERR_BAD_ARG, "the simulation lives on another device");
    if ((int)b->members.size() >= FX_MAX_BATCH) return b->fail(FIREX_ERR_BUDGET, "batch is full");
    if (!b->members.empty() && (b->members[0]->storage != s->storage || b->members[0]->half != s->half))
        return b->fail(FIREX_ERR_UNSUPPORTED, "batch members must share storage precision and pressure storage");
    DeviceGuard dg(b->device);
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventRecord(ev, s->solo->stream);
    cudaStreamWaitEvent(b->stream, ev, 0);  // the batch runs after the sim's queued work
    cudaEventDestroy(ev);
    s->batch = b;
    s->dirty = true;
    b->members.push_back(s);
    b->rebuild_table();
    return FIREX_OK;
}

int firex_batch_remove(firex_batch* b, firex_sim* s) {
    if (!b || !s) return FIREX_ERR_BAD_ARG;
    if (s->batch != b) return b->fail(FIREX_ERR_BAD_ARG, "the simulation is not a member of this batch");
    DeviceGuard dg(b->device);
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventRecord(ev, b->stream);
    cudaStreamWaitEvent(s->solo->stream, ev, 0);  // later sim work runs after the batch's
    cudaEventDestroy(ev);
    auto& m = b->members;
    m.erase(std::remove(m.begin(), m.end(), s), m.end());
    s->batch = nullptr;
    s->dirty = true;
    b->rebuild_table();
    return FIREX_OK;
}

int firex_batch_size(const firex_batch* b, int32_t* n) {
    if (!b || !n) return FIREX_ERR_BAD_ARG;
    *n = (int32_t)b->members.size();
    return FIREX_OK;
}

int firex_batch_step(firex_batch* b, int32_t nsteps, double dt) {
    if (!b) return FIREX_ERR_BAD_ARG;
    if (nsteps < 0 || !std::isfinite(dt) || dt < 0) return b->fail(FIREX_ERR_BAD_ARG, "step count and dt must be finite and non-negative");
    return b->step(nsteps, dt);
}

int firex_batch_sync(firex_batch* b) {
    if (!b) return FIREX_ERR_BAD_ARG;
    DeviceGuard dg(b->device);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return b->poison(e, "batch sync");
    for (firex_sim* s : b->members) {
        if (s->copyStream) {
            e = cudaStreamSynchronize(s->copyStream);
            if (e != cudaSuccess) return b->poison(e, "batch sync (readback)");
            s->copyPending = false;
        }
        const int rc = s->check_device_waits();
        if (rc != FIREX_OK) return b->fail(rc, s->err);
    }
    return FIREX_OK;
}

void* firex_batch_stream(const firex_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"
