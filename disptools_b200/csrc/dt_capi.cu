// Host side of disptools_b200: the C ABI, the error state, the device
// workspace and the device-resident solve loop.
//
// A solve runs as a sequence of "steps"; each step is one gradient launch
// (a no-op for volumes that do not need a new gradient) followed by one trial
// launch whose last block runs the step control of every volume on the
// device.  Steps are captured once into a CUDA graph of K steps and the graph
// is relaunched until every volume reports done; the host reads the small
// state array once per graph launch, never per trial.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "dt_internal.h"

using namespace dtb;

// ---------------------------------------------------------------------------
// Error state: same record and semantics as src/disptools.c:8-43.
// ---------------------------------------------------------------------------
static disptools_error_state g_error = {false, -1, "", "", "", ""};

static void set_error(int line, const char *function, const char *message) {
    g_error.error = true;
    g_error.line = line;
    std::snprintf(g_error.file, sizeof g_error.file, "%s", __FILE__);
    std::snprintf(g_error.function, sizeof g_error.function, "%s", function);
    std::snprintf(g_error.message, sizeof g_error.message, "%s", message);
    g_error.trace[0] = '\0';
}

#define DTB_FAIL(code, msg)                         \
    do {                                            \
        set_error(__LINE__, __func__, (msg));       \
        return (code);                              \
    } while (0)

#define DTB_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            char m_[1024];                                                                     \
            std::snprintf(m_, sizeof m_, "CUDA error %d (%s) in %s", (int) e_,                 \
                          cudaGetErrorString(e_), #call);                                      \
            set_error(__LINE__, __func__, m_);                                                 \
            return DTB_ERR_CUDA;                                                               \
        }                                                                                      \
    } while (0)

extern "C" disptools_error_state *disptools_get_error(void) { return &g_error; }
extern "C" bool disptools_has_error(void) { return g_error.error; }
extern "C" void disptools_clear_error(void) {
    g_error.error = false;
    g_error.line = -1;
    g_error.file[0] = g_error.function[0] = g_error.message[0] = g_error.trace[0] = '\0';
}
extern "C" int get_float_type_size(void) { return 64; }

static std::atomic<unsigned long long> g_launches{0};
static thread_local bool t_capturing = false;
void dtb::set_capturing(bool on) { t_capturing = on; }
void dtb::count_launch(unsigned n) {
    if (!t_capturing) g_launches += n;
}
extern "C" unsigned long long dtb_kernel_launch_count(void) { return g_launches.load(); }

// ---------------------------------------------------------------------------
// Kernel profiling: per-kernel launch counts and device time of the launches
// that did work, measured with CUDA events recorded between the kernels of
// the captured step graph.
// ---------------------------------------------------------------------------
namespace {
enum { PROF_TRIAL = 0, PROF_GRADIENT = 1, PROF_KINDS = 2 + dtb::PROF_MATCH_KINDS };
const char *const kProfNames[PROF_KINDS] = {"trial", "gradient", "match_gradient", "match_cost"};
struct Profile {
    bool on = false;
    long long launches[PROF_KINDS] = {};
    double ms[PROF_KINDS] = {};
};
std::mutex g_prof_mutex;
Profile g_prof;
}  // namespace

bool dtb::profiling_on() {
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    return g_prof.on;
}

void dtb::profile_match(int kind, double ms) {
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    if (!g_prof.on || kind < 0 || kind >= PROF_MATCH_KINDS) return;
    g_prof.launches[2 + kind]++;
    g_prof.ms[2 + kind] += ms;
}

extern "C" int dtb_set_profiling(int on) {
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    g_prof = Profile();
    g_prof.on = on != 0;
    return DTB_OK;
}

extern "C" int dtb_get_profile(dtb_kernel_profile *out, int max) {
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    int n = 0;
    for (int k = 0; k < PROF_KINDS && n < max; ++k, ++n) {
        std::snprintf(out[n].name, sizeof out[n].name, "%s", kProfNames[k]);
        out[n].launches = g_prof.launches[k];
        out[n].total_ms = g_prof.ms[k];
    }
    return n;
}

static int default_precision_init() {
    const char *p = std::getenv("DISPTOOLS_B200_PRECISION");
    if (p && (!std::strcmp(p, "fp64") || !std::strcmp(p, "FP64") || !std::strcmp(p, "double")))
        return DTB_PRECISION_FP64;
    return DTB_PRECISION_MIXED;
}
static int g_default_precision = default_precision_init();

extern "C" int dtb_set_default_precision(int precision) {
    if (precision != DTB_PRECISION_MIXED && precision != DTB_PRECISION_FP64) {
        set_error(__LINE__, __func__, "invalid precision");
        return DTB_ERR_ARGUMENT;
    }
    g_default_precision = precision;
    return DTB_OK;
}
extern "C" int dtb_get_default_precision(void) { return g_default_precision; }

// cuda/device.cu:4-15
extern "C" bool set_device(const int id) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        set_error(__LINE__, __func__, "cannot query the CUDA device count");
        return false;
    }
    if (id < 0 || id >= n) return false;
    if (cudaSetDevice(id) != cudaSuccess) {
        cudaGetLastError();
        set_error(__LINE__, __func__, "cudaSetDevice failed");
        return false;
    }
    return true;
}

// NVTX range over a scope (shows the solver's phases in a timeline profiler;
// header-only NVTX 3, inactive unless a tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// ---------------------------------------------------------------------------
// Device workspace: one growing allocation reused across calls.
// ---------------------------------------------------------------------------
namespace {

struct Workspace {
    void *ptr = nullptr;
    size_t bytes = 0;
};
std::mutex g_ws_mutex;
// Per device: the solver's scratch (pitched buffers, descriptors, partials),
// the staging area of host-array calls and the adjoint's weights.  They grow
// on demand and are kept until dtb_release_device_memory() or the end of the
// process.
std::vector<Workspace> g_ws, g_io, g_adj;
// Per device: recorded after the last adjoint's gather pass, on its stream.
std::vector<cudaEvent_t> g_adj_done;

// Failure-path test hook (dtb_test_drop_tma_load).
struct DropTest {
    long long tile = -1;
    int iteration = -1;
    unsigned wait_limit = 0;
} g_drop;

// Cap on the device memory each of the two areas may hold (0: none).
size_t g_mem_limit = 0;

int grow(std::vector<Workspace> &pool, size_t bytes, char **out) {
    int dev = 0;
    DTB_CUDA(cudaGetDevice(&dev));
    if ((int) pool.size() <= dev) pool.resize(dev + 1);
    Workspace &w = pool[dev];
    if (g_mem_limit && bytes > g_mem_limit)
        DTB_FAIL(DTB_ERR_ALLOC, "the solve needs more device memory than the limit set by "
                                "dtb_set_device_memory_limit");
    if (w.ptr && w.bytes < bytes) {
        cudaFree(w.ptr);
        w.ptr = nullptr;
        w.bytes = 0;
    }
    if (!w.ptr) {
        size_t want = bytes + bytes / 8;
        if (g_mem_limit && want > g_mem_limit) want = g_mem_limit;
        if (cudaMalloc(&w.ptr, want) != cudaSuccess) {
            cudaGetLastError();
            w.ptr = nullptr;
            DTB_FAIL(DTB_ERR_ALLOC, "cannot allocate the device workspace");
        }
        w.bytes = want;
    }
    *out = static_cast<char *>(w.ptr);
    return DTB_OK;
}

// Returns a device buffer of at least `bytes` on the current device.
int workspace(size_t bytes, char **out) { return grow(g_ws, bytes, out); }
// Staging buffer of host-array calls (separate from the workspace, which the
// solve itself carves up).
int io_buffer(size_t bytes, char **out) { return grow(g_io, bytes, out); }

// Bump allocator over a workspace region (256-byte alignment).
struct Carve {
    char *base;
    size_t off = 0;
    template <typename U>
    U *take(size_t count) {
        off = (off + 255) & ~size_t(255);
        U *p = reinterpret_cast<U *>(base + off);
        off += count * sizeof(U);
        return p;
    }
};

bool valid_dims(size_t nx, size_t ny, size_t nz) {
    // The one-sided boundary stencils read two voxels inward (src/headers/
    // jacobian_macros.h:7-99), so every axis needs at least three voxels.
    return nx >= 3 && ny >= 3 && nz >= 3 && nx < (1u << 30) && ny < (1u << 30) && nz < (1u << 30);
}

Geom make_geom(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz, int order = 4) {
    Geom g;
    g.nx = (int) nx;
    g.ny = (int) ny;
    g.nz = (int) nz;
    g.order = order;
    g.ys = (long long) nx;
    g.zs = (long long) nx * ny;
    g.cs = (long long) nx * ny * nz;
    g.ih[0] = 1.0 / dx;  // src/jacobian.c:73-75
    g.ih[1] = 1.0 / dy;
    g.ih[2] = 1.0 / dz;
    g.sp[0] = dx;
    g.sp[1] = dy;
    g.sp[2] = dz;
    return g;
}

// Planes per tile along z for a volume of nz planes.
int bz_for(int nz, int bz) { return nz < bz ? nz : bz; }

int steps_per_graph() {
    const char *e = std::getenv("DISPTOOLS_B200_STEPS_PER_GRAPH");
    if (e) {
        const int v = std::atoi(e);
        if (v > 0) return v;
    }
    return 16;
}

// Device view of one volume for the solver (device pointers of type T).
template <typename T>
struct DevVol {
    Geom g;
    const T *Jt;
    const uint8_t *mask;
    T *field;  // in: initial guess, out: result
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = [] {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &ptr, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            ptr = nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(ptr);
    }();
    return fn;
}

// Tiled map over a pitched [comps][nz][ny][nx] array (comps = 1 gives rank 3).
// The box is box_x x box_y x box_z voxels of every component.
bool encode_map(CUtensorMap *out, CUtensorMapDataType type, size_t esize, const void *base, const Geom &g, int comps,
                uint32_t box_x, uint32_t box_y, uint32_t box_z = 1) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const int rank = comps > 1 ? 4 : 3;
    cuuint64_t dims[4] = {(cuuint64_t) g.nx, (cuuint64_t) g.ny, (cuuint64_t) g.nz, (cuuint64_t) comps};
    cuuint64_t strides[3] = {(cuuint64_t) g.ys * esize, (cuuint64_t) g.zs * esize, (cuuint64_t) g.cs * esize};
    cuuint32_t box[4] = {box_x, box_y, box_z, (cuuint32_t) comps};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(out, type, rank, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map over the adjoint's weights W[c][a][wn] (the field's row and
// plane strides): dimensions x, y, z, a, c; boxes of box_x x box_y voxels
// of one plane, one axis a and all three components.
bool encode_weights_map(CUtensorMap *out, CUtensorMapDataType type, size_t esize, const void *W, const Geom &g,
                        long long wn, uint32_t box_x, uint32_t box_y) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[5] = {(cuuint64_t) g.nx, (cuuint64_t) g.ny, (cuuint64_t) g.nz, 3, 3};
    cuuint64_t strides[4] = {(cuuint64_t) g.ys * esize, (cuuint64_t) g.zs * esize, (cuuint64_t) wn * esize,
                             (cuuint64_t) (3 * wn) * esize};
    cuuint32_t box[5] = {box_x, box_y, 1, 1, 3};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return fn(out, type, 5, const_cast<void *>(W), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Geometry of the solver's own buffers: rows padded to 16 elements so that
// every row starts 16-byte aligned (a TMA requirement for all element types).
Geom pitched(const Geom &g) {
    Geom q = g;
    q.ys = ((long long) g.nx + 15) / 16 * 16;
    q.zs = q.ys * g.ny;
    q.cs = q.zs * g.nz;
    return q;
}

// Copies rows of a dense [rows][nx] array into/out of a pitched one.
template <typename U>
cudaError_t copy_rows(U *dst, size_t dpitch, const U *src, size_t spitch, size_t nx, size_t rows, cudaStream_t s) {
    return cudaMemcpy2DAsync(dst, dpitch * sizeof(U), src, spitch * sizeof(U), nx * sizeof(U), rows,
                             cudaMemcpyDeviceToDevice, s);
}

int num_sms() {
    static int n = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    return n;
}

// Per-device resources that live across solves: the solver's own stream,
// pinned host mirrors, events and the captured step graph (reused while the
// launch configuration is unchanged).
struct GraphKey {
    size_t tsize = 0;
    int algorithm = -1;
    const void *desc = nullptr;
    const int *tile_vol = nullptr;
    int total_tiles = 0, grid_t = 0, grid_g = 0, grid_b = 0, K = 0, threads_y = 0;
    const unsigned char *flags = nullptr;
    bool operator==(const GraphKey &o) const {
        return tsize == o.tsize && algorithm == o.algorithm && desc == o.desc && tile_vol == o.tile_vol &&
               total_tiles == o.total_tiles && grid_t == o.grid_t && grid_g == o.grid_g && grid_b == o.grid_b &&
               K == o.K && threads_y == o.threads_y && flags == o.flags;
    }
};

struct Engine {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_order = nullptr;
    SolverState *h_states = nullptr;
    size_t states_cap = 0;
    unsigned char *h_flags = nullptr;
    unsigned char *d_flags = nullptr;
    size_t flags_cap = 0;
    std::vector<cudaEvent_t> evs;      // profiling events: two sets of nk + 1
    cudaEvent_t ev_done[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // the same steps with either set of events and flags
    GraphKey key;
    int last_cfg[4] = {0, 0, 0, 0};  // tile shapes of the last solve (TileConfig order)
    int last_trial_kind = -1;        // trial kernel of the last solve (TileConfig::trial_kind)
};
std::vector<Engine *> g_engines;

// The engine of the current device (created on first use).
int engine(Engine **out) {
    int dev = 0;
    DTB_CUDA(cudaGetDevice(&dev));
    if ((int) g_engines.size() <= dev) g_engines.resize(dev + 1, nullptr);
    Engine *e = g_engines[dev];
    if (!e) {
        e = new Engine();
        e->device = dev;
        DTB_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        DTB_CUDA(cudaEventCreate(&e->ev0));
        DTB_CUDA(cudaEventCreate(&e->ev1));
        DTB_CUDA(cudaEventCreateWithFlags(&e->ev_order, cudaEventDisableTiming));
        DTB_CUDA(cudaEventCreateWithFlags(&e->ev_done[0], cudaEventDisableTiming));
        DTB_CUDA(cudaEventCreateWithFlags(&e->ev_done[1], cudaEventDisableTiming));
        g_engines[dev] = e;
    }
    *out = e;
    return DTB_OK;
}

// Host copies of the states: two sets of `count` (one per replay in flight).
int ensure_host_states(Engine *e, size_t count) {
    count *= 2;
    if (e->states_cap >= count) return DTB_OK;
    if (e->h_states) cudaFreeHost(e->h_states);
    e->h_states = nullptr;
    e->states_cap = 0;
    DTB_CUDA(cudaMallocHost(&e->h_states, count * sizeof(SolverState)));
    e->states_cap = count;
    return DTB_OK;
}

// Work flags and events of the profiled step graphs: two sets (one per
// replay in flight) of nk flags and nk + 1 events.
int ensure_profiling(Engine *e, size_t nk) {
    if (e->flags_cap < 2 * nk) {
        if (e->h_flags) cudaFreeHost(e->h_flags);
        if (e->d_flags) cudaFree(e->d_flags);
        e->h_flags = e->d_flags = nullptr;
        e->flags_cap = 0;
        DTB_CUDA(cudaMallocHost(&e->h_flags, 2 * nk));
        DTB_CUDA(cudaMalloc(&e->d_flags, 2 * nk));
        e->flags_cap = 2 * nk;
    }
    while (e->evs.size() < 2 * (nk + 1)) {
        cudaEvent_t ev;
        DTB_CUDA(cudaEventCreate(&ev));
        e->evs.push_back(ev);
    }
    return DTB_OK;
}

// Verbose output of the solvers (the reference's verbose_printf lines);
// -1: read DISPTOOLS_B200_VERBOSE on first use.
int g_verbose = -1;
bool verbose_enabled() {
    if (g_verbose < 0) {
        const char *v = std::getenv("DISPTOOLS_B200_VERBOSE");
        g_verbose = (v && std::strcmp(v, "0") != 0 && v[0]) ? 1 : 0;
    }
    return g_verbose != 0;
}

// Tile and block shape of the TMA kernels (gradient method):
//   tile_x    tile width in voxels (32, or 64 for FP32); tiles are TT_Y high
//   trial_ty  thread rows of the trial kernel (16: one tile row and two
//             columns per thread; 8: two rows)
//   grad_ty   thread rows of the gradient kernel (16: one tile row and two
//             columns per thread; 8: two rows)
//   bz        planes of a tile along z (capped at nz)
//   pf        L2 prefetch distance in planes beyond each TMA load (0: off)
//   trial_kind  trial kernel of the gradient method: 0 k_trial_tma (candidate
//             planes formed in a shared ring, one block barrier per plane),
//             1 k_trial_rel (stages held until their plane was the centre,
//             taps formed where read, no barrier in the plane loop)
// The greedy method runs 32 x TT_Y tiles of bz planes.
struct TileConfig {
    int tile_x = 32, trial_ty = 16, grad_ty = 16, bz = 32, pf = 0, trial_kind = 0;
};

// Explicit shapes from the environment (DISPTOOLS_B200_TILE_X = 32 | 64,
// DISPTOOLS_B200_TRIAL_THREADS_Y = 8 | 16, DISPTOOLS_B200_THREADS_Y = 8 | 16,
// DISPTOOLS_B200_BZ > 0).  Returns true when any is set; the autotuner is
// then skipped.
bool env_config(size_t tsize, TileConfig *c) {
    bool any = false;
    auto num = [&](const char *name, int *out, std::initializer_list<int> allowed) {
        const char *e = std::getenv(name);
        if (!e) return;
        const int v = std::atoi(e);
        bool ok = allowed.size() == 0 ? v > 0 : false;
        for (int a : allowed) ok |= v == a;
        if (ok) {
            *out = v;
            any = true;
        }
    };
    num("DISPTOOLS_B200_TILE_X", &c->tile_x, {32, 64});
    num("DISPTOOLS_B200_TRIAL_THREADS_Y", &c->trial_ty, {8, 16});
    num("DISPTOOLS_B200_THREADS_Y", &c->grad_ty, {8, 16});
    num("DISPTOOLS_B200_BZ", &c->bz, {});
    {
        // DISPTOOLS_B200_TRIAL_KERNEL = formed | release
        const char *e = std::getenv("DISPTOOLS_B200_TRIAL_KERNEL");
        if (e && (std::strcmp(e, "formed") == 0 || std::strcmp(e, "release") == 0)) {
            c->trial_kind = std::strcmp(e, "release") == 0 ? 1 : 0;
            any = true;
        }
    }
    {
        const char *e = std::getenv("DISPTOOLS_B200_PREFETCH");
        if (e) {
            const int v = std::atoi(e);
            if (v >= 0 && v <= 16) {
                c->pf = v;
                any = true;
            }
        }
    }
    if (tsize != 4) c->tile_x = 32;
    if (c->tile_x == 64) c->trial_ty = 16, c->grad_ty = 8;
    return any;
}

template <typename T>
int choose_config(Engine *e, int algorithm, const std::vector<DevVol<T>> &vols, const dtb_params &p,
                  int precision, TileConfig *out);

// One solve of `vols` on the engine's stream with tile shapes `cfg` (chosen
// by choose_config when null).  With `tune_ms` set it solves nothing: it
// sets the solve up on zeroed inputs, times one gradient and one trial launch
// of a mid-solve state (best of three after one warm-up) into *tune_ms and
// returns; the caller's arrays are not read.
template <typename T>
int solve_device_on(Engine *e, int algorithm, const std::vector<DevVol<T>> &vols, const dtb_params &p,
                    dtb_solve_stats *stats, int precision, const TileConfig *cfg_in = nullptr,
                    float *tune_ms = nullptr) {
    NvtxRange range(tune_ms ? "dtb tile-shape trial" : "dtb solve");
    cudaStream_t stream = e->stream;
    const int count = (int) vols.size();
    TileConfig cfg;
    if (cfg_in) {
        cfg = *cfg_in;
    } else {
        const int rc0 = choose_config<T>(e, algorithm, vols, p, precision, &cfg);
        if (rc0 != DTB_OK) return rc0;
    }
    e->last_cfg[0] = cfg.tile_x;
    e->last_cfg[1] = cfg.trial_ty;
    e->last_cfg[2] = cfg.grad_ty;
    e->last_cfg[3] = cfg.bz;
    e->last_trial_kind = cfg.trial_kind;
    // The greedy trial kernel exists for 32-wide tiles only.
    const int tile_x = algorithm == DTB_ALGORITHM_GRADIENT ? cfg.tile_x : 32;
    const int threads_y = cfg.grad_ty;
    const int trial_ty = cfg.trial_ty;
    const bool gradient = algorithm == DTB_ALGORITHM_GRADIENT;
    // ---- workspace layout: every buffer of the solve is the library's own,
    // in the pitched layout.
    const long long log_cap = (verbose_enabled() && !tune_ms)
                                  ? std::min<long long>(4 * (std::max<long long>(p.it_max, 0) + 16), 1ll << 20)
                                  : 0;
    std::vector<int> tiles(count), tbegin(count);
    std::vector<Geom> geo(count);
    int total_tiles = 0;
    size_t need = 0;
    auto align = [](size_t b) { return (b + 255) & ~size_t(255); };
    const int tile_y = TT_Y;
    for (int i = 0; i < count; ++i) {
        const Geom g = pitched(vols[i].g);
        geo[i] = g;
        const int bz = bz_for(g.nz, cfg.bz);
        const int t = ((g.nx + tile_x - 1) / tile_x) * ((g.ny + tile_y - 1) / tile_y) * ((g.nz + bz - 1) / bz);
        tiles[i] = t;
        tbegin[i] = total_tiles;
        total_tiles += t;
        const size_t N = (size_t) g.cs;
        need += 3 * align(3 * N * sizeof(T));       // field[0], field[1], gradient
        need += align(N * sizeof(T)) + align(N);     // target map, mask
        need += 2 * align(N * sizeof(T));            // e' (gradient) or error maps (greedy)
        need += align(t * sizeof(double2)) + align(t * sizeof(double));
        need += align(sizeof(SolverState)) + align(7 * sizeof(CUtensorMap));
        need += align((size_t) log_cap * sizeof(IterLog));
    }
    need += align(count * sizeof(VolumeDesc<T>)) + align(total_tiles * sizeof(int)) + align(2 * sizeof(TileQueue));

    char *base = nullptr;
    int rc = workspace(need, &base);
    if (rc != DTB_OK) return rc;
    Carve cv{base};

    std::vector<VolumeDesc<T>> desc(count);
    std::vector<SolverState> hst(count);
    std::vector<int> tile_vol(total_tiles);
    std::vector<CUtensorMap *> d_maps(count);
    for (int i = 0; i < count; ++i) {
        const Geom &g = geo[i];
        const Geom &gu = vols[i].g;  // caller's dense layout
        const size_t N = (size_t) g.cs;
        VolumeDesc<T> &d = desc[i];
        std::memset(&d, 0, sizeof d);
        d.g = g;
        d.field[0] = cv.take<T>(3 * N);
        d.field[1] = cv.take<T>(3 * N);
        d.grad = cv.take<T>(3 * N);
        T *Jt = cv.take<T>(N);
        uint8_t *mask = cv.take<uint8_t>(N);
        d.Jt = Jt;
        d.mask = mask;
        T *aux0 = cv.take<T>(N), *aux1 = cv.take<T>(N);
        if (gradient) {
            d.ep[0] = aux0;
            d.ep[1] = aux1;
        } else {
            d.v[0] = aux0;
            d.v[1] = aux1;
        }
        d.part_t = cv.take<double2>(tiles[i]);
        d.part_g = cv.take<double>(tiles[i]);
        d.st = cv.take<SolverState>(1);
        IterLog *log = log_cap ? cv.take<IterLog>((size_t) log_cap) : nullptr;
        d_maps[i] = cv.take<CUtensorMap>(7);
        const int bz = bz_for(g.nz, cfg.bz);
        d.tiles_x = (g.nx + tile_x - 1) / tile_x;
        d.tiles_y = (g.ny + tile_y - 1) / tile_y;
        d.tiles_z = (g.nz + bz - 1) / bz;
        d.tile_begin = tbegin[i];
        d.ntiles = tiles[i];
        d.bz = bz;
        d.drop_tile = !tune_ms ? (int) g_drop.tile : -1;
        d.drop_it = g_drop.iteration;
        d.wait_limit = g_drop.wait_limit;
        for (int t = 0; t < tiles[i]; ++t) tile_vol[tbegin[i] + t] = i;

        SolverState &s = hst[i];
        std::memset(&s, 0, sizeof s);
        s.epsilon = p.epsilon;
        s.tolerance = p.tolerance;
        s.eta_max = p.eta_max;
        s.alpha = p.alpha;
        s.beta = p.beta;
        s.gamma = p.gamma;
        s.delta = p.delta;
        s.zeta = p.zeta;
        s.theta = p.theta;
        s.iota = p.iota;
        s.it_max = p.it_max;
        s.strict = p.strict;
        s.algorithm = algorithm;
        s.eta = p.eta;
        s.E_last = DBL_MAX;
        s.M_last = DBL_MAX;
        s.phase = PH_EVAL0;
        s.log = log;
        s.log_cap = log_cap;
        s.log_n = 0;

        if (tune_ms) {
            // A step in the main loop: both kernels do all their work.
            s.phase = gradient ? PH_MAIN : PH_GREEDY;
            s.need_gradient = 1;
            DTB_CUDA(cudaMemsetAsync(d.field[0], 0, 3 * N * sizeof(T), stream));
            DTB_CUDA(cudaMemsetAsync(Jt, 0, N * sizeof(T), stream));
            DTB_CUDA(cudaMemsetAsync(mask, 0, N, stream));
        } else {
            // Inputs into the pitched layout.
            const size_t rows = (size_t) gu.ny * gu.nz;
            DTB_CUDA(copy_rows<T>(d.field[0], g.ys, vols[i].field, gu.ys, gu.nx, 3 * rows, stream));
            DTB_CUDA(copy_rows<T>(Jt, g.ys, vols[i].Jt, gu.ys, gu.nx, rows, stream));
            DTB_CUDA(copy_rows<uint8_t>(mask, g.ys, vols[i].mask, gu.ys, gu.nx, rows, stream));
        }
        // The gradient is zero on the boundary voxels, which the gradient
        // kernel never writes (src/displacement_field_gradient.c:26-145 on
        // calloc'd buffers).  For the greedy method the second field buffer
        // and the error maps start at zero as well: its update never writes
        // boundary voxels, so they keep the buffer's content
        // (src/displacement_field_greedy.c:43-65).  The gradient method's
        // trial writes every voxel of the candidate and of e' before they
        // are read.
        DTB_CUDA(cudaMemsetAsync(d.grad, 0, 3 * N * sizeof(T), stream));
        if (!gradient) {
            DTB_CUDA(cudaMemsetAsync(d.field[1], 0, 3 * N * sizeof(T), stream));
            DTB_CUDA(cudaMemsetAsync(aux0, 0, N * sizeof(T), stream));
            DTB_CUDA(cudaMemsetAsync(aux1, 0, N * sizeof(T), stream));
        }

        {
            CUtensorMap h_maps[7];
            const CUtensorMapDataType ft = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
            // Boxes: the tile plus 4 voxels in x (16-byte aligned start) and 2
            // rows in y for the stencil inputs; the bare tile for J_t and the
            // mask.  The greedy method's error maps are read one plane at a
            // time with 3 rows of halo in y (slots 3 and 4).
            const uint32_t bx = (uint32_t) tile_x;
            T *m3 = gradient ? d.ep[0] : d.v[0], *m4 = gradient ? d.ep[1] : d.v[1];
            const uint32_t my = gradient ? TT_Y + 4 : TT_Y + 6, mz = 1;
            bool ok = encode_map(&h_maps[0], ft, sizeof(T), d.field[0], g, 3, bx + 8, TT_Y + 4) &&
                      encode_map(&h_maps[1], ft, sizeof(T), d.field[1], g, 3, bx + 8, TT_Y + 4) &&
                      encode_map(&h_maps[2], ft, sizeof(T), d.grad, g, 3, bx + 8, TT_Y + 4) &&
                      encode_map(&h_maps[3], ft, sizeof(T), m3, g, 1, bx + 8, my, mz) &&
                      encode_map(&h_maps[4], ft, sizeof(T), m4, g, 1, bx + 8, my, mz) &&
                      encode_map(&h_maps[5], ft, sizeof(T), Jt, g, 1, bx, TT_Y) &&
                      encode_map(&h_maps[6], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, mask, g, 1, bx, TT_Y);
            if (!ok) DTB_FAIL(DTB_ERR_CUDA, "cannot encode the TMA descriptors (cuTensorMapEncodeTiled)");
            // From pageable memory: the copy is staged before the call returns.
            DTB_CUDA(cudaMemcpyAsync(d_maps[i], h_maps, sizeof h_maps, cudaMemcpyHostToDevice, stream));
            d.tm_field[0] = d_maps[i] + 0;
            d.tm_field[1] = d_maps[i] + 1;
            d.tm_grad = d_maps[i] + 2;
            if (gradient) {
                d.tm_ep[0] = d_maps[i] + 3;
                d.tm_ep[1] = d_maps[i] + 4;
            } else {
                d.tm_v[0] = d_maps[i] + 3;
                d.tm_v[1] = d_maps[i] + 4;
            }
            d.tm_Jt = d_maps[i] + 5;
            d.tm_mask = d_maps[i] + 6;
        }
    }
    VolumeDesc<T> *d_desc = cv.take<VolumeDesc<T>>(count);
    int *d_tile_vol = cv.take<int>(total_tiles);
    TileQueue *d_queues = cv.take<TileQueue>(2);  // trial, gradient
    DTB_CUDA(cudaMemsetAsync(d_queues, 0, 2 * sizeof(TileQueue), stream));
    std::vector<SolverState *> d_states(count);
    for (int i = 0; i < count; ++i) {
        d_states[i] = desc[i].st;
        DTB_CUDA(cudaMemcpyAsync(desc[i].st, &hst[i], sizeof(SolverState), cudaMemcpyHostToDevice, stream));
        // Greedy method: whether the trial must copy the new buffer's
        // boundary values (they are all +0 unless the initial field's are not).
        if (!gradient && !tune_ms)
            DTB_CUDA(launch_boundary_nonzero<T>(desc[i].field[0], desc[i].g, &desc[i].st->b0_nonzero, stream));
    }
    DTB_CUDA(cudaMemcpyAsync(d_desc, desc.data(), count * sizeof(VolumeDesc<T>), cudaMemcpyHostToDevice, stream));
    DTB_CUDA(cudaMemcpyAsync(d_tile_vol, tile_vol.data(), total_tiles * sizeof(int), cudaMemcpyHostToDevice,
                             stream));


    // Persistent grids: as many blocks as fit on the device at once.
    const bool rel = gradient && cfg.trial_kind == 1;
    const int bps_t = !gradient ? greedy_tma_blocks_per_sm<T>()
                                : (rel ? trial_rel_blocks_per_sm<T>(tile_x, trial_ty)
                                       : trial_tma_blocks_per_sm<T>(tile_x, trial_ty));
    const int grid_t = std::min(total_tiles, std::max(1, bps_t) * num_sms());
    const int grid_g = std::min(total_tiles, std::max(1, gradient_tma_blocks_per_sm<T>(tile_x, threads_y)) * num_sms());
    auto launch_t = [&](unsigned char *flag) -> cudaError_t {
        if (rel)
            return launch_trial_rel<T>(d_desc, d_tile_vol, total_tiles, grid_t, stream, flag, tile_x, trial_ty,
                                       d_queues);
        if (gradient) return launch_trial_tma<T>(d_desc, d_tile_vol, total_tiles, grid_t, stream, flag, tile_x, trial_ty,
                                                    d_queues, cfg.pf);
        return launch_greedy_tma<T>(d_desc, d_tile_vol, total_tiles, grid_t, stream, flag, d_queues);
    };
    auto launch_g = [&](unsigned char *flag) -> cudaError_t {
        return launch_gradient_tma<T>(d_desc, d_tile_vol, total_tiles, grid_g, stream, flag, tile_x, threads_y,
                                      d_queues + 1, cfg.pf);
    };

    cudaEvent_t ev0 = e->ev0, ev1 = e->ev1;
    if (tune_ms) {
        float best = FLT_MAX;
        for (int r = 0; r < 4; ++r) {
            for (int i = 0; i < count; ++i)
                DTB_CUDA(cudaMemcpyAsync(desc[i].st, &hst[i], sizeof(SolverState), cudaMemcpyHostToDevice, stream));
            DTB_CUDA(cudaEventRecord(ev0, stream));
            if (gradient) DTB_CUDA(launch_g(nullptr));
            DTB_CUDA(launch_t(nullptr));
            DTB_CUDA(cudaEventRecord(ev1, stream));
            DTB_CUDA(cudaEventSynchronize(ev1));
            float ms = 0.f;
            DTB_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
            if (r > 0) best = std::min(best, ms);
        }
        *tune_ms = best;
        return DTB_OK;
    }
    DTB_CUDA(cudaEventRecord(ev0, stream));

    // Evaluate the initial fields (launched once, outside the graph; this is
    // also the first launch of each kernel, which sets its attributes).
    DTB_CUDA(launch_t(nullptr));
    if (gradient) DTB_CUDA(launch_g(nullptr));

    // Capture K steps into a graph (reused while the configuration is the
    // same).  With profiling on, event records are captured between the
    // kernels and every kernel gets a flag that it sets when it did work.
    const int K = steps_per_graph();
    const bool prof = g_prof.on;
    const int kernels_per_step = gradient ? 2 : 1;
    const int nk = K * kernels_per_step;
    if (prof) {
        rc = ensure_profiling(e, nk);
        if (rc != DTB_OK) return rc;
    }
    std::vector<cudaEvent_t> &evs = e->evs;
    unsigned char *d_flags = prof ? e->d_flags : nullptr, *h_flags = prof ? e->h_flags : nullptr;
    GraphKey key;
    key.tsize = sizeof(T);
    key.algorithm = algorithm;
    key.desc = d_desc;
    key.tile_vol = d_tile_vol;
    key.total_tiles = total_tiles;
    key.grid_t = grid_t;
    key.grid_g = grid_g;
    key.K = K;
    key.threads_y = (((trial_ty * 100 + threads_y) * 1000 + tile_x) * 100 + cfg.pf) * 2 + (rel ? 1 : 0);
    key.flags = d_flags;
    // Two graphs of the same K steps, each with its own set of profiling
    // events and work flags, so that one replay can be queued while the
    // host reads the results of the other.
    if (!(e->exec[0] && e->exec[1] && e->key == key)) {
        for (cudaGraphExec_t &x : e->exec) {
            if (x) cudaGraphExecDestroy(x);
            x = nullptr;
        }
        for (int b = 0; b < 2; ++b) {
            cudaEvent_t *ev = prof ? &evs[b * (nk + 1)] : nullptr;
            unsigned char *fl = prof ? d_flags + b * nk : nullptr;
            cudaGraph_t graph = nullptr;
            set_capturing(true);
            DTB_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            // Inside a capture only cudaEventRecordExternal turns a record
            // into an event-record node that fires on every replay.
            if (prof) {
                cudaMemsetAsync(fl, 0, nk, stream);
                cudaEventRecordWithFlags(ev[0], stream, cudaEventRecordExternal);
            }
            for (int k = 0, j = 0; k < K; ++k) {
                if (gradient) {
                    launch_g(prof ? fl + j : nullptr);
                    if (prof) cudaEventRecordWithFlags(ev[j + 1], stream, cudaEventRecordExternal);
                    ++j;
                }
                launch_t(prof ? fl + j : nullptr);
                if (prof) cudaEventRecordWithFlags(ev[j + 1], stream, cudaEventRecordExternal);
                ++j;
            }
            cudaError_t cap = cudaStreamEndCapture(stream, &graph);
            set_capturing(false);
            if (cap != cudaSuccess) {
                cudaGetLastError();
                DTB_CUDA(cap);
            }
            cudaError_t inst = cudaGraphInstantiate(&e->exec[b], graph, 0);
            cudaGraphDestroy(graph);
            DTB_CUDA(inst);
        }
        e->key = key;
    }

    // Replays alternate between the two graphs; replay r copies the states
    // (and flags) into host set r % 2 and records ev_done[r % 2].  The host
    // queues replay r + 1 before it waits for replay r, so the device never
    // idles while the host checks.  Kernels of a finished volume return at
    // once, so the one replay queued after the last useful one costs only
    // its launches.
    rc = ensure_host_states(e, count);
    if (rc != DTB_OK) return rc;
    long long max_steps = 0;
    for (int i = 0; i < count; ++i) max_steps = std::max(max_steps, 64 * (p.it_max + 2) + 4096);
    long long steps = 0;
    int status = DTB_OK;
    cudaError_t loop_err = cudaSuccess;
    auto enqueue = [&](long long r) -> cudaError_t {
        const int b = (int) (r & 1);
        cudaError_t err = cudaGraphLaunch(e->exec[b], stream);
        if (err != cudaSuccess) return err;
        count_launch(nk);
        steps += K;
        SolverState *hs = e->h_states + (size_t) b * count;
        for (int i = 0; i < count; ++i)
            cudaMemcpyAsync(&hs[i], d_states[i], sizeof(SolverState), cudaMemcpyDeviceToHost, stream);
        if (prof) cudaMemcpyAsync(h_flags + b * nk, d_flags + b * nk, nk, cudaMemcpyDeviceToHost, stream);
        return cudaEventRecord(e->ev_done[b], stream);
    };
    // Waits for replay r, adds its profile; true when every volume is done.
    auto finish = [&](long long r, bool *all_done) -> cudaError_t {
        const int b = (int) (r & 1);
        cudaError_t err = cudaEventSynchronize(e->ev_done[b]);
        if (err != cudaSuccess) return err;
        if (prof) {
            std::lock_guard<std::mutex> lock(g_prof_mutex);
            const cudaEvent_t *ev = &evs[b * (nk + 1)];
            for (int j = 0; j < nk; ++j) {
                if (!h_flags[b * nk + j]) continue;
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, ev[j], ev[j + 1]) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                const int kind = (gradient && j % 2 == 0) ? PROF_GRADIENT : PROF_TRIAL;
                g_prof.launches[kind]++;
                g_prof.ms[kind] += ms;
            }
        }
        const SolverState *hs = e->h_states + (size_t) b * count;
        bool done = true;
        for (int i = 0; i < count; ++i) done &= hs[i].done != 0;
        *all_done = done;
        return cudaSuccess;
    };
    NvtxRange loop_range("dtb step graphs");
    long long r = 0;
    if ((loop_err = enqueue(0)) != cudaSuccess) status = DTB_ERR_CUDA;
    while (status == DTB_OK) {
        if ((loop_err = enqueue(r + 1)) != cudaSuccess) {
            status = DTB_ERR_CUDA;
            break;
        }
        bool all_done = false;
        if ((loop_err = finish(r, &all_done)) != cudaSuccess) {
            status = DTB_ERR_CUDA;
            break;
        }
        ++r;
        if (all_done) break;
        if (steps > max_steps) {
            status = DTB_ERR_ARGUMENT;
            break;
        }
    }
    // The replay queued last (r): wait for it so its states and profile are read.
    if (status == DTB_OK) {
        bool all_done = false;
        if ((loop_err = finish(r, &all_done)) != cudaSuccess) status = DTB_ERR_CUDA;
    }
    const SolverState *h_states = e->h_states + (size_t) (r & 1) * count;
    const cudaError_t rec_err = cudaEventRecord(ev1, stream);
    if (status == DTB_OK && rec_err != cudaSuccess) {
        status = DTB_ERR_CUDA;
        loop_err = rec_err;
    }
    if (status == DTB_ERR_CUDA) DTB_CUDA(loop_err != cudaSuccess ? loop_err : cudaErrorUnknown);
    if (status != DTB_OK) DTB_FAIL(status, "the solver did not terminate within its step bound");

    // Results: the accepted field is field[old_buf]; copy it back into the
    // caller's dense buffer.
    for (int i = 0; i < count; ++i) {
        const SolverState &s = h_states[i];
        if (s.fault) DTB_FAIL(DTB_ERR_CUDA, "a TMA transfer did not complete within its bound");
        const Geom &gu = vols[i].g;
        DTB_CUDA(copy_rows<T>(vols[i].field, gu.ys, desc[i].field[s.old_buf], geo[i].ys, gu.nx,
                              3 * (size_t) gu.ny * gu.nz, stream));
    }
    DTB_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev0, ev1) != cudaSuccess) ms = -1.f;
    cudaGetLastError();
    if (log_cap) {
        // The reference's verbose lines (src/displacement_field_gradient.c:377-410,
        // src/displacement_field_greedy.c:184-228), printed after the solve.
        for (int i = 0; i < count; ++i) {
            const SolverState &s = h_states[i];
            std::vector<IterLog> lines((size_t) std::min(s.log_n, log_cap));
            if (!lines.empty())
                DTB_CUDA(cudaMemcpy(lines.data(), s.log, lines.size() * sizeof(IterLog), cudaMemcpyDeviceToHost));
            if (count > 1) std::printf("Volume %d\n", i);
            for (const IterLog &l : lines) {
                if (l.kind == 0)
                    std::printf("Iteration %5lld:  total error %6e  max voxel error %6e  eta %6e\n", l.it, l.E, l.M,
                                l.eta);
                else
                    std::printf("Error not decreasing, reducing step size to %.4e\n", l.eta);
            }
            switch (s.reason) {
            case DTB_STOP_ERROR_EXPLODED: std::printf("Terminating: error exploded.\n"); break;
            case DTB_STOP_ETA:
            case DTB_STOP_THETA: std::printf("Error not decreasing, terminating.\n"); break;
            case DTB_STOP_MAX_EXPLODED: std::printf("Terminating: voxel error exploded.\n"); break;
            case DTB_STOP_EPSILON: std::printf("Terminating: reached desired tolerance.\n"); break;
            default: break;
            }
            // Printed when the loop counter equals it_max on exit (:418).
            if (s.it == p.it_max) std::printf("Terminating: reached maximum number of iterations.\n");
        }
        std::fflush(stdout);
    }
    if (stats) {
        for (int i = 0; i < count; ++i) {
            const SolverState &s = h_states[i];
            dtb_solve_stats &o = stats[i];
            o.iterations = s.it;
            o.trials = s.trials;
            o.gradients = s.gradients;
            o.reason = s.reason;
            o.precision = precision;
            o.error = s.ret_E;
            o.max_error = s.ret_M;
            o.cand_error = s.E;
            o.cand_max_error = s.M;
            o.eta = s.eta;
            o.device_ms = ms;
        }
    }
    return DTB_OK;
}

// ---------------------------------------------------------------------------
// Autotuner of the tile shapes: the first gradient solve of a problem shape
// on a device times each candidate shape on the solve's own geometry (see
// solve_device_on's tuning mode) and keeps the fastest for later solves of
// that shape.  Solves of fewer than AUTOTUNE_MIN_VOXELS voxels, greedy solves
// and solves with shapes set in the environment take the fixed shapes.
// ---------------------------------------------------------------------------
struct TuneKey {
    int device;
    size_t tsize;
    int count;
    long long voxels;
    int mx, my, mz;
    bool operator<(const TuneKey &o) const {
        return std::tie(device, tsize, count, voxels, mx, my, mz) <
               std::tie(o.device, o.tsize, o.count, o.voxels, o.mx, o.my, o.mz);
    }
};
std::map<TuneKey, TileConfig> g_tuned;  // guarded by g_ws_mutex
int g_autotune = -1;                     // -1: read DISPTOOLS_B200_AUTOTUNE on first use
constexpr long long AUTOTUNE_MIN_VOXELS = 1ll << 21;

bool autotune_enabled() {
    if (g_autotune < 0) {
        const char *v = std::getenv("DISPTOOLS_B200_AUTOTUNE");
        g_autotune = (v && std::strcmp(v, "0") == 0) ? 0 : 1;
    }
    return g_autotune != 0;
}

// Planes per z tile that fill the waves of a persistent grid of `slots`
// resident blocks.  The launch is modelled as ceil(tiles / slots) waves of
// bz + 6 plane-times (a tile forms bz + 4 planes, plus its fixed cost), with
// tiles(bz) = sum over volumes of (x-y tiles) x ceil(nz / bz); the cheapest
// bz in [12, 64] wins, the larger one on ties.  At 256^3 with 32 x 16 tiles
// and 296 slots this gives 29 planes (1152 tiles, 3.9 waves) where 32
// planes leave the fourth wave less than half full (1024 tiles, 3.5 waves).
int wave_filled_bz(const std::vector<Geom> &geo, int tile_x, int slots) {
    int mz = 0;
    for (const Geom &g : geo) mz = std::max(mz, g.nz);
    int best = std::min(mz, 32);
    double best_t = DBL_MAX;
    for (int bz = std::min(64, mz); bz >= 12; --bz) {
        long long tiles = 0;
        for (const Geom &g : geo) {
            const int b = std::min(bz, g.nz);
            tiles += (long long) ((g.nx + tile_x - 1) / tile_x) * ((g.ny + TT_Y - 1) / TT_Y) * ((g.nz + b - 1) / b);
        }
        const double t = (double) ((tiles + slots - 1) / slots) * (bz + 6);
        if (t < best_t) {
            best_t = t;
            best = bz;
        }
    }
    return best;
}

// Candidate shapes, the one every other must beat by 1 % first: the default
// x-y shape at `bzw` (the wave-filled depth of the solve, 0: none), which
// measured 2 % faster than the fixed 32 planes at 256^3 (0.2275 against
// 0.233 ms a trial), else the fixed default.
std::vector<TileConfig> tile_candidates(size_t tsize, int bzw) {
    std::vector<TileConfig> c;
    const bool wave = bzw > 0 && bzw != 16 && bzw != 32 && bzw != 64;
    if (wave) c.push_back({32, 16, 16, bzw});
    const std::vector<TileConfig> fixed = {{32, 16, 16, 32}, {32, 16, 8, 32}, {32, 16, 16, 16}, {32, 16, 16, 64},
                                           {32, 8, 16, 32}};
    c.insert(c.end(), fixed.begin(), fixed.end());
    if (tsize == 4) c.push_back({64, 16, 8, 32});
    if (wave) c.push_back({32, 16, 8, bzw});
    // The trial kernel without the per-plane barrier (trial_kind 1) is not a
    // candidate: at 256^3 it took 0.305-0.315 ms a launch against 0.227-0.233
    // ms for the formed-plane kernel.  The environment can still select it.
    return c;
}

template <typename T>
int choose_config(Engine *e, int algorithm, const std::vector<DevVol<T>> &vols, const dtb_params &p,
                  int precision, TileConfig *out) {
    TileConfig c;
    if (env_config(sizeof(T), &c) || algorithm != DTB_ALGORITHM_GRADIENT || !autotune_enabled()) {
        *out = c;
        return DTB_OK;
    }
    TuneKey key{e->device, sizeof(T), (int) vols.size(), 0, 0, 0, 0};
    for (const DevVol<T> &v : vols) {
        key.voxels += (long long) v.g.nx * v.g.ny * v.g.nz;
        key.mx = std::max(key.mx, v.g.nx);
        key.my = std::max(key.my, v.g.ny);
        key.mz = std::max(key.mz, v.g.nz);
    }
    if (key.voxels < AUTOTUNE_MIN_VOXELS) {
        *out = c;
        return DTB_OK;
    }
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
        *out = it->second;
        return DTB_OK;
    }
    NvtxRange range("dtb autotune");
    TileConfig best = c;
    float best_ms = FLT_MAX;
    std::vector<Geom> geo;
    for (const DevVol<T> &v : vols) geo.push_back(v.g);
    const int slots = std::max(1, trial_tma_blocks_per_sm<T>(32, 16)) * num_sms();
    for (const TileConfig &cand : tile_candidates(sizeof(T), wave_filled_bz(geo, 32, slots))) {
        float ms = FLT_MAX;
        const int rc = solve_device_on<T>(e, algorithm, vols, p, nullptr, precision, &cand, &ms);
        if (rc != DTB_OK) return rc;
        // A shape must beat the best so far by 1 % to replace it, so timing
        // noise does not move the choice away from the default.
        if (best_ms == FLT_MAX || ms < 0.99f * best_ms) {
            best = cand;
            best_ms = ms;
        }
    }
    g_tuned[key] = best;
    *out = best;
    return DTB_OK;
}

// Device-resident solve of `vols` (all inputs already on the device), on the
// engine's own non-blocking stream (graph capture is not allowed on the
// legacy default stream), ordered after the caller's stream and before
// anything the caller enqueues next.
template <typename T>
int solve_device(int algorithm, const std::vector<DevVol<T>> &vols, const dtb_params &p,
                 dtb_solve_stats *stats, int precision, cudaStream_t user) {
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    Engine *e = nullptr;
    int rc = engine(&e);
    if (rc != DTB_OK) return rc;
    DTB_CUDA(cudaEventRecord(e->ev_order, user));
    DTB_CUDA(cudaStreamWaitEvent(e->stream, e->ev_order, 0));
    rc = solve_device_on<T>(e, algorithm, vols, p, stats, precision);
    if (cudaEventRecord(e->ev_order, e->stream) == cudaSuccess) cudaStreamWaitEvent(user, e->ev_order, 0);
    cudaStreamSynchronize(e->stream);
    cudaGetLastError();
    return rc;
}

bool check_params(const dtb_params &p, const char **why) {
    // ASSERT_PARAMETERS, src/headers/disptools.h:107-152, as errors.
    if (!(p.alpha > 0.0)) return *why = "alpha must be positive", false;
    if (!(p.beta > 0.0)) return *why = "beta must be positive", false;
    if (!(p.gamma > 0.0)) return *why = "gamma must be positive", false;
    if (!(p.delta > 0.0)) return *why = "delta must be positive", false;
    if (!(p.zeta > 0.0)) return *why = "zeta must be positive", false;
    if (!(p.eta > 0.0)) return *why = "eta must be positive", false;
    if (!(p.eta_max > 0.0)) return *why = "eta_max must be positive", false;
    if (!(p.theta >= 0.0)) return *why = "theta must be non-negative", false;
    if (!(p.iota >= 0.0)) return *why = "iota must be non-negative", false;
    if (!(p.tolerance >= 0.0)) return *why = "tolerance must be non-negative", false;
    if (!(p.epsilon > 0.0)) return *why = "epsilon must be positive", false;
    if (p.it_max < 0) return *why = "it_max must be non-negative", false;
    return true;
}

// Host-array solve: upload (converting to T), solve on the device, download.
// Everything runs on the device's engine stream; the device buffers come from
// the growing staging area, so a call allocates nothing once the area is large
// enough, and the host waits once, when the results have arrived.
template <typename T>
int solve_host(int algorithm, int count, const dtb_volume *vols, const dtb_params &p, dtb_solve_stats *stats,
               int precision) {
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    NvtxRange range("dtb solve (host arrays)");
    Engine *e = nullptr;
    int rc = engine(&e);
    if (rc != DTB_OK) return rc;
    cudaStream_t stream = e->stream;
    constexpr bool is_double = std::is_same<T, double>::value;
    auto align = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t need = 0, stage_elems = 0;
    for (int i = 0; i < count; ++i) {
        const size_t N = vols[i].nx * vols[i].ny * vols[i].nz;
        need += align(3 * N * sizeof(T)) + align(N * sizeof(T)) + align(N);
        stage_elems = std::max(stage_elems, 3 * N);
    }
    if (!is_double) need += align(stage_elems * sizeof(double));
    char *base = nullptr;
    rc = io_buffer(need, &base);
    if (rc != DTB_OK) return rc;
    Carve cv{base};
    double *stage = is_double ? nullptr : cv.take<double>(stage_elems);
    std::vector<DevVol<T>> dv(count);
    for (int i = 0; i < count; ++i) {
        const dtb_volume &v = vols[i];
        const size_t N = v.nx * v.ny * v.nz;
        T *field = cv.take<T>(3 * N);
        T *Jt = cv.take<T>(N);
        uint8_t *mask = cv.take<uint8_t>(N);
        if (is_double) {
            DTB_CUDA(cudaMemcpyAsync(field, v.field, 3 * N * sizeof(double), cudaMemcpyHostToDevice, stream));
            DTB_CUDA(cudaMemcpyAsync(Jt, v.J, N * sizeof(double), cudaMemcpyHostToDevice, stream));
        } else {
            // The stage is reused by every volume: stream order puts each
            // copy after the previous conversion.
            DTB_CUDA(cudaMemcpyAsync(stage, v.field, 3 * N * sizeof(double), cudaMemcpyHostToDevice, stream));
            DTB_CUDA(launch_convert<T>(stage, 1, field, 3 * (long long) N, stream));
            DTB_CUDA(cudaMemcpyAsync(stage, v.J, N * sizeof(double), cudaMemcpyHostToDevice, stream));
            DTB_CUDA(launch_convert<T>(stage, 1, Jt, (long long) N, stream));
        }
        static_assert(sizeof(bool) == 1, "bool must be one byte");
        DTB_CUDA(cudaMemcpyAsync(mask, v.mask, N, cudaMemcpyHostToDevice, stream));
        dv[i] = DevVol<T>{make_geom(v.nx, v.ny, v.nz, v.dx, v.dy, v.dz), Jt, mask, field};
    }
    rc = solve_device_on<T>(e, algorithm, dv, p, stats, precision);
    if (rc != DTB_OK) {
        cudaStreamSynchronize(stream);
        cudaGetLastError();
        return rc;
    }
    for (int i = 0; i < count; ++i) {
        const dtb_volume &v = vols[i];
        const size_t N = v.nx * v.ny * v.nz;
        if (is_double) {
            DTB_CUDA(cudaMemcpyAsync(v.field, dv[i].field, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, stream));
        } else {
            DTB_CUDA(launch_to_double<T>(dv[i].field, stage, 3 * (long long) N, stream));
            DTB_CUDA(cudaMemcpyAsync(v.field, stage, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, stream));
        }
    }
    DTB_CUDA(cudaStreamSynchronize(stream));
    return DTB_OK;
}

int check_volumes(int count, const dtb_volume *vols) {
    if (count < 1 || !vols) DTB_FAIL(DTB_ERR_ARGUMENT, "no volumes");
    for (int i = 0; i < count; ++i) {
        const dtb_volume &v = vols[i];
        if (!valid_dims(v.nx, v.ny, v.nz)) DTB_FAIL(DTB_ERR_ARGUMENT, "every axis needs at least 3 voxels");
        if (!v.J || !v.mask || !v.field) DTB_FAIL(DTB_ERR_ARGUMENT, "null array");
        if (!(v.dx > 0.0 && v.dy > 0.0 && v.dz > 0.0)) DTB_FAIL(DTB_ERR_ARGUMENT, "spacing must be positive");
    }
    return DTB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Explicit entry points.
// ---------------------------------------------------------------------------
extern "C" int dtb_generate_displacement_batched(int algorithm, int precision, int count,
                                                 const dtb_volume *volumes, const dtb_params *params,
                                                 dtb_solve_stats *stats) {
    disptools_clear_error();
    if (algorithm != DTB_ALGORITHM_GRADIENT && algorithm != DTB_ALGORITHM_GREEDY)
        DTB_FAIL(DTB_ERR_ARGUMENT, "invalid algorithm");
    if (precision != DTB_PRECISION_MIXED && precision != DTB_PRECISION_FP64)
        DTB_FAIL(DTB_ERR_ARGUMENT, "invalid precision");
    if (!params) DTB_FAIL(DTB_ERR_ARGUMENT, "null parameters");
    const char *why = nullptr;
    if (!check_params(*params, &why)) DTB_FAIL(DTB_ERR_ARGUMENT, why);
    int rc = check_volumes(count, volumes);
    if (rc != DTB_OK) return rc;
    if (precision == DTB_PRECISION_FP64) return solve_host<double>(algorithm, count, volumes, *params, stats, precision);
    return solve_host<float>(algorithm, count, volumes, *params, stats, precision);
}

extern "C" int dtb_generate_displacement(int algorithm, int precision, size_t nx, size_t ny, size_t nz, double dx,
                                         double dy, double dz, const double *J, const bool *mask,
                                         const dtb_params *params, double *field, dtb_solve_stats *stats) {
    if (algorithm == DTB_ALGORITHM_MATCHING) {
        disptools_clear_error();
        if (!params) DTB_FAIL(DTB_ERR_ARGUMENT, "null parameters");
        const char *why = nullptr;
        if (!check_params(*params, &why)) DTB_FAIL(DTB_ERR_ARGUMENT, why);
        return dtb_volume_matching(nx, ny, nz, dx, dy, dz, J, mask, params, field, stats);
    }
    const dtb_volume v = {nx, ny, nz, dx, dy, dz, J, mask, field};
    return dtb_generate_displacement_batched(algorithm, precision, 1, &v, params, stats);
}

extern "C" int dtb_generate_displacement_batched_device(int algorithm, int precision, int count,
                                                        const dtb_device_volume *volumes,
                                                        const dtb_params *params, dtb_solve_stats *stats,
                                                        void *stream) {
    disptools_clear_error();
    if (algorithm == DTB_ALGORITHM_MATCHING) {
        // The matching solver, one volume after the other, on float64 arrays.
        if (precision != DTB_PRECISION_FP64)
            DTB_FAIL(DTB_ERR_ARGUMENT, "the matching solver takes float64 device arrays");
        if (!params || count < 1 || !volumes) DTB_FAIL(DTB_ERR_ARGUMENT, "null argument");
        const char *why = nullptr;
        if (!check_params(*params, &why)) DTB_FAIL(DTB_ERR_ARGUMENT, why);
        for (int i = 0; i < count; ++i) {
            const dtb_device_volume &v = volumes[i];
            const int rc = dtb_volume_matching_device(v.nx, v.ny, v.nz, v.dx, v.dy, v.dz,
                                                      static_cast<const double *>(v.J), params,
                                                      static_cast<double *>(v.field), stats ? &stats[i] : nullptr,
                                                      stream);
            if (rc != DTB_OK) return rc;
        }
        return DTB_OK;
    }
    if (algorithm != DTB_ALGORITHM_GRADIENT && algorithm != DTB_ALGORITHM_GREEDY)
        DTB_FAIL(DTB_ERR_ARGUMENT, "invalid algorithm");
    if (precision != DTB_PRECISION_MIXED && precision != DTB_PRECISION_FP64)
        DTB_FAIL(DTB_ERR_ARGUMENT, "invalid precision");
    if (!params || count < 1 || !volumes) DTB_FAIL(DTB_ERR_ARGUMENT, "null argument");
    const char *why = nullptr;
    if (!check_params(*params, &why)) DTB_FAIL(DTB_ERR_ARGUMENT, why);
    for (int i = 0; i < count; ++i) {
        const dtb_device_volume &v = volumes[i];
        if (!valid_dims(v.nx, v.ny, v.nz)) DTB_FAIL(DTB_ERR_ARGUMENT, "every axis needs at least 3 voxels");
        if (!v.J || !v.mask || !v.field) DTB_FAIL(DTB_ERR_ARGUMENT, "null array");
        if (!(v.dx > 0.0 && v.dy > 0.0 && v.dz > 0.0)) DTB_FAIL(DTB_ERR_ARGUMENT, "spacing must be positive");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == DTB_PRECISION_FP64) {
        std::vector<DevVol<double>> dv(count);
        for (int i = 0; i < count; ++i) {
            const dtb_device_volume &v = volumes[i];
            dv[i] = DevVol<double>{make_geom(v.nx, v.ny, v.nz, v.dx, v.dy, v.dz), static_cast<const double *>(v.J),
                                   static_cast<const uint8_t *>(v.mask), static_cast<double *>(v.field)};
        }
        return solve_device<double>(algorithm, dv, *params, stats, precision, s);
    }
    std::vector<DevVol<float>> dv(count);
    for (int i = 0; i < count; ++i) {
        const dtb_device_volume &v = volumes[i];
        dv[i] = DevVol<float>{make_geom(v.nx, v.ny, v.nz, v.dx, v.dy, v.dz), static_cast<const float *>(v.J),
                              static_cast<const uint8_t *>(v.mask), static_cast<float *>(v.field)};
    }
    return solve_device<float>(algorithm, dv, *params, stats, precision, s);
}

// ---------------------------------------------------------------------------
// Reference-named solver entry points (FLOATING = double).
// ---------------------------------------------------------------------------
static void reference_solve(int algorithm, size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
                            const double *J, const bool *mask, double epsilon, double tolerance, double eta,
                            double eta_max, double alpha, double beta, double gamma, double delta, double zeta,
                            double theta, double iota, bool strict, size_t it_max, double *field) {
    dtb_params p;
    p.epsilon = epsilon;
    p.tolerance = tolerance;
    p.eta = eta;
    p.eta_max = eta_max;
    p.alpha = alpha;
    p.beta = beta;
    p.gamma = gamma;
    p.delta = delta;
    p.zeta = zeta;
    p.theta = theta;
    p.iota = iota;
    p.strict = strict ? 1 : 0;
    p.it_max = (long long) it_max;
    dtb_generate_displacement(algorithm, g_default_precision, nx, ny, nz, dx, dy, dz, J, mask, &p, field, nullptr);
}

extern "C" void generate_displacement_gradient_cuda(
    const size_t nx, const size_t ny, const size_t nz, const double dx, const double dy, const double dz,
    const double *J, const bool *mask, const double epsilon, const double tolerance, double eta,
    const double eta_max, const double alpha, const double beta, const double gamma, const double delta,
    const double zeta, const double theta, const double iota, const bool strict, const size_t it_max,
    double *field) {
    reference_solve(DTB_ALGORITHM_GRADIENT, nx, ny, nz, dx, dy, dz, J, mask, epsilon, tolerance, eta, eta_max, alpha,
                    beta, gamma, delta, zeta, theta, iota, strict, it_max, field);
}

extern "C" void generate_displacement_greedy_cuda(
    const size_t nx, const size_t ny, const size_t nz, const double dx, const double dy, const double dz,
    const double *J, const bool *mask, const double epsilon, const double tolerance, double eta,
    const double eta_max, const double alpha, const double beta, const double gamma, const double delta,
    const double zeta, const double theta, const double iota, const bool strict, const size_t it_max,
    double *field) {
    reference_solve(DTB_ALGORITHM_GREEDY, nx, ny, nz, dx, dy, dz, J, mask, epsilon, tolerance, eta, eta_max, alpha,
                    beta, gamma, delta, zeta, theta, iota, strict, it_max, field);
}

// ---------------------------------------------------------------------------
// Jacobian (device pointers) and its adjoint.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
int jacobian_device_impl(const Geom &g, const T *field, T *J, cudaStream_t s) {
    // TMA kernel: fourth order, rows a multiple of 16 bytes long, a 16-byte
    // aligned field and pair-aligned J.  It takes its tensor map as a kernel
    // parameter and needs no device memory of its own: no lock, no wait.
    if (g.order == 4 && (g.ys * (long long) sizeof(T)) % 16 == 0 && reinterpret_cast<uintptr_t>(field) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(J) % (2 * sizeof(T)) == 0) {
        CUtensorMap tm;
        const CUtensorMapDataType ft = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        if (encode_map(&tm, ft, sizeof(T), field, g, 3, 32 + 2 * 4, TT_Y + 2 * 2)) {
            DTB_CUDA(launch_jacobian_tma<T>(tm, g, J, g.ys, g.zs, num_sms(), s));
            return DTB_OK;
        }
    }
    // Other layouts and order 2: the plain-load kernel, with its descriptor
    // in the shared workspace.
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    const int bz = bz_for(g.nz, 32);
    const int ntiles = ((g.nx + BX - 1) / BX) * ((g.ny + BY - 1) / BY) * ((g.nz + bz - 1) / bz);
    char *base = nullptr;
    int rc = workspace(1024 + sizeof(VolumeDesc<T>) + (size_t) ntiles * sizeof(int), &base);
    if (rc != DTB_OK) return rc;
    Carve cv{base};
    VolumeDesc<T> *d_desc = cv.take<VolumeDesc<T>>(1);
    int *d_tv = cv.take<int>(ntiles);
    VolumeDesc<T> d;
    std::memset(&d, 0, sizeof d);
    d.g = g;
    d.field[0] = const_cast<T *>(field);
    d.jout = J;
    d.tiles_x = (g.nx + BX - 1) / BX;
    d.tiles_y = (g.ny + BY - 1) / BY;
    d.tiles_z = (g.nz + bz - 1) / bz;
    d.tile_begin = 0;
    d.ntiles = ntiles;
    d.bz = bz;
    DTB_CUDA(cudaMemcpyAsync(d_desc, &d, sizeof d, cudaMemcpyHostToDevice, s));
    DTB_CUDA(cudaMemsetAsync(d_tv, 0, (size_t) ntiles * sizeof(int), s));
    DTB_CUDA(launch_jacobian<T>(d_desc, d_tv, ntiles, ntiles, s));
    // The descriptor lives in the shared workspace: finish before releasing it.
    DTB_CUDA(cudaStreamSynchronize(s));
    return DTB_OK;
}

// The adjoint's path: the weight pass and gather by default, the fused TMA
// kernel (order 4, a 16-byte-aligned field whose rows are a multiple of 16
// bytes long) when DISPTOOLS_B200_ADJOINT=fused asks for it.
bool adjoint_fused_allowed() {
    const char *e = std::getenv("DISPTOOLS_B200_ADJOINT");
    return e && std::strcmp(e, "fused") == 0;
}

template <typename T>
int adjoint_device_impl(const Geom &g, const T *field, const T *gJ, T *gout, cudaStream_t s) {
    // Fused kernel: the weights stay on chip, the tensor map is a kernel
    // parameter, no device memory of its own: no lock, no wait.
    if (adjoint_fused_allowed() && g.order == 4 && (g.ys * (long long) sizeof(T)) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(field) % 16 == 0) {
        CUtensorMap tm;
        const CUtensorMapDataType ft = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        if (encode_map(&tm, ft, sizeof(T), field, g, 3, 32 + 2 * 4, TT_Y + 2 * 4)) {
            DTB_CUDA(launch_adjoint_tma<T>(tm, g, gJ, gout, num_sms(), s));
            return DTB_OK;
        }
    }
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    // Weights W[9][wn] in the adjoint's own buffer, each component 256-byte
    // aligned.  Calls are ordered on the device, not on the host: this
    // call's stream waits for the previous call's gather (any stream) before
    // it overwrites W.  Growing the buffer frees the old one, which waits
    // for the device.
    const long long wn = ((long long) g.cs + 63) / 64 * 64;
    char *base = nullptr;
    int rc = grow(g_adj, 9 * (size_t) wn * sizeof(T) + 256, &base);
    if (rc != DTB_OK) return rc;
    int dev = 0;
    DTB_CUDA(cudaGetDevice(&dev));
    if ((int) g_adj_done.size() <= dev) g_adj_done.resize(dev + 1, nullptr);
    if (!g_adj_done[dev]) DTB_CUDA(cudaEventCreateWithFlags(&g_adj_done[dev], cudaEventDisableTiming));
    DTB_CUDA(cudaStreamWaitEvent(s, g_adj_done[dev], 0));
    T *W = reinterpret_cast<T *>(base);
    // The weight pass on the TMA stencil kernel when the layout allows it
    // (as for the Jacobian map), else on the plain-load kernel.  The gather
    // pass streams W by TMA after a TMA weight pass (W then has rows a
    // multiple of 16 bytes long) into a pair-aligned gradient.
    bool w_done = false;
    const CUtensorMapDataType ft = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    if (g.order == 4 && (g.ys * (long long) sizeof(T)) % 16 == 0 && reinterpret_cast<uintptr_t>(field) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(gJ) % (2 * sizeof(T)) == 0) {
        CUtensorMap tm;
        if (encode_map(&tm, ft, sizeof(T), field, g, 3, 32 + 2 * 4, TT_Y + 2 * 2)) {
            DTB_CUDA(launch_jacobian_tma<T>(tm, g, nullptr, g.ys, g.zs, num_sms(), s, gJ, W, wn));
            w_done = true;
        }
    }
    CUtensorMap tw[3];
    if (w_done && reinterpret_cast<uintptr_t>(gout) % (2 * sizeof(T)) == 0 &&
        encode_weights_map(&tw[0], ft, sizeof(T), W, g, wn, 32 + 2 * 4, TT_Y) &&
        encode_weights_map(&tw[1], ft, sizeof(T), W, g, wn, 32, TT_Y + 2 * 2) &&
        encode_weights_map(&tw[2], ft, sizeof(T), W, g, wn, 32, TT_Y))
        DTB_CUDA(launch_gather_tma<T>(tw[0], tw[1], tw[2], g, gout, num_sms(), s));
    else
        DTB_CUDA(launch_adjoint<T>(g, field, gJ, W, wn, gout, w_done, s));
    DTB_CUDA(cudaEventRecord(g_adj_done[dev], s));
    return DTB_OK;
}

}  // namespace

extern "C" int dtb_jacobian_device(int precision, int order, size_t nx, size_t ny, size_t nz, double dx, double dy,
                                   double dz, const void *field, void *J, void *stream) {
    disptools_clear_error();
    if (!valid_dims(nx, ny, nz)) DTB_FAIL(DTB_ERR_ARGUMENT, "every axis needs at least 3 voxels");
    if (!field || !J) DTB_FAIL(DTB_ERR_ARGUMENT, "null array");
    if (order != 4 && order != 2) DTB_FAIL(DTB_ERR_ARGUMENT, "order must be 4 or 2");
    const Geom g = make_geom(nx, ny, nz, dx, dy, dz, order);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == DTB_PRECISION_FP64)
        return jacobian_device_impl<double>(g, static_cast<const double *>(field), static_cast<double *>(J), s);
    if (precision == DTB_PRECISION_MIXED)
        return jacobian_device_impl<float>(g, static_cast<const float *>(field), static_cast<float *>(J), s);
    DTB_FAIL(DTB_ERR_ARGUMENT, "invalid precision");
}

extern "C" int dtb_jacobian_adjoint_device(int precision, int order, size_t nx, size_t ny, size_t nz, double dx,
                                           double dy, double dz, const void *field, const void *grad_J,
                                           void *grad_field, void *stream) {
    disptools_clear_error();
    if (!valid_dims(nx, ny, nz)) DTB_FAIL(DTB_ERR_ARGUMENT, "every axis needs at least 3 voxels");
    if (!field || !grad_J || !grad_field) DTB_FAIL(DTB_ERR_ARGUMENT, "null array");
    if (order != 4 && order != 2) DTB_FAIL(DTB_ERR_ARGUMENT, "order must be 4 or 2");
    const Geom g = make_geom(nx, ny, nz, dx, dy, dz, order);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == DTB_PRECISION_FP64)
        return adjoint_device_impl<double>(g, static_cast<const double *>(field), static_cast<const double *>(grad_J),
                                           static_cast<double *>(grad_field), s);
    if (precision == DTB_PRECISION_MIXED)
        return adjoint_device_impl<float>(g, static_cast<const float *>(field), static_cast<const float *>(grad_J),
                                          static_cast<float *>(grad_field), s);
    DTB_FAIL(DTB_ERR_ARGUMENT, "invalid precision");
}

namespace {

// The cofactor path of the differentiable Jacobian: fourth order, rows a
// multiple of 16 bytes long, a 16-byte-aligned field, C and gJ, pair-aligned
// J and gradient.
template <typename T>
bool cof_layout_ok(const Geom &g, const void *a16_0, const void *a16_1, const void *pair) {
    return g.order == 4 && (g.ys * (long long) sizeof(T)) % 16 == 0 && reinterpret_cast<uintptr_t>(a16_0) % 16 == 0 &&
           reinterpret_cast<uintptr_t>(a16_1) % 16 == 0 && reinterpret_cast<uintptr_t>(pair) % (2 * sizeof(T)) == 0;
}

template <typename T>
int jacobian_cof_impl(const Geom &g, const T *field, T *J, T *C, cudaStream_t s) {
    if (!cof_layout_ok<T>(g, field, C, J)) DTB_FAIL(DTB_ERR_ARGUMENT, "layout not supported by the cofactor path");
    const CUtensorMapDataType ft = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUtensorMap tm;
    if (!encode_map(&tm, ft, sizeof(T), field, g, 3, 32 + 2 * 4, TT_Y + 2 * 2))
        DTB_FAIL(DTB_ERR_CUDA, "cannot encode the TMA descriptor (cuTensorMapEncodeTiled)");
    DTB_CUDA(launch_jacobian_tma<T>(tm, g, J, g.ys, g.zs, num_sms(), s, nullptr, C, g.cs));
    return DTB_OK;
}

template <typename T>
int adjoint_cof_impl(const Geom &g, const T *C, const T *gJ, T *gout, cudaStream_t s) {
    if (!cof_layout_ok<T>(g, C, gJ, gout)) DTB_FAIL(DTB_ERR_ARGUMENT, "layout not supported by the cofactor path");
    const CUtensorMapDataType ft = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUtensorMap tw[3], tg;
    if (!(encode_weights_map(&tw[0], ft, sizeof(T), C, g, g.cs, 32 + 2 * 4, TT_Y) &&
          encode_weights_map(&tw[1], ft, sizeof(T), C, g, g.cs, 32, TT_Y + 2 * 2) &&
          encode_weights_map(&tw[2], ft, sizeof(T), C, g, g.cs, 32, TT_Y) &&
          encode_map(&tg, ft, sizeof(T), gJ, g, 1, 32 + 2 * 4, TT_Y + 2 * 2)))
        DTB_FAIL(DTB_ERR_CUDA, "cannot encode the TMA descriptors (cuTensorMapEncodeTiled)");
    DTB_CUDA(launch_gather_tma<T>(tw[0], tw[1], tw[2], g, gout, num_sms(), s, &tg));
    return DTB_OK;
}

}  // namespace

extern "C" int dtb_jacobian_cof_device(int precision, size_t nx, size_t ny, size_t nz, double dx, double dy,
                                       double dz, const void *field, void *J, void *C, void *stream) {
    disptools_clear_error();
    if (!valid_dims(nx, ny, nz)) DTB_FAIL(DTB_ERR_ARGUMENT, "every axis needs at least 3 voxels");
    if (!field || !J || !C) DTB_FAIL(DTB_ERR_ARGUMENT, "null array");
    const Geom g = make_geom(nx, ny, nz, dx, dy, dz, 4);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == DTB_PRECISION_FP64)
        return jacobian_cof_impl<double>(g, static_cast<const double *>(field), static_cast<double *>(J),
                                         static_cast<double *>(C), s);
    if (precision == DTB_PRECISION_MIXED)
        return jacobian_cof_impl<float>(g, static_cast<const float *>(field), static_cast<float *>(J),
                                        static_cast<float *>(C), s);
    DTB_FAIL(DTB_ERR_ARGUMENT, "invalid precision");
}

extern "C" int dtb_jacobian_adjoint_cof_device(int precision, size_t nx, size_t ny, size_t nz, double dx, double dy,
                                               double dz, const void *C, const void *grad_J, void *grad_field,
                                               void *stream) {
    disptools_clear_error();
    if (!valid_dims(nx, ny, nz)) DTB_FAIL(DTB_ERR_ARGUMENT, "every axis needs at least 3 voxels");
    if (!C || !grad_J || !grad_field) DTB_FAIL(DTB_ERR_ARGUMENT, "null array");
    const Geom g = make_geom(nx, ny, nz, dx, dy, dz, 4);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == DTB_PRECISION_FP64)
        return adjoint_cof_impl<double>(g, static_cast<const double *>(C), static_cast<const double *>(grad_J),
                                        static_cast<double *>(grad_field), s);
    if (precision == DTB_PRECISION_MIXED)
        return adjoint_cof_impl<float>(g, static_cast<const float *>(C), static_cast<const float *>(grad_J),
                                       static_cast<float *>(grad_field), s);
    DTB_FAIL(DTB_ERR_ARGUMENT, "invalid precision");
}

extern "C" int dtb_set_device_memory_limit(size_t bytes) {
    disptools_clear_error();
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    g_mem_limit = bytes;
    return DTB_OK;
}

extern "C" int dtb_test_drop_tma_load(long long tile, int iteration, unsigned wait_limit) {
    disptools_clear_error();
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    g_drop.tile = tile;
    g_drop.iteration = iteration;
    g_drop.wait_limit = tile >= 0 ? wait_limit : 0;
    return DTB_OK;
}

extern "C" int dtb_set_verbose(int on) {
    disptools_clear_error();
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    const int prev = verbose_enabled() ? 1 : 0;
    g_verbose = on ? 1 : 0;
    return prev;
}

extern "C" int dtb_set_autotune(int on) {
    disptools_clear_error();
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    const int prev = autotune_enabled() ? 1 : 0;
    g_autotune = on ? 1 : 0;
    return prev;
}

extern "C" int dtb_get_tile_config(int *shape) {
    disptools_clear_error();
    if (!shape) DTB_FAIL(DTB_ERR_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    int dev = 0;
    DTB_CUDA(cudaGetDevice(&dev));
    if ((int) g_engines.size() <= dev || !g_engines[dev] || g_engines[dev]->last_cfg[0] == 0)
        DTB_FAIL(DTB_ERR_ARGUMENT, "no solve has run on this device");
    for (int k = 0; k < 4; ++k) shape[k] = g_engines[dev]->last_cfg[k];
    return DTB_OK;
}

extern "C" int dtb_get_trial_kernel(void) {
    disptools_clear_error();
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    int dev = 0;
    DTB_CUDA(cudaGetDevice(&dev));
    if ((int) g_engines.size() <= dev || !g_engines[dev] || g_engines[dev]->last_trial_kind < 0)
        DTB_FAIL(DTB_ERR_ARGUMENT, "no solve has run on this device");
    return g_engines[dev]->last_trial_kind;
}

extern "C" int dtb_release_device_memory(void) {
    disptools_clear_error();
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    int dev = 0;
    DTB_CUDA(cudaGetDevice(&dev));
    for (std::vector<Workspace> *pool : {&g_ws, &g_io, &g_adj}) {
        if ((int) pool->size() > dev && (*pool)[dev].ptr) {
            cudaFree((*pool)[dev].ptr);
            (*pool)[dev] = Workspace{};
        }
    }
    // The cached step graph points into the freed workspace.
    if ((int) g_engines.size() > dev && g_engines[dev]) {
        for (cudaGraphExec_t &x : g_engines[dev]->exec) {
            if (x) cudaGraphExecDestroy(x);
            x = nullptr;
        }
        g_engines[dev]->key = GraphKey{};
    }
    cudaGetLastError();
    return DTB_OK;
}

// src/jacobian.c:7-21, on the device in FP64.
extern "C" void jacobian_dynamic(const size_t nx, const size_t ny, const size_t nz, const double dx, const double dy,
                                 const double dz, const double *f, double *J) {
    disptools_clear_error();
    if (!valid_dims(nx, ny, nz)) {
        set_error(__LINE__, __func__, "every axis needs at least 3 voxels");
        return;
    }
    const size_t N = nx * ny * nz;
    double *df = nullptr, *dJ = nullptr;
    if (cudaMalloc(&df, 3 * N * sizeof(double)) != cudaSuccess || cudaMalloc(&dJ, N * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(df);
        set_error(__LINE__, __func__, "cannot allocate device buffers");
        return;
    }
    cudaError_t e = cudaMemcpy(df, f, 3 * N * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && dtb_jacobian_device(DTB_PRECISION_FP64, 4, nx, ny, nz, dx, dy, dz, df, dJ, nullptr) == DTB_OK)
        e = cudaMemcpy(J, dJ, N * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(__LINE__, __func__, cudaGetErrorString(e));
    }
    cudaFree(df);
    cudaFree(dJ);
}

// src/jacobian.c:29-55, on the device.
extern "C" void regularise(const size_t nx, const size_t ny, const size_t nz, double *J, double epsilon) {
    disptools_clear_error();
    const size_t N = nx * ny * nz;
    if (N == 0) return;
    double *dJ = nullptr;
    if (cudaMalloc(&dJ, N * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        set_error(__LINE__, __func__, "cannot allocate device buffers");
        return;
    }
    cudaError_t e = cudaMemcpy(dJ, J, N * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_regularise<double>(dJ, (long long) N, epsilon, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(J, dJ, N * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(__LINE__, __func__, cudaGetErrorString(e));
    }
    cudaFree(dJ);
}
