// snow_b200.cu -- host orchestration and C ABI of libsnowb200.so (see include/snow_b200.h).
//
// snow_simulation (cuda_simulation.cu:4861-5157) is restated as a sequence of fused
// kernels on one stream.  Set sizes live on the device (DevState), so a substep needs no
// host round trip; the host reads them back once per call to honour the reference's
// contract (ParticleSet::setSize).  Sorting follows the reference's sort points exactly,
// but a set whose predicted positions have not changed since its last sort is not
// sorted again (the result would be identical).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "sort.cuh"
#include "solver.cuh"
#include "phase.cuh"
#include "adjoint.cuh"
#include "export.cuh"
#include "render.cuh"
#include "ssfr.cuh"

namespace snowb {

// ------------------------------------------------------------------ error state
static thread_local int g_err = SNOWB_OK;
static thread_local std::string g_msg;

static int fail(int code, const std::string& msg)
{
    g_err = code;
    g_msg = msg;
    return code;
}
#define CUDA_TRY(x)                                                                          \
    do {                                                                                     \
        cudaError_t _e = (x);                                                                \
        if (_e != cudaSuccess)                                                               \
            return fail(SNOWB_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e));    \
    } while (0)
#define TRY(x)                      \
    do {                            \
        int _r = (x);               \
        if (_r != SNOWB_OK) return _r; \
    } while (0)

// ------------------------------------------------------------------ global state
static std::mutex g_mu;
static bool g_have_params = false;
static snowb_sim_params g_sim;
static DevParams g_P;
static float g_domain[5] = {-1.f, 1.f, -1.f, 1.f, 0.f};   // x_min, x_max, z_min, z_max, floor_y
static int g_quirks = SNOWB_QUIRKS_REFERENCE;
static cudaStream_t g_stream = 0;
static int g_max_blocks = 148 * 16;
static int g_sms = 148;

static float smallest_with_sqrt_ge(float t)   // min x: sqrtf(x) >= t
{
    float x = t * t;
    while (x > 0.f && std::sqrt(x) >= t) x = std::nextafter(x, 0.f);
    while (std::sqrt(x) < t) x = std::nextafter(x, INFINITY);
    return x;
}
static float smallest_with_sqrt_gt(float t)   // min x: sqrtf(x) > t
{
    float x = t * t;
    while (x > 0.f && std::sqrt(x) > t) x = std::nextafter(x, 0.f);
    while (!(std::sqrt(x) > t)) x = std::nextafter(x, INFINITY);
    return x;
}

static DevParams derive(const snowb_sim_params& s)
{
    DevParams P;
    std::memset(&P, 0, sizeof(P));
    P.h = s.effective_radius; P.r = s.particle_radius; P.two_r = 2.f * s.particle_radius;
    P.poly6 = s.poly6; P.poly6_G = s.poly6_G; P.spiky_G = s.spiky_G; P.visc_lap = s.viscosity_laplacian;
    P.keps = s.kernel_epsilon; P.pbd_eps = s.pbd_epsilon; P.rho0 = s.rest_density;
    P.inv_rho0 = 1.f / s.rest_density; P.eps = s.epsilon; P.scorr_coeff = s.scorr_coeff;
    P.scorr_div = s.scorr_divisor;
    {   // W_poly6(0) evaluated as the kernel does
        float h2 = P.h * P.h, d2 = 0.f * 0.f, q = h2 - d2;
        float q3 = q * q;
        q3 = q3 * q;
        P.W0 = P.poly6 * q3;
    }
    P.gx = s.gravity[0]; P.gy = s.gravity[1]; P.gz = s.gravity[2];
    P.damping = s.global_damping; P.max_speed = s.maximum_speed; P.min_speed = s.minimum_speed;
    P.b_damping = s.boundary_damping; P.mu_s = s.static_friction; P.mu_k = s.kinematic_friction;
    P.k_stretch = s.k_stretch; P.k_water = s.k_water; P.k_snow = s.k_snow; P.C_water = s.C_water;
    P.C_snow = s.C_snow; P.Tf = s.freezing_point; P.blending = s.blending_speed; P.sor = s.sor_coeff;
    P.sph_visc = s.sph_viscosity; P.dem_visc = s.dem_viscosity; P.Th = s.T_homogeneous;
    P.k_ref = s.k_refreezing; P.brk = s.break_threshold;
    P.ox = s.world_origin[0]; P.oy = s.world_origin[1]; P.oz = s.world_origin[2];
    P.csx = s.cell_size[0]; P.csy = s.cell_size[1]; P.csz = s.cell_size[2];
    P.gsx = s.grid_size[0]; P.gsy = s.grid_size[1]; P.gsz = s.grid_size[2];
    P.ncells = s.num_cells; P.maxc = s.maximum_connection;
    P.sgx = P.gsx; P.sgz = P.gsz; P.batch_nx = 1; P.batch_shift = 0; P.scene_mask = 0;
    P.wx0 = g_domain[0]; P.wx1 = g_domain[1]; P.wz0 = g_domain[2]; P.wz1 = g_domain[3]; P.floor_y = g_domain[4];
    P.h2_lt = smallest_with_sqrt_ge(P.h);
    P.r2_lt = smallest_with_sqrt_ge(P.two_r);
    P.r2_le = smallest_with_sqrt_gt(P.two_r);
    P.h2_cull = P.h2_lt * (1.f + 1e-5f);
    P.r2_cull = P.r2_le * (1.f + 1e-5f);
    P.quirks = SNOWB_QUIRKS_REFERENCE;
    {   // the s_corr term is -0 inside the support when scorr_coeff is +0 and its quotient
        // W / scorr_divisor (at most W(0) / scorr_divisor) stays finite to the fourth power
        uint32_t bits;
        std::memcpy(&bits, &s.scorr_coeff, sizeof bits);
        const double xmax = (double)P.W0 / (double)s.scorr_divisor;
        const bool finite = std::isfinite(s.scorr_coeff) && std::isfinite(s.scorr_divisor) && s.scorr_divisor > 0.f &&
                            std::isfinite(xmax) && xmax * xmax * xmax * xmax < 1e30;
        P.scorr_off = bits == 0u && finite;
        P.scorr_cpl_off = (bits >> 31) == 0u && finite;
    }
    return P;
}

// ------------------------------------------------------------------ context
template <class T>
static int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T)));
    return SNOWB_OK;
}

struct SetBufs {
    uint32_t *key = nullptr, *slot = nullptr, *tmp = nullptr, *cnt = nullptr, *off = nullptr, *bsum = nullptr;
    uint32_t* val = nullptr;
    float4* p4 = nullptr;
    float *invm = nullptr, *contrib = nullptr, *lambda = nullptr, *mass = nullptr;
    uint32_t* sid = nullptr;   // scene id per sorted particle (batched runs)
};

struct Ctx {
    int device = -1;
    uint32_t cap = 0, bcap = 0, ncells = 0, maxc = 0;
    SetBufs s[2];          // 0 = water (SPH), 1 = snow (DEM)
    SetBufs b;             // boundary
    SetBufs gen;           // scratch for the standalone sort entry points
    uint32_t gen_cap = 0;
    uint32_t *fl_s = nullptr, *fl_d = nullptr, *rk_s = nullptr, *rk_d = nullptr, *sbsum = nullptr;
    uint8_t* active = nullptr;
    uint32_t *sc_flag = nullptr, *sc_list = nullptr;   // link super-cell lists (SCList)
    uint32_t *fs = nullptr, *fe = nullptr;
    snowb_float3* tmp_vel = nullptr;
    uint32_t *nl_e = nullptr, *nl_cnt = nullptr;
    uint32_t *nl2_e = nullptr, *nl2_cnt = nullptr;   // the first density pass's snow lists (link formation)
    // link formation's copy of the snow set's sorted view, taken after the sort point that
    // precedes it, so that the first iteration's sort may run beside it
    float4* lf_p4 = nullptr;
    snowb_float3* lf_sp = nullptr;
    uint32_t *lf_gi = nullptr, *lf_gh = nullptr, *lf_sid = nullptr, *lf_cs = nullptr, *lf_ce = nullptr,
             *lf_off = nullptr;
    float4* link_terms = nullptr;         // one interlink term per slot (k_link_terms)
    float4* contact = nullptr;            // two snow contact sums per particle (k_dem_corr<true>)
    // the snow set's phase-change buffer (the caller's serves the water set), so that the two
    // sets' compactions run side by side
    snowb_particle_data pbuf{};
    uint32_t* psid = nullptr;
    double* epart = nullptr;
    double* eout = nullptr;
    DevState* S = nullptr;
    DevState* S_host = nullptr;
    uint32_t* err_dev = nullptr;
    cudaStream_t side = nullptr;          // second stream for the water sort (see sort_pair)
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaStream_t side2 = nullptr;         // third stream (the water PBF pass beside the snow passes)
    cudaEvent_t fork2 = nullptr, join2 = nullptr;
    cudaStream_t side3 = nullptr;         // fourth stream (the snow contact sums beside the snow PBF pass)
    cudaEvent_t fork3 = nullptr, join3 = nullptr;
    cudaStream_t side4 = nullptr;         // fifth stream (link formation beside the integration and iteration 1)
    cudaEvent_t fork4 = nullptr, ev_view = nullptr, ev_links = nullptr;
};
static Ctx g_ctx;
static uint64_t g_ctx_gen = 0;   // bumped whenever the scratch buffers are (re)allocated

static void free_set(SetBufs& s)
{
    void* ptrs[] = {s.key, s.slot, s.tmp, s.cnt, s.off, s.bsum, s.val, s.p4, s.invm, s.contrib, s.lambda, s.mass,
                    s.sid};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    s = SetBufs();
}
static void free_ctx(Ctx& c)
{
    for (auto& s : c.s) free_set(s);
    free_set(c.b);
    free_set(c.gen);
    void* ptrs[] = {c.fl_s, c.fl_d, c.rk_s, c.rk_d, c.sbsum, c.active, c.sc_flag, c.sc_list, c.fs, c.fe, c.tmp_vel,
                    c.epart, c.eout, c.link_terms, c.contact, c.psid,
                    c.pbuf.positions, c.pbuf.predict_positions, c.pbuf.new_positions, c.pbuf.velocity, c.pbuf.force,
                    c.pbuf.correction, c.pbuf.mass, c.pbuf.massInv, c.pbuf.contrib, c.pbuf.density, c.pbuf.C,
                    c.pbuf.lambda, c.pbuf.T, c.pbuf.new_T, c.pbuf.trackId, c.pbuf.iter_end, c.pbuf.connect_record,
                    c.pbuf.connect_length,
                    c.S, c.err_dev, c.nl_e, c.nl_cnt, c.nl2_e, c.nl2_cnt, c.lf_p4, c.lf_sp, c.lf_gi, c.lf_gh,
                    c.lf_sid, c.lf_cs, c.lf_ce, c.lf_off};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c.S_host) cudaFreeHost(c.S_host);
    if (c.side) cudaStreamDestroy(c.side);
    if (c.fork) cudaEventDestroy(c.fork);
    if (c.join) cudaEventDestroy(c.join);
    if (c.side2) cudaStreamDestroy(c.side2);
    if (c.fork2) cudaEventDestroy(c.fork2);
    if (c.join2) cudaEventDestroy(c.join2);
    if (c.side3) cudaStreamDestroy(c.side3);
    if (c.fork3) cudaEventDestroy(c.fork3);
    if (c.join3) cudaEventDestroy(c.join3);
    if (c.side4) cudaStreamDestroy(c.side4);
    if (c.fork4) cudaEventDestroy(c.fork4);
    if (c.ev_view) cudaEventDestroy(c.ev_view);
    if (c.ev_links) cudaEventDestroy(c.ev_links);
    c = Ctx();
}
static int alloc_sort(SetBufs& s, uint32_t cap, uint32_t ncells, bool attrs)
{
    TRY(dalloc(&s.key, cap)); TRY(dalloc(&s.slot, cap)); TRY(dalloc(&s.tmp, cap)); TRY(dalloc(&s.val, cap));
    TRY(dalloc(&s.cnt, ncells)); TRY(dalloc(&s.off, ncells + 1));
    TRY(dalloc(&s.bsum, ncells / SCAN_CHUNK + 2));
    CUDA_TRY(cudaMemset(s.cnt, 0, sizeof(uint32_t) * ncells));
    CUDA_TRY(cudaMemset(s.bsum, 0, sizeof(uint32_t) * (ncells / SCAN_CHUNK + 2)));
    if (attrs) {
        TRY(dalloc(&s.p4, cap)); TRY(dalloc(&s.invm, cap)); TRY(dalloc(&s.contrib, cap)); TRY(dalloc(&s.lambda, cap));
        TRY(dalloc(&s.sid, cap));
    }
    return SNOWB_OK;
}
// (Re)create the context for the current device with room for `full` particles per set,
// `nb` boundary particles and `ncells` cells.
static int ensure_ctx(uint32_t full, uint32_t nb, uint32_t ncells)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    Ctx& c = g_ctx;
    const uint32_t maxc = g_sim.maximum_connection > 0 ? g_sim.maximum_connection : 1;
    if (c.device == dev && c.cap >= full && c.bcap >= nb && c.ncells == ncells && c.maxc >= maxc) return SNOWB_OK;
    free_ctx(c);
    ++g_ctx_gen;
    c.device = dev;
    c.cap = full > 0 ? full : 1;
    c.bcap = nb > 0 ? nb : 1;
    c.ncells = ncells;
    for (auto& s : c.s) TRY(alloc_sort(s, c.cap, ncells, true));
    TRY(dalloc(&c.b.p4, c.bcap)); TRY(dalloc(&c.b.invm, c.bcap)); TRY(dalloc(&c.b.mass, c.bcap));
    TRY(dalloc(&c.b.lambda, c.bcap)); TRY(dalloc(&c.b.sid, c.bcap));
    TRY(dalloc(&c.fl_s, c.cap)); TRY(dalloc(&c.fl_d, c.cap)); TRY(dalloc(&c.rk_s, c.cap)); TRY(dalloc(&c.rk_d, c.cap));
    TRY(dalloc(&c.sbsum, 4 * (c.cap / SCAN_CHUNK + 2)));
    TRY(dalloc(&c.active, c.cap));
    TRY(dalloc(&c.sc_flag, ncells / 8 + 1)); TRY(dalloc(&c.sc_list, ncells / 8 + 1));
    CUDA_TRY(cudaMemset(c.sc_flag, 0, sizeof(uint32_t) * (ncells / 8 + 1)));
    TRY(dalloc(&c.fs, ncells)); TRY(dalloc(&c.fe, ncells));
    TRY(dalloc(&c.tmp_vel, c.cap));
    TRY(dalloc(&c.nl_e, (size_t)NLIST_K * 2 * c.cap));
    TRY(dalloc(&c.nl_cnt, 2 * (size_t)c.cap));
    TRY(dalloc(&c.nl2_e, (size_t)NLIST_K * 2 * c.cap));
    TRY(dalloc(&c.nl2_cnt, 2 * (size_t)c.cap));
    TRY(dalloc(&c.lf_p4, c.cap)); TRY(dalloc(&c.lf_sp, c.cap)); TRY(dalloc(&c.lf_gi, c.cap));
    TRY(dalloc(&c.lf_gh, c.cap)); TRY(dalloc(&c.lf_sid, c.cap)); TRY(dalloc(&c.lf_cs, (size_t)c.ncells));
    TRY(dalloc(&c.lf_ce, (size_t)c.ncells)); TRY(dalloc(&c.lf_off, (size_t)c.ncells + 1));
    c.maxc = maxc;
    TRY(dalloc(&c.link_terms, (size_t)c.cap * maxc));
    TRY(dalloc(&c.contact, (size_t)c.cap * 2));
    {
        snowb_particle_data& b = c.pbuf;
        snowb_float3** v3[] = {&b.positions, &b.predict_positions, &b.new_positions, &b.velocity, &b.force,
                               &b.correction};
        for (auto p : v3) TRY(dalloc(p, c.cap));
        float** f1[] = {&b.mass, &b.massInv, &b.contrib, &b.density, &b.C, &b.lambda, &b.T, &b.new_T};
        for (auto p : f1) TRY(dalloc(p, c.cap));
        TRY(dalloc(&b.trackId, c.cap)); TRY(dalloc(&b.iter_end, c.cap));
        TRY(dalloc(&b.connect_record, (size_t)c.cap * maxc)); TRY(dalloc(&b.connect_length, (size_t)c.cap * maxc));
        TRY(dalloc(&c.psid, c.cap));
    }
    TRY(dalloc(&c.epart, 4 * 1024)); TRY(dalloc(&c.eout, 4));
    TRY(dalloc(&c.S, 1)); TRY(dalloc(&c.err_dev, 1));
    CUDA_TRY(cudaMemset(c.S, 0, sizeof(DevState)));
    CUDA_TRY(cudaMemset(c.err_dev, 0, sizeof(uint32_t)));
    CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&c.S_host), sizeof(DevState)));
    CUDA_TRY(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming));
    CUDA_TRY(cudaStreamCreateWithFlags(&c.side2, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&c.fork2, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&c.join2, cudaEventDisableTiming));
    {   // the snow contact sums are the longest of the passes after the density pass when the
        // neighbour lists grow long: their stream has the highest priority too
        int least = 0, greatest = 0;
        CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUDA_TRY(cudaStreamCreateWithPriority(&c.side3, cudaStreamNonBlocking, greatest));
    }
    CUDA_TRY(cudaEventCreateWithFlags(&c.fork3, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&c.join3, cudaEventDisableTiming));
    {   // link formation's serial chains run beside the density pass, which would otherwise
        // take the SMs first: its stream has the highest priority
        int least = 0, greatest = 0;
        CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUDA_TRY(cudaStreamCreateWithPriority(&c.side4, cudaStreamNonBlocking, greatest));
    }
    CUDA_TRY(cudaEventCreateWithFlags(&c.fork4, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&c.ev_view, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&c.ev_links, cudaEventDisableTiming));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g_max_blocks = sms * 16;
    g_sms = sms;
    return SNOWB_OK;
}
// the link passes' super-cell lists (warp form only: maximum_connection <= SNOWB_MAXC_FAST)
static SCList sc_lists(const DevParams& P)
{
    if (P.maxc > SNOWB_MAXC_FAST) return SCList{nullptr, nullptr, nullptr, 0u};
    return SCList{g_ctx.sc_flag, g_ctx.sc_list, g_ctx.S->sc_count, P.ncells / 64u};
}
static int ensure_gen(uint32_t n, uint32_t ncells)
{
    Ctx& c = g_ctx;
    if (c.gen.key && c.gen_cap >= n && c.ncells == ncells) return SNOWB_OK;
    free_set(c.gen);
    c.gen_cap = n > 0 ? n : 1;
    return alloc_sort(c.gen, c.gen_cap, ncells, false);
}

// ------------------------------------------------------------------ launch helpers
// Every kernel launch goes through KL: it counts launches and, while profiling is on,
// brackets the launch with CUDA events on the library's stream.
struct ProfRec {
    const char* name;
    cudaEvent_t a, b;
};
static bool g_prof = false;
static uint64_t g_launches = 0;
static std::vector<ProfRec> g_prof_pool;
static size_t g_prof_used = 0;
static size_t g_prof_last_substep = 0;   // pool index of the last substep run outside a graph
static bool g_capturing = false;

static void prof_begin(const char* name)
{
    ++g_launches;
    if (!g_prof) return;
    if (g_prof_used == g_prof_pool.size()) {
        ProfRec r{name, nullptr, nullptr};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        g_prof_pool.push_back(r);
    }
    g_prof_pool[g_prof_used].name = name;
    // inside a stream capture the record must become an event node of the graph
    cudaEventRecordWithFlags(g_prof_pool[g_prof_used].a, g_stream, g_capturing ? cudaEventRecordExternal : 0);
}
static void prof_end()
{
    if (!g_prof) return;
    cudaEventRecordWithFlags(g_prof_pool[g_prof_used].b, g_stream, g_capturing ? cudaEventRecordExternal : 0);
    ++g_prof_used;
}
// accumulated per-kernel times (name, launches, ms) of the current profiling window
static std::vector<std::string> g_acc_name;
static std::vector<uint64_t> g_acc_count;
static std::vector<double> g_acc_ms;
static int prof_accumulate(size_t first, size_t last)
{
    for (size_t k = first; k < last; ++k) {
        float ms = 0.f;
        cudaError_t e = cudaEventElapsedTime(&ms, g_prof_pool[k].a, g_prof_pool[k].b);
        if (e != cudaSuccess) return -1;
        const std::string nm = g_prof_pool[k].name;
        size_t idx = 0;
        while (idx < g_acc_name.size() && g_acc_name[idx] != nm) ++idx;
        if (idx == g_acc_name.size()) { g_acc_name.push_back(nm); g_acc_count.push_back(0); g_acc_ms.push_back(0.0); }
        g_acc_count[idx] += 1;
        g_acc_ms[idx] += ms;
    }
    return 0;
}

static inline unsigned blocks_for(uint64_t work, int tpb)
{
    uint64_t b = (work + tpb - 1) / tpb;
    if (b < 1) b = 1;
    if (b > (uint64_t)g_max_blocks) b = g_max_blocks;
    return (unsigned)b;
}
#define KL(kernel, grid, tpb, ...)                                                         \
    do {                                                                                   \
        prof_begin(#kernel);                                                               \
        kernel<<<(grid), (tpb), 0, g_stream>>>(__VA_ARGS__);                               \
        prof_end();                                                                        \
        cudaError_t _e = cudaGetLastError();                                               \
        if (_e != cudaSuccess)                                                             \
            return fail(SNOWB_ERR_CUDA, std::string(#kernel) + ": " + cudaGetErrorString(_e)); \
    } while (0)
#define LAUNCH(kernel, work, tpb, ...) KL(kernel, blocks_for((work), (tpb)), (tpb), __VA_ARGS__)

// ------------------------------------------------------------------ autotuner
// Launch shapes of the tunable kernels (threads per block, grid cap in blocks per SM),
// chosen per kernel and work-size bucket (floor(log2(threads of work))) by
// snowb_autotune, which times every candidate shape from CUDA-event nodes inside the
// substep's graph.  Launch shapes never change results: every thread's work and every
// reduction order are independent of the block and grid shape.
struct TuneEntry {
    std::string name;
    int bucket, tpb, capm;
};
static std::vector<TuneEntry> g_tune;
static uint64_t g_tune_gen = 0;        // bumped when the table or the forced shape changes (graph key)
static int g_tune_force_tpb = 0, g_tune_force_capm = 0;
static std::vector<std::pair<std::string, int>> g_tune_seen;   // (kernel, bucket) launched while forcing
static inline int ilog2_u64(uint64_t x)
{
    int b = 0;
    while (x > 1) { x >>= 1; ++b; }
    return b;
}
static void tune_pick(const char* name, uint64_t work, int tpb0, int max_tpb, int& tpb, unsigned& grid)
{
    const int bucket = ilog2_u64(work ? work : 1);
    tpb = tpb0;
    int capm = 0;
    if (g_tune_force_tpb) {
        tpb = g_tune_force_tpb < max_tpb ? g_tune_force_tpb : max_tpb;
        capm = g_tune_force_capm;
        bool seen = false;
        for (auto& e : g_tune_seen) seen |= e.first == name && e.second == bucket;
        if (!seen) g_tune_seen.emplace_back(name, bucket);
    } else {
        for (const auto& e : g_tune)
            if (e.bucket == bucket && e.name == name) { tpb = e.tpb; capm = e.capm; break; }
        if (tpb > max_tpb) tpb = max_tpb;
    }
    uint64_t b = (work + tpb - 1) / tpb;
    if (b < 1) b = 1;
    const uint64_t cap = capm ? (uint64_t)capm * g_sms : (uint64_t)g_max_blocks;
    if (b > cap) b = cap;
    grid = (unsigned)b;
}
#define TLAUNCH(kernel, max_tpb, work, tpb0, ...)                                            \
    do {                                                                                     \
        int _tpb;                                                                            \
        unsigned _grid;                                                                      \
        tune_pick(#kernel, (work), (tpb0), (max_tpb), _tpb, _grid);                          \
        KL(kernel, _grid, _tpb, __VA_ARGS__);                                                \
    } while (0)
// tunable only when `tunable` holds (else the built-in shape)
#define TLAUNCH_IF(tunable, kernel, max_tpb, work, tpb0, ...)                                \
    do {                                                                                     \
        if (tunable) TLAUNCH(kernel, max_tpb, work, tpb0, __VA_ARGS__);                       \
        else LAUNCH(kernel, work, tpb0, __VA_ARGS__);                                        \
    } while (0)
#define LAUNCH1(kernel, ...) KL(kernel, 1, 32, __VA_ARGS__)

static inline unsigned scan_blocks(uint32_t n) { return (n + SCAN_CHUNK - 1) / SCAN_CHUNK + (n == 0); }

// exclusive scan of in[0, n) (n from the device when n_ptr is set; `cap` bounds it)
static int scan(const uint32_t* in, const uint32_t* n_ptr, uint32_t n_fixed, uint32_t cap, uint32_t* bsum,
                uint32_t* out, uint32_t* total, const uint32_t* cond)
{
    const uint32_t nb = scan_blocks(n_ptr ? cap : n_fixed);
    KL(k_scan_sums, nb, SCAN_TPB, in, n_ptr, n_fixed, bsum, cond);
    KL(k_scan_apply, nb, SCAN_TPB, in, n_ptr, n_fixed, bsum, out, total, cond);
    return SNOWB_OK;
}

// hash + stable sort + reorder of one set (sort_and_reorder :398-420), writing the
// caller's cell data and the compact sorted copies.  cond: skip unless *cond != 0.
// gate.S set: a sort point of the substep, which decides for itself whether the set keeps
// its last sort (cond then points at that decision, DevState::resort)
static int sort_set(const DevParams& P, SetBufs& B, const snowb_particle_data& D, const snowb_cell_data& cd,
                    const uint32_t* n_ptr, uint32_t cap, const uint32_t* cond, bool clear_all,
                    const uint32_t* sid_o = nullptr, SortGate gate = SortGate{nullptr, 0, 0})
{
    const uint32_t nc = P.ncells;
    const unsigned nb = (nc + SCAN_CHUNK - 1) / SCAN_CHUNK;
    // chunk counts come from the hash pass (bsum is all zero between sorts)
    LAUNCH(k_hash_count, cap, 256, P, D.predict_positions, n_ptr, 0u, B.key, B.slot, B.cnt, cond, sid_o, B.bsum,
           gate);
    KL(k_cell_scan, nb, SCAN_TPB, B.cnt, B.bsum, nc, B.off, cd.cell_start, n_ptr, 0u, clear_all ? 1 : 0, cond,
       gate.S ? &gate.S->moved[gate.set] : nullptr);
    LAUNCH(k_scatter, cap, 256, B.key, B.slot, B.off, B.tmp, n_ptr, 0u, cond, B.bsum, nb);
    LAUNCH(k_rank_reorder, cap, 256, B.key, B.off, B.tmp, D.predict_positions, D.mass, D.massInv, D.contrib, cd, B.p4,
           B.invm, B.contrib, n_ptr, 0u, cond, sid_o, sid_o ? B.sid : nullptr);
    return SNOWB_OK;
}

static SetView make_view(const snowb_cell_data& cd, const float4* p4, const float* wsrc,
                         const uint32_t* sid_sorted = nullptr)
{
    SetView v;
    v.sid = sid_sorted;
    v.cs = cd.cell_start; v.ce = cd.cell_end; v.gi = cd.grid_index; v.gh = cd.grid_hash; v.p4 = p4;
    v.sp = cd.sorted_pos;
    v.wsrc = wsrc; v.n = 0;
    return v;
}

struct StepArgs {
    snowb_particle_data *sph, *dem, *bnd, *buf;
    uint32_t nb, full;
    snowb_cell_data scd, dcd, bcd;
    float dt;
    int iterations;
    int correct_dem, sph_sph, friction, temperature, change_phase, freezing, melting, dem_visc, interlink,
        dynamic, cd_on;
    float dTe;
    int stop_after;
    const uint32_t *sid_sph, *sid_dem, *sid_bnd;   // batched runs: scene id per slot (else null)
    uint32_t* sid_buf;
    int xsph_thread[2];   // XSPH of the water / snow set in the one-thread form (sizes at the call)
};


// ------------------------------------------------------------------ adjoint tape
// While recording (snowb_adjoint_begin .. snowb_adjoint_end) every substep saves what its
// reverse needs: the state at its start, the positions after integration, the input
// and corrected positions of every solver iteration with the interlink records seen by
// that iteration, and the velocities after finalize and after the water XSPH.  Sizes
// are those of the recorded substeps (no phase change may happen while recording).
struct TapeStep {
    std::vector<void*> bufs;
    float *x0[2], *v0[2], *T0[2], *x0p[2], *vf[2], *vw1;
    std::vector<float*> xit[2], xmid[2];
    std::vector<uint32_t*> rec;
    std::vector<float*> len;
    uint32_t* rec_pre;   // records at the substep's start (before link formation)
};
struct Tape {
    bool recording = false;
    std::vector<TapeStep> steps;   // allocated entries, reused across recordings
    size_t used = 0;
    uint32_t full = 0, n[2] = {0, 0}, nb = 0, maxc = 0;
    int iterations = 0;
    int device = -1;
    // forward context of the recorded substeps
    snowb_particle_data sph{}, dem{}, bnd{};
    snowb_cell_data bcd{};
    DevParams P{};
    float dt = 0.f;
    int friction = 0, temperature = 0, correct_dem = 0, interlink = 0, dem_visc = 0, cd_on = 0;
    uint32_t* viol = nullptr;      // device flag: a phase change or contrib != 1 while recording
};
static Tape g_tape;

static void tape_free_steps()
{
    for (auto& st : g_tape.steps)
        for (void* p : st.bufs) cudaFree(p);
    g_tape.steps.clear();
    g_tape.used = 0;
}
static int tape_alloc_step(TapeStep& T)
{
    const size_t f3n = (size_t)g_tape.full * 3, f1n = g_tape.full;
    auto F = [&](float** p, size_t n) -> int { TRY(dalloc(p, n)); T.bufs.push_back(*p); return SNOWB_OK; };
    for (int s = 0; s < 2; ++s) {
        TRY(F(&T.x0[s], f3n)); TRY(F(&T.v0[s], f3n)); TRY(F(&T.T0[s], f1n)); TRY(F(&T.x0p[s], f3n));
        TRY(F(&T.vf[s], f3n));
        T.xit[s].assign(g_tape.iterations, nullptr);
        T.xmid[s].assign(g_tape.iterations, nullptr);
        for (int it = 0; it < g_tape.iterations; ++it) { TRY(F(&T.xit[s][it], f3n)); TRY(F(&T.xmid[s][it], f3n)); }
    }
    TRY(F(&T.vw1, f3n));
    TRY(dalloc(&T.rec_pre, (size_t)g_tape.full * g_tape.maxc)); T.bufs.push_back(T.rec_pre);
    T.rec.assign(g_tape.iterations, nullptr);
    T.len.assign(g_tape.iterations, nullptr);
    for (int it = 0; it < g_tape.iterations; ++it) {
        TRY(dalloc(&T.rec[it], (size_t)g_tape.full * g_tape.maxc)); T.bufs.push_back(T.rec[it]);
        TRY(F(&T.len[it], (size_t)g_tape.full * g_tape.maxc));
    }
    return SNOWB_OK;
}
static int tape_copy(void* dst, const void* src, size_t bytes)
{
    if (bytes) CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, g_stream));
    return SNOWB_OK;
}
// kind: 0 substep start, 1 after integration, 2 iteration start, 3 after the iteration's
// apply, 4 after finalize, 5 after the water XSPH, 6 substep end
static int tape_hook(const StepArgs& a, int kind, int it)
{
    Tape& tp = g_tape;
    if (kind == 0 && tp.used == tp.steps.size()) {
        tp.steps.emplace_back();
        TRY(tape_alloc_step(tp.steps.back()));
    }
    TapeStep& T = tp.steps[tp.used];
    const size_t b3[2] = {(size_t)tp.n[0] * 12, (size_t)tp.n[1] * 12};
    const snowb_particle_data* D[2] = {a.sph, a.dem};
    switch (kind) {
    case 0:
        for (int s = 0; s < 2; ++s) {
            TRY(tape_copy(T.x0[s], D[s]->positions, b3[s]));
            TRY(tape_copy(T.v0[s], D[s]->velocity, b3[s]));
            TRY(tape_copy(T.T0[s], D[s]->T, (size_t)tp.n[s] * 4));
        }
        TRY(tape_copy(T.rec_pre, a.dem->connect_record, (size_t)tp.n[1] * tp.maxc * 4));
        LAUNCH(ka_check_contrib, tp.n[0] + tp.n[1], 256, tp.n[0], tp.n[1], a.sph->contrib, a.dem->contrib, tp.viol);
        break;
    case 1:
        for (int s = 0; s < 2; ++s) TRY(tape_copy(T.x0p[s], D[s]->positions, b3[s]));
        break;
    case 2:
        for (int s = 0; s < 2; ++s) TRY(tape_copy(T.xit[s][it], D[s]->predict_positions, b3[s]));
        TRY(tape_copy(T.rec[it], a.dem->connect_record, (size_t)tp.n[1] * tp.maxc * 4));
        TRY(tape_copy(T.len[it], a.dem->connect_length, (size_t)tp.n[1] * tp.maxc * 4));
        break;
    case 3:
        for (int s = 0; s < 2; ++s) TRY(tape_copy(T.xmid[s][it], D[s]->predict_positions, b3[s]));
        break;
    case 4:
        for (int s = 0; s < 2; ++s) TRY(tape_copy(T.vf[s], D[s]->velocity, b3[s]));
        break;
    case 5:
        TRY(tape_copy(T.vw1, a.sph->velocity, b3[0]));
        break;
    case 6:
        LAUNCH1(ka_check_phase, g_ctx.S, tp.viol);
        ++tp.used;
        break;
    }
    return SNOWB_OK;
}
#define TAPE_HOOK(kind, it) do { if (g_tape.recording) TRY(tape_hook(a, (kind), (it))); } while (0)

// One substep (cuda_simulation.cu:4861-5157) given step flags derived from the scene time.
// Returns SNOWB_OK; stops early after stage `stop_after` (0 = complete).
static int substep(const DevParams& P, const StepArgs& a, bool step_sph, bool step_dem)
{
    if (g_prof && !g_capturing) g_prof_last_substep = g_prof_used;
    Ctx& c = g_ctx;
    DevState* S = c.S;
    const uint32_t full = a.full, cap = g_ctx.cap;
    const bool ref = P.quirks == SNOWB_QUIRKS_REFERENCE;
    Sets X{*a.sph, *a.dem, *a.bnd};
    const bool batched = a.sid_sph != nullptr;
    SetView vs = make_view(a.scd, c.s[0].p4, a.sph->mass, batched ? c.s[0].sid : nullptr);
    SetView vd = make_view(a.dcd, c.s[1].p4, a.dem->mass, batched ? c.s[1].sid : nullptr);
    SetView vb = make_view(a.bcd, c.b.p4, a.bnd->volume, batched ? c.b.sid : nullptr);
    SceneIds scn{const_cast<uint32_t*>(a.sid_sph), const_cast<uint32_t*>(a.sid_dem), a.sid_buf};
    Sorted ss{c.s[0].invm, c.s[0].contrib, c.s[0].lambda, nullptr};
    Sorted sd{c.s[1].invm, c.s[1].contrib, c.s[1].lambda, nullptr};
    Sorted sb{c.b.invm, nullptr, c.b.lambda, c.b.mass};
    StageFlags F{a.correct_dem, a.sph_sph, a.interlink, step_sph ? 1 : 0, step_dem ? 1 : 0};
    NList NL{c.nl_e, c.nl_cnt, 2 * cap, cap};
    // the substep's first density pass lists the snow-snow candidates for link formation in
    // a list of their own, which the iterations' density passes leave alone
    NList NL2{c.nl2_e, c.nl2_cnt, 2 * cap, cap};
    // the friction pass may replay the density+lambda lists when a contact (d <= 2r) after a
    // move of at most FR_LIST_MOVE per particle was within h before it
    const bool fr_lists = P.two_r + 2.f * FR_LIST_MOVE < 0.9f * P.h;
    const uint32_t* n_s = &S->n_sph;
    const uint32_t* n_d = &S->n_dem;
    const uint32_t work3 = 2 * full + a.nb;
    // dirty_*: the host knows the set may have moved since its last sort (no launch at all
    // otherwise).  On the device, each sort point's hash pass turns the writers' moved flag
    // into the decision: a set whose particles all kept their cells keeps its permutation and
    // cell table, its hash, scan and scatter launches return at once and the rank pass only
    // refreshes the gathered outputs.
    bool dirty_s = true, dirty_d = true;
    auto track = [&](int set) { return SortTrack{c.s[set].key, set ? a.sid_dem : a.sid_sph, &S->moved[set]}; };
    const SortTrack track_s = track(0), track_d = track(1);
    // a sort point of one set: the full sort when the set moved, else only the refresh of the
    // gathered outputs
    auto sort_if = [&](int set, bool begin) -> int {
        TRY(sort_set(P, c.s[set], set ? *a.dem : *a.sph, set ? a.dcd : a.scd, set ? n_d : n_s, cap, &S->resort[set],
                     !ref, set ? a.sid_dem : a.sid_sph, SortGate{S, set, begin ? 1 : 0}));
        return SNOWB_OK;
    };
    // launches on a side stream forked from the main one; join_side makes the main stream
    // wait for them
    auto on_side = [&](cudaStream_t st, cudaEvent_t ev, auto&& launch) -> int {
        const cudaStream_t main_stream = g_stream;
        CUDA_TRY(cudaEventRecord(ev, main_stream));
        CUDA_TRY(cudaStreamWaitEvent(st, ev, 0));
        g_stream = st;
        const int rc = launch();
        g_stream = main_stream;
        return rc;
    };
    auto join_side = [&](cudaStream_t st, cudaEvent_t ev) -> int {
        CUDA_TRY(cudaEventRecord(ev, st));
        CUDA_TRY(cudaStreamWaitEvent(g_stream, ev, 0));
        return SNOWB_OK;
    };
    // Inside an iteration the water PBF pass (water corrections) and the interlink terms (the
    // per-slot term buffer, link deletions) share no buffer with the density, snow PBF and
    // contact passes, so they run beside them on the side streams when the substep runs
    // whole (a stage stop keeps every launch on the main stream).
    const bool beside = a.stop_after == 0;
    // The two sets' sorts share no buffer: the water sort runs on a side stream beside the
    // snow sort (a fork and a join of the captured graph), so the small set's chain of
    // latency-bound launches overlaps the large one's.  after_phase: the sort point after
    // the phase change, where only a compaction (which marks both sets moved) alters the
    // result.
    // begin: the substep's first sort point, whose snow hash pass also opens the substep
    // (both sets are dirty there)
    // defer_water: the friction sort point, whose passes read no water data: its water sort
    // stays on the side stream beside the friction and apply passes, joined by the next
    // sort point or by join_water
    bool water_pending = false;
    auto join_water = [&]() -> int {
        if (water_pending) TRY(join_side(c.side, c.join));
        water_pending = false;
        return SNOWB_OK;
    };
    // link formation beside the integration and the first iteration (see below): the snow
    // sort waits for link formation's copy of the snow view, the first interlink terms for
    // the links
    bool view_pending = false, links_pending = false;
    auto sort_pair = [&](bool after_phase, bool begin = false, bool defer_water = false) -> int {
        TRY(join_water());
        const bool need_s = dirty_s || after_phase, need_d = dirty_d || after_phase;
        if (!need_s && !need_d) return SNOWB_OK;
        if (need_s) TRY(on_side(c.side, c.fork, [&]() { return sort_if(0, false); }));
        if (need_d && view_pending) {
            CUDA_TRY(cudaStreamWaitEvent(g_stream, c.ev_view, 0));
            view_pending = false;
        }
        if (need_d) TRY(sort_if(1, begin));
        if (need_s) {
            if (defer_water) water_pending = true;
            else TRY(join_side(c.side, c.join));
        }
        dirty_s = dirty_d = false;
        return SNOWB_OK;
    };
#define STOP(k) do { if (a.stop_after == (k)) return SNOWB_OK; } while (0)

    TAPE_HOOK(0, 0);
    TRY(sort_pair(false, true));
    STOP(1);
    // The substep's first density pass feeds the heat pass and the link formation, which
    // read the water and snow densities only; the boundary's values are rewritten by the
    // iterations' density+lambda passes before anything reads them, so a whole substep with
    // iterations leaves the boundary out here.
    const int bnd_first = !(beside && a.iterations > 0);
    TLAUNCH(k_density<false>, 256, bnd_first ? work3 : 2 * full, 128, P, S, vs, vd, vb, X, ss, sd, sb, NL2, bnd_first);
    STOP(2);
    // in a whole substep the phase flags pass commits the new temperatures itself
    const int commit_in_flags = beside && a.temperature && a.change_phase;
    if (a.temperature) {
        TLAUNCH(k_heat, 256, 2 * full, 128, P, S, vs, vd, X, a.dt);
        if (!commit_in_flags) LAUNCH(k_heat_commit, 2 * full, 256, S, X, a.dTe, step_sph ? 1 : 0, step_dem ? 1 : 0);
    }
    STOP(3);
    if (a.change_phase) {
        LAUNCH(k_phase_flags, 2 * full, 256, P, S, *a.sph, *a.dem, a.freezing, a.melting, c.fl_s, c.fl_d,
               commit_in_flags, a.dTe, step_sph ? 1 : 0, step_dem ? 1 : 0);
        const uint32_t sb_stride = cap / SCAN_CHUNK + 2;
        // the two sets' scans share nothing: in a whole substep the snow set's runs beside
        auto scan_pair = [&](auto&& scan_s, auto&& scan_d) -> int {
            if (beside) {
                TRY(on_side(c.side, c.fork, scan_d));
                TRY(scan_s());
                TRY(join_side(c.side, c.join));
            } else {
                TRY(scan_s());
                TRY(scan_d());
            }
            return SNOWB_OK;
        };
        TRY(scan_pair([&]() { return scan(c.fl_s, n_s, 0, cap, c.sbsum, c.rk_s, &S->n_freeze, nullptr); },
                      [&]() { return scan(c.fl_d, n_d, 0, cap, c.sbsum + sb_stride, c.rk_d, &S->n_melt, nullptr); }));
        LAUNCH(k_phase_move, 2 * full, 256, P, S, *a.sph, *a.dem, c.fl_s, c.rk_s, c.fl_d, c.rk_d, scn);
        // compact_and_clean (:4495-4589): predicate scans run every substep (they define
        // scan_index), the data movement only after a phase change.
        TRY(scan_pair(
            [&]() { return scan(a.sph->predicate, nullptr, full, full, c.sbsum, a.sph->scan_index, &S->new_sph, nullptr); },
            [&]() {
                return scan(a.dem->predicate, nullptr, full, full, c.sbsum + sb_stride, a.dem->scan_index, &S->new_dem,
                            nullptr);
            }));
        const uint64_t cw = (uint64_t)full * (P.maxc + 1);   // a thread per particle and per link slot
        // the water set loses the freezing particles, the snow set the melting ones; in a whole
        // substep the water set compacts through the caller's buffer beside the snow set
        // compacting through the library's
        auto compact_water = [&]() -> int {
            LAUNCH(k_copy_to_buffer, cw, 256, P, S, *a.sph, *a.buf, full, scn.sph, scn.buf, &S->n_freeze);
            LAUNCH(k_scatter_set, cw, 256, P, S, *a.sph, *a.buf, full, scn.sph, scn.buf, 0, &S->n_freeze);
            return SNOWB_OK;
        };
        const snowb_particle_data& dbuf = beside ? c.pbuf : *a.buf;
        uint32_t* dsid = beside ? c.psid : scn.buf;
        if (beside) TRY(on_side(c.side, c.fork, compact_water));
        else TRY(compact_water());
        LAUNCH(k_copy_to_buffer, cw, 256, P, S, *a.dem, dbuf, full, scn.dem, dsid, &S->n_melt);
        LAUNCH(k_scatter_set, cw, 256, P, S, *a.dem, dbuf, full, scn.dem, dsid, ref ? 0 : 1, &S->n_melt);
        if (beside) TRY(join_side(c.side, c.join));
        LAUNCH(k_compact_finish, 2 * full + (uint64_t)P.maxc * full, 256, P, S, *a.sph, *a.dem, full, 1);
        LAUNCH1(k_commit_sizes, S);
    }
    STOP(4);
    if (a.change_phase) {   // the reference sorts again; only a phase change alters the result
        TRY(sort_pair(true));
    }
    STOP(5);
    if (a.interlink) {
        // link formation over a view of the snow set: the set's own, or its copy
        auto form = [&](const SetView& v, const uint32_t* off) -> int {
            const SCList scl = sc_lists(P);
            TLAUNCH(k_link_filter, 256, full, 128, P, S, v, *a.dem, a.dynamic, c.active, NL2, scl);
            const uint32_t nsc = (P.gsx / 4) * (P.gsy / 4) * (P.gsz / 4);   // super-cells per colour
            for (uint32_t col = 0; col < 8; ++col) {
                if (P.maxc <= SNOWB_MAXC_FAST)
                    TLAUNCH(k_link_colour_warp, 256, (uint64_t)nsc * 32, 128, P, S, v, *a.dem, off, off + 1, c.active,
                            col, a.dynamic, NL2, scl);
                else
                    TLAUNCH(k_link_colour, 128, nsc, 64, P, S, v, *a.dem, off, off + 1, c.active, col, a.dynamic);
            }
            if (a.dynamic) LAUNCH1(k_adjust_links, P, S, *a.dem, full);
            return SNOWB_OK;
        };
        // Link formation reads the snow set's sorted view, its links and temperatures and
        // writes its links; the integration and the first iteration's sort points, density,
        // PBF and contact passes touch none of the links.  In a whole substep it therefore
        // runs beside them, over a copy of the view (the first snow sort rewrites the view),
        // and the first interlink terms wait for it.
        const bool links_early = beside && a.iterations > 0 && !g_tape.recording;
        if (links_early) {
            SetView vl = vd;
            vl.p4 = c.lf_p4; vl.sp = c.lf_sp; vl.gi = c.lf_gi; vl.gh = c.lf_gh; vl.cs = c.lf_cs; vl.ce = c.lf_ce;
            vl.sid = vd.sid ? c.lf_sid : nullptr;
            TRY(on_side(c.side4, c.fork4, [&]() -> int {
                LAUNCH(k_copy_link_view, (full > P.ncells + 1 ? full : P.ncells + 1), 256, vd, full, P.ncells,
                       c.s[1].off, c.lf_p4, c.lf_sp, c.lf_gi, c.lf_gh, c.lf_sid, c.lf_cs, c.lf_ce, c.lf_off);
                CUDA_TRY(cudaEventRecord(c.ev_view, g_stream));
                TRY(form(vl, c.lf_off));
                CUDA_TRY(cudaEventRecord(c.ev_links, g_stream));
                return SNOWB_OK;
            }));
            view_pending = links_pending = true;
        } else {
            TRY(form(vd, c.s[1].off));
        }
    }
    STOP(6);
    if (step_sph || step_dem) {
        LAUNCH(k_integrate, 2 * full, 256, P, S, X, full, a.dt, a.cd_on, step_sph ? 1 : 0, step_dem ? 1 : 0, track_s,
               track_d);
        if (step_sph) dirty_s = true;
        if (step_dem) dirty_d = true;
    }
    TAPE_HOOK(1, 0);
    STOP(7);
    for (int it = 0; it < a.iterations; ++it) {
        const int base = 10 + 10 * it;
        TRY(sort_pair(false));
        TAPE_HOOK(2, it);
        STOP(base + 0);
        // the interlink terms read the predicted positions and the link records only
        auto link_terms = [&]() -> int {
            if (links_pending) {
                CUDA_TRY(cudaStreamWaitEvent(g_stream, c.ev_links, 0));
                links_pending = false;
            }
            TLAUNCH(k_link_terms, 256, (uint64_t)P.maxc * full, 256, P, S, *a.dem, c.link_terms);
            return SNOWB_OK;
        };
        const bool links_beside = beside && a.interlink;
        if (links_beside) TRY(on_side(c.side, c.fork, link_terms));
        // density + lambda in one pass (stage boundaries base+1 and base+2 coincide)
        TLAUNCH(k_density<true>, 256, work3, 128, P, S, vs, vd, vb, X, ss, sd, sb, NL, 1);
        STOP(base + 2);
        // with the interlink pass beside, the passes that finish a correction apply it (no
        // k_apply launch): the water PBF passes for the water, k_link_apply for the snow
        const int apply_w = links_beside && step_sph ? 1 : 0;
        auto pbf_water = [&]() -> int {
            TLAUNCH(k_pbf_water_warp, 256, (uint64_t)full * 32, 128, P, S, vs, vd, vb, X, ss, sd, sb, a.dt, F, apply_w,
                    track_s);
            return SNOWB_OK;
        };
        if (beside) TRY(on_side(c.side2, c.fork2, pbf_water));
        else TRY(pbf_water());
        // the snow contact sums, kept apart for k_link_apply, beside the snow PBF pass
        if (links_beside)
            TRY(on_side(c.side3, c.fork3, [&]() -> int {
                TLAUNCH(k_dem_corr<true>, 256, full, 128, P, S, vs, vd, vb, X, ss, sd, sb, F, NL, c.contact);
                return SNOWB_OK;
            }));
        // the reference's snow PBF pass adds into repeated targets with float atomics (Q3):
        // its order follows the launch shape, so that pass keeps the built-in shape
        TLAUNCH_IF(!ref, k_pbf, 256, 2 * full, 128, P, S, vs, vd, vb, X, ss, sd, sb, a.dt, F, NL, apply_w, track_s);
        STOP(base + 3);
        if (!links_beside) TLAUNCH(k_dem_corr<false>, 256, full, 128, P, S, vs, vd, vb, X, ss, sd, sb, F, NL, nullptr);
        if (a.interlink) {
            if (links_beside) {
                TRY(join_side(c.side3, c.join3));
                TRY(join_side(c.side, c.join));
            } else {
                TRY(link_terms());
            }
            if (links_beside)
                TLAUNCH(k_link_apply, 256, full, 128, P, S, vd, *a.dem, c.link_terms, c.contact, F.correct_dem,
                        step_dem ? 1 : 0, track_d);
            else
                TLAUNCH(k_link_sum, 256, full, 128, P, S, *a.dem, c.link_terms);
        }
        if (beside) TRY(join_side(c.side2, c.join2));
        STOP(base + 5);
        if (links_beside) {
            if (step_sph) dirty_s = true;
            if (step_dem) dirty_d = true;
        } else if (step_sph || step_dem) {
            TLAUNCH(k_apply, 1024, 2 * full, 256, P, S, vs, vd, X, step_sph ? 1 : 0, step_dem ? 1 : 0, track_s,
                    track_d);
            if (step_sph) dirty_s = true;
            if (step_dem) dirty_d = true;
        }
        TAPE_HOOK(3, it);
        STOP(base + 6);
        if (a.friction && step_dem) {
            TRY(sort_pair(false, false, beside));
            // a whole substep applies the friction correction in the friction pass itself
            if (beside) {
                TLAUNCH(k_friction<true>, 256, full, 128, P, S, vd, vb, X, sd, sb, NL, fr_lists ? 1 : 0, track_d);
            } else {
                TLAUNCH(k_friction<false>, 256, full, 128, P, S, vd, vb, X, sd, sb, NL, fr_lists ? 1 : 0, track_d);
                TLAUNCH(k_apply, 1024, full, 256, P, S, vs, vd, X, 0, 1, track_s, track_d);
            }
            dirty_d = true;
        }
        STOP(base + 7);
    }
    TRY(join_water());
    if (step_sph || step_dem)
        LAUNCH(k_finalize, 2 * full, 256, P, S, X, a.dt, step_sph ? 1 : 0, step_dem ? 1 : 0);
    TAPE_HOOK(4, 0);
    STOP(90);
    // apply_XSPH_viscosity (:3663-3711), Jacobi
    // both forms give the same results; the choice only follows the set sizes at the call
    if (step_sph) {
        if (a.xsph_thread[0])
            TLAUNCH(k_xsph_thread, 256, full, 128, P, S, vs, vd, *a.sph, *a.dem, 1, P.sph_visc, c.tmp_vel);
        else
            TLAUNCH(k_xsph_warp, 256, (uint64_t)full * 32, 128, P, S, vs, vd, *a.sph, *a.dem, 1, P.sph_visc, c.tmp_vel);
        LAUNCH(k_xsph_commit, full, 256, P, S, vs, 1, c.tmp_vel, a.sph->velocity);
    }
    TAPE_HOOK(5, 0);
    if (a.dem_visc && step_dem) {
        if (a.xsph_thread[1])
            TLAUNCH(k_xsph_thread, 256, full, 128, P, S, vd, vs, *a.dem, *a.sph, 0, P.dem_visc, c.tmp_vel);
        else
            TLAUNCH(k_xsph_warp, 256, (uint64_t)full * 32, 128, P, S, vd, vs, *a.dem, *a.sph, 0, P.dem_visc, c.tmp_vel);
        LAUNCH(k_xsph_commit, full, 256, P, S, vd, 0, c.tmp_vel, a.dem->velocity);
    }
    TAPE_HOOK(6, 0);
#undef STOP
    return SNOWB_OK;
}


// ------------------------------------------------------------------ adjoint: recording
// Checks of a call made while recording; the first recorded call fixes the context.
static int tape_start_call(const DevParams& P, snowb_particle_data* sph, uint32_t ns, snowb_particle_data* dem,
                           uint32_t nd, snowb_particle_data* bnd, uint32_t nb, uint32_t full, snowb_cell_data bcd,
                           float dt, int iterations, const int* fl, const snowb_step_options& opt,
                           const snowb_batch* batch)
{
    Tape& tp = g_tape;
    if (opt.quirks != SNOWB_QUIRKS_FIXED) return fail(SNOWB_ERR_INVALID, "adjoint recording needs SNOWB_QUIRKS_FIXED");
    if (opt.use_graph || opt.stop_after || batch)
        return fail(SNOWB_ERR_INVALID, "adjoint recording runs plain substeps (no graph, no stop, no batch)");
    // flags: sph_dem, sph_sph, friction, temperature, change_phase, freezing, melting, dem_visc,
    // interlink, dynamic, cd_on
    if (fl[1] || fl[9]) return fail(SNOWB_ERR_INVALID, "adjoint: sph_sph_correction and dynamic links must be off");
    if (P.scorr_coeff != 0.f) return fail(SNOWB_ERR_INVALID, "adjoint: scorr_coeff must be 0");
    if (iterations < 1) return fail(SNOWB_ERR_INVALID, "adjoint: at least one iteration");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    const bool first = tp.used == 0;
    const bool same = tp.device == dev && tp.full == full && tp.n[0] == ns && tp.n[1] == nd && tp.nb == nb &&
                      tp.maxc == P.maxc && tp.iterations == iterations;
    if (!first && !same) return fail(SNOWB_ERR_INVALID, "adjoint: recorded calls must keep sizes and iterations");
    if (first && !same) {
        tape_free_steps();
        tp.device = dev; tp.full = full; tp.n[0] = ns; tp.n[1] = nd; tp.nb = nb; tp.maxc = P.maxc;
        tp.iterations = iterations;
    }
    if (!tp.viol) {
        TRY(dalloc(&tp.viol, 1));
        CUDA_TRY(cudaMemset(tp.viol, 0, sizeof(uint32_t)));
    }
    tp.sph = *sph; tp.dem = *dem; tp.bnd = *bnd; tp.bcd = bcd; tp.P = P; tp.dt = dt;
    tp.correct_dem = fl[0]; tp.friction = fl[2]; tp.temperature = fl[3]; tp.dem_visc = fl[7];
    tp.interlink = fl[8]; tp.cd_on = fl[10];
    return SNOWB_OK;
}

// ------------------------------------------------------------------ adjoint: reverse pass
struct AdjBufs {
    int device = -1;
    uint32_t cap = 0, bcap = 0, ncells = 0;
    snowb_cell_data cd[2] = {};
    SetBufs sb[2];
    float4* bp4 = nullptr;
    float *binvm = nullptr, *bmass = nullptr;
    float* f[3][7] = {};            // rho, C, S, lam, lamb, rhob, Sb
    float *XB[2] = {}, *U[2] = {}, *X0B[2] = {}, *VB[2] = {}, *XBX[2] = {}, *XH[2] = {}, *T0B[2] = {};
    float* GVW = nullptr;
    uint32_t* nbuf = nullptr;
    double* gp = nullptr;
    std::vector<void*> bufs;
};
static AdjBufs g_adj;

static void adj_free()
{
    for (auto& s : g_adj.sb) free_set(s);
    for (void* p : g_adj.bufs) cudaFree(p);
    g_adj = AdjBufs();
}
static int adj_ensure(uint32_t cap, uint32_t bcap, uint32_t ncells)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    AdjBufs& B = g_adj;
    if (B.device == dev && B.cap >= cap && B.bcap >= bcap && B.ncells == ncells) return SNOWB_OK;
    adj_free();
    B.device = dev; B.cap = cap; B.bcap = bcap; B.ncells = ncells;
    auto A = [&](auto** p, size_t n) -> int { TRY(dalloc(p, n)); B.bufs.push_back(*p); return SNOWB_OK; };
    for (int s = 0; s < 2; ++s) {
        TRY(alloc_sort(B.sb[s], cap, ncells, true));
        TRY(A(&B.cd[s].grid_hash, cap)); TRY(A(&B.cd[s].grid_index, cap));
        TRY(A(&B.cd[s].cell_start, ncells)); TRY(A(&B.cd[s].cell_end, ncells));
        TRY(A(&B.cd[s].sorted_pos, cap));
        for (float** q : {&B.XB[s], &B.U[s], &B.X0B[s], &B.VB[s], &B.XBX[s], &B.XH[s]}) TRY(A(q, (size_t)cap * 3));
        TRY(A(&B.T0B[s], cap));
    }
    for (int s = 0; s < 3; ++s)
        for (int k = 0; k < 7; ++k) TRY(A(&B.f[s][k], s == 2 ? bcap : cap));
    TRY(A(&B.bp4, bcap)); TRY(A(&B.binvm, bcap)); TRY(A(&B.bmass, bcap));
    TRY(A(&B.GVW, (size_t)cap * 3));
    TRY(A(&B.nbuf, 4)); TRY(A(&B.gp, 4));
    return SNOWB_OK;
}
static inline snowb_float3* F3(float* p) { return reinterpret_cast<snowb_float3*>(p); }
static inline const snowb_float3* F3(const float* p) { return reinterpret_cast<const snowb_float3*>(p); }
static int zero(void* p, size_t bytes)
{
    if (bytes) CUDA_TRY(cudaMemsetAsync(p, 0, bytes, g_stream));
    return SNOWB_OK;
}
static int dcopy(void* dst, const void* src, size_t bytes)
{
    if (bytes) CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, g_stream));
    return SNOWB_OK;
}

// reverse of one recorded substep; gx/gv/gT (per set) hold the adjoint of the state after
// it on entry and the adjoint of the state before it on return
static int adj_substep(const TapeStep& T, float* const gx[2], float* const gv[2], float* const gT[2], float* gL)
{
    Tape& tp = g_tape;
    AdjBufs& B = g_adj;
    const DevParams& P = tp.P;
    const uint32_t n[2] = {tp.n[0], tp.n[1]}, nw = n[0], ns = n[1], nb = tp.nb, cap = B.cap;
    const size_t b3[2] = {(size_t)nw * 12, (size_t)ns * 12};
    const int last = tp.iterations - 1;
    Sets X{tp.sph, tp.dem, tp.bnd};
    AdjField F[3];
    for (int s = 0; s < 3; ++s)
        F[s] = AdjField{B.f[s][0], B.f[s][1], B.f[s][2], B.f[s][3], B.f[s][4], B.f[s][5], B.f[s][6]};
    const size_t fb[3] = {(size_t)nw * 4, (size_t)ns * 4, (size_t)nb * 4};
    AdjParams G{B.gp};
    SetView vw = make_view(B.cd[0], B.sb[0].p4, tp.sph.mass);
    SetView vs = make_view(B.cd[1], B.sb[1].p4, tp.dem.mass);
    SetView vb = make_view(tp.bcd, B.bp4, tp.bnd.volume);
    auto sort2 = [&](const float* pw, const float* ps) -> int {
        snowb_particle_data dw = tp.sph, ds = tp.dem;
        dw.predict_positions = const_cast<snowb_float3*>(F3(pw));
        ds.predict_positions = const_cast<snowb_float3*>(F3(ps));
        TRY(sort_set(P, B.sb[0], dw, B.cd[0], B.nbuf + 0, cap, nullptr, true));
        TRY(sort_set(P, B.sb[1], ds, B.cd[1], B.nbuf + 1, cap, nullptr, true));
        return SNOWB_OK;
    };
    auto zero_rhob = [&]() -> int {
        for (int s = 0; s < 3; ++s) TRY(zero(F[s].rhob, fb[s]));
        return SNOWB_OK;
    };
    auto fields = [&]() -> int {
        LAUNCH(ka_fields, nw + ns + nb, 128, P, nw, ns, nb, vw, vs, vb, X, F[0], F[1], F[2]);
        return SNOWB_OK;
    };
    // 1. fields at the last iteration's input positions (densities read by the XSPH)
    TRY(sort2(T.xit[0][last], T.xit[1][last]));
    TRY(fields());
    TRY(zero_rhob());
    // 2. XSPH at the positions of the last sort (after the friction pass's sort)
    const float* xx[2] = {tp.friction ? T.xmid[0][last] : T.xit[0][last],
                          tp.friction ? T.xmid[1][last] : T.xit[1][last]};
    if (tp.friction) TRY(sort2(xx[0], xx[1]));
    for (int s = 0; s < 2; ++s) { TRY(zero(B.VB[s], b3[s])); TRY(zero(B.XBX[s], b3[s])); }
    TRY(dcopy(B.GVW, gv[0], b3[0]));
    if (tp.dem_visc)
        LAUNCH(ka_xsph_rev, ns + nw, 128, P, ns, nw, vs, vw, F3(T.vf[1]), F3(T.vw1), tp.dem.mass, tp.sph.mass,
               F[1].rho, F[0].rho, P.dem_visc, F3(gv[1]), F3(B.VB[1]), F3(B.GVW), F3(B.XBX[1]), F3(B.XBX[0]),
               F[1].rhob, F[0].rhob);
    else
        TRY(dcopy(B.VB[1], gv[1], b3[1]));
    LAUNCH(ka_xsph_rev, nw + ns, 128, P, nw, ns, vw, vs, F3(T.vf[0]), F3(T.vf[1]), tp.sph.mass, tp.dem.mass, F[0].rho,
           F[1].rho, P.sph_visc, F3(B.GVW), F3(B.VB[0]), F3(B.VB[1]), F3(B.XBX[0]), F3(B.XBX[1]), F[0].rhob,
           F[1].rhob);
    // 3. finalize: x = x_new, v = (x_new - x0p)/dt
    for (int s = 0; s < 2; ++s) {
        TRY(dcopy(B.XB[s], gx[s], b3[s]));
        TRY(zero(B.X0B[s], b3[s]));
        LAUNCH(ka_finalize_rev, n[s], 256, n[s], tp.dt, F3(B.VB[s]), F3(B.XB[s]), F3(B.X0B[s]));
    }
    AdjSet AW{F3(B.XB[0]), F3(B.U[0]), F3(B.X0B[0]), F3(T.x0p[0])};
    AdjSet AS{F3(B.XB[1]), F3(B.U[1]), F3(B.X0B[1]), F3(T.x0p[1])};
    // 4. solver iterations, last to first
    for (int it = last; it >= 0; --it) {
        if (tp.friction) {
            if (it != last) TRY(sort2(T.xmid[0][it], T.xmid[1][it]));
            LAUNCH(ka_scale3, ns, 256, ns, F3(B.U[1]), P.sor, F3(B.XB[1]));
            LAUNCH(ka_friction_rev, ns, 128, P, ns, nb, vs, vb, X, AS);
        }
        if (it == last && tp.friction)
            for (int s = 0; s < 2; ++s) LAUNCH(ka_axpy3, n[s], 256, n[s], F3(B.XB[s]), F3(B.XB[s]), 1.f, F3(B.XBX[s]));
        TRY(sort2(T.xit[0][it], T.xit[1][it]));
        TRY(fields());
        for (int s = 0; s < 2; ++s) LAUNCH(ka_scale3, n[s], 256, n[s], F3(B.U[s]), P.sor, F3(B.XB[s]));
        LAUNCH(ka_pbf_lambar, nw + ns + nb, 128, P, nw, ns, nb, vw, vs, vb, X, F[0], F[1], F[2], AW);
        LAUNCH(ka_pos_rev, nw + ns, 128, P, nw, ns, nb, vw, vs, vb, X, F[0], F[1], F[2], AW, AS, G, 1,
               tp.correct_dem);
        if (tp.interlink)
            LAUNCH(ka_interlink_rev, ns, 128, P, ns, F3(T.xit[1][it]), T.rec[it], T.len[it], tp.dem.massInv, AS, G,
                   gL);
        if (it == last && !tp.friction)
            for (int s = 0; s < 2; ++s) LAUNCH(ka_axpy3, n[s], 256, n[s], F3(B.XB[s]), F3(B.XB[s]), 1.f, F3(B.XBX[s]));
        TRY(zero_rhob());
    }
    // 5. heat and link formation at the substep's start positions
    for (int s = 0; s < 2; ++s) TRY(zero(B.XH[s], b3[s]));
    if (tp.interlink)
        LAUNCH(ka_linkform_rev, ns, 128, P, ns, F3(T.x0[1]), T.rec_pre, T.rec[0], gL, F3(B.XH[1]));
    if (tp.temperature) {
        TRY(sort2(T.x0[0], T.x0[1]));
        TRY(fields());
        AdjSet HW{F3(B.XH[0]), F3(B.U[0]), F3(B.X0B[0]), F3(T.x0p[0])};
        AdjSet HS{F3(B.XH[1]), F3(B.U[1]), F3(B.X0B[1]), F3(T.x0p[1])};
        LAUNCH(ka_heat_rev, nw + ns, 128, P, nw, ns, vw, vs, X, T.T0[0], T.T0[1], gT[0], gT[1], B.T0B[0], B.T0B[1],
               F[0], F[1], HW, HS, G, tp.dt);
        LAUNCH(ka_pos_rev, nw + ns, 128, P, nw, ns, nb, vw, vs, vb, X, F[0], F[1], F[2], HW, HS, G, 0, 0);
        TRY(zero_rhob());
        for (int s = 0; s < 2; ++s) TRY(dcopy(gT[s], B.T0B[s], fb[s]));
    }
    // 6. integration (velocity adjoint written to gv, positions added to XH)
    for (int s = 0; s < 2; ++s) {
        LAUNCH(ka_integrate_rev, n[s], 256, P, n[s], tp.dt, tp.cd_on, F3(T.x0[s]), F3(T.v0[s]), F3(B.XB[s]),
               F3(B.X0B[s]), F3(B.XH[s]), F3(gv[s]));
        TRY(dcopy(gx[s], B.XH[s], b3[s]));
    }
    return SNOWB_OK;
}

static int adjoint_backward(const snowb_adjoint_io* io)
{
    Tape& tp = g_tape;
    if (tp.recording) return fail(SNOWB_ERR_INVALID, "adjoint: call snowb_adjoint_end before the backward pass");
    if (tp.used == 0) return fail(SNOWB_ERR_INVALID, "adjoint: nothing recorded");
    if (!io || !io->gx_sph || !io->gv_sph || !io->gT_sph || !io->gx_dem || !io->gv_dem || !io->gT_dem ||
        !io->gL_dem)
        return fail(SNOWB_ERR_INVALID, "adjoint: null gradient buffer");
    uint32_t viol = 0;
    CUDA_TRY(cudaMemcpyAsync(&viol, tp.viol, sizeof(uint32_t), cudaMemcpyDeviceToHost, g_stream));
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    if (viol & 1u) return fail(SNOWB_ERR_INVALID, "adjoint: a particle changed phase while recording");
    if (viol & 2u) return fail(SNOWB_ERR_INVALID, "adjoint: recorded particles need contrib == 1");
    TRY(adj_ensure(tp.full, tp.nb, tp.P.ncells));
    AdjBufs& B = g_adj;
    const uint32_t nh[4] = {tp.n[0], tp.n[1], tp.nb, 0};
    CUDA_TRY(cudaMemcpyAsync(B.nbuf, nh, sizeof(nh), cudaMemcpyHostToDevice, g_stream));
    CUDA_TRY(cudaMemsetAsync(B.gp, 0, 4 * sizeof(double), g_stream));
    LAUNCH(k_boundary_prep, tp.nb, 256, tp.bcd, tp.bnd.volume, tp.bnd.massInv, tp.bnd.mass, tp.nb, B.bp4, B.binvm,
           B.bmass, nullptr, nullptr);
    float* gx[2] = {io->gx_sph, io->gx_dem};
    float* gv[2] = {io->gv_sph, io->gv_dem};
    float* gT[2] = {io->gT_sph, io->gT_dem};
    for (size_t k = tp.used; k-- > 0;) TRY(adj_substep(tp.steps[k], gx, gv, gT, io->gL_dem));
    double g[4];
    CUDA_TRY(cudaMemcpyAsync(g, B.gp, sizeof(g), cudaMemcpyDeviceToHost, g_stream));
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    snowb_adjoint_io* w = const_cast<snowb_adjoint_io*>(io);
    for (int k = 0; k < 4; ++k) w->grad_params[k] += g[k];
    tp.used = 0;
    CUDA_TRY(cudaMemsetAsync(tp.viol, 0, sizeof(uint32_t), g_stream));
    return SNOWB_OK;
}

static int check_params()
{
    if (!g_have_params) return fail(SNOWB_ERR_NO_PARAMS, "snowb_set_sim_params has not been called");
    return SNOWB_OK;
}

// ------------------------------------------------------------------ CUDA graph of a substep
// One substep's launch sequence is fixed by its arguments (all sizes live on the device),
// so it is captured once on a library-owned stream and replayed; the caller's stream and
// the capture stream are ordered with events.  Graphs are cached by their arguments, so a
// host that alternates between several scenes (or batches) replays each scene's graph
// without capturing it again; the least recently used graph goes when the cache is full.
struct GraphEntry {
    std::vector<unsigned char> key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t nodes = 0;        // kernels per replay
    size_t prof_pairs = 0;     // profiling event pairs recorded by one replay
    bool prof = false;         // captured with profiling event nodes
    uint64_t last_use = 0;
};
struct GraphCache {
    std::vector<GraphEntry> entries;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int device = -1;
    uint64_t tick = 0;
    bool prof_replayed = false;   // a profiling graph ran since snowb_profile_begin
    size_t prof_pairs = 0;        // its event pairs (already accumulated after each replay)
};
static GraphCache g_graph;
static constexpr size_t kGraphCacheMax = 256;

static void graph_destroy(GraphEntry& e)
{
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (e.graph) cudaGraphDestroy(e.graph);
    e.exec = nullptr;
    e.graph = nullptr;
}
// drop cached graphs (only the profiling ones if prof_only)
static void graph_reset(bool prof_only = false)
{
    auto& v = g_graph.entries;
    for (auto& e : v)
        if (!prof_only || e.prof) graph_destroy(e);
    v.erase(std::remove_if(v.begin(), v.end(), [](const GraphEntry& e) { return e.exec == nullptr; }), v.end());
}
static void graph_free()
{
    graph_reset();
    if (g_graph.stream) cudaStreamDestroy(g_graph.stream);
    if (g_graph.ev_in) cudaEventDestroy(g_graph.ev_in);
    if (g_graph.ev_out) cudaEventDestroy(g_graph.ev_out);
    g_graph = GraphCache();
}
template <class T>
static void key_add(std::vector<unsigned char>& k, const T& v)
{
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    k.insert(k.end(), p, p + sizeof(T));
}

// Run `count` substeps by replaying the captured graph (capturing it first if needed).
static int graph_substeps(const DevParams& P, const StepArgs& a, bool step_sph, bool step_dem, int count)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (g_graph.device != dev) {
        graph_free();
        g_graph.device = dev;
    }
    if (!g_graph.stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&g_graph.stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&g_graph.ev_in, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&g_graph.ev_out, cudaEventDisableTiming));
    }
    std::vector<unsigned char> key;
    key_add(key, P);
    key_add(key, a);
    key_add(key, *a.sph);
    key_add(key, *a.dem);
    key_add(key, *a.bnd);
    key_add(key, *a.buf);
    key_add(key, step_sph);
    key_add(key, step_dem);
    key_add(key, g_ctx.S);
    key_add(key, g_ctx_gen);
    key_add(key, g_prof);
    key_add(key, g_tune_gen);
    const cudaStream_t user = g_stream;
    GraphEntry* ent = nullptr;
    for (auto& e : g_graph.entries)
        if (e.key == key) { ent = &e; break; }
    if (!ent) {
        if (g_graph.entries.size() >= kGraphCacheMax) {
            auto lru = std::min_element(g_graph.entries.begin(), g_graph.entries.end(),
                                        [](const GraphEntry& x, const GraphEntry& y) { return x.last_use < y.last_use; });
            graph_destroy(*lru);
            g_graph.entries.erase(lru);
        }
        g_stream = g_graph.stream;
        // with profiling on, the events recorded around each launch become event nodes of
        // the graph, which time every kernel without host gaps between launches
        g_prof_used = 0;
        cudaError_t e0 = cudaStreamBeginCapture(g_graph.stream, cudaStreamCaptureModeThreadLocal);
        const uint64_t before = g_launches;
        g_capturing = true;
        int rc = e0 == cudaSuccess ? substep(P, a, step_sph, step_dem) : SNOWB_ERR_CUDA;
        g_capturing = false;
        const uint64_t nodes = g_launches - before;
        g_launches = before;
        cudaGraph_t gr = nullptr;
        cudaError_t e1 = cudaStreamEndCapture(g_graph.stream, &gr);
        g_stream = user;
        if (e0 != cudaSuccess) return fail(SNOWB_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e0));
        if (rc != SNOWB_OK) { if (gr) cudaGraphDestroy(gr); return rc; }
        if (e1 != cudaSuccess) return fail(SNOWB_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e1));
        GraphEntry e;
        e.key = std::move(key);
        e.graph = gr;
        e.nodes = nodes;
        e.prof = g_prof;
        e.prof_pairs = g_prof_used;
        // kernel nodes keep the priorities of the streams they were captured from
        cudaError_t e2 = cudaGraphInstantiate(&e.exec, gr, cudaGraphInstantiateFlagUseNodePriority);
        if (e2 != cudaSuccess) {
            cudaGraphDestroy(gr);
            return fail(SNOWB_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e2));
        }
        g_graph.entries.push_back(std::move(e));
        ent = &g_graph.entries.back();
    }
    ent->last_use = ++g_graph.tick;
    if (ent->prof) {
        g_graph.prof_replayed = true;
        g_graph.prof_pairs = ent->prof_pairs;
    }
    CUDA_TRY(cudaEventRecord(g_graph.ev_in, user));
    CUDA_TRY(cudaStreamWaitEvent(g_graph.stream, g_graph.ev_in, 0));
    for (int k = 0; k < count; ++k) {
        CUDA_TRY(cudaGraphLaunch(ent->exec, g_graph.stream));
        if (ent->prof) {
            CUDA_TRY(cudaStreamSynchronize(g_graph.stream));
            if (prof_accumulate(0, ent->prof_pairs) != 0) return fail(SNOWB_ERR_CUDA, "profile events");
        }
    }
    CUDA_TRY(cudaEventRecord(g_graph.ev_out, g_graph.stream));
    CUDA_TRY(cudaStreamWaitEvent(user, g_graph.ev_out, 0));
    g_launches += (uint64_t)count * ent->nodes;
    return SNOWB_OK;
}

// Grid of a batch: the scene grid repeated scenes_x times along x and scenes_z times along z.
static int batch_layout(DevParams& P, const snowb_batch* b)
{
    if (!b) return fail(SNOWB_ERR_INVALID, "null batch");
    const uint32_t nx = b->scenes_x, nz = b->scenes_z;
    if (nx == 0 || nz == 0 || (nx & (nx - 1)) || (nz & (nz - 1)))
        return fail(SNOWB_ERR_INVALID, "scenes_x and scenes_z must be powers of two");
    const uint64_t cells = (uint64_t)P.gsx * nx * P.gsy * P.gsz * nz;
    if (cells >= (1ull << 31)) return fail(SNOWB_ERR_INVALID, "batched cell grid too large");
    P.sgx = P.gsx; P.sgz = P.gsz;
    P.gsx *= nx; P.gsz *= nz;
    P.ncells = (uint32_t)cells;
    P.batch_nx = nx;
    P.batch_shift = (uint32_t)__builtin_ctz(nx);
    P.scene_mask = nx * nz - 1u;
    return SNOWB_OK;
}

static int run_steps(snowb_particle_data* sph, uint32_t* sph_size, snowb_particle_data* dem, uint32_t* dem_size,
                     snowb_particle_data* bnd, uint32_t nb, uint32_t full, snowb_particle_data* buf,
                     snowb_cell_data scd, snowb_cell_data dcd, snowb_cell_data bcd, snowb_scene_params* scene,
                     float dt, int iterations, const int* fl, float dTe, const snowb_step_options& opt,
                     const snowb_batch* batch = nullptr)
{
    TRY(check_params());
    if (!sph || !dem || !bnd || !buf || !sph_size || !dem_size || !scene)
        return fail(SNOWB_ERR_INVALID, "null argument");
    if (*sph_size > full || *dem_size > full) return fail(SNOWB_ERR_INVALID, "set size exceeds full_size");
    if (opt.substeps < 1) return fail(SNOWB_ERR_INVALID, "substeps must be >= 1");
    DevParams P = g_P;
    P.quirks = opt.quirks;
    if (P.gsx < 4 || P.gsy < 4 || P.gsz < 4) return fail(SNOWB_ERR_INVALID, "grid must be at least 4 cells per axis");
    if (full >= (1u << 25) || nb >= (1u << 25)) return fail(SNOWB_ERR_INVALID, "more than 2^25 particles per set");
    if (batch) {
        if (opt.quirks != SNOWB_QUIRKS_FIXED)
            return fail(SNOWB_ERR_INVALID, "batched scenes need SNOWB_QUIRKS_FIXED (the reference's quirks depend "
                                           "on whole-set sizes)");
        if (!batch->scene_sph || !batch->scene_dem || !batch->scene_boundary || !batch->scene_buffer)
            return fail(SNOWB_ERR_INVALID, "batch scene id arrays missing");
        TRY(batch_layout(P, batch));
    }
    TRY(ensure_ctx(full, nb, P.ncells));
    Ctx& c = g_ctx;
    if (g_tape.recording) TRY(tape_start_call(P, sph, *sph_size, dem, *dem_size, bnd, nb, full, bcd, dt, iterations,
                                              fl, opt, batch));
    // XSPH's thread form for sets past XSPH_WARP_MAX (the snow set's reference-mode launch
    // covers only the water set's launch size, Q6)
    const uint32_t xs_s = *sph_size;
    const uint32_t xs_d = opt.quirks == SNOWB_QUIRKS_REFERENCE ? umin32(coverage(*sph_size), *dem_size) : *dem_size;
    StepArgs a{sph, dem, bnd, buf, nb, full, scd, dcd, bcd, dt, iterations,
               fl[0], fl[1], fl[2], fl[3], fl[4], fl[5], fl[6], fl[7], fl[8], fl[9], fl[10], dTe, opt.stop_after,
               batch ? batch->scene_sph : nullptr, batch ? batch->scene_dem : nullptr,
               batch ? batch->scene_boundary : nullptr, batch ? batch->scene_buffer : nullptr,
               {xs_s > XSPH_WARP_MAX ? 1 : 0, xs_d > XSPH_WARP_MAX ? 1 : 0}};
    LAUNCH1(k_set_state, c.S, *sph_size, *dem_size, nb);
    if (batch)
        LAUNCH(k_check_scenes, full > nb ? full : nb, 256, P, c.S, a.sid_sph, a.sid_dem, a.sid_bnd);
    LAUNCH(k_boundary_prep, nb, 256, bcd, bnd->volume, bnd->massInv, bnd->mass, nb, c.b.p4, c.b.invm, c.b.mass,
           a.sid_bnd, a.sid_bnd ? c.b.sid : nullptr);
    int k = 0;
    while (k < opt.substeps) {
        const bool step_sph = scene->current_time >= scene->fluid_start_time;
        const bool step_dem = scene->current_time >= scene->solid_start_time;
        if (opt.use_graph && opt.stop_after == 0) {
            // replay as many substeps as keep the same step flags
            int run = 0;
            float t = scene->current_time;
            while (k + run < opt.substeps && (t >= scene->fluid_start_time) == step_sph &&
                   (t >= scene->solid_start_time) == step_dem) {
                ++run;
                t += dt;
            }
            TRY(graph_substeps(P, a, step_sph, step_dem, run));
            for (int r = 0; r < run; ++r) scene->current_time += dt;
            k += run;
            continue;
        }
        TRY(substep(P, a, step_sph, step_dem));
        if (opt.stop_after != 0) break;
        scene->current_time += dt;
        ++k;
    }
    if (opt.sync) {
        CUDA_TRY(cudaMemcpyAsync(c.S_host, c.S, sizeof(DevState), cudaMemcpyDeviceToHost, g_stream));
        CUDA_TRY(cudaStreamSynchronize(g_stream));
        *sph_size = c.S_host->n_sph;
        *dem_size = c.S_host->n_dem;
        if (c.S_host->err) return fail(SNOWB_ERR_DEVICE, "device error flag " + std::to_string(c.S_host->err));
    }
    return SNOWB_OK;
}

// ------------------------------------------------------- set-up passes (one or many scenes)
static int calc_hash(const DevParams& P, snowb_cell_data cd, const snowb_float3* pos, const uint32_t* sid, uint32_t n)
{
    if (n == 0) return SNOWB_OK;
    if (!pos || !cd.grid_hash || !cd.grid_index) return fail(SNOWB_ERR_INVALID, "null pointer");
    LAUNCH(k_calc_hash, n, 256, P, cd, pos, n, sid);
    return SNOWB_OK;
}

// stable sort of (grid_hash, grid_index) pairs by hash over a table of nc cells
static int sort_pairs(uint32_t nc, snowb_cell_data cd, uint32_t n)
{
    if (n < 2) return SNOWB_OK;
    if (!cd.grid_hash || !cd.grid_index) return fail(SNOWB_ERR_INVALID, "null pointer");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (g_ctx.device != dev || g_ctx.ncells != nc) TRY(ensure_ctx(1, 1, nc));
    TRY(ensure_gen(n, nc));
    SetBufs& B = g_ctx.gen;
    CUDA_TRY(cudaMemsetAsync(g_ctx.err_dev, 0, sizeof(uint32_t), g_stream));
    LAUNCH(k_key_count, n, 256, cd.grid_hash, cd.grid_index, n, nc, B.key, B.val, B.slot, B.cnt, g_ctx.err_dev);
    const unsigned nb = (nc + SCAN_CHUNK - 1) / SCAN_CHUNK;
    KL(k_block_sums, nb, SCAN_TPB, B.cnt, nc, B.bsum, nullptr);
    // cell_start is not touched by a plain sort: clear nothing (clear_all = 0, n = 0)
    KL(k_cell_scan, nb, SCAN_TPB, B.cnt, B.bsum, nc, B.off, nullptr, nullptr, 0u, 0, nullptr);
    LAUNCH(k_scatter, n, 256, B.key, B.slot, B.off, B.tmp, nullptr, n, nullptr);
    LAUNCH(k_rank_pairs, n, 256, B.key, B.val, B.off, B.tmp, cd.grid_hash, cd.grid_index, n);
    uint32_t err = 0;
    CUDA_TRY(cudaMemcpyAsync(&err, g_ctx.err_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, g_stream));
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    if (err) return fail(SNOWB_ERR_INVALID, "grid_hash holds keys >= num_cells");
    return SNOWB_OK;
}

static int reorder(uint32_t table_cells, snowb_cell_data cd, const snowb_float3* old_pos, uint32_t n,
                   uint32_t num_cells)
{
    if (!cd.cell_start || !cd.cell_end || !cd.grid_hash || !cd.grid_index || !cd.sorted_pos)
        return fail(SNOWB_ERR_INVALID, "null pointer");
    if (num_cells > table_cells) return fail(SNOWB_ERR_INVALID, "num_cells exceeds the cell table");
    if (num_cells) CUDA_TRY(cudaMemsetAsync(cd.cell_start, 0xff, sizeof(uint32_t) * num_cells, g_stream));
    if (n == 0) return SNOWB_OK;
    if (!old_pos) return fail(SNOWB_ERR_INVALID, "null pointer");
    LAUNCH(k_reorder, n, 256, cd, old_pos, n);
    return SNOWB_OK;
}

static int boundary_volume(const DevParams& P, snowb_cell_data cd, float* mass, float* volume, const uint32_t* sid,
                           uint32_t n)
{
    if (n == 0) return SNOWB_OK;
    if (!mass || !volume) return fail(SNOWB_ERR_INVALID, "null pointer");
    LAUNCH(k_boundary_volume, n, 128, P, cd, mass, volume, n, sid);
    return SNOWB_OK;
}

// connect_and_record over a sorted snow set (sid: its scene ids in original order, or null)
static int connect_links(const DevParams& P, snowb_particle_data* dem, uint32_t n, snowb_cell_data dcd, int dynamic,
                         const uint32_t* sid)
{
    if (!dem) return fail(SNOWB_ERR_INVALID, "null pointer");
    if (n == 0) return SNOWB_OK;
    if (P.gsx < 4 || P.gsy < 4 || P.gsz < 4) return fail(SNOWB_ERR_INVALID, "grid must be at least 4 cells per axis");
    TRY(ensure_ctx(g_ctx.cap > n ? g_ctx.cap : n, g_ctx.bcap ? g_ctx.bcap : 1, P.ncells));
    Ctx& c = g_ctx;
    LAUNCH1(k_set_state, c.S, 0u, n, 0u);
    CUDA_TRY(cudaMemsetAsync(c.fs, 0, sizeof(uint32_t) * P.ncells, g_stream));
    CUDA_TRY(cudaMemsetAsync(c.fe, 0, sizeof(uint32_t) * P.ncells, g_stream));
    LAUNCH(k_fresh_ranges, n, 256, dcd.grid_hash, n, c.fs, c.fe);
    // the view's compact copy (and sorted scene ids) are filled from sorted_pos
    LAUNCH(k_boundary_prep, n, 256, dcd, dem->mass, dem->massInv, dem->mass, n, c.s[1].p4, c.s[1].invm, c.s[1].lambda,
           sid, sid ? c.s[1].sid : nullptr);
    SetView vd = make_view(dcd, c.s[1].p4, dem->mass, sid ? c.s[1].sid : nullptr);
    const SCList scl = sc_lists(P);
    LAUNCH(k_link_filter, n, 128, P, c.S, vd, *dem, dynamic, c.active, NList{nullptr, nullptr, 0u, 0u}, scl);
    const uint32_t nsc = (P.gsx / 4) * (P.gsy / 4) * (P.gsz / 4);
    for (uint32_t col = 0; col < 8; ++col) {
        if (P.maxc <= SNOWB_MAXC_FAST)
            LAUNCH(k_link_colour_warp, (uint64_t)nsc * 32, 128, P, c.S, vd, *dem, c.fs, c.fe, c.active, col, dynamic,
                   NList{nullptr, nullptr, 0u, 0u}, scl);
        else
            LAUNCH(k_link_colour, nsc, 64, P, c.S, vd, *dem, c.fs, c.fe, c.active, col, dynamic);
    }
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    return SNOWB_OK;
}

}  // namespace snowb

using namespace snowb;

// =========================================================================== C ABI
extern "C" {

int snowb_last_error(void) { return g_err; }
const char* snowb_last_error_string(void) { return g_msg.c_str(); }

int snowb_allocate_array(void** dev_ptr, size_t size)
{
    if (!dev_ptr) return fail(SNOWB_ERR_INVALID, "null pointer");
    CUDA_TRY(cudaMalloc(dev_ptr, size));
    return SNOWB_OK;
}

int snowb_set_sim_params(const snowb_sim_params* params)
{
    if (!params) return fail(SNOWB_ERR_INVALID, "null params");
    for (int k = 0; k < 3; ++k) {
        uint32_t g = params->grid_size[k];
        if (g == 0 || (g & (g - 1))) return fail(SNOWB_ERR_INVALID, "grid sizes must be powers of two");
    }
    if ((uint64_t)params->grid_size[0] * params->grid_size[1] * params->grid_size[2] != params->num_cells)
        return fail(SNOWB_ERR_INVALID, "num_cells must equal the grid volume");
    std::lock_guard<std::mutex> lk(g_mu);
    g_sim = *params;
    g_P = derive(g_sim);
    g_have_params = true;
    return SNOWB_OK;
}

int snowb_set_domain(float x_min, float x_max, float z_min, float z_max, float floor_y)
{
    if (!(x_min < x_max) || !(z_min < z_max) || !std::isfinite(x_min) || !std::isfinite(x_max) ||
        !std::isfinite(z_min) || !std::isfinite(z_max) || !std::isfinite(floor_y))
        return fail(SNOWB_ERR_INVALID, "domain needs finite x_min < x_max, z_min < z_max and floor_y");
    std::lock_guard<std::mutex> lk(g_mu);
    g_domain[0] = x_min; g_domain[1] = x_max; g_domain[2] = z_min; g_domain[3] = z_max; g_domain[4] = floor_y;
    if (g_have_params) g_P = derive(g_sim);
    return SNOWB_OK;
}

int snowb_compute_grid_size(uint32_t n, uint32_t block_size, uint32_t* num_blocks, uint32_t* num_threads)
{
    if (!num_blocks || !num_threads) return fail(SNOWB_ERR_INVALID, "null pointer");
    if (n == 0) { *num_blocks = 0; *num_threads = 0; return SNOWB_OK; }
    if (block_size == 0) return fail(SNOWB_ERR_INVALID, "block_size must be > 0");
    *num_threads = block_size < n ? block_size : n;
    *num_blocks = (n % *num_threads != 0) ? (n / *num_threads + 1) : (n / *num_threads);
    return SNOWB_OK;
}

int snowb_calculate_hash(snowb_cell_data cd, const snowb_float3* pos, uint32_t n)
{
    TRY(check_params());
    return calc_hash(g_P, cd, pos, nullptr, n);
}

int snowb_sort_particles(snowb_cell_data cd, uint32_t n)
{
    TRY(check_params());
    return sort_pairs(g_P.ncells, cd, n);
}

// ---------------------------------------------------------------------------
// Sort without allocation.  Some callers cannot call cudaMalloc: a renderer or game loop
// that forbids allocation after start-up (cudaMalloc may synchronise the device and stall
// the frame), a plugin whose host owns every device allocation, or a process running under
// a fixed device-memory budget.  snowb_sort_particles_static does the same stable sort as
// snowb_sort_particles, but all its scratch lives in the fixed array below, which the
// module reserves once on every device that loads this library and keeps until exit.
// In host code the array's name is only a host-side stand-in, so its device address is
// taken with cudaGetSymbolAddress once per device (on the first call made with that
// device current; that first call should come before any stream capture).  All calls
// share the array: calls that overlap on the GPU (other streams, other host threads)
// race and must be serialised by the caller.  The address is kept for the life of the
// process; a cudaDeviceReset in between is not supported (the library's other device
// state does not survive one either).  The limits are in include/snow_b200.h.
static constexpr size_t kStaticBsum = SNOWB_STATIC_SORT_MAX_CELLS / SCAN_CHUNK + 2;
static constexpr size_t kStaticWords = 4ull * SNOWB_STATIC_SORT_MAX_PARTICLES + SNOWB_STATIC_SORT_MAX_CELLS +
                                       (SNOWB_STATIC_SORT_MAX_CELLS + 1) + kStaticBsum + 1;
static __device__ __align__(256) uint32_t g_static_sort_scratch[kStaticWords];
static uint32_t* g_static_sort_ptr[64] = {};   // device address of the array, per device

static int static_sort_scratch(uint32_t** out)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(SNOWB_ERR_INVALID, "device index out of range for the static scratch table");
    if (!g_static_sort_ptr[dev]) {
        void* p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_static_sort_scratch));
        g_static_sort_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_static_sort_ptr[dev];
    return SNOWB_OK;
}
#define KL_PLAIN(kernel, grid, tpb, ...)                                                   \
    do {                                                                                   \
        kernel<<<(grid), (tpb), 0, g_stream>>>(__VA_ARGS__);                               \
        cudaError_t _e = cudaGetLastError();                                               \
        if (_e != cudaSuccess)                                                             \
            return fail(SNOWB_ERR_CUDA, std::string(#kernel) + ": " + cudaGetErrorString(_e)); \
    } while (0)

int snowb_sort_particles_static(snowb_cell_data cd, uint32_t n)
{
    TRY(check_params());
    if (n < 2) return SNOWB_OK;
    if (!cd.grid_hash || !cd.grid_index) return fail(SNOWB_ERR_INVALID, "null pointer");
    const uint32_t nc = g_P.ncells;
    if (n > SNOWB_STATIC_SORT_MAX_PARTICLES)
        return fail(SNOWB_ERR_INVALID, "snowb_sort_particles_static: " + std::to_string(n) +
                                           " particles exceed the static scratch limit of " +
                                           std::to_string(SNOWB_STATIC_SORT_MAX_PARTICLES));
    if (nc > SNOWB_STATIC_SORT_MAX_CELLS)
        return fail(SNOWB_ERR_INVALID, "snowb_sort_particles_static: " + std::to_string(nc) +
                                           " cells exceed the static scratch limit of " +
                                           std::to_string(SNOWB_STATIC_SORT_MAX_CELLS));
    uint32_t* base = nullptr;
    TRY(static_sort_scratch(&base));
    const uint32_t M = SNOWB_STATIC_SORT_MAX_PARTICLES;
    uint32_t* key = base;
    uint32_t* val = key + M;
    uint32_t* slot = val + M;
    uint32_t* tmp = slot + M;
    uint32_t* cnt = tmp + M;
    uint32_t* off = cnt + SNOWB_STATIC_SORT_MAX_CELLS;
    uint32_t* bsum = off + (SNOWB_STATIC_SORT_MAX_CELLS + 1);
    uint32_t* err = bsum + kStaticBsum;
    // the per-cell counters and the error word must start at zero on every call
    CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * nc, g_stream));
    CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(uint32_t), g_stream));
    const unsigned nb = (nc + SCAN_CHUNK - 1) / SCAN_CHUNK;
    KL_PLAIN(k_key_count, blocks_for(n, 256), 256, cd.grid_hash, cd.grid_index, n, nc, key, val, slot, cnt, err);
    KL_PLAIN(k_block_sums, nb, SCAN_TPB, cnt, nc, bsum, nullptr);
    KL_PLAIN(k_cell_scan, nb, SCAN_TPB, cnt, bsum, nc, off, nullptr, nullptr, 0u, 0, nullptr);
    KL_PLAIN(k_scatter, blocks_for(n, 256), 256, key, slot, off, tmp, nullptr, n, nullptr);
    KL_PLAIN(k_rank_pairs, blocks_for(n, 256), 256, key, val, off, tmp, cd.grid_hash, cd.grid_index, n);
    uint32_t herr = 0;
    CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, g_stream));
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    if (herr) return fail(SNOWB_ERR_INVALID, "grid_hash holds keys >= num_cells");
    return SNOWB_OK;
}

int snowb_reorder_data(snowb_cell_data cd, const snowb_float3* old_pos, uint32_t n, uint32_t num_cells)
{
    TRY(check_params());
    return reorder(g_P.ncells, cd, old_pos, n, num_cells);
}

int snowb_compute_boundary_volume(snowb_cell_data cd, float* mass, float* volume, uint32_t n)
{
    TRY(check_params());
    return boundary_volume(g_P, cd, mass, volume, nullptr, n);
}

int snowb_integrate_pbd(snowb_particle_data* particles, float dt, uint32_t n, int cd_on)
{
    TRY(check_params());
    if (!particles) return fail(SNOWB_ERR_INVALID, "null pointer");
    if (n == 0) return SNOWB_OK;
    TRY(ensure_ctx(g_ctx.cap ? g_ctx.cap : 1, g_ctx.bcap ? g_ctx.bcap : 1, g_P.ncells));
    DevParams P = g_P;
    P.quirks = SNOWB_QUIRKS_FIXED;   // exactly n particles (the caller owns the launch size)
    LAUNCH1(k_set_state, g_ctx.S, n, 0u, 0u);
    Sets X{*particles, *particles, *particles};
    LAUNCH(k_integrate, n, 256, P, g_ctx.S, X, n, dt, cd_on, 1, 0, SortTrack{}, SortTrack{});
    return SNOWB_OK;
}

int snowb_connect_and_record(snowb_particle_data* dem, uint32_t n, snowb_cell_data dcd, int dynamic)
{
    TRY(check_params());
    return connect_links(g_P, dem, n, dcd, dynamic, nullptr);
}

static snowb_step_options default_options()
{
    snowb_step_options o;
    o.quirks = g_quirks; o.substeps = 1; o.stop_after = 0; o.use_graph = 0; o.sync = 1;
    return o;
}

int snowb_snow_simulation(snowb_particle_data* sph, uint32_t* sph_size, snowb_particle_data* dem, uint32_t* dem_size,
                          snowb_particle_data* boundary, uint32_t boundary_size, uint32_t full_size,
                          snowb_particle_data* buffer, snowb_cell_data scd, snowb_cell_data dcd, snowb_cell_data bcd,
                          snowb_scene_params* scene, float dt, int iterations, int sph_dem_correction,
                          int sph_sph_correction, int dem_friction, int compute_temperature, int change_phase,
                          int simulate_freezing, int simulate_melting, int dem_viscosity, int use_interlink,
                          int dynamic_max_connections, int cd_on, float temperature_variation)
{
    const int fl[11] = {sph_dem_correction, sph_sph_correction, dem_friction, compute_temperature, change_phase,
                        simulate_freezing, simulate_melting, dem_viscosity, use_interlink, dynamic_max_connections,
                        cd_on};
    snowb_step_options o = default_options();
    return run_steps(sph, sph_size, dem, dem_size, boundary, boundary_size, full_size, buffer, scd, dcd, bcd, scene,
                     dt, iterations, fl, temperature_variation, o);
}

int snowb_snow_simulation_ex(snowb_particle_data* sph, uint32_t* sph_size, snowb_particle_data* dem,
                             uint32_t* dem_size, snowb_particle_data* boundary, uint32_t boundary_size,
                             uint32_t full_size, snowb_particle_data* buffer, snowb_cell_data scd,
                             snowb_cell_data dcd, snowb_cell_data bcd, snowb_scene_params* scene, float dt,
                             int iterations, int sph_dem_correction, int sph_sph_correction, int dem_friction,
                             int compute_temperature, int change_phase, int simulate_freezing, int simulate_melting,
                             int dem_viscosity, int use_interlink, int dynamic_max_connections, int cd_on,
                             float temperature_variation, const snowb_step_options* options)
{
    const int fl[11] = {sph_dem_correction, sph_sph_correction, dem_friction, compute_temperature, change_phase,
                        simulate_freezing, simulate_melting, dem_viscosity, use_interlink, dynamic_max_connections,
                        cd_on};
    snowb_step_options o = options ? *options : default_options();
    if (o.quirks != SNOWB_QUIRKS_REFERENCE && o.quirks != SNOWB_QUIRKS_FIXED)
        return fail(SNOWB_ERR_INVALID, "unknown quirk mode");
    return run_steps(sph, sph_size, dem, dem_size, boundary, boundary_size, full_size, buffer, scd, dcd, bcd, scene,
                     dt, iterations, fl, temperature_variation, o);
}

// ------------------------------------------------------------------ batched scenes
static int batch_P(const snowb_batch* b, DevParams& P)
{
    TRY(check_params());
    P = g_P;
    return batch_layout(P, b);
}

int snowb_batch_num_cells(const snowb_batch* b, uint32_t* num_cells)
{
    if (!num_cells) return fail(SNOWB_ERR_INVALID, "null pointer");
    DevParams P;
    TRY(batch_P(b, P));
    *num_cells = P.ncells;
    return SNOWB_OK;
}

int snowb_batch_calculate_hash(const snowb_batch* b, snowb_cell_data cd, const snowb_float3* pos,
                               const uint32_t* scene_of, uint32_t n)
{
    DevParams P;
    TRY(batch_P(b, P));
    if (n && !scene_of) return fail(SNOWB_ERR_INVALID, "null scene ids");
    return calc_hash(P, cd, pos, scene_of, n);
}

int snowb_batch_sort_particles(const snowb_batch* b, snowb_cell_data cd, uint32_t n)
{
    DevParams P;
    TRY(batch_P(b, P));
    return sort_pairs(P.ncells, cd, n);
}

int snowb_batch_reorder_data(const snowb_batch* b, snowb_cell_data cd, const snowb_float3* old_pos, uint32_t n)
{
    DevParams P;
    TRY(batch_P(b, P));
    return reorder(P.ncells, cd, old_pos, n, P.ncells);
}

int snowb_batch_compute_boundary_volume(const snowb_batch* b, snowb_cell_data cd, float* mass, float* volume,
                                        uint32_t n)
{
    DevParams P;
    TRY(batch_P(b, P));
    if (n && !b->scene_boundary) return fail(SNOWB_ERR_INVALID, "null scene ids");
    return boundary_volume(P, cd, mass, volume, b->scene_boundary, n);
}

int snowb_batch_connect_and_record(const snowb_batch* b, snowb_particle_data* dem, uint32_t n,
                                   snowb_cell_data dcd, int dynamic)
{
    DevParams P;
    TRY(batch_P(b, P));
    if (n && !b->scene_dem) return fail(SNOWB_ERR_INVALID, "null scene ids");
    return connect_links(P, dem, n, dcd, dynamic, b->scene_dem);
}

int snowb_batch_snow_simulation(const snowb_batch* b, snowb_particle_data* sph, uint32_t* sph_size,
                                snowb_particle_data* dem, uint32_t* dem_size, snowb_particle_data* boundary,
                                uint32_t boundary_size, uint32_t full_size, snowb_particle_data* buffer,
                                snowb_cell_data scd, snowb_cell_data dcd, snowb_cell_data bcd,
                                snowb_scene_params* scene, float dt, int iterations, int sph_dem_correction,
                                int sph_sph_correction, int dem_friction, int compute_temperature, int change_phase,
                                int simulate_freezing, int simulate_melting, int dem_viscosity, int use_interlink,
                                int dynamic_max_connections, int cd_on, float temperature_variation,
                                const snowb_step_options* options)
{
    if (!b) return fail(SNOWB_ERR_INVALID, "null batch");
    const int fl[11] = {sph_dem_correction, sph_sph_correction, dem_friction, compute_temperature, change_phase,
                        simulate_freezing, simulate_melting, dem_viscosity, use_interlink, dynamic_max_connections,
                        cd_on};
    snowb_step_options o = options ? *options : default_options();
    return run_steps(sph, sph_size, dem, dem_size, boundary, boundary_size, full_size, buffer, scd, dcd, bcd, scene,
                     dt, iterations, fl, temperature_variation, o, b);
}

// ------------------------------------------------------------------ autotuner
int snowb_autotune(snowb_particle_data* sph, uint32_t* sph_size, snowb_particle_data* dem, uint32_t* dem_size,
                   snowb_particle_data* boundary, uint32_t boundary_size, uint32_t full_size,
                   snowb_particle_data* buffer, snowb_cell_data scd, snowb_cell_data dcd, snowb_cell_data bcd,
                   snowb_scene_params* scene, float dt, int iterations, int sph_dem_correction,
                   int sph_sph_correction, int dem_friction, int compute_temperature, int change_phase,
                   int simulate_freezing, int simulate_melting, int dem_viscosity, int use_interlink,
                   int dynamic_max_connections, int cd_on, float temperature_variation, int quirks,
                   int substeps, const snowb_batch* batch)
{
    if (substeps < 1) return fail(SNOWB_ERR_INVALID, "autotune: substeps must be >= 1");
    if (g_prof || g_tape.recording) return fail(SNOWB_ERR_INVALID, "autotune: profiling or adjoint recording active");
    if (quirks != SNOWB_QUIRKS_REFERENCE && quirks != SNOWB_QUIRKS_FIXED)
        return fail(SNOWB_ERR_INVALID, "unknown quirk mode");
    const int fl[11] = {sph_dem_correction, sph_sph_correction, dem_friction, compute_temperature, change_phase,
                        simulate_freezing, simulate_melting, dem_viscosity, use_interlink, dynamic_max_connections,
                        cd_on};
    static const int tpbs[3] = {64, 128, 256};
    static const int caps[3] = {8, 16, 64};
    snowb_step_options o;
    o.quirks = quirks; o.stop_after = 0; o.use_graph = 1; o.sync = 1;
    std::vector<std::string> names;
    std::vector<std::vector<double>> ms;   // [name][candidate]
    g_tune_seen.clear();
    int rc = SNOWB_OK;
    for (int c = 0; c < 9 && rc == SNOWB_OK; ++c) {
        g_tune_force_tpb = tpbs[c / 3];
        g_tune_force_capm = caps[c % 3];
        ++g_tune_gen;
        o.substeps = 1;   // capture and warm the candidate's graph, untimed
        rc = run_steps(sph, sph_size, dem, dem_size, boundary, boundary_size, full_size, buffer, scd, dcd, bcd, scene,
                       dt, iterations, fl, temperature_variation, o, batch);
        if (rc != SNOWB_OK) break;
        snowb_profile_begin();
        o.substeps = substeps;
        rc = run_steps(sph, sph_size, dem, dem_size, boundary, boundary_size, full_size, buffer, scd, dcd, bcd, scene,
                       dt, iterations, fl, temperature_variation, o, batch);
        const int rc2 = snowb_profile_end(nullptr, 0);
        if (rc == SNOWB_OK) rc = rc2;
        for (size_t k = 0; k < g_acc_name.size(); ++k) {
            size_t idx = 0;
            while (idx < names.size() && names[idx] != g_acc_name[k]) ++idx;
            if (idx == names.size()) { names.push_back(g_acc_name[k]); ms.emplace_back(9, -1.0); }
            ms[idx][c] = g_acc_ms[k];
        }
    }
    g_tune_force_tpb = 0;
    g_tune_force_capm = 0;
    ++g_tune_gen;
    if (rc != SNOWB_OK) return rc;
    for (const auto& sb : g_tune_seen) {
        size_t idx = 0;
        while (idx < names.size() && names[idx] != sb.first) ++idx;
        if (idx == names.size()) continue;
        int best = -1;
        for (int c = 0; c < 9; ++c)
            if (ms[idx][c] >= 0.0 && (best < 0 || ms[idx][c] < ms[idx][best])) best = c;
        if (best < 0) continue;
        bool found = false;
        for (auto& e : g_tune)
            if (e.name == sb.first && e.bucket == sb.second) {
                e.tpb = tpbs[best / 3]; e.capm = caps[best % 3]; found = true;
            }
        if (!found) g_tune.push_back(TuneEntry{sb.first, sb.second, tpbs[best / 3], caps[best % 3]});
    }
    ++g_tune_gen;
    return SNOWB_OK;
}

int snowb_autotune_table(char* out, size_t cap)
{
    if (!out || cap == 0) return fail(SNOWB_ERR_INVALID, "null buffer");
    std::string txt;
    for (const auto& e : g_tune)
        txt += e.name + " " + std::to_string(e.bucket) + " " + std::to_string(e.tpb) + " " + std::to_string(e.capm) +
               "\n";
    const size_t n = txt.size() < cap - 1 ? txt.size() : cap - 1;
    std::memcpy(out, txt.data(), n);
    out[n] = 0;
    if (txt.size() >= cap) return fail(SNOWB_ERR_INVALID, "table buffer too small");
    return SNOWB_OK;
}

int snowb_autotune_load(const char* table)
{
    if (!table) return fail(SNOWB_ERR_INVALID, "null table");
    std::vector<TuneEntry> t;
    const char* p = table;
    while (*p) {
        const char* eol = std::strchr(p, '\n');
        std::string line(p, eol ? (size_t)(eol - p) : std::strlen(p));
        p = eol ? eol + 1 : p + line.size();
        if (line.empty()) continue;
        char name[128];
        int bucket, tpb, capm;
        if (std::sscanf(line.c_str(), "%127s %d %d %d", name, &bucket, &tpb, &capm) != 4)
            return fail(SNOWB_ERR_INVALID, "autotune table: bad line '" + line + "'");
        if (bucket < 0 || bucket > 63 || (tpb != 32 && tpb != 64 && tpb != 128 && tpb != 256 && tpb != 512 && tpb != 1024) ||
            capm < 0 || capm > 1024)
            return fail(SNOWB_ERR_INVALID, "autotune table: value out of range in '" + line + "'");
        t.push_back(TuneEntry{name, bucket, tpb, capm});
    }
    g_tune = t;
    ++g_tune_gen;
    return SNOWB_OK;
}

int snowb_autotune_reset(void)
{
    g_tune.clear();
    ++g_tune_gen;
    return SNOWB_OK;
}

// ------------------------------------------------------------------ point-sprite rendering
static int render_cam(const snowb_camera* cam, RenderCam& c)
{
    if (!cam) return fail(SNOWB_ERR_INVALID, "null camera");
    if (cam->width == 0 || cam->height == 0 || (uint64_t)cam->width * cam->height > (1ull << 28))
        return fail(SNOWB_ERR_INVALID, "image size out of range");
    std::memcpy(c.V, cam->view, sizeof(c.V));
    std::memcpy(c.Pm, cam->projection, sizeof(c.Pm));
    std::memcpy(c.cam, cam->camera_pos, sizeof(c.cam));
    std::memcpy(c.light, cam->light_pos, sizeof(c.light));
    c.point_size = cam->point_size;
    c.W = cam->width;
    c.H = cam->height;
    return SNOWB_OK;
}

int snowb_render_clear(const snowb_camera* cam, float* rgba, unsigned long long* zbuf)
{
    RenderCam c;
    TRY(render_cam(cam, c));
    if (!rgba || !zbuf) return fail(SNOWB_ERR_INVALID, "null image");
    LAUNCH(kr_clear, (uint64_t)c.W * c.H, 256, c.W * c.H, zbuf, rgba, make_float4(0.f, 0.f, 0.f, 0.f));
    return SNOWB_OK;
}

int snowb_render_clear_colour(const snowb_camera* cam, const float* clear_rgba, float* rgba, unsigned long long* zbuf)
{
    RenderCam c;
    TRY(render_cam(cam, c));
    if (!rgba || !zbuf || !clear_rgba) return fail(SNOWB_ERR_INVALID, "null pointer");
    LAUNCH(kr_clear, (uint64_t)c.W * c.H, 256, c.W * c.H, zbuf, rgba,
           make_float4(clear_rgba[0], clear_rgba[1], clear_rgba[2], clear_rgba[3]));
    return SNOWB_OK;
}

int snowb_render_points(const snowb_particle_data* set, uint32_t n, const snowb_camera* cam,
                        const snowb_point_colour* colour, uint32_t draw, float* rgba, unsigned long long* zbuf)
{
    RenderCam c;
    TRY(render_cam(cam, c));
    if (!set || !colour || !rgba || !zbuf) return fail(SNOWB_ERR_INVALID, "null pointer");
    if (draw > 31) return fail(SNOWB_ERR_INVALID, "at most 32 draws between clears");
    if (n >= (1u << 27)) return fail(SNOWB_ERR_INVALID, "more than 2^27 particles in one draw");
    if (n == 0) return SNOWB_OK;
    RenderColour rc;
    std::memcpy(rc.rgb, colour->rgb, sizeof(rc.rgb));
    rc.temp = colour->use_temperature ? 1 : 0;
    std::memcpy(rc.cool, colour->coolest_rgb, sizeof(rc.cool));
    std::memcpy(rc.hot, colour->hottest_rgb, sizeof(rc.hot));
    rc.t_cool = colour->coolest_T;
    rc.t_hot = colour->hottest_T;
    const float* T = rc.temp ? set->T : nullptr;
    LAUNCH(kr_depth, n, 128, c, rc, set->positions, T, n, draw, zbuf);
    LAUNCH(kr_shade, (uint64_t)c.W * c.H, 256, c, rc, set->positions, T, draw, zbuf, rgba);
    return SNOWB_OK;
}

// ------------------------------------------------------------------ screen-space fluid
// 4x4 column-major product A * B in glm's order: column c = ((A0 b0 + A1 b1) + A2 b2) + A3 b3
static void mat_mul(const float* A, const float* B, float* out)
{
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r)
            out[c * 4 + r] = ((A[r] * B[c * 4] + A[4 + r] * B[c * 4 + 1]) + A[8 + r] * B[c * 4 + 2]) +
                             A[12 + r] * B[c * 4 + 3];
}
// inverse of a column-major 4x4 (Gauss-Jordan with partial pivoting in double, rounded to
// float); false when singular
static bool mat_inv(const float* M, float* out)
{
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            a[r][c] = M[c * 4 + r];
            a[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    for (int k = 0; k < 4; ++k) {
        int piv = k;
        for (int r = k + 1; r < 4; ++r)
            if (std::fabs(a[r][k]) > std::fabs(a[piv][k])) piv = r;
        if (a[piv][k] == 0.0) return false;
        if (piv != k)
            for (int c = 0; c < 8; ++c) std::swap(a[k][c], a[piv][c]);
        const double d = a[k][k];
        for (int c = 0; c < 8; ++c) a[k][c] /= d;
        for (int r = 0; r < 4; ++r) {
            if (r == k) continue;
            const double f = a[r][k];
            if (f != 0.0)
                for (int c = 0; c < 8; ++c) a[r][c] -= f * a[k][c];
        }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) out[c * 4 + r] = (float)a[r][4 + c];
    return true;
}
static int ssfr_cam(const snowb_camera* cam, const snowb_ssfr* ss, SsfrCam& c)
{
    RenderCam rc;
    TRY(render_cam(cam, rc));
    std::memcpy(c.V, cam->view, sizeof(c.V));
    std::memcpy(c.P, cam->projection, sizeof(c.P));
    mat_mul(c.P, c.V, c.PV);
    if (!mat_inv(c.P, c.Pinv) || !mat_inv(c.V, c.Vinv)) return fail(SNOWB_ERR_INVALID, "singular camera matrix");
    c.point_size = cam->point_size;
    c.radius = ss ? ss->sphere_radius : 0.f;
    c.W = cam->width;
    c.H = cam->height;
    return SNOWB_OK;
}
static int ssfr_shade(const snowb_ssfr* ss, SsfrShade& s)
{
    if (!ss) return fail(SNOWB_ERR_INVALID, "null ssfr parameters");
    if (!(ss->filter_radius >= 0.f && ss->filter_radius <= 256.f)) return fail(SNOWB_ERR_INVALID, "filter radius out of 0..256");
    s.filter_radius = ss->filter_radius;
    s.blur_scale = ss->blur_scale;
    s.falloff = ss->blur_depth_falloff;
    std::memcpy(s.light, ss->light_color, sizeof(s.light));
    std::memcpy(s.clear, ss->clear_color, sizeof(s.clear));
    return SNOWB_OK;
}

int snowb_ssfr_matrices(const snowb_camera* cam, float* out80)
{
    SsfrCam c;
    TRY(ssfr_cam(cam, nullptr, c));
    if (!out80) return fail(SNOWB_ERR_INVALID, "null output");
    std::memcpy(out80, c.PV, 64);
    std::memcpy(out80 + 16, c.V, 64);
    std::memcpy(out80 + 32, c.P, 64);
    std::memcpy(out80 + 48, c.Pinv, 64);
    std::memcpy(out80 + 64, c.Vinv, 64);
    return SNOWB_OK;
}

int snowb_ssfr_clear(const snowb_camera* cam, float* depth, unsigned long long* thick)
{
    SsfrCam c;
    TRY(ssfr_cam(cam, nullptr, c));
    if (!depth && !thick) return SNOWB_OK;
    LAUNCH(ks_fill, (uint64_t)c.W * c.H, 256, c.W * c.H, reinterpret_cast<uint32_t*>(depth), 0x3f800000u, thick);
    return SNOWB_OK;
}

int snowb_ssfr_sphere_depth(const snowb_particle_data* set, uint32_t n, const snowb_camera* cam, const snowb_ssfr* ssfr,
                            float* depth)
{
    SsfrCam c;
    TRY(ssfr_cam(cam, ssfr, c));
    if (!set || !ssfr || !depth) return fail(SNOWB_ERR_INVALID, "null pointer");
    if (n == 0) return SNOWB_OK;
    LAUNCH(ks_sphere_depth, n, 128, c, set->positions, n, reinterpret_cast<uint32_t*>(depth));
    return SNOWB_OK;
}

int snowb_ssfr_thickness(const snowb_particle_data* set, uint32_t n, const snowb_camera* cam, unsigned long long* thick)
{
    SsfrCam c;
    TRY(ssfr_cam(cam, nullptr, c));
    if (!set || !thick) return fail(SNOWB_ERR_INVALID, "null pointer");
    if (n == 0) return SNOWB_OK;
    LAUNCH(ks_thickness, n, 128, c, set->positions, n, thick);
    return SNOWB_OK;
}

int snowb_ssfr_smooth(const snowb_camera* cam, const snowb_ssfr* ssfr, const float* depth, float* tmp, float* out)
{
    SsfrCam c;
    SsfrShade s;
    TRY(ssfr_cam(cam, ssfr, c));
    TRY(ssfr_shade(ssfr, s));
    if (!depth || !tmp || !out || tmp == depth || tmp == out) return fail(SNOWB_ERR_INVALID, "bad buffers");
    const uint64_t np = (uint64_t)c.W * c.H;
    LAUNCH(ks_bilateral, np, 256, c, s, depth, tmp, 0);
    LAUNCH(ks_bilateral, np, 256, c, s, tmp, out, 1);
    return SNOWB_OK;
}

int snowb_ssfr_compose(const snowb_camera* cam, const snowb_ssfr* ssfr, const float* depth,
                       const unsigned long long* thick, const float* scene_rgba, const float* scene_depth, float* rgba)
{
    SsfrCam c;
    SsfrShade s;
    TRY(ssfr_cam(cam, ssfr, c));
    TRY(ssfr_shade(ssfr, s));
    if (!depth || !thick || !scene_rgba || !scene_depth || !rgba) return fail(SNOWB_ERR_INVALID, "null pointer");
    LAUNCH(ks_compose, (uint64_t)c.W * c.H, 256, c, s, depth, thick, scene_rgba, scene_depth, rgba);
    return SNOWB_OK;
}

int snowb_ssfr_workspace_bytes(const snowb_camera* cam, uint64_t* bytes)
{
    RenderCam c;
    TRY(render_cam(cam, c));
    if (!bytes) return fail(SNOWB_ERR_INVALID, "null output");
    *bytes = (uint64_t)c.W * c.H * 48u;
    return SNOWB_OK;
}

int snowb_render_fluid(const snowb_particle_data* sph, uint32_t n_sph, const snowb_particle_data* dem, uint32_t n_dem,
                       const snowb_camera* cam, const snowb_point_colour* snow_colour, const snowb_ssfr* ssfr,
                       void* workspace, float* rgba)
{
    if (!sph || !dem || !snow_colour || !ssfr || !workspace || !rgba) return fail(SNOWB_ERR_INVALID, "null pointer");
    if ((reinterpret_cast<uintptr_t>(workspace) & 15u) != 0) return fail(SNOWB_ERR_INVALID, "workspace not 16-byte aligned");
    RenderCam rc;
    TRY(render_cam(cam, rc));
    const uint64_t np = (uint64_t)rc.W * rc.H;
    char* w = static_cast<char*>(workspace);
    unsigned long long* zbuf = reinterpret_cast<unsigned long long*>(w);
    unsigned long long* thick = zbuf + np;
    float* scene = reinterpret_cast<float*>(thick + np);
    float* scene_depth = scene + 4 * np;
    float* fdepth = scene_depth + np;
    float* tmp = fdepth + np;
    float* smooth = tmp + np;
    // scene: the snow as point sprites over the clear colour, and its sphere depth
    TRY(snowb_render_clear_colour(cam, ssfr->clear_color, scene, zbuf));
    TRY(snowb_render_points(dem, n_dem, cam, snow_colour, 0, scene, zbuf));
    TRY(snowb_ssfr_clear(cam, scene_depth, thick));
    TRY(snowb_ssfr_clear(cam, fdepth, nullptr));
    TRY(snowb_ssfr_sphere_depth(dem, n_dem, cam, ssfr, scene_depth));
    // water: sphere depth, smoothed, thickness, composite
    TRY(snowb_ssfr_sphere_depth(sph, n_sph, cam, ssfr, fdepth));
    TRY(snowb_ssfr_smooth(cam, ssfr, fdepth, tmp, smooth));
    TRY(snowb_ssfr_thickness(sph, n_sph, cam, thick));
    TRY(snowb_ssfr_compose(cam, ssfr, smooth, thick, scene, scene_depth, rgba));
    return SNOWB_OK;
}

// ------------------------------------------------------------------ .bgeo export
int snowb_write_bgeo_host(const float* positions, uint32_t n, const char* path, const float* rgb, float pscale,
                          int label, int float_label)
{
    if (!path || !rgb || (n && !positions)) return fail(SNOWB_ERR_INVALID, "null pointer");
    std::string err;
    if (bgeo_write(path, positions, n, rgb, pscale, label, float_label, err) != 0) return fail(SNOWB_ERR_INVALID, err);
    return SNOWB_OK;
}

int snowb_export_bgeo(const snowb_particle_data* set, uint32_t n, const char* path, const float* rgb, float pscale,
                      int label, int float_label)
{
    if (!set || !path || !rgb) return fail(SNOWB_ERR_INVALID, "null pointer");
    float* h = nullptr;
    if (n) {
        CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&h), (size_t)n * 12));
        cudaError_t e = cudaMemcpyAsync(h, set->positions, (size_t)n * 12, cudaMemcpyDeviceToHost, g_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
        if (e != cudaSuccess) { cudaFreeHost(h); return fail(SNOWB_ERR_CUDA, cudaGetErrorString(e)); }
    }
    std::string err;
    const int rc = bgeo_write(path, h, n, rgb, pscale, label, float_label, err);
    if (h) cudaFreeHost(h);
    if (rc != 0) return fail(SNOWB_ERR_INVALID, err);
    return SNOWB_OK;
}

int snowb_export_bgeo_async(const snowb_particle_data* set, uint32_t n, const char* path, const float* rgb,
                            float pscale, int label, int float_label)
{
    if (!set || !path || !rgb) return fail(SNOWB_ERR_INVALID, "null pointer");
    ExportJob* job = new ExportJob();
    if (n) {
        cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&job->staging), (size_t)n * 12);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&job->ev, cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(job->staging, set->positions, (size_t)n * 12, cudaMemcpyDeviceToHost, g_stream);
        if (e == cudaSuccess) e = cudaEventRecord(job->ev, g_stream);
        if (e != cudaSuccess) {
            if (job->staging) cudaFreeHost(job->staging);
            if (job->ev) cudaEventDestroy(job->ev);
            delete job;
            return fail(SNOWB_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    const std::string file(path);
    const float col[3] = {rgb[0], rgb[1], rgb[2]};
    job->th = std::thread([job, file, n, col, pscale, label, float_label]() {
        if (job->ev && cudaEventSynchronize(job->ev) != cudaSuccess) { job->rc = -1; job->err = "copy failed"; return; }
        job->rc = bgeo_write(file.c_str(), job->staging, n, col, pscale, label, float_label, job->err);
    });
    g_exports.push_back(job);
    return SNOWB_OK;
}

int snowb_export_wait(void)
{
    int rc = SNOWB_OK;
    std::string err;
    for (ExportJob* job : g_exports) {
        job->th.join();
        if (job->rc != 0 && rc == SNOWB_OK) { rc = SNOWB_ERR_INVALID; err = job->err; }
        if (job->staging) cudaFreeHost(job->staging);
        if (job->ev) cudaEventDestroy(job->ev);
        delete job;
    }
    g_exports.clear();
    if (rc != SNOWB_OK) return fail(rc, err);
    return SNOWB_OK;
}

// ------------------------------------------------------------------ adjoint
int snowb_adjoint_begin(void)
{
    if (g_tape.recording) return fail(SNOWB_ERR_INVALID, "adjoint: already recording");
    g_tape.recording = true;
    g_tape.used = 0;
    if (g_tape.viol) CUDA_TRY(cudaMemsetAsync(g_tape.viol, 0, sizeof(uint32_t), g_stream));
    return SNOWB_OK;
}

int snowb_adjoint_end(uint32_t* substeps)
{
    if (!g_tape.recording) return fail(SNOWB_ERR_INVALID, "adjoint: not recording");
    g_tape.recording = false;
    if (substeps) *substeps = (uint32_t)g_tape.used;
    return SNOWB_OK;
}

int snowb_adjoint_backward(snowb_adjoint_io* io)
{
    return adjoint_backward(io);
}

int snowb_adjoint_release(void)
{
    g_tape.recording = false;
    tape_free_steps();
    if (g_tape.viol) cudaFree(g_tape.viol);
    g_tape = Tape();
    adj_free();
    return SNOWB_OK;
}

int snowb_read_sizes(uint32_t* sph_size, uint32_t* dem_size)
{
    if (!g_ctx.S) return fail(SNOWB_ERR_INVALID, "no step has run");
    CUDA_TRY(cudaMemcpyAsync(g_ctx.S_host, g_ctx.S, sizeof(DevState), cudaMemcpyDeviceToHost, g_stream));
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    if (sph_size) *sph_size = g_ctx.S_host->n_sph;
    if (dem_size) *dem_size = g_ctx.S_host->n_dem;
    return SNOWB_OK;
}

int snowb_device_counters(uint32_t* out, int n)
{
    if (!out || n <= 0) return fail(SNOWB_ERR_INVALID, "null pointer");
    if (!g_ctx.S) return fail(SNOWB_ERR_INVALID, "no step has run");
    CUDA_TRY(cudaMemcpyAsync(g_ctx.S_host, g_ctx.S, sizeof(DevState), cudaMemcpyDeviceToHost, g_stream));
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    const uint32_t* src = reinterpret_cast<const uint32_t*>(g_ctx.S_host);
    const int m = (int)(sizeof(DevState) / sizeof(uint32_t));
    for (int k = 0; k < n; ++k) out[k] = k < m ? src[k] : 0u;
    return SNOWB_OK;
}

int snowb_set_quirks(int mode)
{
    if (mode != SNOWB_QUIRKS_REFERENCE && mode != SNOWB_QUIRKS_FIXED) return fail(SNOWB_ERR_INVALID, "unknown quirk mode");
    g_quirks = mode;
    return SNOWB_OK;
}

int snowb_set_stream(void* stream)
{
    g_stream = reinterpret_cast<cudaStream_t>(stream);
    return SNOWB_OK;
}

int snowb_synchronize(void)
{
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    return SNOWB_OK;
}

int snowb_energy_momentum(const snowb_particle_data* sph, uint32_t ns, const snowb_particle_data* dem, uint32_t nd,
                          double out[4])
{
    TRY(check_params());
    if (!sph || !dem || !out) return fail(SNOWB_ERR_INVALID, "null pointer");
    TRY(ensure_ctx(g_ctx.cap ? g_ctx.cap : 1, g_ctx.bcap ? g_ctx.bcap : 1, g_P.ncells));
    const int nb = 512;
    KL(k_energy_partial, nb, 256, *sph, ns, *dem, nd, (double)g_sim.C_water, (double)g_sim.C_snow, g_ctx.epart);
    KL(k_energy_final, 1, 32, g_ctx.epart, nb, g_ctx.eout);
    CUDA_TRY(cudaMemcpyAsync(out, g_ctx.eout, 4 * sizeof(double), cudaMemcpyDeviceToHost, g_stream));
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    return SNOWB_OK;
}

int snowb_launch_count(uint64_t* count)
{
    if (!count) return fail(SNOWB_ERR_INVALID, "null pointer");
    *count = g_launches;
    return SNOWB_OK;
}

int snowb_profile_begin(void)
{
    g_prof = true;
    g_prof_used = 0;
    g_graph.prof_replayed = false;
    g_graph.prof_pairs = 0;
    g_acc_name.clear(); g_acc_count.clear(); g_acc_ms.clear();
    return SNOWB_OK;
}

int snowb_profile_end(char* out, size_t cap)
{
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    if (g_graph.stream) CUDA_TRY(cudaStreamSynchronize(g_graph.stream));
    // launches issued directly (not through a graph) are still pending in the pool
    const size_t done = g_graph.prof_replayed ? g_graph.prof_pairs : 0;
    if (!g_graph.prof_replayed || g_prof_used > done)
        if (prof_accumulate(done, g_prof_used) != 0) return fail(SNOWB_ERR_CUDA, "profile events");
    g_prof = false;
    g_prof_used = 0;
    g_graph.prof_replayed = false;
    g_graph.prof_pairs = 0;
    graph_reset(true);   // profiling graphs carry event nodes; the plain ones stay cached
    std::string txt;
    for (size_t i = 0; i < g_acc_name.size(); ++i)
        txt += g_acc_name[i] + " " + std::to_string(g_acc_count[i]) + " " + std::to_string(g_acc_ms[i]) + "\n";
    if (out && cap) {
        size_t n = txt.size() < cap - 1 ? txt.size() : cap - 1;
        std::memcpy(out, txt.data(), n);
        out[n] = 0;
        if (txt.size() >= cap) return fail(SNOWB_ERR_INVALID, "profile buffer too small");
    }
    return SNOWB_OK;
}

int snowb_profile_timeline(char* out, size_t cap)
{
    if (!out || cap == 0) return fail(SNOWB_ERR_INVALID, "null buffer");
    if (!g_prof) return fail(SNOWB_ERR_INVALID, "profiling is off");
    CUDA_TRY(cudaStreamSynchronize(g_stream));
    if (g_graph.stream) CUDA_TRY(cudaStreamSynchronize(g_graph.stream));
    // a graph replay re-records its events: they hold the last replay's times
    const size_t n = g_graph.prof_replayed ? g_graph.prof_pairs : g_prof_used;
    const size_t first = g_graph.prof_replayed ? 0 : (g_prof_last_substep < n ? g_prof_last_substep : 0);
    std::string txt;
    for (size_t k = first; k < n; ++k) {
        float t0 = 0.f, t1 = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&t0, g_prof_pool[first].a, g_prof_pool[k].a));
        CUDA_TRY(cudaEventElapsedTime(&t1, g_prof_pool[first].a, g_prof_pool[k].b));
        char line[160];
        std::snprintf(line, sizeof line, "%s %.4f %.4f\n", g_prof_pool[k].name, t0, t1);
        txt += line;
    }
    const size_t m = txt.size() < cap - 1 ? txt.size() : cap - 1;
    std::memcpy(out, txt.data(), m);
    out[m] = 0;
    if (txt.size() >= cap) return fail(SNOWB_ERR_INVALID, "timeline buffer too small");
    return SNOWB_OK;
}

int snowb_release(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    graph_free();
    free_ctx(g_ctx);
    tape_free_steps();
    adj_free();
    return SNOWB_OK;
}

}  // extern "C"
