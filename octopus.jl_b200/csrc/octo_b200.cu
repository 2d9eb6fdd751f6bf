// libocto_b200: host runtime and C ABI of the B200 strong-strong PIC collision backend.
//
// One collide is: device slicing of both beams (one small readback of the slice table),
// a host-built collision-time wavefront schedule (slicing.jl:561-647) uploaded once, and
// per wavefront a fixed sequence of batched kernels -- bounds, on-device grid/Green-cache
// planning, Green spectra, luminosity, fixed-point deposition, the Hockney FFT convolution
// with the field derivative fused into the inverse pass, and the synchro-beam kick.  The
// luminosity parts and status are read back once at the end.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/octo_b200.h"
#include "k_gauss.cuh"
#include "k_line.cuh"
#include "k_moments.cuh"
#include "k_misc.cuh"
#include "k_learned.cuh"
#include "k_pic.cuh"
#include "k_replay.cuh"
#include "k_slicing.cuh"
#include "k_umma.cuh"
#include "noalloc_cache.h"

using namespace octo;

namespace {

struct CudaFail {
    std::string msg;
};
struct OctoFail {
    int code;
    std::string msg;
};

#define CK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) throw CudaFail{std::string(#call) + ": " + cudaGetErrorString(e_)};         \
    } while (0)

// Launch a kernel of the collide path with programmatic stream serialization: it may begin launching
// while its predecessor in the stream drains, and its first statement (pdl_wait) holds it until that
// grid has completed.  A predecessor that is a copy, a memset or an event wait stays a full dependency.
template <class... P, class... A>
void launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A &&...args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

// Inverse error function: Winitzki start, Halley steps on erf / erfc.  Used only for the
// :normal_quantile slice quantiles sqrt(2)*erfinv(2s/ns-1) (slicing.jl:425).
double erfinv_host(double x) {
    if (std::isnan(x) || x < -1.0 || x > 1.0) return NAN;
    if (x == 1.0) return INFINITY;
    if (x == -1.0) return -INFINITY;
    if (x == 0.0) return x;
    double ax = std::fabs(x);
    const double a = 0.147, pi = 3.141592653589793;
    double ln = std::log1p(-ax * ax);
    double t1 = 2.0 / (pi * a) + ln / 2.0;
    double y = std::sqrt(std::sqrt(t1 * t1 - ln / a) - t1);
    const double c = 1.1283791670955126;  // 2/sqrt(pi)
    for (int it = 0; it < 4; ++it) {
        double f = (ax < 0.5) ? (std::erf(y) - ax) : ((1.0 - ax) - std::erfc(y));
        double step = f / (c * std::exp(-y * y));
        y = y - step / (1.0 + y * step);
    }
    return x < 0 ? -y : y;
}

struct OrderEntry {
    double t;
    int i, j;
};

// slicing.jl:561-568 (stable sort by collision time -(c1+c2)/2)
std::vector<OrderEntry> collision_order(const double *c1, int ns1, const double *c2, int ns2) {
    std::vector<OrderEntry> o;
    o.reserve((size_t)ns1 * ns2);
    for (int i = 0; i < ns1; ++i)
        for (int j = 0; j < ns2; ++j) o.push_back({-(c1[i] + c2[j]) / 2, i + 1, j + 1});
    std::stable_sort(o.begin(), o.end(), [](const OrderEntry &a, const OrderEntry &b) { return a.t < b.t; });
    return o;
}

// slicing.jl:601-647 : greedy ready, conflict-free batches.
std::vector<std::vector<OrderEntry>> pair_batches(const std::vector<OrderEntry> &pairs, int ns1, int ns2) {
    std::vector<std::vector<OrderEntry>> batches;
    std::vector<std::vector<int>> by_i(ns1 + 1), by_j(ns2 + 1);
    for (size_t k = 0; k < pairs.size(); ++k) {
        by_i[pairs[k].i].push_back((int)k);
        by_j[pairs[k].j].push_back((int)k);
    }
    std::vector<size_t> next_i(ns1 + 1, 0), next_j(ns2 + 1, 0);
    std::vector<char> done(pairs.size(), 0);
    size_t remaining = pairs.size();
    while (remaining > 0) {
        std::vector<OrderEntry> cur;
        std::vector<char> used_i(ns1 + 1, 0), used_j(ns2 + 1, 0);
        for (size_t k = 0; k < pairs.size(); ++k) {
            if (done[k]) continue;
            const OrderEntry &p = pairs[k];
            if (used_i[p.i] || used_j[p.j]) continue;
            bool ri = next_i[p.i] < by_i[p.i].size() && by_i[p.i][next_i[p.i]] == (int)k;
            bool rj = next_j[p.j] < by_j[p.j].size() && by_j[p.j][next_j[p.j]] == (int)k;
            if (ri && rj) {
                cur.push_back(p);
                used_i[p.i] = 1; used_j[p.j] = 1; done[k] = 1;
                next_i[p.i]++; next_j[p.j]++;
                --remaining;
            }
        }
        if (cur.empty()) throw OctoFail{OCTO_ERR_ARG, "internal collision scheduler error: no ready slice pair"};
        batches.push_back(cur);
    }
    return batches;
}

// Run f with the particle real type of the context: double (plain form) or float (precision form).
template <class F>
void with_real(bool fp32, F f) {
    if (fp32) f(float(0));
    else f(double(0));
}

// Bumped whenever a workspace buffer is (re)allocated or freed: a captured collide graph holds the buffers'
// addresses and is replayed only while the epoch it was built at is current.
static std::atomic<long long> g_alloc_epoch{0};

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    void ensure(size_t m) {
        if (m <= n) return;
        g_alloc_epoch.fetch_add(1);
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        CK(cudaMalloc(&p, std::max<size_t>(m, 1) * sizeof(T)));
        n = m;
    }
    void release() {
        if (p) { g_alloc_epoch.fetch_add(1); cudaFree(p); }
        p = nullptr;
        n = 0;
    }
};

template <class T>
struct PinBuf {
    T *p = nullptr;
    size_t n = 0;
    void ensure(size_t m) {
        if (m <= n) return;
        g_alloc_epoch.fetch_add(1);
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        CK(cudaMallocHost(&p, std::max<size_t>(m, 1) * sizeof(T)));
        n = m;
    }
    void release() {
        if (p) { g_alloc_epoch.fetch_add(1); cudaFreeHost(p); }
        p = nullptr;
        n = 0;
    }
};

constexpr int kAlign = 32;           // slice start alignment (elements)
constexpr long long kChunk = 8192;   // particles per slicing block

struct BeamWS {
    DevBuf<double> s[6];  // slice-sorted coordinates (sized in doubles; float elements in the precision form)
    DevBuf<double> t[6];  // the spatially ordered copy (plain PIC), swapped into s once written
    DevBuf<unsigned long long> box;  // spatial order: slice boxes
    DevBuf<int> cursor;              // spatial order: bin counts / cursors
    DevBuf<long long> hist;          // :equal_area histogram
    DevBuf<unsigned long long> rkey, rkey_sorted;  // :equal_count rank sort
    DevBuf<int> rval, rval_sorted;
    DevBuf<char> sort_tmp;
    DevBuf<int> dest;  // caller index -> slice-sorted position
    DevBuf<SliceInfo> info;
    DevBuf<double> lane_sum, lane_min, lane_max, lanes, q;
    DevBuf<int> counts;
    DevBuf<long long> blockoff;
    long long total = 0;
    void release() {
        for (auto &b : s) b.release();
        for (auto &b : t) b.release();
        box.release(); cursor.release(); hist.release(); rkey.release(); rkey_sorted.release(); rval.release();
        rval_sorted.release(); sort_tmp.release();
        dest.release(); info.release(); lane_sum.release(); lane_min.release(); lane_max.release();
        lanes.release(); q.release(); counts.release(); blockoff.release();
    }
};

}  // namespace

// ---------------------------------------------------------------- tensor-core GEMM launch
namespace octo {
namespace nn {
// Picks the tile width from N (32, 64, 128 or 256 columns of fp32 accumulator in TMEM).
void launch_gemm(const GemmArgs &g, int splits, cudaStream_t st) {
    const int bn = g.N <= 32 ? 32 : (g.N <= 64 ? 64 : (g.N <= 128 ? 128 : 256));
    const int tiles_m = (g.M + kBM - 1) / kBM, cols = ((g.N + bn - 1) / bn) * splits;
    const size_t smem = umma_smem_bytes(bn);
    static std::atomic<int> resident[4] = {{0}, {0}, {0}, {0}};  // CTAs per SM of each tile width (one arch)
    const int slot = bn == 32 ? 0 : (bn == 64 ? 1 : (bn == 128 ? 2 : 3));
    auto go = [&](void (*kernel)(const GemmArgs)) {
        CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // all of the unified L1 / shared array as shared memory, so two CTAs fit on an SM
        CK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        // persistent CTAs: as many as are resident at once, spread over the (n, split) columns
        int dev = 0, sms = 0, per_sm = resident[slot].load();
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (per_sm == 0) {
            // shared memory decides: the kernel's launch bounds guarantee two CTAs' registers, and each CTA
            // holds its stages, about 1 KB of static shared memory and the 1 KB the driver reserves
            int sm_bytes = 0;
            CK(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
            per_sm = std::max(1, std::min(2, sm_bytes / (int)(smem + 2048)));
            resident[slot].store(per_sm);
        }
        const int slots = std::max(1, sms * std::max(1, per_sm));
        const int gx = std::max(1, std::min(tiles_m, (slots + cols - 1) / cols));
        const dim3 grid((unsigned)gx, (unsigned)((g.N + bn - 1) / bn), (unsigned)splits);
        launch_pdl(kernel, grid, kGemmThreads, smem, st, g);
    };
    if (bn == 32) go(k_umma_gemm<32>);
    else if (bn == 64) go(k_umma_gemm<64>);
    else if (bn == 128) go(k_umma_gemm<128>);
    else go(k_umma_gemm<256>);
}
}  // namespace nn
}  // namespace octo

#include "cnn_host.cuh"

struct octo_cnn {
    nn::Cnn net;
    std::string err;
};

struct octo_ctx {
    int device = 0;
    int num_sms = 148;  // the device's SM count (block-count policies)
    // launch shape (octo_pic_autotune): the deposit launches at least dep_waves waves of the SMs per front,
    // the kick sizes its blocks to fill kick_slots times the resident block slots
    int dep_waves = 1, kick_slots = 1;
    // plain PIC: group each slice's particles by transverse position in the working copy (octo_set_particle_order)
    int spatial = 0;
    octo_pic_options opt{};
    std::vector<double> pos[2];
    DevOptions dopt{};
    std::string err;
    int ns[2] = {0, 0};
    BeamWS bw[2];
    DevBuf<double2> tw_x, tw_y;  // FP64 twiddles (Green spectra; plain-form convolution)
    DevBuf<float2> twf_x, twf_y; // FP32 twiddles (precision-form convolution)
    int fp32 = 0;                // precision form: float particles, field planes and FFTs
    DevBuf<Task> tasks;
    DevBuf<Plane> planes;
    DevBuf<LumJob> lumjobs;
    DevBuf<TaskGeom> geom;
    DevBuf<int2> blockmap;
    DevBuf<FirstLum> first_lum;
    DevBuf<unsigned> lum_tick;
    DevBuf<CacheEntry> cache;
    DevBuf<NodeMesh> nodes;
    DevBuf<LumGeom> lumgeom;
    DevBuf<unsigned long long> bnd, lumb, nodebox_s, nodebox_f;
    DevBuf<int> nanflag, nodenan;
    DevBuf<DevStatus> status;
    DevBuf<double2> ghat;
    DevBuf<long long> qgrid, lq;
    DevBuf<double2> spec;
    DevBuf<double2> fields;
    DevBuf<double> lum_parts, lum_partial, node_ref, stats, partial;
    DevBuf<HybridTask> hyb;            // Gaussian-subtracted hybrid state per task
    DevBuf<double> hmom, hprof, hsum;  // its moment partials, node profiles and profile sums
    DevBuf<double> esum;               // grid_extent = :sigma: per-block sums of the drifted offsets
    DevBuf<unsigned long long> ubox;   // :source_slice: union box per (direction, source slice)
    DevBuf<int> uflag;                 // ... and its non-finite flags
    DevBuf<long long> slr;             // ... both beams' slice ranges (start, count)
    DevBuf<double> mom_partial, mom_means;  // beam moment rows: block partials and the means
    // soft-Gaussian solver: slices, their moments, kick tasks, block maps, partial sums
    DevBuf<GSlice> g_slices;
    DevBuf<GMoments> g_mom;
    DevBuf<GTask> g_tasks;
    DevBuf<int2> g_bmap;
    DevBuf<int> g_index;
    DevBuf<double> g_partial, g_lum_partial;
    DevBuf<unsigned long long> qtot;   // per-plane total fixed-point charge
    DevBuf<double *> soa_ptrs;
    PinBuf<char> stage;
    PinBuf<double> h_lum;
    PinBuf<DevStatus> h_status;
    PinBuf<double> h_noderef;
    PinBuf<SliceInfo> h_slices;
    long long gstride = 0;
    int nslots = 0;
    int cache_ready = 0;
    std::vector<int> trace_i, trace_j;
    std::vector<double> trace_lum;
    long long last_launches = 0;
    // per-phase device timing (octo_set_timing): event pairs recorded around each launch group
    // second stream of the collide: each front's luminosity work overlaps its field solve (forked after the
    // front's bounds, joined before its kick)
    cudaStream_t lum_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int timing = 0;
    unsigned timing_mask = ~0u;  // phases timed when timing is on (octo_set_timing_phases)
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_marks;
    double phase_ms[OCTO_NPHASES] = {0};
    long long phase_launches[OCTO_NPHASES] = {0};
    double phase_bytes[OCTO_NPHASES] = {0};
    // learned field correction (octo_set_field_correction): the attached network (an octo_cnn), the scale of
    // its outputs, the tolerance of the per-plane correction estimate, the untouched border, and the count of
    // planes over tolerance in the last collide
    octo_cnn *cnn = nullptr;
    float cnn_scale = 1.f, cnn_tol = INFINITY;
    int cnn_edge = 2;
    DevBuf<int> cnn_flags;
    DevBuf<long long> cnn_q;  // total fixed-point charge per plane of the front
    PinBuf<int> h_cnn_flags;
    // octo_capture_charge_plane: one field-solve charge grid of the next collide, copied right after its
    // deposit, with the mesh it was deposited on
    int cap_armed = 0, cap_taken = 0, cap_i = 0, cap_j = 0, cap_dir = 0, cap_kind = 0, cap_bits = 0;
    DevBuf<long long> cap_q;
    DevBuf<Grid> cap_grid;  // [0] the source mesh the plane was deposited on, [1] the field mesh of its task
    // captured collide graph (octo_set_collide_graph): captured after two ordinary collides with the same
    // schedule, replayed behind its device guard (k_replay_check) while the buffers and the key hold
    struct Replay {
        int enabled = 1;            // octo_set_collide_graph
        int valid = 0;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        long long epoch = -1;       // g_alloc_epoch at capture
        // what the captured kernels hold besides the schedule tables
        const void *beam[2][6] = {};
        long long n[2] = {0, 0};
        double kbb1 = 0, kbb2 = 0, klum = 0;
        int compute_lum = -1, dep_waves = 0, kick_slots = 0, spatial = 0;
        // the host side of the captured collide, for finish()
        std::vector<OrderEntry> order;
        std::vector<std::vector<OrderEntry>> batches;
        std::vector<char> ran;
        std::vector<Task> tasks;
        int ntasks = 0, npairs_total = 0;
        long long body_launches = 0;
        std::vector<int> pos_of;          // pair index (i-1)*ns2 + (j-1) -> its position in the captured order
        std::vector<long long> sig;       // schedule of the captured collide (k_replay_check's layout)
        std::vector<long long> last_sig;  // schedule of the last ordinary collide
        long long builds = 0, replays = 0, declined = 0, failures = 0;
    } rp;
    DevBuf<long long> rp_sig;
    DevBuf<FrontKick> rp_fronts;
    DevBuf<int> rp_ok;
    PinBuf<int> h_rp_ok;
    cudaStream_t cap_stream = nullptr;  // the stream graphs are captured on (never the legacy default stream)
    int in_autotune = 0;
};

namespace {

bool replay_eligible(const octo_ctx *c);

// ---- per-phase timing: a scope records an event pair on the stream around a launch group
cudaEvent_t take_event(octo_ctx *c) {
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}
struct PhaseScope {
    octo_ctx *c;
    int phase;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    int nlaunch;
    double bytes;
    PhaseScope(octo_ctx *c_, int ph, cudaStream_t s, int nl = 1, double b = 0.0) : c(c_), phase(ph), st(s), nlaunch(nl), bytes(b) {
        if (c->timing && ((c->timing_mask >> phase) & 1u)) { a = take_event(c); CK(cudaEventRecord(a, st)); }
    }
    ~PhaseScope() {
        if (c->timing && a) {
            cudaEvent_t b = take_event(c);
            if (cudaEventRecord(b, st) == cudaSuccess) c->ev_marks.push_back({phase, {a, b}});
            c->phase_launches[phase] += nlaunch;
            c->phase_bytes[phase] += bytes;
        }
    }
};
void harvest_timing(octo_ctx *c) {
    if (!c->timing) return;
    for (auto &m : c->ev_marks) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, m.second.first, m.second.second) == cudaSuccess) c->phase_ms[m.first] += ms;
    }
    c->ev_marks.clear();
    c->ev_used = 0;
}

void set_error(octo_ctx *c, const std::string &m) { c->err = m; }

bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }
// Grid sizes the shared-memory FFTs take: 2^a or 3 * 2^a cells per axis (padded lines 2^(a+1), 3 * 2^(a+1)).
bool fft_size_ok(int v) { return is_pow2(v) || (v % 3 == 0 && is_pow2(v / 3)); }

int validate_options(const octo_pic_options &o, std::string &msg) {
    if (o.nx < 5 || o.ny < 5) { msg = "PICPoissonSolver grid must be at least (5, 5)"; return OCTO_ERR_ARG; }
    if (!fft_size_ok(o.nx) || !fft_size_ok(o.ny) || o.nx < 8 || o.ny % 8 != 0 || o.nx > 512 || o.ny > 512) {
        msg = "this backend's FFT needs grid dimensions of the form 2^a or 3*2^a in 8..512, ny a multiple of 8";
        return OCTO_ERR_UNSUPPORTED;
    }
    if (o.deposit_method != OCTO_CIC && o.deposit_method != OCTO_TSC) { msg = "deposit_method must be :CIC or :TSC"; return OCTO_ERR_ARG; }
    int lm = o.lum_deposit_method < 0 ? o.deposit_method : o.lum_deposit_method;
    if (lm != OCTO_CIC && lm != OCTO_TSC) { msg = "luminosity_deposit_method must resolve to :CIC or :TSC"; return OCTO_ERR_ARG; }
    int lnx = o.lum_nx > 0 ? o.lum_nx : o.nx, lny = o.lum_ny > 0 ? o.lum_ny : o.ny;
    if (lnx < 3 || lny < 3) { msg = "luminosity_grid dimensions must both be at least 3"; return OCTO_ERR_ARG; }
    if (o.green_type != OCTO_GREEN_INTEGRATED && o.green_type != OCTO_GREEN_STANDARD) {
        msg = "green_type must be :integrated or :standard on this backend (:lattice is an experimental CPU study kernel)";
        return OCTO_ERR_UNSUPPORTED;
    }
    if (o.green_cache != OCTO_CACHE_NONE && o.green_cache != OCTO_CACHE_SLICE_PAIR) { msg = "green_cache must be :none or :slice_pair"; return OCTO_ERR_ARG; }
    if (o.field_derivative != 2 && o.field_derivative != 4) { msg = "field_derivative must be :second or :fourth"; return OCTO_ERR_ARG; }
    if (o.slice_interpolation != 0 && o.slice_interpolation != 1) { msg = "slice_interpolation must be :linear or :quadratic"; return OCTO_ERR_ARG; }
    if (o.interaction_grid != OCTO_GRID_SLICE_PAIR && o.interaction_grid != OCTO_GRID_SOURCE_SLICE &&
        o.interaction_grid != OCTO_GRID_NODE) {
        msg = "interaction_grid must be :slice_pair, :source_slice or :node";
        return OCTO_ERR_ARG;
    }
    if (o.grid_extent != 0 && o.grid_extent != 1) { msg = "grid_extent must be :extrema or :sigma"; return OCTO_ERR_ARG; }
    if (o.grid_extent == 1 && o.interaction_grid != OCTO_GRID_SLICE_PAIR) {  // pic_cpu.jl:545-558
        msg = "grid_extent = :sigma is implemented for interaction_grid = :slice_pair only: :source_slice and :node "
              "size their meshes from union or per-node extrema and apply no extent estimator";
        return OCTO_ERR_UNSUPPORTED;
    }
    if (o.grid_extent == 1 && !(o.grid_extent_sigma > 0.0)) { msg = "grid_extent_sigma must be positive"; return OCTO_ERR_ARG; }
    if (o.interaction_grid == OCTO_GRID_NODE && o.slice_interpolation != 0) {
        msg = "slice_interpolation = :quadratic is not implemented for interaction_grid = :node";
        return OCTO_ERR_UNSUPPORTED;
    }
    if (!(o.green_min_ratio > 0.0 && o.green_min_ratio <= 1.0)) { msg = "slice_pair_green_min_ratio must be in (0, 1]"; return OCTO_ERR_ARG; }
    if (!(o.green_growth >= 0.0)) { msg = "slice_pair_green_growth must be non-negative"; return OCTO_ERR_ARG; }
    if (!(o.grid_quantize >= 0.0)) { msg = "grid_quantize must be non-negative"; return OCTO_ERR_ARG; }
    for (int b = 0; b < 2; ++b) {
        int ns = b == 0 ? o.nslices1 : o.nslices2;
        int m = b == 0 ? o.slicing_method1 : o.slicing_method2;
        if (ns < 1 || ns > kMaxSlices) { msg = "nslices must be in 1..64 on this backend"; return OCTO_ERR_ARG; }
        if (m < OCTO_SLICING_NORMAL_QUANTILE || m > OCTO_SLICING_EQUAL_WIDTH) {
            msg = "slicing method must be :normal_quantile, :specified, :equal_area, :equal_count or :equal_width";
            return OCTO_ERR_ARG;
        }
        const int res = b == 0 ? o.resolution1 : o.resolution2;
        if (res < 0) { msg = "slicing resolution must be positive"; return OCTO_ERR_ARG; }
        if (m == OCTO_SLICING_EQUAL_AREA && (long long)ns * (res > 0 ? res : 100) > 16384) {
            msg = "this backend's :equal_area histogram holds at most 16384 bins (nslices * resolution)";
            return OCTO_ERR_UNSUPPORTED;
        }
        const double *p = b == 0 ? o.positions1 : o.positions2;
        if (m == OCTO_SLICING_SPECIFIED && ns > 1 && !p) { msg = "specified slicing requires nslices-1 internal positions"; return OCTO_ERR_ARG; }
    }
    if (o.gaussian) {  // GaussianPICPoissonSolver (gaussian_pic.jl:94-110, 140-151)
        if (o.interaction_grid != OCTO_GRID_SLICE_PAIR || o.slice_interpolation != 0) {
            msg = "GaussianPICPoissonSolver uses linear slice interpolation on the :slice_pair grid; "
                  "interaction_grid and slice_interpolation must keep their defaults";
            return OCTO_ERR_UNSUPPORTED;
        }
        if (!(o.margin_sigma >= 0.0)) { msg = "margin_sigma must be non-negative"; return OCTO_ERR_ARG; }
        if (!(o.coupling_tol >= 0.0)) { msg = "coupling_tol must be non-negative (INFINITY: uncoupled)"; return OCTO_ERR_ARG; }
    }
    if (o.precision != 0 && o.precision != 1) {
        msg = "precision must be 0 (FP64 plain form) or 1 (FP32 precision form)";
        return OCTO_ERR_ARG;
    }
    if (o.solver != OCTO_SOLVER_PIC && o.solver != OCTO_SOLVER_SOFT_GAUSSIAN) {
        msg = "solver must be OCTO_SOLVER_PIC or OCTO_SOLVER_SOFT_GAUSSIAN";
        return OCTO_ERR_ARG;
    }
    if (o.solver == OCTO_SOLVER_SOFT_GAUSSIAN) {  // GaussianPoissonSolver{T} (interface.jl:976-1000)
        if (!(std::isfinite(o.min_sigma) && o.min_sigma >= 0.0)) { msg = "min_sigma must be finite and nonnegative"; return OCTO_ERR_ARG; }
        if (o.gaussian_when_luminosity != 1 && o.gaussian_when_luminosity != 2) {
            msg = "gaussian_when_luminosity must be 1 or 2";
            return OCTO_ERR_ARG;
        }
        if (o.virtual_drift < 0 || o.virtual_drift > 2) {
            msg = "virtual_drift must be 0 (:hirata), 1 (:chromatic) or 2 (:exact)";
            return OCTO_ERR_ARG;
        }
        if (o.include_sigma_xy != 0 && o.include_sigma_xy != 1) {
            msg = "include_sigma_xy must be 0 or 1";
            return OCTO_ERR_ARG;
        }
        if (o.gaussian) {
            msg = "the soft-Gaussian solver runs without the PIC hybrid (gaussian = 0)";
            return OCTO_ERR_UNSUPPORTED;
        }
    }
    return OCTO_OK;
}

void upload_twiddles(DevBuf<double2> &buf, int L) {
    std::vector<double2> h(L / 2);
    for (int k = 0; k < L / 2; ++k) {
        double a = 2.0 * 3.141592653589793238462643 * (double)k / (double)L;
        h[k] = make_double2(std::cos(a), -std::sin(a));
    }
    buf.ensure(L / 2);
    CK(cudaMemcpy(buf.p, h.data(), sizeof(double2) * (L / 2), cudaMemcpyHostToDevice));
}
// FP32 twiddles: the FP64 values rounded once.
void upload_twiddles(DevBuf<float2> &buf, int L) {
    std::vector<float2> h(L / 2);
    for (int k = 0; k < L / 2; ++k) {
        double a = 2.0 * 3.141592653589793238462643 * (double)k / (double)L;
        h[k] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    buf.ensure(L / 2);
    CK(cudaMemcpy(buf.p, h.data(), sizeof(float2) * (L / 2), cudaMemcpyHostToDevice));
}

// Coefficients of Weideman's N = 32 rational approximation of w(z) (SIAM J. Numer. Anal. 31, 1994), from the
// paper's construction: a_m = Re(DFT of f(t_k) = exp(-t_k^2)(L^2 + t_k^2) on t_k = L tan(k pi / 2M))_m / 2M.
void upload_weideman() {
    constexpr int N = kWeidemanN, M = 2 * N, M2 = 2 * M;
    const double pi = 3.141592653589793238462643;
    double h[N + 1];
    const double L = std::sqrt((double)N / std::sqrt(2.0));
    h[0] = L;
    double f[M2];
    for (int idx = 0; idx < M2; ++idx) {
        const int k = idx - M;
        if (k == -M) { f[idx] = 0.0; continue; }
        const double t = L * std::tan(0.5 * (double)k * pi / (double)M);
        f[idx] = std::exp(-t * t) * (L * L + t * t);
    }
    for (int m = 1; m <= N; ++m) {
        double re = 0.0;
        for (int n = 0; n < M2; ++n) re += f[(n + M) % M2] * std::cos(2.0 * pi * (double)((long)m * n % M2) / (double)M2);
        h[1 + N - m] = re / (double)M2;
    }
    CK(cudaMemcpyToSymbol(c_weideman, h, sizeof h));
}

long long padded_total(long long n, int ns) { return n + (long long)ns * kAlign; }

__global__ void k_init_bounds(unsigned long long *bnd, int ntasks, unsigned long long *lumb, int npairs, int *nanflag,
                              DevStatus *st, int reset_status) {
    pdl_wait();
    pdl_release();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntasks) {
        for (int k = 0; k < 8; ++k) bnd[(long long)t * 8 + k] = (k & 1) ? kOrdMaxInit : kOrdMinInit;
        nanflag[t] = 0;
    }
    if (t < npairs)
        for (int k = 0; k < 4; ++k) lumb[(long long)t * 4 + k] = (k & 1) ? kOrdMaxInit : kOrdMinInit;
    if (t == 0 && reset_status) {
        st->first_bad = ~0ull;
        st->code = 0;
        st->role = 0;
        st->dropped = 0;
    }
}

__global__ void k_init_boxes(unsigned long long *a, long long na, unsigned long long *b, long long nb) {
    pdl_wait();
    pdl_release();
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < na) a[t] = (t & 1) ? kOrdMaxInit : kOrdMinInit;
    else if (t < na + nb) b[t - na] = (t & 1) ? kOrdMaxInit : kOrdMinInit;
}

// Device slicing of both beams in shared launches; returns after enqueueing (the slice tables are read
// back by the caller).
void slice_beams(octo_ctx *c, const octo_beam &b1, const octo_beam &b2, cudaStream_t st, long long &launches) {
    long long nblk_max = 1;
    int ns_max = 1;
    for (int b = 0; b < 2; ++b) {
        BeamWS &W = c->bw[b];
        const long long n = (b == 0 ? b1 : b2).n;
        const int ns = c->ns[b];
        const long long total = padded_total(n, ns);
        for (auto &a : W.s) a.ensure(total);
        W.dest.ensure(n);
        W.info.ensure(1);
        W.lane_sum.ensure(kFoldLanes); W.lane_min.ensure(kFoldLanes); W.lane_max.ensure(kFoldLanes);
        W.lanes.ensure((size_t)kFoldLanes * ns);
        const long long nblocks = (n + kChunk - 1) / kChunk;
        W.counts.ensure((size_t)nblocks * ns);
        W.blockoff.ensure((size_t)nblocks * ns);
        W.total = total;
        nblk_max = std::max(nblk_max, nblocks);
        ns_max = std::max(ns_max, ns);
    }
    with_real(c->fp32, [&](auto r) {
        using R = decltype(r);
        SliceArgs<R> A{};
        for (int b = 0; b < 2; ++b) {
            BeamWS &W = c->bw[b];
            const octo_beam &B = b == 0 ? b1 : b2;
            const void *cc[6] = {B.x, B.px, B.y, B.py, B.z, B.pz};
            for (int k = 0; k < 6; ++k) { A.c[b][k] = (const R *)cc[k]; A.s[b][k] = (R *)W.s[k].p; }
            A.dest[b] = W.dest.p;
            A.info[b] = W.info.p;
            A.lane_sum[b] = W.lane_sum.p; A.lane_min[b] = W.lane_min.p; A.lane_max[b] = W.lane_max.p;
            A.lanes[b] = W.lanes.p;
            A.q[b] = W.q.p;
            A.counts[b] = W.counts.p;
            A.blockoff[b] = W.blockoff.p;
            A.n[b] = B.n;
            A.nblocks[b] = (B.n + kChunk - 1) / kChunk;
            A.method[b] = b == 0 ? c->opt.slicing_method1 : c->opt.slicing_method2;
            A.ns[b] = c->ns[b];
            A.cpos[b] = b == 0 ? c->opt.center_position1 : c->opt.center_position2;
            const int res = b == 0 ? c->opt.resolution1 : c->opt.resolution2;
            A.resolution[b] = res > 0 ? res : 100;
            if (A.method[b] == kEqualArea) {
                W.hist.ensure((size_t)A.ns[b] * A.resolution[b]);
                CK(cudaMemsetAsync(W.hist.p, 0, sizeof(long long) * A.ns[b] * A.resolution[b], st));
                A.hist[b] = W.hist.p;
            }
            if (A.method[b] == kEqualCount) {
                W.rkey.ensure(B.n); W.rkey_sorted.ensure(B.n); W.rval.ensure(B.n); W.rval_sorted.ensure(B.n);
                A.rkey[b] = W.rkey.p; A.rkey_sorted[b] = W.rkey_sorted.p;
                A.rval[b] = W.rval.p; A.rval_sorted[b] = W.rval_sorted.p;
            }
        }
        const bool any_area = A.method[0] == kEqualArea || A.method[1] == kEqualArea;
        const bool any_count = A.method[0] == kEqualCount || A.method[1] == kEqualCount;
        const long long iters = (std::max(b1.n, b2.n) + kFoldLanes - 1) / kFoldLanes;
        const int rows = (int)std::min<long long>(kLaneFoldRows, std::max<long long>(1, iters));
        const size_t fold_smem = sizeof(double) * 33 * (size_t)rows;
        launch_pdl(k_lane_fold<R>, dim3(kFoldLanes / 32, 1, 2), kLaneFoldThreads, fold_smem, st, A, 0, rows);
        launch_pdl(k_fold_stats<R>, 2, 1024, 0, st, A, 0);
        launch_pdl(k_lane_fold<R>, dim3(kFoldLanes / 32, 1, 2), kLaneFoldThreads, fold_smem, st, A, 1, rows);
        launch_pdl(k_fold_stats<R>, 2, 1024, 0, st, A, 1);
        if (any_area) {  // :equal_area boundaries from the z histogram
            long long bins = 1;
            for (int b = 0; b < 2; ++b)
                if (A.method[b] == kEqualArea) bins = std::max<long long>(bins, (long long)A.ns[b] * A.resolution[b]);
            CK(cudaFuncSetAttribute(k_area_hist<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * bins)));
            CK(cudaFuncSetAttribute(k_area_bounds<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(8 * bins)));
            launch_pdl(k_area_hist<R>, dim3((unsigned)nblk_max, 1, 2), 256, (size_t)(4 * bins), st, A, kChunk);
            launch_pdl(k_area_bounds<R>, 2, 1024, (size_t)(8 * bins), st, A);
            launches += 2;
        }
        if (any_count) {  // :equal_count: rank order by a stable radix sort of z, then the rank scatter
            const unsigned kb = (unsigned)std::min<long long>(148 * 8, (std::max(b1.n, b2.n) + 255) / 256);
            launch_pdl(k_rank_keys<R>, dim3(kb, 1, 2), 256, 0, st, A);
            for (int b = 0; b < 2; ++b) {
                if (A.method[b] != kEqualCount) continue;
                BeamWS &W = c->bw[b];
                const int n = (int)(b == 0 ? b1.n : b2.n);
                size_t tmp = 0;
                CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, W.rkey.p, W.rkey_sorted.p, W.rval.p, W.rval_sorted.p, n,
                                                   0, 64, st));
                W.sort_tmp.ensure(tmp);
                CK(cub::DeviceRadixSort::SortPairs((void *)W.sort_tmp.p, tmp, W.rkey.p, W.rkey_sorted.p, W.rval.p,
                                                   W.rval_sorted.p, n, 0, 64, st));
                launches += 4;
            }
            launch_pdl(k_rank_bounds<R>, 2, 32, 0, st, A, kAlign);
            launch_pdl(k_rank_scatter<R>, dim3(kb, 1, 2), 256, 0, st, A);
            launches += 3;
        }
        launch_pdl(k_slice_count<R>, dim3((unsigned)nblk_max, 1, 2), 256, 0, st, A, kChunk);
        launch_pdl(k_slice_offsets<R>, 2, 1024, 0, st, A, kAlign);
        launch_pdl(k_slice_scatter<R>, dim3((unsigned)nblk_max, 1, 2), kScatterThreads, 0, st, A, kChunk);
        launch_pdl(k_slice_lanes<R>, dim3(kFoldLanes / 256, ns_max, 2), 256, 0, st, A);
        launch_pdl(k_slice_finish<R>, dim3(ns_max, 2), 1024, 0, st, A);
    });
    launches += 9;
    // plain PIC: the working copy in spatial order (the centroid lanes above used the stable copy)
    if (c->spatial && c->opt.solver == OCTO_SOLVER_PIC && !c->opt.gaussian) {
        with_real(c->fp32, [&](auto r) {
            using R = decltype(r);
            SpatialArgs<R> S{};
            for (int b = 0; b < 2; ++b) {
                BeamWS &W = c->bw[b];
                const octo_beam &B = b == 0 ? b1 : b2;
                for (auto &a : W.t) a.ensure(W.total);
                W.box.ensure((size_t)4 * c->ns[b]);
                W.cursor.ensure((size_t)kSpatialCells * c->ns[b]);
                CK(cudaMemsetAsync(W.cursor.p, 0, sizeof(int) * kSpatialCells * c->ns[b], st));
                const void *cc[6] = {B.x, B.px, B.y, B.py, B.z, B.pz};
                for (int k = 0; k < 6; ++k) { S.c[b][k] = (const R *)cc[k]; S.t[b][k] = (R *)W.t[k].p; }
                S.dest[b] = W.dest.p;
                S.info[b] = W.info.p;
                S.box[b] = W.box.p;
                S.cursor[b] = W.cursor.p;
                S.n[b] = B.n;
                S.nblocks[b] = (B.n + kChunk - 1) / kChunk;
            }
            launch_pdl(k_init_boxes, (unsigned)((4 * (c->ns[0] + c->ns[1]) + 255) / 256), 256, 0, st, c->bw[0].box.p,
                       (long long)4 * c->ns[0], c->bw[1].box.p, (long long)4 * c->ns[1]);
            launch_pdl(k_spatial_boxes<R>, dim3((unsigned)nblk_max, 1, 2), 256, 0, st, S, kChunk);
            launch_pdl(k_spatial_count<R>, dim3((unsigned)nblk_max, 1, 2), 256, 0, st, S, kChunk);
            launch_pdl(k_spatial_scan<R>, dim3(ns_max, 2), 1024, 0, st, S);
            launch_pdl(k_spatial_scatter<R>, dim3((unsigned)nblk_max, 1, 2), 256, 0, st, S, kChunk);
        });
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 6; ++k) std::swap(c->bw[b].s[k], c->bw[b].t[k]);
        launches += 5;
    }
    CK(cudaGetLastError());
}

long long first_nonfinite_host(const octo_beam &beam, cudaStream_t st, bool z_only) {
    const size_t esz = beam.dtype == 1 ? sizeof(float) : sizeof(double);
    std::vector<unsigned char> h((size_t)beam.n * esz);
    void *arr[6] = {beam.x, beam.px, beam.y, beam.py, beam.z, beam.pz};
    long long first = -1;
    for (int k = 0; k < 6; ++k) {
        if (z_only && k != 4) continue;
        CK(cudaMemcpyAsync(h.data(), arr[k], esz * beam.n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (long long i = 0; i < beam.n; ++i) {
            const double v = beam.dtype == 1 ? (double)((const float *)h.data())[i] : ((const double *)h.data())[i];
            if (!std::isfinite(v)) { if (first < 0 || i < first) first = i; break; }
        }
    }
    return first;
}

// dtype: the element type the call requires (0 float64, 1 float32), or -1 for either.
int check_beam(const octo_beam *b, std::string &msg, int dtype = 0) {
    if (!b) { msg = "beam pointer is NULL"; return OCTO_ERR_ARG; }
    if (b->n <= 0) { msg = "longitudinal slicing requires at least one particle"; return OCTO_ERR_ARG; }
    if (b->n >= (1LL << 31) - 4096) { msg = "beam too large for 32-bit particle indices"; return OCTO_ERR_ARG; }
    if (b->dtype != 0 && b->dtype != 1) { msg = "beam dtype must be 0 (float64) or 1 (float32)"; return OCTO_ERR_ARG; }
    if (dtype >= 0 && b->dtype != dtype) {
        msg = dtype == 0 ? "this call needs float64 beams (the plain form's element type)"
                         : "the precision form (precision = 1) needs float32 beams";
        return OCTO_ERR_ARG;
    }
    if (!b->x || !b->px || !b->y || !b->py || !b->z || !b->pz) { msg = "beam coordinate pointer is NULL"; return OCTO_ERR_ARG; }
    return OCTO_OK;
}

template <class F>
void launch_method(int method, F f) {
    if (method == 0) f(std::integral_constant<int, 0>());
    else f(std::integral_constant<int, 1>());
}


// Dynamic shared memory of the FFT kernels for line length L (4 warps per block), complex elements of
// `real` bytes per component (8 FP64, 4 FP32).
size_t fft_smem(int L, size_t real = sizeof(double), int lines = 4) { return 2 * real * (size_t)(L / 2 + lines * L); }
// k_conv_cols: a second line per warp when the padded column length is 3 * 2^a.
size_t cols_smem(int L, size_t real) { return fft_smem(L, real, L % 3 == 0 ? 8 : 4); }
// k_green_rows (FP64): twiddles + 4 lines + the (kGreenRows+1) x (NX+1) corner lattice of F.
size_t green_smem(int NX) { return fft_smem(NX) + sizeof(double) * (size_t)(kGreenRows + 1) * (NX + 1); }
// k_conv_field: twiddles (NX/2) + 4 lines (4*NX) complex, plus a (tile+4) x nx phi tile; NX = 2*nx.
size_t field_smem(int NX, size_t real = sizeof(double)) {
    return fft_smem(NX, real) + real * (size_t)(kFieldTile + 4) * (NX / 2);
}
// Register-FFT kernels (rfft.cuh): twiddle tables + one 256-element scratch per warp.
size_t rf_smem(int G, size_t real, int warps = 4) {
    const int tables = G == 32 ? RfGeom<32>::kTables : G == 16 ? RfGeom<16>::kTables : RfGeom<8>::kTables;
    return 2 * real * (size_t)(tables + warps * RfGeom<8>::kWarpScratch);
}
template <class F>
void with_rf(int G, F f) {
    if (G == 32) f(std::integral_constant<int, 32>());
    else if (G == 16) f(std::integral_constant<int, 16>());
    else f(std::integral_constant<int, 8>());
}
// Lanes per line of the register FFT for the x-lines (rows, field) and y-lines (columns), 0 where the
// shared-memory FFT of fft.cuh runs.  The Green spectra are stored in the column transform's order, so
// k_green_cols* and k_conv_cols* always take the same path (both decide from NY alone).
int rf_rows(int nx) { return rf_lanes(2 * nx); }
int rf_cols(int ny) { return rf_lanes(2 * ny); }
constexpr size_t kSmemLimit = 227 * 1024;

// Raise the dynamic shared-memory limit of every kernel launched with more than 48 KB to the B200 opt-in
// maximum (the attribute only permits; occupancy follows the size each launch asks for).
void set_smem_limits() {
    const int lim = (int)kSmemLimit;
    CK(cudaFuncSetAttribute(k_green_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    CK(cudaFuncSetAttribute(k_green_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    auto per_real = [&](auto r) {
        using R = decltype(r);
        CK(cudaFuncSetAttribute(k_deposit<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_deposit<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_lum_deposit<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_lum_deposit<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        if constexpr (sizeof(R) == 4) {
            CK(cudaFuncSetAttribute(k_deposit_node3<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            CK(cudaFuncSetAttribute(k_deposit_node3<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        }
        CK(cudaFuncSetAttribute(k_conv_rows<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_conv_cols<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_conv_field<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_lane_fold<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                lim - (int)(2 * kLaneFoldThreads * sizeof(double))));
    };
    per_real(double(0));
    per_real(float(0));
    auto per_g = [&](auto g) {
        constexpr int G = decltype(g)::value;
        CK(cudaFuncSetAttribute(k_green_rows_r<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_green_cols_r<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        auto per_r = [&](auto r) {
            using R = decltype(r);
            CK(cudaFuncSetAttribute(k_conv_rows_r<R, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            CK(cudaFuncSetAttribute(k_conv_cols_r<R, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
            CK(cudaFuncSetAttribute(k_conv_field_r<R, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        };
        per_r(double(0));
        per_r(float(0));
    };
    per_g(std::integral_constant<int, 8>());
    per_g(std::integral_constant<int, 16>());
    per_g(std::integral_constant<int, 32>());
}

// Green spectra of `count` meshes (mode 0: the front's tasks from `base`; mode 1: node meshes).
void launch_green(const octo_ctx *c, const Collide &C, int mode, int base, int count, cudaStream_t st) {
    const int nx = c->opt.nx, ny = c->opt.ny, NX = 2 * nx, NY = 2 * ny;
    const int gx = rf_rows(nx), gy = rf_cols(ny);
    if (gx && ny % (8 * (32 / gx)) == 0) {  // a block's rows never straddle the wrap at row ny
        with_rf(gx, [&](auto g) {
            constexpr int G = decltype(g)::value, ROWS = 8 * (32 / G);
            const size_t sm = rf_smem(G, sizeof(double)) + sizeof(double) * (size_t)(ROWS + 1) * (NX + 1);
            launch_pdl(k_green_rows_r<G>, dim3(NY / ROWS, count), 128, sm, st, C, mode, base, 0);
        });
    } else {
        launch_pdl(k_green_rows, dim3(NY / kGreenRows, count), 128, green_smem(NX), st, C, mode, base, 0);
    }
    if (gy) {
        with_rf(gy, [&](auto g) {
            constexpr int G = decltype(g)::value, PER = 4 * (32 / G);
            launch_pdl(k_green_cols_r<G>, dim3((nx + 1 + PER - 1) / PER, count), 128, rf_smem(G, sizeof(double)), st, C, mode, base, 0);
        });
    } else {
        launch_pdl(k_green_cols, dim3((nx + 1 + 3) / 4, count), 128, fft_smem(NY), st, C, mode, base, 0);
    }
}

// Particles per block for a launch whose rows (planes or slice sides) take ceil(n / share) blocks each, one block
// resident per SM (it holds its rows' whole grids): for w = min_waves .. 8 waves the share is the smallest that
// fits the blocks into w waves of the SMs, and the w with the least (waves run) x (share + a block's fixed cost,
// `fixed` particles' worth of clearing and merging its grid) is taken.
long long wave_share(const std::vector<long long> &rn, long long fixed, long long sms, int min_waves) {
    long long sum = 0, mx = 1;
    for (long long n : rn) { sum += n; mx = std::max(mx, n); }
    const long long rows = (long long)rn.size();
    long long share = std::max<long long>(1024, mx);
    double best = 1e300;
    for (int w = std::max(1, min_waves); w <= 8; ++w) {
        const long long room = std::max<long long>(1, sms * w - rows);
        const long long pb = std::max<long long>(1024, (sum + room - 1) / room);
        long long T = 0;
        for (long long n : rn) T += std::min<long long>(32, std::max<long long>(1, (n + pb - 1) / pb));
        const double cost = (double)((T + sms - 1) / sms) * (double)(pb + fixed);
        if (cost < best) { best = cost; share = pb; }
    }
    return share;
}
// The grid's blocks per row for that share: enough for the largest row (at most 32).
unsigned share_blocks(const std::vector<long long> &rn, long long share) {
    long long mx = 1;
    for (long long n : rn) mx = std::max(mx, n);
    return (unsigned)std::max<long long>(1, std::min<long long>(32, (mx + share - 1) / share));
}

// Enqueue the node meshes of both directions (pic_cpu.jl:1404-1419) with no host synchronisation: the
// per-direction drift tables and slice counts are staged in pinned memory owned by the context, and
// mesh validity is known on the host from the slice counts (node_mesh_valid).
void build_node_meshes(octo_ctx *c, Collide &C, const SliceInfo &S1, const SliceInfo &S2, cudaStream_t st,
                       long long &launches, bool capture, bool padded, long long &node_cap) {
    const int ns1 = c->ns[0], ns2 = c->ns[1];
    const int nnode = ns1 * (ns2 + 1) + ns2 * (ns1 + 1);
    c->nodes.ensure(nnode);
    c->nodenan.ensure(1);
    CK(cudaMemsetAsync(c->nodenan.p, 0, sizeof(int), st));
    // staging: the drift references of each beam's rows ([slice][2*o + 1], o = the other beam's slice
    // count: o + 1 node drifts, then the o field-role centres), then both beams' slice counts
    const int nref1 = 2 * ns2 + 1, nref2 = 2 * ns1 + 1;
    const size_t off2 = (size_t)ns1 * nref1, offc = off2 + (size_t)ns2 * nref2;
    const size_t cap = 2 * (size_t)kMaxSlices * (2 * kMaxSlices + 1) + 2 * kMaxSlices;
    c->h_noderef.ensure(cap);
    c->node_ref.ensure(cap);
    double *href = c->h_noderef.p;
    for (int bm = 0; bm < 2; ++bm) {
        const SliceInfo &SS = bm == 0 ? S1 : S2, &SO = bm == 0 ? S2 : S1;
        const int ns = bm ? ns2 : ns1, o = bm ? ns1 : ns2, nref = 2 * o + 1;
        double *r = href + (bm ? off2 : 0);
        for (int sl = 0; sl < ns; ++sl) {
            for (int b = 0; b <= o; ++b) r[(size_t)sl * nref + b] = 0.5 * (SS.center[sl] - SO.boundary[b]);
            for (int i = 0; i < o; ++i) r[(size_t)sl * nref + o + 1 + i] = SO.center[i];
        }
    }
    long long *hcnt = (long long *)(href + offc);
    for (int s = 0; s < ns1; ++s) hcnt[s] = S1.count[s];
    for (int s = 0; s < ns2; ++s) hcnt[ns1 + s] = S2.count[s];
    // a captured collide's drift references are refreshed on the device by its guard (k_replay_check)
    if (!capture) CK(cudaMemcpyAsync(c->node_ref.p, href, sizeof(double) * (offc + ns1 + ns2), cudaMemcpyHostToDevice, st));
    const long long *dcnt = (const long long *)(c->node_ref.p + offc);
    const int nbox_s = std::max(ns1 * (ns2 + 1), ns2 * (ns1 + 1)), nbox_f = ns1 * ns2;
    c->nodebox_s.ensure((size_t)2 * nbox_s * 4);
    c->nodebox_f.ensure((size_t)2 * nbox_f * 4);
    unsigned long long *sbox1 = c->nodebox_s.p, *sbox2 = c->nodebox_s.p + (size_t)nbox_s * 4;
    unsigned long long *fbox1 = c->nodebox_f.p, *fbox2 = c->nodebox_f.p + (size_t)nbox_f * 4;
    const long long ns8 = 8ll * nbox_s, nf8 = 8ll * nbox_f;
    launch_pdl(k_init_boxes, (unsigned)((ns8 + nf8 + 255) / 256), 256, 0, st, c->nodebox_s.p, ns8, c->nodebox_f.p, nf8);
    // one pass over both beams: beam 0's source role is direction 1, its field role direction 2
    NodeBoxArgs A{};
    long long maxn = 1;
    for (int bm = 0; bm < 2; ++bm) {
        const BeamWS &W = c->bw[bm];
        const SliceInfo &SS = bm == 0 ? S1 : S2;
        A.x[bm] = W.s[0].p; A.px[bm] = W.s[1].p; A.y[bm] = W.s[2].p; A.py[bm] = W.s[3].p; A.z[bm] = W.s[4].p;
        A.info[bm] = W.info.p;
        for (int s = 0; s < c->ns[bm]; ++s) maxn = std::max(maxn, SS.count[s]);
        A.ns[bm] = c->ns[bm];
    }
    // a collide that may be captured keeps this chunking for later turns: room for slices a sixteenth larger
    // (the graph's guard checks that every slice still fits)
    if (padded) maxn += maxn / 16 + kBoxTile;
    A.ref[0] = c->node_ref.p; A.ref[1] = c->node_ref.p + off2;
    A.sbox[0] = sbox1; A.sbox[1] = sbox2;
    A.fbox[0] = fbox2; A.fbox[1] = fbox1;
    A.nanf = c->nodenan.p;
    const long long bx = std::min<long long>(256, (maxn + 4095) / 4096);
    A.chunk = ((maxn + bx - 1) / bx + kBoxTile - 1) / kBoxTile * kBoxTile;
    node_cap = bx * A.chunk;
    const int gz = (std::max(nref1, nref2) + kBoxLanes * kBoxGroups - 1) / (kBoxLanes * kBoxGroups);
    with_real(c->fp32, [&](auto r) {
        launch_pdl(k_node_boxes<decltype(r)>, dim3((unsigned)bx, ns1 + ns2, gz), kBoxThreads, 0, st, A);
    });
    launch_pdl(k_node_plan, (ns1 * (ns2 + 1) + 63) / 64, 64, 0, st, c->dopt, sbox1, fbox1, ns1, ns2 + 1, dcnt, c->nodenan.p,
                                                           c->nodes.p, c->status.p);
    launch_pdl(k_node_plan, (ns2 * (ns1 + 1) + 63) / 64, 64, 0, st, c->dopt, sbox2, fbox2, ns2, ns1 + 1, dcnt + ns1,
                                                           c->nodenan.p, c->nodes.p + ns1 * (ns2 + 1), c->status.p);
    launches += 4;
    // Green spectra of every valid node mesh
    C.nodes = c->nodes.p;
    launch_green(c, C, 1, 0, nnode, st);
    launches += 2;
}

// Validity of node mesh (source slice src0, node b1 in 1..nsf+1) as k_node_plan decides it for finite
// inputs: the source slice is non-empty and one of the field slices adjacent to the node is non-empty.
bool node_mesh_valid(const SliceInfo &SS, const SliceInfo &SF, int nsf, int src0, int b1) {
    if (SS.count[src0] == 0) return false;
    for (int adj = b1 - 1; adj <= b1; ++adj)
        if (1 <= adj && adj <= nsf && SF.count[adj - 1] > 0) return true;
    return false;
}

// One collide as three stages, so a batch of independent collides can interleave them:
// begin() validates and enqueues the slicing and the copy of the slice tables to pinned memory; run()
// waits for those tables, builds the schedule and enqueues every wavefront, the write-back and the copy
// of the results; finish() waits for the results, reports errors and folds the luminosity.
struct CollideJob {
    octo_ctx *c;
    octo_beam *b1, *b2;
    const octo_beam_params *p1, *p2;
    int64_t turn;
    int compute_lum;
    octo_collide_report *rep;
    cudaStream_t st;
    long long launches = 0;
    bool fp32 = false;
    size_t rsz = sizeof(double);
    long long n1 = 0, n2 = 0;
    double kbb1 = 0, kbb2 = 0, klum = 0;
    double kbb1p = 0, kbb2p = 0;  // per beam, before the division by the other beam's macroparticles
    std::vector<OrderEntry> order;
    std::vector<std::vector<OrderEntry>> batches;
    std::vector<char> ran;
    std::vector<Task> tasks;
    int ntasks = 0, npairs_total = 0;
    // capture: enqueue this collide's kernels into a graph being captured on st -- the slice tables were read
    // by the ordinary collide just run, the schedule tables are resident on the device -- with no host
    // synchronisation, no uploads and no copies back (the captured graph's own nodes do those)
    bool capture = false;
    int nplanes_total = 0, nlum_total = 0, nfirst_total = 0;  // the schedule tables' lengths (run)
    std::vector<int> slot;  // replayed graph: order position -> the captured position its pair's results use
    std::vector<FrontKick> fkick;  // per wavefront: its tasks and kick block map entries (run)
    long long node_cap = 0;        // :node: the largest slice the node-box chunking covers (run)
    void begin();
    void run();
    void run_gaussian(const SliceInfo &S1, const SliceInfo &S2);
    void write_back();
    double finish();
};

void CollideJob::begin() {
    const octo_pic_options &o = c->opt;
    std::string msg;
    int rc = check_beam(b1, msg, c->fp32);
    if (rc == OCTO_OK) rc = check_beam(b2, msg, c->fp32);
    if (rc != OCTO_OK) throw OctoFail{rc, msg};
    if (!p1 || !p2) throw OctoFail{OCTO_ERR_ARG, "beam params pointer is NULL"};
    fp32 = c->fp32 != 0;
    rsz = fp32 ? sizeof(float) : sizeof(double);
    CK(cudaSetDevice(c->device));
    // kbb and luminosity scale (slicing.jl:77-91, pic_cpu.jl:821-829)
    if (!o.has_kbb1 && !(std::isfinite(p1->E0) && p1->E0 != 0))
        throw OctoFail{OCTO_ERR_ARG, "beam1 E0 must be finite and nonzero when kbb1 is not specified"};
    if (!o.has_kbb2 && !(std::isfinite(p2->E0) && p2->E0 != 0))
        throw OctoFail{OCTO_ERR_ARG, "beam2 E0 must be finite and nonzero when kbb2 is not specified"};
    n1 = b1->n;
    n2 = b2->n;
    const double kbb1p = o.has_kbb1 ? o.kbb1 : p1->charge * p2->charge * p1->r0 * p2->npart * p1->mc2 / p1->E0;
    const double kbb2p = o.has_kbb2 ? o.kbb2 : p1->charge * p2->charge * p2->r0 * p1->npart * p2->mc2 / p2->E0;
    kbb1 = kbb1p / (double)n2;
    kbb2 = kbb2p / (double)n1;
    this->kbb1p = kbb1p;
    this->kbb2p = kbb2p;
    klum = o.has_lum_scale ? o.lum_scale : p1->npart * p2->npart / (double)(n1 * n2);

    // ---- slicing (one readback of the slice tables, into pinned memory so the copy is asynchronous)
    {
        PhaseScope ps(c, OCTO_PHASE_SLICING, st, 9);
        slice_beams(c, *b1, *b2, st, launches);
    }
    c->h_slices.ensure(2);
    CK(cudaMemcpyAsync(c->h_slices.p + 0, c->bw[0].info.p, sizeof(SliceInfo), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c->h_slices.p + 1, c->bw[1].info.p, sizeof(SliceInfo), cudaMemcpyDeviceToHost, st));
}

void CollideJob::run() {
    const octo_pic_options &o = c->opt;
    CK(cudaSetDevice(c->device));
    if (!capture) CK(cudaStreamSynchronize(st));
    for (int b = 0; b < 2; ++b) {
        if (c->h_slices.p[b].nonfinite) {
            long long first = first_nonfinite_host(b == 0 ? *b1 : *b2, st, true);
            if (rep) { rep->role = 3; rep->first_index = first + 1; }
            char m[192];
            snprintf(m, sizeof m, "non-finite beam%d coordinate z at particle %lld (longitudinal slicing, turn %lld)",
                     b + 1, first + 1, (long long)turn);
            throw OctoFail{OCTO_ERR_NONFINITE, m};
        }
    }
    const SliceInfo S1 = c->h_slices.p[0], S2 = c->h_slices.p[1];
    if (o.solver == OCTO_SOLVER_SOFT_GAUSSIAN) {
        run_gaussian(S1, S2);
        write_back();
        return;
    }
    const int ns1 = c->ns[0], ns2 = c->ns[1];
    const int nx = o.nx, ny = o.ny, NX = 2 * nx, NY = 2 * ny;
    const int gx = rf_rows(nx), gy = rf_cols(ny);
    const int lnx = c->dopt.lnx, lny = c->dopt.lny;
    const bool node = o.interaction_grid == OCTO_GRID_NODE;
    const bool lk = o.longitudinal_kick != 0;
    const bool quad = o.slice_interpolation == 1;
    const int method = o.deposit_method;
    const int lmethod = c->dopt.lum_method;
    // a collide that may be captured sizes what depends on the slice counts with room to spare (the kick's
    // block map, the node boxes' chunking), so that its graph fits later turns whose counts differ a little
    const bool padded = replay_eligible(c);

    Collide C{};
    C.o = c->dopt;
    C.o.dep_rotate = (c->spatial && !c->opt.gaussian) ? 1 : 0;  // spatially ordered slices (slice_beams)
    C.klum = klum;
    for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 6; ++k) C.beam[b].c[k] = c->bw[b].s[k].p;
    C.tw_x = c->tw_x.p;
    C.tw_y = c->tw_y.p;
    C.twr_x = fp32 ? (const void *)c->twf_x.p : (const void *)c->tw_x.p;
    C.twr_y = fp32 ? (const void *)c->twf_y.p : (const void *)c->tw_y.p;
    C.gstride = c->gstride;

    // ---- Green slots / cache / status
    const int maxw = std::min(ns1, ns2);
    const int nnode = node ? ns1 * (ns2 + 1) + ns2 * (ns1 + 1) : 0;
    const int nslots = node ? nnode : (o.green_cache ? 2 * ns1 * ns2 : 2 * maxw);
    if ((size_t)nslots * c->gstride > c->ghat.n) c->ghat.ensure((size_t)nslots * c->gstride);
    c->status.ensure(1);
    if (!c->cache_ready) {
        DevStatus z{};
        z.first_bad = ~0ull;
        CK(cudaMemcpyAsync(c->status.p, &z, sizeof z, cudaMemcpyHostToDevice, st));
        if (!node && o.green_cache) {
            c->cache.ensure((size_t)2 * ns1 * ns2);
            CK(cudaMemsetAsync(c->cache.p, 0, sizeof(CacheEntry) * 2 * ns1 * ns2, st));
        }
        CK(cudaStreamSynchronize(st));
        c->cache_ready = 1;
    }
    C.cache = c->cache.p;
    C.status = c->status.p;
    C.ghat = c->ghat.p;

    // ---- schedule (slicing.jl:561-647), skipping pairs with an empty slice (pic_cpu.jl:302)
    order = collision_order(S1.center, ns1, S2.center, ns2);
    // :source_slice runs one pair per front in collision order (pic_cpu.jl:54, 240-248): a source slice's union
    // box is taken at its first use, from the beams as that pair finds them
    const bool shared = c->dopt.shared_grid != 0;
    if (shared) {
        batches.clear();
        for (const OrderEntry &e : order) batches.push_back({e});
    } else {
        batches = pair_batches(order, ns1, ns2);
    }
    std::vector<char> ub_seen(shared ? ns1 + ns2 : 0, 0);
    std::vector<int> pos_of((size_t)ns1 * ns2);
    for (size_t p = 0; p < order.size(); ++p) pos_of[(size_t)(order[p].i - 1) * ns2 + (order[p].j - 1)] = (int)p;

    // ---- status reset for this call (cache counters stay cumulative)
    launch_pdl(k_init_bounds, 1, 1, 0, st, nullptr, 0, nullptr, 0, nullptr, c->status.p, 1);
    launches += 1;
    if (c->cnn) {
        c->cnn_flags.ensure(1);
        CK(cudaMemsetAsync(c->cnn_flags.p, 0, sizeof(int), st));
    }

    // ---- node meshes at turn start
    if (node) {
        PhaseScope ps(c, OCTO_PHASE_NODE, st, 16);
        build_node_meshes(c, C, S1, S2, st, launches, capture, padded, node_cap);
    }
    auto node_id = [&](int dir, int src_slice0, int node1) {
        return dir == 1 ? src_slice0 * (ns2 + 1) + (node1 - 1) : ns1 * (ns2 + 1) + src_slice0 * (ns1 + 1) + (node1 - 1);
    };

    std::vector<Plane> planes;
    std::vector<LumJob> lumjobs;
    std::vector<int2> blockmap;
    // nb: the front's kick block map entries; cap: with the spare entries (the kick's grid)
    struct Front { int t0, nt, p0, np, l0, nl, b0, nb; long long maxsrc, maxlum; int kchunk; int cap; };
    std::vector<Front> fronts;
    const int nplanes_task = node ? (lk ? 3 : 2) : (quad ? 3 : 2);
    ran.assign(order.size(), 0);
    tasks.clear();
    for (size_t f = 0; f < batches.size(); ++f) {
        Front F{(int)tasks.size(), 0, (int)planes.size(), 0, (int)lumjobs.size(), 0, (int)blockmap.size(), 0, 1, 1,
                kKickChunk, 0};
        for (const OrderEntry &pr : batches[f]) {
            const int i = pr.i, j = pr.j;
            if (S1.count[i - 1] == 0 || S2.count[j - 1] == 0) continue;
            if (node) {
                bool ok = node_mesh_valid(S1, S2, ns2, i - 1, j) && node_mesh_valid(S1, S2, ns2, i - 1, j + 1) &&
                          node_mesh_valid(S2, S1, ns1, j - 1, i) && node_mesh_valid(S2, S1, ns1, j - 1, i + 1);
                if (!ok) continue;
            }
            const int p = pos_of[(size_t)(i - 1) * ns2 + (j - 1)];
            ran[p] = 1;
            for (int dir = 1; dir <= 2; ++dir) {
                Task T{};
                T.dir = dir; T.i = i; T.j = j;
                T.src_beam = dir - 1;
                T.fld_beam = 2 - dir;
                const SliceInfo &SS = dir == 1 ? S1 : S2, &SF = dir == 1 ? S2 : S1;
                const int ss = dir == 1 ? i - 1 : j - 1, sf = dir == 1 ? j - 1 : i - 1;
                // :source_slice keeps one cache entry per (source slice, direction), the keys (i, 0, 1) and
                // (j, 0, 2) of pic_cpu.jl:372-373, in the slot of partner slice 1
                T.key = shared ? (dir == 1 ? (i - 1) * ns2 : ns1 * ns2 + (j - 1))
                               : ((dir - 1) * ns1 + (i - 1)) * ns2 + (j - 1);
                T.ub = dir == 1 ? i - 1 : ns1 + (j - 1);
                T.ub_first = shared && !ub_seen[T.ub];
                if (shared) ub_seen[T.ub] = 1;
                T.pair = p;
                T.front = (int)f;
                T.src_start = SS.start[ss]; T.src_n = SS.count[ss];
                T.fld_start = SF.start[sf]; T.fld_n = SF.count[sf];
                T.c_src = SS.center[ss];
                T.c_fld = SF.center[sf];
                T.lb_fld = SF.boundary[sf];
                T.rb_fld = SF.boundary[sf + 1];
                T.sL = 0.5 * (T.c_src - T.lb_fld);
                T.sR = 0.5 * (T.c_src - T.rb_fld);
                T.sM = 0.5 * (T.c_src - T.c_fld);
                T.ks = 2.0 * (dir == 1 ? kbb2 : kbb1);
                const double denom = T.rb_fld - T.lb_fld;  // pic_cpu.jl:1540-1548
                if (!std::isfinite(denom) || denom == 0.0) { T.hzi = 0.0; T.zbias = 0.5; }
                else { T.hzi = 1.0 / denom; T.zbias = T.rb_fld * T.hzi; }
                T.nodeL = node ? node_id(dir, ss, sf + 1) : -1;
                T.nodeR = node ? node_id(dir, ss, sf + 2) : -1;
                T.plane0 = (int)planes.size();
                T.nplanes = nplanes_task;
                const int tid = (int)tasks.size();
                const int bits = fp32 ? fixed_bits_for32(T.src_n) : fixed_bits_for(T.src_n);
                for (int k = 0; k < nplanes_task; ++k) {
                    Plane P{};
                    P.task = tid;
                    P.src_beam = T.src_beam;
                    P.src_start = T.src_start;
                    P.src_n = T.src_n;
                    P.fixed_bits = bits;
                    if (node) {
                        // L: sL on gL ; R: sR on gR ; Z: sR on gL (pic_cpu.jl:1506-1516)
                        P.kind = k == 0 ? 0 : (k == 1 ? 1 : 3);
                        P.s = k == 0 ? T.sL : T.sR;
                        P.geom = (k == 1) ? T.nodeR : T.nodeL;
                        P.green = P.geom;
                        P.count_dropped = k < 2 ? 1 : 0;
                        if (fp32 && k == 2) { P.other_delta = -2; P.self_first = 0; }  // L - Z
                    } else {
                        P.kind = k == 0 ? 0 : (k == 1 ? 1 : 2);
                        P.s = k == 0 ? T.sL : (k == 1 ? T.sR : 0.5 * (T.sL + T.sR));
                        P.geom = -1;
                        P.green = -1;
                        // :sigma and :source_slice meshes need not cover the source: count particles outside at
                        // either drift once (the L plane checks both)
                        P.count_dropped = ((c->dopt.grid_extent || shared) && k == 0) ? 2 : 0;
                        if (fp32 && !quad && k == 1) { P.other_delta = -1; P.self_first = 0; }  // L - R
                        if (fp32 && quad && k < 2) { P.other_delta = 2 - k; P.self_first = 1; }  // L - M, R - M
                    }
                    planes.push_back(P);
                }
                F.maxsrc = std::max<long long>(F.maxsrc, T.src_n);
                tasks.push_back(T);
            }
            if (compute_lum) {
                LumJob J{};
                J.pair = p;
                J.s1_start = S1.start[i - 1]; J.s1_n = S1.count[i - 1];
                J.s2_start = S2.start[j - 1]; J.s2_n = S2.count[j - 1];
                J.sM1 = 0.5 * (S1.center[i - 1] - S2.center[j - 1]);
                J.sM2 = 0.5 * (S2.center[j - 1] - S1.center[i - 1]);
                J.bits1 = fp32 ? fixed_bits_for32(J.s1_n) : fixed_bits_for(J.s1_n);
                J.bits2 = fp32 ? fixed_bits_for32(J.s2_n) : fixed_bits_for(J.s2_n);
                F.maxlum = std::max<long long>(F.maxlum, std::max<long long>(J.s1_n, J.s2_n));
                lumjobs.push_back(J);
            }
        }
        F.nt = (int)tasks.size() - F.t0;
        // kick blocks of kchunk field particles: 2048, or fewer where the front would not fill the GPU's
        // resident block slots (two per SM in FP64, four in FP32)
        long long nfld = 0;
        for (int t = F.t0; t < F.t0 + F.nt; ++t) nfld += tasks[t].fld_n;
        const long long slots = (long long)c->num_sms * (fp32 ? 4 : 2) * c->kick_slots;
        const long long want = (nfld + slots - 1) / slots;
        F.kchunk = (int)std::min<long long>(kKickChunk, std::max<long long>(kKickThreads, (want + kKickThreads - 1) /
                                                                                           kKickThreads * kKickThreads));
        for (int t = F.t0; t < F.t0 + F.nt; ++t)
            for (long long off = 0; off < tasks[t].fld_n; off += F.kchunk) blockmap.push_back(make_int2(t, (int)off));
        F.nb = (int)blockmap.size() - F.b0;
        if (padded && F.nt) {  // room for one more block per task and a sixteenth more, unused here
            const int spare = F.nt + F.nb / 16;
            for (int k = 0; k < spare; ++k) blockmap.push_back(make_int2(-1, 0));
        }
        F.cap = (int)blockmap.size() - F.b0;
        F.np = (int)planes.size() - F.p0;
        F.nl = (int)lumjobs.size() - F.l0;
        if (F.nt) fronts.push_back(F);
    }
    fkick.clear();
    for (const Front &F : fronts) fkick.push_back(FrontKick{F.t0, F.nt, F.b0, F.cap, F.kchunk, 0});
    ntasks = (int)tasks.size();
    npairs_total = (int)order.size();
    // :node with luminosity: each kick reduces its field slice's virtual positions for that slice's next pair,
    // and one turn-start pass covers every slice's first pair (no per-front bounds pass).
    for (auto &T : tasks) { T.next_pair = -1; T.next_task = -1; T.next_sM = 0.0; }
    std::vector<FirstLum> first_lum;
    const bool fused_lum_bounds = node && compute_lum;
    if (fused_lum_bounds) {
        // lumjob k belongs to tasks 2k (direction 1) and 2k + 1
        std::vector<std::vector<int>> lj_of[2];
        lj_of[0].resize(ns1);
        lj_of[1].resize(ns2);
        for (int k = 0; k < (int)lumjobs.size(); ++k) {
            lj_of[0][tasks[2 * k].i - 1].push_back(k);
            lj_of[1][tasks[2 * k].j - 1].push_back(k);
        }
        for (int t = 0; t < ntasks; ++t) {
            Task &T = tasks[t];
            const int fb = T.fld_beam, sl = fb == 0 ? T.i - 1 : T.j - 1;
            const std::vector<int> &L = lj_of[fb][sl];
            const auto it = std::upper_bound(L.begin(), L.end(), t / 2);
            if (it == L.end()) continue;
            const LumJob &J = lumjobs[*it];
            T.next_pair = J.pair;
            T.next_task = 2 * *it;
            T.next_sM = fb == 0 ? J.sM1 : J.sM2;
        }
        for (int b = 0; b < 2; ++b)
            for (int sl = 0; sl < (b == 0 ? ns1 : ns2); ++sl) {
                if (lj_of[b][sl].empty()) continue;
                const LumJob &J = lumjobs[lj_of[b][sl][0]];
                FirstLum F{};
                F.start = b == 0 ? J.s1_start : J.s2_start;
                F.count = b == 0 ? J.s1_n : J.s2_n;
                F.sM = b == 0 ? J.sM1 : J.sM2;
                F.beam = b;
                F.pair = J.pair;
                F.task = 2 * lj_of[b][sl][0];
                first_lum.push_back(F);
            }
    }
    int max_planes = 1, max_lum = 1;
    for (auto &F : fronts) { max_planes = std::max(max_planes, F.np); max_lum = std::max(max_lum, F.nl); }

    // ---- device buffers and one upload of the whole schedule
    nplanes_total = (int)planes.size();
    nlum_total = (int)lumjobs.size();
    nfirst_total = (int)first_lum.size();
    c->tasks.ensure(std::max(ntasks, 1));
    c->planes.ensure(std::max<size_t>(planes.size(), 1));
    c->lumjobs.ensure(std::max<size_t>(lumjobs.size(), 1));
    c->geom.ensure(std::max(ntasks, 1));
    c->blockmap.ensure(std::max<size_t>(blockmap.size(), 1));
    c->bnd.ensure((size_t)std::max(ntasks, 1) * 8);
    c->nanflag.ensure(std::max(ntasks, 1));
    c->lumb.ensure((size_t)std::max(npairs_total, 1) * 4);
    c->lumgeom.ensure(std::max(npairs_total, 1));
    c->lum_parts.ensure(std::max(npairs_total, 1));
    const size_t cells = (size_t)nx * ny;
    const size_t lcells = (size_t)(lnx + 1) * (lny + 1);
    if (c->qgrid.n < (size_t)max_planes * cells) {
        c->qgrid.ensure((size_t)max_planes * cells);
        CK(cudaMemsetAsync(c->qgrid.p, 0, sizeof(long long) * c->qgrid.n, st));
    }
    c->spec.ensure((size_t)max_planes * (nx + 1) * ny);
    c->fields.ensure((size_t)max_planes * (fp32 ? 1 : 2) * cells);  // double2 units: 32 B (FP64) / 16 B (FP32) per cell
    c->lum_partial.ensure((size_t)max_lum * kLumSplit);
    if (c->lum_tick.n < (size_t)max_lum) {
        c->lum_tick.ensure((size_t)max_lum);
        CK(cudaMemsetAsync(c->lum_tick.p, 0, sizeof(unsigned) * c->lum_tick.n, st));
    }
    if (c->lq.n < (size_t)2 * max_lum * lcells) {
        c->lq.ensure((size_t)2 * max_lum * lcells);
        CK(cudaMemsetAsync(c->lq.p, 0, sizeof(long long) * c->lq.n, st));
    }
    c->first_lum.ensure(std::max<size_t>(first_lum.size(), 1));
    std::vector<long long> slr;
    if (shared) {
        slr.assign((size_t)2 * kMaxSlices * 2, 0);
        for (int b = 0; b < 2; ++b)
            for (int sl = 0; sl < (b == 0 ? ns1 : ns2); ++sl) {
                const SliceInfo &SB = b == 0 ? S1 : S2;
                slr[((size_t)b * kMaxSlices + sl) * 2] = SB.start[sl];
                slr[((size_t)b * kMaxSlices + sl) * 2 + 1] = SB.count[sl];
            }
        c->ubox.ensure((size_t)(ns1 + ns2) * kUnionRow);
        c->uflag.ensure(ns1 + ns2);
        c->slr.ensure(slr.size());
    }
    const size_t bytes = sizeof(Task) * tasks.size() + sizeof(Plane) * planes.size() + sizeof(LumJob) * lumjobs.size() +
                         sizeof(int2) * blockmap.size() + sizeof(FirstLum) * first_lum.size() +
                         sizeof(long long) * slr.size() + 64;
    c->stage.ensure(bytes);
    char *h = c->stage.p;
    auto put = [&](void *dst, const void *src, size_t nbytes) {
        if (!nbytes || capture) return;
        std::memcpy(h, src, nbytes);
        CK(cudaMemcpyAsync(dst, h, nbytes, cudaMemcpyHostToDevice, st));
        h += nbytes;
    };
    put(c->tasks.p, tasks.data(), sizeof(Task) * tasks.size());
    put(c->planes.p, planes.data(), sizeof(Plane) * planes.size());
    put(c->lumjobs.p, lumjobs.data(), sizeof(LumJob) * lumjobs.size());
    put(c->blockmap.p, blockmap.data(), sizeof(int2) * blockmap.size());
    put(c->first_lum.p, first_lum.data(), sizeof(FirstLum) * first_lum.size());
    if (shared) {
        put(c->slr.p, slr.data(), sizeof(long long) * slr.size());
        const long long nu = (long long)(ns1 + ns2) * kUnionRow;
        launch_pdl(k_init_boxes, (unsigned)((nu + 255) / 256), 256, 0, st, c->ubox.p, nu, (unsigned long long *)nullptr, 0ll);
        CK(cudaMemsetAsync(c->uflag.p, 0, sizeof(int) * (ns1 + ns2), st));
        launches += 1;
        C.ubox = c->ubox.p;
        C.uflag = c->uflag.p;
        C.slr = c->slr.p;
    }
    CK(cudaMemsetAsync(c->lum_parts.p, 0, sizeof(double) * npairs_total, st));
    launch_pdl(k_init_bounds, (std::max(ntasks, npairs_total) + 255) / 256, 256, 0, st, c->bnd.p, ntasks, c->lumb.p, npairs_total,
                                                                                c->nanflag.p, c->status.p, 0);
    launches += 1;
    C.tasks = c->tasks.p;
    C.planes = c->planes.p;
    C.lumjobs = c->lumjobs.p;
    C.geom = c->geom.p;
    C.lumgeom = c->lumgeom.p;
    C.bnd = c->bnd.p;
    C.lumb = c->lumb.p;
    C.nanflag = c->nanflag.p;
    C.qgrid = c->qgrid.p;
    C.spec = c->spec.p;
    C.fields = c->fields.p;
    C.lq = c->lq.p;
    C.lum_parts = c->lum_parts.p;
    C.lum_partial = c->lum_partial.p;
    C.lum_tick = c->lum_tick.p;
    C.nodes = c->nodes.p;
    const bool gaussian = c->dopt.gaussian != 0;
    if (!c->lum_stream) {
        CK(cudaStreamCreateWithFlags(&c->lum_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    }
    // nothing an earlier (failed) collide left on the luminosity stream may overlap this one (a captured graph
    // forks and joins that stream within itself)
    if (!capture) {
        CK(cudaEventRecord(c->ev_join, c->lum_stream));
        CK(cudaStreamWaitEvent(st, c->ev_join, 0));
    }
    if (c->dopt.grid_extent) {
        c->esum.ensure((size_t)std::max(ntasks, 1) * kMaxBoundBlocks * 8);
        C.esum = c->esum.p;
    }
    if (gaussian) {
        c->hyb.ensure(std::max(ntasks, 1));
        c->hmom.ensure((size_t)std::max(ntasks, 1) * kMaxBoundBlocks * kMomentSums);
        c->qtot.ensure(max_planes);
        c->hprof.ensure((size_t)max_planes * 3 * (nx + ny));
        c->hsum.ensure((size_t)max_planes * 2);
        C.hyb = c->hyb.p;
        C.hmom = c->hmom.p;
        C.qtot = c->qtot.p;
        C.hprof = c->hprof.p;
        C.hsum = c->hsum.p;
    }

    if (!first_lum.empty()) {
        PhaseScope ps(c, OCTO_PHASE_BOUNDS, st, 1, (double)(n1 + n2) * 4 * rsz);
        long long maxn = 1;
        for (auto &F : first_lum) maxn = std::max<long long>(maxn, F.count);
        const unsigned bx = (unsigned)std::max<long long>(1, std::min<long long>(kMaxBoundBlocks, (maxn + 2047) / 2048));
        with_real(fp32, [&](auto r) {
            launch_pdl(k_first_lum_bounds<decltype(r)>, dim3(bx, (unsigned)first_lum.size()), 256, 0, st, C, c->first_lum.p);
        });
        launches += 1;
    }

    const size_t qsz = fp32 ? sizeof(int) : sizeof(long long);  // the block-private grids' element
    const size_t dep_bytes = c->dopt.dep_global ? 0 : cells * qsz;
    const size_t lum_bytes = c->dopt.lum_global ? 0 : lcells * qsz;

    // ---- wavefronts
    for (const Front &F : fronts) {
        const int npf = F.nt / 2;
        double slice_bytes = 0.0, src_bytes = 0.0, fld_bytes = 0.0;
        for (int t = F.t0; t < F.t0 + F.nt; t += 2) slice_bytes += (double)(tasks[t].src_n + tasks[t].fld_n);
        for (int t = F.t0; t < F.t0 + F.nt; ++t) { src_bytes += (double)tasks[t].src_n; fld_bytes += (double)tasks[t].fld_n; }
        const unsigned bps = (unsigned)std::max<long long>(1, std::min<long long>(kMaxBoundBlocks, (F.maxsrc + 2047) / 2048));
        bool union_first = false;
        for (int t = F.t0; t < F.t0 + F.nt; ++t) union_first = union_first || tasks[t].ub_first;
        if (union_first) {
            // the source slice's union box at its first use: the whole partner beam, then the source slice
            double pbytes = 0.0;
            long long pmax = 1;
            for (int t = F.t0; t < F.t0 + F.nt; ++t) {
                if (!tasks[t].ub_first) continue;
                const SliceInfo &SP = tasks[t].fld_beam == 0 ? S1 : S2;
                for (int sl = 0; sl < (tasks[t].fld_beam == 0 ? ns1 : ns2); ++sl) {
                    pbytes += (double)SP.count[sl];
                    pmax = std::max<long long>(pmax, SP.count[sl]);
                }
                pbytes += (double)tasks[t].src_n;
            }
            PhaseScope ps(c, OCTO_PHASE_BOUNDS, st, 2, pbytes * 5 * rsz);
            const unsigned bxp = (unsigned)std::max<long long>(1, std::min<long long>(kMaxBoundBlocks, (pmax + 2047) / 2048));
            with_real(fp32, [&](auto r) {
                launch_pdl(k_union_partner<decltype(r)>, dim3(bxp, (unsigned)std::max(ns1, ns2), (unsigned)F.nt), 256, 0, st, C,
                           F.t0);
                launch_pdl(k_union_source<decltype(r)>, dim3(bps, (unsigned)F.nt), 256, 0, st, C, F.t0);
            });
            launches += 2;
        }
        if (!node) {
            PhaseScope ps(c, OCTO_PHASE_BOUNDS, st, gaussian ? 2 : 1, slice_bytes * 5 * rsz);
            with_real(fp32, [&](auto r) { launch_pdl(k_pair_bounds<decltype(r)>, dim3(bps, 2 * npf), 256, 0, st, C, F.t0); });
            if (gaussian) {
                with_real(fp32, [&](auto r) { launch_pdl(k_hyb_moments<decltype(r)>, dim3(bps, 2 * npf), 256, 0, st, C, F.t0); });
                launch_pdl(k_hyb_fold, (F.nt * 32 + 127) / 128, 128, 0, st, C, F.t0, F.nt, (int)bps);
            }
            launches += gaussian ? 3 : 1;
        }
        bool lum_forked = false;
        if (compute_lum && F.nl) {
            CK(cudaEventRecord(c->ev_fork, st));
            CK(cudaStreamWaitEvent(c->lum_stream, c->ev_fork, 0));
            {
                PhaseScope ps(c, OCTO_PHASE_LUMINOSITY, c->lum_stream, 2, slice_bytes * 4 * rsz);
                // uniform blocks per side: this stream runs beside the front's deposit and convolution and wants
                // parallelism (blocks in proportion to each side's slice, sized to whole waves, measured slower)
                unsigned bpp = (unsigned)std::max<long long>(1, std::min<long long>(8, (F.maxlum + 32767) / 32768));
                with_real(fp32, [&](auto r) {
                    launch_method(lmethod, [&](auto M) {
                        launch_pdl(k_lum_deposit<decltype(r), decltype(M)::value>, dim3(bpp, 2 * F.nl), 1024, lum_bytes, c->lum_stream, 
                            C, F.l0, F.t0);
                    });
                });
                launch_pdl(k_lum_overlap, dim3(kLumSplit, F.nl), 256, 0, c->lum_stream, C, F.l0);
            }
            CK(cudaEventRecord(c->ev_join, c->lum_stream));
            lum_forked = true;
            launches += 2;
        }
        if (!node) {
            {
                PhaseScope ps(c, OCTO_PHASE_PLAN, st, 1);
                with_real(fp32, [&](auto r) {
                    launch_pdl(k_plan<decltype(r)>, (F.nt + 63) / 64, 64, 0, st, C, F.t0, F.nt, 0, (int)bps);
                });
            }
            PhaseScope ps(c, OCTO_PHASE_GREEN, st, gaussian ? 3 : 2);
            launch_green(c, C, 0, F.t0, F.nt, st);
            if (gaussian) {
                launch_pdl(k_hyb_profiles, F.np, 256, 0, st, C, F.p0);
                CK(cudaMemsetAsync(c->qtot.p, 0, sizeof(unsigned long long) * F.np, st));
            }
            launches += gaussian ? 4 : 3;
        }
        {
            PhaseScope ps(c, OCTO_PHASE_DEPOSIT, st, 1, src_bytes * 4 * rsz);
            // the precision form's :node planes of a task in one pass when their three int32 grids fit shared
            // memory (k_deposit_node3)
            const int ppt = c->dopt.longitudinal_kick ? 3 : 2;  // :node planes per task (L, R and Z)
            const bool node3 = fp32 && node && !c->dopt.dep_global && !c->dopt.dep_rotate && ppt * cells * sizeof(int) <= kSmemLimit;
            const int rows = node3 ? F.np / ppt : F.np;
            // k_deposit_node3 (a task's three int32 planes per block): a row gets ceil(src_n / per_block) blocks,
            // so rows of large slices get more blocks than rows of small ones.  One block runs per SM (it holds its
            // planes' whole grids); for w = dep_waves .. 8 waves per_block is the smallest share that fits the
            // front's blocks into w waves, and the w with the least (waves run) x (share + the block's fixed cost:
            // clearing and merging its grids, counted as cells / 4 particles per grid) is taken.  k_deposit (one
            // plane per row) keeps a uniform count per row: 32768-particle shares, and at least dep_waves waves
            // for the narrow fronts (its 64-bit atomic loop measured 19 % slower with the per-row stride).
            std::vector<long long> rn(rows);
            for (int r = 0; r < rows; ++r) rn[r] = planes[F.p0 + r * (node3 ? ppt : 1)].src_n;
            const long long per_block = wave_share(rn, (long long)cells * (node3 ? ppt : 1) / 4, c->num_sms, c->dep_waves);
            unsigned bpp = share_blocks(rn, per_block);
            if (!node3) {
                const long long wave = ((long long)c->num_sms * c->dep_waves + rows - 1) / rows;
                bpp = (unsigned)std::max<long long>(1, std::min<long long>(32, std::max<long long>((F.maxsrc + 32767) / 32768, wave)));
            }
            if (node3) {
                launch_method(method, [&](auto M) {
                    launch_pdl(k_deposit_node3<float, decltype(M)::value>, dim3(bpp, rows), 1024, ppt * cells * sizeof(int), st, C,
                               F.p0, ppt, per_block);
                });
            } else {
                with_real(fp32, [&](auto r) {
                    launch_method(method, [&](auto M) {
                        launch_pdl(k_deposit<decltype(r), decltype(M)::value>, dim3(bpp, F.np), 1024, dep_bytes, st, C, F.p0);
                    });
                });
            }
        }
        const bool learned = c->cnn != nullptr;
        if (learned) {  // the learned correction's input from the front's charge grids, and the network
            if (F.np > c->cnn->net.maxB)
                throw OctoFail{OCTO_ERR_ARG, "the field-correction network's max_batch is smaller than a wavefront's "
                                             "plane count (" + std::to_string(F.np) + ")"};
            c->cnn_q.ensure((size_t)c->cnn->net.maxB);
            launch_pdl(k_cnn_prep, F.np, 256, 0, st, C, F.p0, c->cnn->net.x0.p, c->cnn_q.p);
            c->cnn->net.forward(F.np, st, false);
            launches += 1 + 17;
        }
        if (c->cap_armed && !c->cap_taken) {
            for (int t = F.t0; t < F.t0 + F.nt; ++t) {
                const Task &T = tasks[t];
                if (T.i != c->cap_i || T.j != c->cap_j || T.dir != c->cap_dir || c->cap_kind >= T.nplanes) continue;
                const Plane &P = planes[T.plane0 + c->cap_kind];
                c->cap_q.ensure(cells);
                c->cap_grid.ensure(2);
                CK(cudaMemcpyAsync(c->cap_q.p, c->qgrid.p + (size_t)(T.plane0 + c->cap_kind - F.p0) * cells,
                                   sizeof(long long) * cells, cudaMemcpyDeviceToDevice, st));
                const Grid *mesh = P.geom >= 0 ? &(c->nodes.p + P.geom)->sg : &(c->geom.p + t)->sg;
                const Grid *fmesh = P.geom >= 0 ? &(c->nodes.p + P.geom)->fg : &(c->geom.p + t)->fg;
                CK(cudaMemcpyAsync(c->cap_grid.p, mesh, sizeof(Grid), cudaMemcpyDeviceToDevice, st));
                CK(cudaMemcpyAsync(c->cap_grid.p + 1, fmesh, sizeof(Grid), cudaMemcpyDeviceToDevice, st));
                c->cap_bits = P.fixed_bits;
                c->cap_taken = 1;
            }
        }
        {
            PhaseScope ps(c, OCTO_PHASE_FFT, st, 2);
            with_real(fp32, [&](auto r) {
                using R = decltype(r);
                if (gx) {
                    with_rf(gx, [&](auto g) {
                        constexpr int G = decltype(g)::value, PER = 4 * (32 / G);
                        launch_pdl(k_conv_rows_r<R, G>, dim3((ny / 2 + PER - 1) / PER, F.np), 128, rf_smem(G, rsz), st, C, F.p0);
                    });
                } else {
                    launch_pdl(k_conv_rows<R>, dim3((ny / 2 + 3) / 4, F.np), 128, fft_smem(NX, rsz), st, C, F.p0);
                }
                if (fp32)  // the precision form reads partner grids, so the front's grids are cleared here
                    CK(cudaMemsetAsync(c->qgrid.p, 0, sizeof(long long) * cells * F.np, st));
                if (gy) {
                    with_rf(gy, [&](auto g) {
                        constexpr int G = decltype(g)::value, PER = 4 * (32 / G);
                        launch_pdl(k_conv_cols_r<R, G>, dim3((nx + 1 + PER - 1) / PER, F.np), 128, rf_smem(G, rsz), st, C, F.p0);
                    });
                } else {
                    launch_pdl(k_conv_cols<R>, dim3((nx + 1 + 3) / 4, F.np), 128, cols_smem(NY, rsz), st, C, F.p0);
                }
            });
        }
        {
            PhaseScope ps(c, OCTO_PHASE_FIELD, st, 1);
            with_real(fp32, [&](auto r) {
                using R = decltype(r);
                if (gx) {
                    with_rf(gx, [&](auto g) {
                        constexpr int G = decltype(g)::value;
                        const size_t sm = rf_smem(G, rsz, kFieldWarpsR) + rsz * (size_t)(kFieldTileR + 4) * nx;
                        launch_pdl(k_conv_field_r<R, G>, dim3((ny + kFieldTileR - 1) / kFieldTileR, F.np), 32 * kFieldWarpsR, sm,
                                               st, C, F.p0);
                    });
                } else {
                    launch_pdl(k_conv_field<R>, dim3((ny + kFieldTile - 1) / kFieldTile, F.np), 128, field_smem(NX, rsz), st, C, F.p0);
                }
            });
        }
        if (learned) {
            with_real(fp32, [&](auto r) {
                launch_pdl(k_cnn_apply<decltype(r)>, F.np, 256, 0, st, C, F.p0, (const float *)c->cnn->net.out.p,
                           (const long long *)c->cnn_q.p, 1.0f / c->cnn_scale, c->cnn_edge, c->cnn_tol, c->cnn_flags.p);
            });
            launches += 1;
        }
        if (lum_forked) CK(cudaStreamWaitEvent(st, c->ev_join, 0));  // the kick changes what the luminosity read
        {
            PhaseScope ps(c, OCTO_PHASE_KICK, st, 1, fld_bytes * 11 * rsz);
            with_real(fp32, [&](auto r) {
                launch_method(method, [&](auto M) {
                    using R = decltype(r);
                    constexpr int MM = decltype(M)::value;
                    // F.cap blocks: the front's block map, spare entries included (they return at once)
                    if (gaussian) launch_pdl(k_kick<R, MM, true>, F.cap, kKickThreads, 0, st, C, F.p0, c->blockmap.p + F.b0, F.kchunk);
                    else launch_pdl(k_kick<R, MM, false>, F.cap, kKickThreads, 0, st, C, F.p0, c->blockmap.p + F.b0, F.kchunk);
                });
            });
        }
        launches += 5;
    }
    CK(cudaGetLastError());
    write_back();
}

// Slice-sorted coordinates back to caller order, and the copies of the pair luminosities and the status.
void CollideJob::write_back() {
    // ---- back to caller order
    {
        PhaseScope ps(c, OCTO_PHASE_UNSORT, st, 1, (double)(n1 + n2) * 10 * rsz);
        with_real(fp32, [&](auto r) {
            using R = decltype(r);
            UnsortArgs<R> A{};
            for (int b = 0; b < 2; ++b) {
                const BeamWS &W = c->bw[b];
                const octo_beam &B = b == 0 ? *b1 : *b2;
                void *cc[5] = {B.x, B.px, B.y, B.py, B.pz};
                const int sk[5] = {0, 1, 2, 3, 5};
                A.dest[b] = W.dest.p;
                for (int k = 0; k < 5; ++k) { A.s[b][k] = (const R *)W.s[sk[k]].p; A.c[b][k] = (R *)cc[k]; }
                // the soft-Gaussian solver's chromatic and exact virtual drifts move z
                const bool moves_z = c->opt.solver == OCTO_SOLVER_SOFT_GAUSSIAN && c->opt.virtual_drift != 0 &&
                                     c->opt.longitudinal_kick;
                A.sz[b] = moves_z ? (const R *)W.s[4].p : nullptr;
                A.cz[b] = moves_z ? (R *)B.z : nullptr;
                A.n[b] = B.n;
            }
            const long long nmax = std::max(n1, n2);
            launch_pdl(k_unsort<R>, dim3((unsigned)((nmax + 255) / 256), 2), 256, 0, st, A);
        });
        launches++;
    }
    c->h_lum.ensure(std::max(npairs_total, 1));
    c->h_status.ensure(1);
    if (capture) return;
    CK(cudaMemcpyAsync(c->h_lum.p, c->lum_parts.p, sizeof(double) * npairs_total, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c->h_status.p, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
}

// The soft-Gaussian solver (gaussian.jl:7-57): every slice pair in collision order -- all pairs, empty slices
// included, as the reference runs them -- one wavefront of conflict-free pairs at a time.  Task 2k kicks the
// beam-2 slice of pair k with the Gaussian of its beam-1 slice (the reference's lum1 direction), task 2k + 1
// the beam-1 slice with the Gaussian of the beam-2 slice (lum2).
void CollideJob::run_gaussian(const SliceInfo &S1, const SliceInfo &S2) {
    const octo_pic_options &o = c->opt;
    const int ns1 = c->ns[0], ns2 = c->ns[1];
    // luminosity scales (slicing.jl:93-102)
    const double klum1 = o.has_lum_scale ? o.lum_scale : p1->npart * p2->npart / (double)n1;
    const double klum2 = o.has_lum_scale ? o.lum_scale : p1->npart * p2->npart / (double)n2;
    const bool sample_beam1 = o.gaussian_when_luminosity == 1;
    order = collision_order(S1.center, ns1, S2.center, ns2);
    batches = pair_batches(order, ns1, ns2);
    std::vector<int> pos_of((size_t)ns1 * ns2);
    for (size_t p = 0; p < order.size(); ++p) pos_of[(size_t)(order[p].i - 1) * ns2 + (order[p].j - 1)] = (int)p;
    ran.assign(order.size(), 1);
    npairs_total = (int)order.size();

    std::vector<GSlice> gs;
    std::vector<GTask> gt;
    std::vector<int2> smap, kmap;             // sums blocks, kick blocks
    std::vector<int> sfirst, scount;          // per slice: its sums blocks
    std::vector<int> ltask, lfirst, lcount;   // per sampling task: its kick blocks
    struct Front { int s0, ns, sb0, nsb, t0, nt, kb0, nkb, l0, nl; };
    std::vector<Front> fronts;
    tasks.clear();
    for (size_t f = 0; f < batches.size(); ++f) {
        Front F{(int)gs.size(), 0, (int)smap.size(), 0, (int)gt.size(), 0, (int)kmap.size(), 0, (int)ltask.size(), 0};
        for (const OrderEntry &pr : batches[f]) {
            const int i = pr.i, j = pr.j, p = pos_of[(size_t)(i - 1) * ns2 + (j - 1)];
            const int t0 = (int)gt.size();
            // the two slices (moments 2p' and 2p' + 1 of this front: beam 1 slice i, beam 2 slice j)
            for (int b = 0; b < 2; ++b) {
                const SliceInfo &SI = b == 0 ? S1 : S2;
                const int sl = b == 0 ? i - 1 : j - 1;
                GSlice G{SI.start[sl], SI.count[sl], b, t0 + b};
                sfirst.push_back((int)smap.size());
                for (long long off = 0; off < G.n; off += kGaussChunk) smap.push_back(make_int2((int)gs.size(), (int)off));
                scount.push_back((int)smap.size() - sfirst.back());
                gs.push_back(G);
            }
            const int m1 = (int)gs.size() - 2, m2 = (int)gs.size() - 1;
            for (int dir = 1; dir <= 2; ++dir) {
                GTask T{};
                const bool fld2 = dir == 1;  // direction 1: beam-1 source kicks the beam-2 slice
                const SliceInfo &SF = fld2 ? S2 : S1, &SS = fld2 ? S1 : S2;
                const int sf = fld2 ? j - 1 : i - 1, ss = fld2 ? i - 1 : j - 1;
                T.fld_start = SF.start[sf];
                T.fld_n = SF.count[sf];
                T.fld_beam = fld2 ? 1 : 0;
                T.mom = fld2 ? m1 : m2;
                T.pair = p;
                T.lum = compute_lum && (fld2 ? sample_beam1 : !sample_beam1);
                T.center = SS.center[ss];
                T.kbb = SS.weight[ss] * (fld2 ? kbb2p : kbb1p);
                T.klum = SS.weight[ss] * (fld2 ? klum2 : klum1);
                const int tid = (int)gt.size();
                if (T.lum) {
                    ltask.push_back(tid);
                    lfirst.push_back((int)kmap.size());
                }
                for (long long off = 0; off < T.fld_n; off += kGaussChunk) kmap.push_back(make_int2(tid, (int)off));
                if (T.lum) lcount.push_back((int)kmap.size() - lfirst.back());
                gt.push_back(T);
                Task PT{};  // for error reports
                PT.dir = dir; PT.i = i; PT.j = j; PT.src_beam = fld2 ? 0 : 1; PT.fld_beam = T.fld_beam; PT.pair = p;
                tasks.push_back(PT);
            }
        }
        F.ns = (int)gs.size() - F.s0;
        F.nsb = (int)smap.size() - F.sb0;
        F.nt = (int)gt.size() - F.t0;
        F.nkb = (int)kmap.size() - F.kb0;
        F.nl = (int)ltask.size() - F.l0;
        if (F.ns) fronts.push_back(F);
    }
    ntasks = (int)tasks.size();
    // device copies: slices, tasks, block maps, and the index arrays [sfirst | scount | ltask | lfirst | lcount]
    c->g_slices.ensure(std::max<size_t>(gs.size(), 1));
    c->g_mom.ensure(std::max<size_t>(gs.size(), 1));
    c->g_tasks.ensure(std::max<size_t>(gt.size(), 1));
    c->g_bmap.ensure(std::max<size_t>(smap.size() + kmap.size(), 1));
    std::vector<int> idx;
    idx.insert(idx.end(), sfirst.begin(), sfirst.end());
    idx.insert(idx.end(), scount.begin(), scount.end());
    idx.insert(idx.end(), ltask.begin(), ltask.end());
    idx.insert(idx.end(), lfirst.begin(), lfirst.end());
    idx.insert(idx.end(), lcount.begin(), lcount.end());
    c->g_index.ensure(std::max<size_t>(idx.size(), 1));
    c->g_partial.ensure(std::max<size_t>(smap.size(), 1) * kGaussSums);
    c->g_lum_partial.ensure(std::max<size_t>(kmap.size(), 1));
    c->lum_parts.ensure(std::max(npairs_total, 1));
    c->status.ensure(1);
    if (!gs.empty()) CK(cudaMemcpyAsync(c->g_slices.p, gs.data(), sizeof(GSlice) * gs.size(), cudaMemcpyHostToDevice, st));
    if (!gt.empty()) CK(cudaMemcpyAsync(c->g_tasks.p, gt.data(), sizeof(GTask) * gt.size(), cudaMemcpyHostToDevice, st));
    if (!smap.empty()) CK(cudaMemcpyAsync(c->g_bmap.p, smap.data(), sizeof(int2) * smap.size(), cudaMemcpyHostToDevice, st));
    if (!kmap.empty())
        CK(cudaMemcpyAsync(c->g_bmap.p + smap.size(), kmap.data(), sizeof(int2) * kmap.size(), cudaMemcpyHostToDevice, st));
    if (!idx.empty()) CK(cudaMemcpyAsync(c->g_index.p, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(c->lum_parts.p, 0, sizeof(double) * std::max(npairs_total, 1), st));
    {
        DevStatus z{};
        z.first_bad = ~0ull;
        c->h_status.ensure(1);
        *c->h_status.p = z;
        CK(cudaMemcpyAsync(c->status.p, c->h_status.p, sizeof z, cudaMemcpyHostToDevice, st));
    }
    const int *d_sfirst = c->g_index.p, *d_scount = d_sfirst + sfirst.size();
    const int *d_ltask = d_scount + scount.size(), *d_lfirst = d_ltask + ltask.size(), *d_lcount = d_lfirst + lfirst.size();
    GaussArgs A{};
    for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 6; ++k) A.c[b][k] = (void *)c->bw[b].s[k].p;
    A.slices = c->g_slices.p;
    A.mom = c->g_mom.p;
    A.tasks = c->g_tasks.p;
    A.partial = c->g_partial.p;
    A.lum_partial = c->g_lum_partial.p;
    A.lum_parts = c->lum_parts.p;
    A.status = c->status.p;
    A.min_sigma = o.min_sigma;
    A.ignore_centroid[0] = o.ignore_centroid1 != 0;
    A.ignore_centroid[1] = o.ignore_centroid2 != 0;
    A.longitudinal = o.longitudinal_kick != 0;
    A.drift = o.virtual_drift;
    A.coupled = o.include_sigma_xy;
    for (const Front &F : fronts) {
        {
            PhaseScope ps(c, OCTO_PHASE_BOUNDS, st, 2);
            GaussArgs As = A;
            As.blockmap = c->g_bmap.p + F.sb0;
            As.partial = c->g_partial.p + (size_t)F.sb0 * kGaussSums;
            with_real(fp32, [&](auto r) {
                if (F.nsb) launch_pdl(k_gauss_sums<decltype(r)>, F.nsb, kGaussThreads, 0, st, As);
            });
            // moments: first[] is relative to the front's first sums block
            GaussArgs Am = A;
            Am.slices = c->g_slices.p + F.s0;
            Am.mom = c->g_mom.p + F.s0;
            with_real(fp32, [&](auto r) {
                launch_pdl(k_gauss_moments<decltype(r)>, F.ns, 32, 0, st, Am, d_sfirst + F.s0, d_scount + F.s0);
            });
            launches += (F.nsb ? 1 : 0) + 1;
        }
        {
            PhaseScope ps(c, OCTO_PHASE_KICK, st, 2);
            GaussArgs Ak = A;
            Ak.blockmap = c->g_bmap.p + smap.size() + F.kb0;
            Ak.lum_partial = c->g_lum_partial.p + F.kb0;
            with_real(fp32, [&](auto r) {
                if (F.nkb) launch_pdl(k_gauss_kick<decltype(r)>, F.nkb, kGaussThreads, 0, st, Ak);
            });
            // the fold reads the kick partials by their index over all fronts (lfirst)
            if (F.nl) launch_pdl(k_gauss_lum, (F.nl + 31) / 32, 32, 0, st, A, d_ltask + F.l0, d_lfirst + F.l0,
                                 d_lcount + F.l0, F.nl);
            launches += (F.nkb ? 1 : 0) + (F.nl ? 1 : 0);
        }
    }
    CK(cudaGetLastError());
}

double CollideJob::finish() {
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    harvest_timing(c);
    const DevStatus DS = *c->h_status.p;
    c->last_launches = launches;
    if (rep) {
        rep->n_batches = (int)batches.size();
        rep->turn = turn;
        rep->dropped = DS.dropped;
        rep->green_hits = DS.hits;
        rep->green_misses = DS.misses;
        rep->green_rebuilds = DS.rebuilds;
        rep->kernel_launches = launches;
    }
    if (DS.first_bad != ~0ull) {
        const int t = (int)(DS.first_bad >> 16), code = (int)((DS.first_bad >> 8) & 0xff), role = (int)(DS.first_bad & 0xff);
        char m[256];
        if (role == 4) {  // non-finite coordinate at the node-mesh build (turn start)
            long long f1 = first_nonfinite_host(*b1, st, false), f2 = first_nonfinite_host(*b2, st, false);
            const int bb = f1 >= 0 ? 1 : 2;
            const long long first = f1 >= 0 ? f1 : f2;
            if (rep) { rep->role = 4; rep->first_index = first + 1; }
            snprintf(m, sizeof m, "non-finite coordinate at particle %lld of beam%d (node-mesh build, turn %lld)", first + 1,
                     bb, (long long)turn);
            throw OctoFail{OCTO_ERR_NONFINITE, m};
        }
        if (code == OCTO_ERR_NONFINITE && t < ntasks && role == 0) {  // :source_slice union box (pic_cpu.jl:665-712)
            const Task &T = tasks[t];
            long long f2 = first_nonfinite_host(*b2, st, false), f1 = first_nonfinite_host(*b1, st, false);
            const int bb = f2 >= 0 ? 2 : 1;
            const long long first = f2 >= 0 ? f2 : f1;
            if (rep) { rep->role = 5; rep->pair_i = T.i; rep->pair_j = T.j; rep->direction = T.dir; rep->first_index = first + 1; }
            snprintf(m, sizeof m, "non-finite coordinate at particle %lld of beam%d (source-slice union bounds, slice pair "
                                  "(%d, %d), turn %lld)", first + 1, bb, T.i, T.j, (long long)turn);
            throw OctoFail{OCTO_ERR_NONFINITE, m};
        }
        if (code == OCTO_ERR_NONFINITE && t < ntasks) {
            const Task &T = tasks[t];
            if (rep) { rep->role = role; rep->pair_i = T.i; rep->pair_j = T.j; rep->direction = T.dir; }
            const octo_beam &B = (role == 1 ? T.src_beam : T.fld_beam) == 0 ? *b1 : *b2;
            long long first = first_nonfinite_host(B, st, false);
            if (rep) rep->first_index = first + 1;
            snprintf(m, sizeof m, "non-finite %s coordinate at particle %lld of beam%d (slice pair (%d, %d), direction %d, turn %lld)",
                     role == 1 ? "source" : "field", first + 1, (role == 1 ? T.src_beam : T.fld_beam) + 1, T.i, T.j, T.dir,
                     (long long)turn);
            throw OctoFail{OCTO_ERR_NONFINITE, m};
        }
        snprintf(m, sizeof m, "PIC interaction grid requires finite, positive transverse extents; supply a positive "
                              "min_transverse_extent for every degenerate axis (turn %lld)", (long long)turn);
        throw OctoFail{code ? code : OCTO_ERR_EXTENT, m};
    }
    // luminosity fold in collision order (pic_cpu.jl:258-271)
    c->trace_i.clear(); c->trace_j.clear(); c->trace_lum.clear();
    double lum = NAN;
    if (compute_lum) {
        lum = 0.0;
        for (size_t p = 0; p < order.size(); ++p) {
            // a replayed graph stores each pair's luminosity in the slot of its place in the captured order
            const size_t q = slot.empty() ? p : (size_t)slot[p];
            if (!ran[q]) continue;
            lum += c->h_lum.p[q];
            c->trace_i.push_back(order[p].i);
            c->trace_j.push_back(order[p].j);
            c->trace_lum.push_back(c->h_lum.p[q]);
        }
    }
    return lum;
}

int fail(octo_ctx *c, int code, const std::string &m) {
    if (c) c->err = m;
    return code;
}

// ---- captured collide graph
// Plain PIC only: the hybrid's and the learned correction's extra state, :sigma extents, :source_slice's
// sequential union boxes, per-phase timing and a charge-plane capture keep the ordinary path.
bool replay_eligible(const octo_ctx *c) {
    const octo_pic_options &o = c->opt;
    // the hybrid's moments and :sigma's extents are FP64 sums over blocks whose split follows the slice counts
    return c->rp.enabled && o.solver == OCTO_SOLVER_PIC && !o.gaussian && !c->dopt.grid_extent && !c->cnn &&
           !c->dopt.shared_grid && !c->timing && !c->cap_armed && !c->in_autotune &&
           c->ns[0] * c->ns[1] <= kReplayMaxPairs;
}

void drop_replay(octo_ctx *c) {
    auto &R = c->rp;
    if (R.exec) cudaGraphExecDestroy(R.exec);
    if (R.graph) cudaGraphDestroy(R.graph);
    R.exec = nullptr;
    R.graph = nullptr;
    R.valid = 0;
}

// The schedule of a collide in k_replay_check's layout: which slices of both beams hold particles, then for
// every pair index (i-1)*ns2 + (j-1) its wavefront and its place in it.
std::vector<long long> schedule_sig(const octo_ctx *c, const SliceInfo &S1, const SliceInfo &S2,
                                    const std::vector<std::vector<OrderEntry>> &batches) {
    const int ns1 = c->ns[0], ns2 = c->ns[1];
    std::vector<long long> v;
    v.reserve((size_t)(ns1 + ns2) + (size_t)ns1 * ns2);
    for (int k = 0; k < ns1; ++k) v.push_back(S1.count[k] > 0);
    for (int k = 0; k < ns2; ++k) v.push_back(S2.count[k] > 0);
    const size_t base = v.size();
    v.resize(base + (size_t)ns1 * ns2, -1);
    for (size_t f = 0; f < batches.size(); ++f)
        for (size_t q = 0; q < batches[f].size(); ++q)
            v[base + (size_t)(batches[f][q].i - 1) * ns2 + (batches[f][q].j - 1)] = (long long)f * 65536 + (long long)q;
    return v;
}

void beam_ptrs(const octo_beam *b, const void *p[6]) {
    p[0] = b->x; p[1] = b->px; p[2] = b->y; p[3] = b->py; p[4] = b->z; p[5] = b->pz;
}

// The captured kernels hold the beams' addresses, the interaction scales, the launch shape and every workspace
// address: the graph fits a collide only while all of them are unchanged.
bool replay_key_matches(const octo_ctx *c, const CollideJob &J) {
    const auto &R = c->rp;
    if (!R.valid || R.epoch != g_alloc_epoch.load()) return false;
    const octo_beam *b[2] = {J.b1, J.b2};
    for (int k = 0; k < 2; ++k) {
        const void *p[6];
        beam_ptrs(b[k], p);
        for (int q = 0; q < 6; ++q)
            if (p[q] != R.beam[k][q]) return false;
        if (b[k]->n != R.n[k]) return false;
    }
    return R.kbb1 == J.kbb1 && R.kbb2 == J.kbb2 && R.klum == J.klum && R.compute_lum == (J.compute_lum != 0) &&
           R.dep_waves == c->dep_waves && R.kick_slots == c->kick_slots && R.spatial == c->spatial;
}

// Capture the ordinary collide just finished (its schedule tables are resident, its slice tables still in
// pinned memory) as: guard kernel -> IF(body: the collide's kernels) -> copies of the pair luminosities, the
// status and the guard's result.  Any failure leaves the ordinary path in charge.
void build_replay(octo_ctx *c, const CollideJob &job, const std::vector<long long> &sig) {
    auto &R = c->rp;
    drop_replay(c);
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    bool capturing = false;
    try {
        if (!c->cap_stream) CK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
        c->rp_sig.ensure(sig.size());
        c->rp_fronts.ensure(std::max<size_t>(job.fkick.size(), 1));
        c->rp_ok.ensure(1);
        c->h_rp_ok.ensure(1);
        c->h_lum.ensure(std::max(job.npairs_total, 1));
        c->h_status.ensure(1);
        CK(cudaMemcpy(c->rp_sig.p, sig.data(), sizeof(long long) * sig.size(), cudaMemcpyHostToDevice));
        if (!job.fkick.empty())
            CK(cudaMemcpy(c->rp_fronts.p, job.fkick.data(), sizeof(FrontKick) * job.fkick.size(), cudaMemcpyHostToDevice));
        CK(cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle h;
        CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
        ReplayCheck A{};
        A.info[0] = c->bw[0].info.p;
        A.info[1] = c->bw[1].info.p;
        A.sig = c->rp_sig.p;
        A.ns1 = c->ns[0];
        A.ns2 = c->ns[1];
        A.tasks = c->tasks.p;
        A.ntasks = job.ntasks;
        A.planes = c->planes.p;
        A.nplanes = job.nplanes_total;
        A.lumjobs = c->lumjobs.p;
        A.nlum = job.nlum_total;
        A.first = c->first_lum.p;
        A.nfirst = job.nfirst_total;
        A.node_ref = c->dopt.node ? c->node_ref.p : nullptr;
        A.fp32 = c->fp32;
        A.fronts = c->rp_fronts.p;
        A.nfronts = (int)job.fkick.size();
        A.blockmap = c->blockmap.p;
        A.node_cap = job.node_cap;
        // k_node_plan reads the slice counts staged after the drift references (build_node_meshes)
        A.node_counts = c->dopt.node ? (long long *)(c->node_ref.p + (size_t)c->ns[0] * (2 * c->ns[1] + 1) +
                                                     (size_t)c->ns[1] * (2 * c->ns[0] + 1))
                                     : nullptr;
        A.ok = c->rp_ok.p;
        A.handle = h;
        void *args[] = {&A};
        cudaKernelNodeParams kp{};
        kp.func = (void *)k_replay_check;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(1024);
        kp.kernelParams = args;
        cudaGraphNode_t nk, nc, m;
        CK(cudaGraphAddKernelNode(&nk, g, nullptr, 0, &kp));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        CK(cudaGraphAddNode(&nc, g, &nk, 1, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaGraphAddMemcpyNode1D(&m, g, &nc, 1, c->h_lum.p, c->lum_parts.p,
                                    sizeof(double) * std::max(job.npairs_total, 1), cudaMemcpyDeviceToHost));
        CK(cudaGraphAddMemcpyNode1D(&m, g, &nc, 1, c->h_status.p, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost));
        CK(cudaGraphAddMemcpyNode1D(&m, g, &nc, 1, c->h_rp_ok.p, c->rp_ok.p, sizeof(int), cudaMemcpyDeviceToHost));
        // the body: the same collide's kernels, enqueued in capture mode on the capture stream
        CollideJob J2 = job;
        J2.capture = true;
        J2.st = c->cap_stream;
        J2.launches = 0;
        J2.rep = nullptr;
        CK(cudaStreamBeginCaptureToGraph(c->cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        capturing = true;
        J2.run();
        cudaGraph_t cap = nullptr;
        capturing = false;
        CK(cudaStreamEndCapture(c->cap_stream, &cap));
        // the captured kernels index the resident schedule tables: the capture's plan must be that one, byte for
        // byte (the guard rewrites only the drifts, from the same expressions)
        if (J2.ntasks != job.ntasks || J2.nplanes_total != job.nplanes_total || J2.nlum_total != job.nlum_total ||
            J2.nfirst_total != job.nfirst_total || J2.npairs_total != job.npairs_total ||
            J2.tasks.size() != job.tasks.size() ||
            std::memcmp(J2.tasks.data(), job.tasks.data(), sizeof(Task) * job.tasks.size()) != 0)
            throw CudaFail{"collide graph capture: the captured schedule differs from the resident one"};
        CK(cudaGraphInstantiate(&ex, g, 0));
        R.graph = g;
        R.exec = ex;
        R.valid = 1;
        R.sig = sig;
        R.pos_of.assign((size_t)c->ns[0] * c->ns[1], -1);
        for (size_t q = 0; q < job.order.size(); ++q)
            R.pos_of[(size_t)(job.order[q].i - 1) * c->ns[1] + (job.order[q].j - 1)] = (int)q;
        R.order = job.order;
        R.batches = job.batches;
        R.ran = job.ran;
        R.tasks = job.tasks;
        R.ntasks = job.ntasks;
        R.npairs_total = job.npairs_total;
        R.body_launches = J2.launches;
        const octo_beam *b[2] = {job.b1, job.b2};
        for (int k = 0; k < 2; ++k) { beam_ptrs(b[k], R.beam[k]); R.n[k] = b[k]->n; }
        R.kbb1 = job.kbb1;
        R.kbb2 = job.kbb2;
        R.klum = job.klum;
        R.compute_lum = job.compute_lum != 0;
        R.dep_waves = c->dep_waves;
        R.kick_slots = c->kick_slots;
        R.spatial = c->spatial;
        R.epoch = g_alloc_epoch.load();
        R.builds++;
    } catch (...) {
        if (capturing) {
            cudaGraph_t cap = nullptr;
            cudaStreamEndCapture(c->cap_stream, &cap);
        }
        cudaGetLastError();
        if (ex) cudaGraphExecDestroy(ex);
        if (g) cudaGraphDestroy(g);
        R.exec = nullptr;
        R.graph = nullptr;
        R.valid = 0;
        if (++R.failures >= 2) R.enabled = 0;  // this context keeps the ordinary path
    }
}

// After an ordinary collide: capture it once the same schedule has come twice in a row and no current graph
// fits it.
void maybe_build_replay(octo_ctx *c, const CollideJob &job) {
    auto &R = c->rp;
    std::vector<long long> sig = schedule_sig(c, c->h_slices.p[0], c->h_slices.p[1], job.batches);
    const bool repeat = sig == R.last_sig;
    R.last_sig = sig;
    if (!repeat) return;
    if (R.valid && R.sig == sig && replay_key_matches(c, job)) return;
    build_replay(c, job, sig);
}

// ---------------------------------------------------------------- line elements
uint64_t splitmix64_host(uint64_t x) {
    uint64_t z = x + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// _linear6d_symplectic_error (linear6d.jl:147-204): the worst row of M^T J M - J against a componentwise
// forward-error bound, 64 eps max(1, row scale).  Returns the ratio (> 1 rejects; non-finite entries: inf).
double linear6d_symplectic_ratio(const double *m) {
    const double inf = std::numeric_limits<double>::infinity();
    for (int k = 0; k < 36; ++k)
        if (!std::isfinite(m[k])) return inf;
    double worst = 0.0;
    for (int i = 0; i < 6; ++i) {
        double row_res = 0.0, row_scale = 0.0;
        for (int j = 0; j < 6; ++j) {
            double value = 0.0, pscale = 0.0;
            for (int q = 0; q < 6; q += 2) {
                const double pos = m[q * 6 + i] * m[(q + 1) * 6 + j];
                const double neg = m[(q + 1) * 6 + i] * m[q * 6 + j];
                if (!std::isfinite(pos) || !std::isfinite(neg)) return inf;
                value = (value + pos) - neg;
                pscale += std::fabs(pos) + std::fabs(neg);
            }
            const double target = (i % 2 == 0 && j == i + 1) ? 1.0 : (i % 2 == 1 && j == i - 1) ? -1.0 : 0.0;
            row_res += std::fabs(value - target);
            row_scale += std::max(std::fabs(target), pscale);
        }
        const double tol = 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, row_scale);
        if (!std::isfinite(row_res) || !std::isfinite(tol)) return inf;
        const double ratio = tol > 0.0 ? row_res / tol : (row_res == 0.0 ? 0.0 : inf);
        worst = std::max(worst, ratio);
    }
    return worst;
}

bool all_finite(const double *v, int n) {
    for (int k = 0; k < n; ++k)
        if (!std::isfinite(v[k])) return false;
    return true;
}

// 1 / sqrt(1 + r1 r4 - r2 r3) of a coupling block, with the XYCoupling constructor's check
// (linear_maps.jl:296-310).
bool coupling_scale(const double *r, double &g, std::string &msg, const char *who) {
    const double det = 1.0 + r[0] * r[3] - r[1] * r[2];
    if (std::isfinite(det) && det <= 0.0) {
        char b[256];
        snprintf(b, sizeof b, "%s: XYCoupling is not invertible: 1 + r1*r4 - r2*r3 = %.17g must be positive", who, det);
        msg = b;
        return false;
    }
    g = 1.0 / std::sqrt(det);
    return true;
}

// kZeroZeta / kZeroEta / kZeroR for a frame's zeta[4], eta[4], R[4] (contiguous).
int zero_frame_flags(const double *zer) {
    auto zero4 = [](const double *v) { return v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0 && v[3] == 0.0; };
    return (zero4(zer) ? kZeroZeta : 0) | (zero4(zer + 4) ? kZeroEta : 0) | (zero4(zer + 8) ? kZeroR : 0);
}

// Compiles one element into its constant form (the compile_runtime step of each element's constructor),
// validating as those constructors do.
int compile_line_op(const octo_element &e, int rng, uint64_t seed, LineOp &op, std::string &msg) {
    std::memset(&op, 0, sizeof op);
    op.kind = e.kind;
    const double *p = e.p;
    char b[320];
    switch (e.kind) {
        case OCTO_ELEM_LINEAR6D: {
            const double ratio = linear6d_symplectic_ratio(p);
            if (!(ratio <= 1.0)) {
                snprintf(b, sizeof b,
                         "Linear6D runtime matrix must be finite and canonical symplectic in (x, px, y, py, z, pz) "
                         "order: ratio=%.6g",
                         ratio);
                msg = b;
                return OCTO_ERR_ARG;
            }
            for (int k = 0; k < 36; ++k) op.a[k] = p[k];
            return OCTO_OK;
        }
        case OCTO_ELEM_THIN_CRAB_CAVITY: {
            if (!std::isfinite(p[0]) || p[0] == 0.0) {
                snprintf(b, sizeof b, "thin crab-cavity frequency must be finite and nonzero; got %.17g", p[0]);
                msg = b;
                return OCTO_ERR_ARG;
            }
            if (e.nharm < 1 || e.nharm > OCTO_CRAB_MAX_HARMONICS) {
                msg = "thin crab-cavity harmonic count must be 1.." + std::to_string(OCTO_CRAB_MAX_HARMONICS);
                return OCTO_ERR_ARG;
            }
            // kcc = 2 pi f / c (crab_cavity.jl:93), i kcc per harmonic (:133); harmonics with both strengths
            // zero are dropped (their terms are zeros for finite particles; the kernel keeps their NaN spread)
            const double kcc = 2.0 * 3.14159265358979323846 * p[0] / 299792458.0;
            op.n = 0;
            for (int h = 0; h < e.nharm; ++h) {
                if (p[1 + h] == 0.0 && p[9 + h] == 0.0) {
                    op.flags |= kCrabDropped;
                    continue;
                }
                op.a[op.n] = (double)(h + 1) * kcc;
                op.a[8 + op.n] = p[1 + h];
                op.a[16 + op.n] = p[9 + h];
                op.a[24 + op.n] = p[17 + h];
                ++op.n;
            }
            return OCTO_OK;
        }
        case OCTO_ELEM_LORENTZ_BOOST:
        case OCTO_ELEM_REV_LORENTZ_BOOST: {
            if (!std::isfinite(p[0])) { msg = "Lorentz boost angle must be finite"; return OCTO_ERR_ARG; }
            // _lorentz_boost (lorentz_boost.jl:168-174)
            const double c = std::cos(p[0]), s = std::sin(p[0]);
            op.a[0] = c;
            op.a[1] = s;
            op.a[2] = s / c;
            return OCTO_OK;
        }
        case OCTO_ELEM_CHROMATICITY_KICK: {
            if (!all_finite(p, 18)) { msg = "chromaticity kick parameters must be finite"; return OCTO_ERR_ARG; }
            // ChromaticityKick(spec) (chromaticity_kick.jl:74-96)
            for (int k = 0; k < 6; ++k) op.a[k] = p[k];
            op.a[6] = (1.0 + p[4] * p[4]) / p[2];
            op.a[7] = (1.0 + p[5] * p[5]) / p[3];
            for (int k = 0; k < 12; ++k) op.a[8 + k] = p[6 + k];
            op.flags = zero_frame_flags(p + 6);
            return coupling_scale(p + 14, op.a[20], msg, "chromaticity kick") ? OCTO_OK : OCTO_ERR_ARG;
        }
        case OCTO_ELEM_LUMPED_RAD: {
            // LumpedRad(spec) and _validate_lumped_rad_parameters (radiation.jl:83-160)
            for (int i = 0; i < 3; ++i)
                if (!(p[i] > 0.0)) {
                    snprintf(b, sizeof b, "damping_turns[%d] must be positive, got %.17g", i + 1, p[i]);
                    msg = b;
                    return OCTO_ERR_ARG;
                }
            static const char *names[6] = {"beta", "alpha", "sigma", "zeta", "eta", "R"};
            static const int off[6] = {3, 6, 9, 12, 16, 20}, len[6] = {3, 3, 3, 4, 4, 4};
            for (int g = 0; g < 6; ++g)
                for (int i = 0; i < len[g]; ++i)
                    if (!std::isfinite(p[off[g] + i])) {
                        snprintf(b, sizeof b, "%s[%d] must be finite, got %.17g", names[g], i + 1, p[off[g] + i]);
                        msg = b;
                        return OCTO_ERR_ARG;
                    }
            for (int i = 0; i < 3; ++i)
                if (!(p[3 + i] > 0.0)) {
                    snprintf(b, sizeof b, "beta[%d] must be positive, got %.17g", i + 1, p[3 + i]);
                    msg = b;
                    return OCTO_ERR_ARG;
                }
            const bool enabled = p[9] >= 0.0 && p[10] >= 0.0 && p[11] >= 0.0;
            const bool disabled = p[9] < 0.0 && p[10] < 0.0 && p[11] < 0.0;
            if (!enabled && !disabled) {
                msg = "sigma must be nonnegative in all three planes to enable excitation or negative in all three "
                      "planes to disable it";
                return OCTO_ERR_ARG;
            }
            if (e.mode < OCTO_RAD_RADIATION || e.mode > OCTO_RAD_DIFFUSION) {
                msg = "LumpedRad supports Radiation6DMap, Damping6DMap, or Diffusion6DMap";
                return OCTO_ERR_ARG;
            }
            // _lumped_rad_effective_components (radiation.jl:162-171)
            const bool damp = e.is_damping != 0 && e.mode != OCTO_RAD_DIFFUSION;
            const bool exc = e.is_excitation != 0 && enabled && e.mode != OCTO_RAD_DAMPING;
            op.flags = (damp ? kRadDamping : 0) | (exc ? kRadExcitation : 0) | zero_frame_flags(p + 12);
            for (int i = 0; i < 3; ++i) {
                op.a[i] = std::exp(-1.0 / p[i]);
                // _radiation_excitation (radiation.jl:286-299) with scale sqrt(-expm1(-2/tau)) (:110-113)
                const double scale = std::sqrt(-std::expm1(-2.0 / p[i]));
                const double sigma = p[9 + i];
                const double amp = sigma < 0.0 ? 0.0 : sigma * scale;
                const double slope = sigma < 0.0 ? 0.0 : amp / p[3 + i];
                op.a[3 + 3 * i] = amp;
                op.a[4 + 3 * i] = slope;
                op.a[5 + 3 * i] = sigma < 0.0 ? 0.0 : -slope * p[6 + i];
            }
            for (int k = 0; k < 12; ++k) op.a[12 + k] = p[12 + k];
            if (!coupling_scale(p + 20, op.a[24], msg, "lumped radiation")) return OCTO_ERR_ARG;
            // component keys (counter_rng.jl:187-205 for Philox, :284-291 for SplitMix)
            for (int c = 1; c <= 6; ++c)
                op.key[c - 1] = rng == OCTO_RNG_PHILOX
                                    ? splitmix64_host(seed) ^ splitmix64_host(e.rng_id + 0x9e3779b97f4a7c15ull) ^
                                          splitmix64_host((uint64_t)c + 0xbf58476d1ce4e5b9ull)
                                    : seed ^ splitmix64_host(e.rng_id + 0xbf58476d1ce4e5b9ull) ^
                                          splitmix64_host((uint64_t)c + 0xD2B74407B1CE6E93ull);
            return OCTO_OK;
        }
        case OCTO_ELEM_CRAB_DISPERSION:
        case OCTO_ELEM_MOMENTUM_DISPERSION:
            if (!all_finite(p, 4)) { msg = "dispersion coefficients must be finite"; return OCTO_ERR_ARG; }
            for (int k = 0; k < 4; ++k) op.a[k] = p[k];
            return OCTO_OK;
        case OCTO_ELEM_XY_COUPLING:
            if (e.mode < 0 || e.mode > 2) { msg = "XYCoupling mode must be 0 (undefined), 1 (A) or 2 (B)"; return OCTO_ERR_ARG; }
            for (int k = 0; k < 4; ++k) op.a[k] = p[k];
            op.n = e.mode;
            if (e.mode == 0) return OCTO_OK;
            return coupling_scale(p, op.a[4], msg, "xy coupling") ? OCTO_OK : OCTO_ERR_ARG;
        default:
            msg = "unknown line element kind " + std::to_string(e.kind);
            return OCTO_ERR_ARG;
    }
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int32_t octo_version(void) { return 1; }

double octo_erfinv(double x) { return erfinv_host(x); }

double octo_normal_quantile(int32_t s, int32_t ns) {
    return std::sqrt(2.0) * erfinv_host((double)(2 * s) / (double)ns - 1.0);
}

octo_ctx *octo_create(int32_t device, const octo_pic_options *options) {
    if (!options) return nullptr;
    octo_ctx *c = new octo_ctx();
    c->device = device;
    c->opt = *options;
    std::string msg;
    int rc = validate_options(c->opt, msg);
    if (rc != OCTO_OK) { c->err = msg; c->opt.nx = 0; return c; }
    for (int b = 0; b < 2; ++b) {
        int ns = b == 0 ? options->nslices1 : options->nslices2;
        const double *p = b == 0 ? options->positions1 : options->positions2;
        int m = b == 0 ? options->slicing_method1 : options->slicing_method2;
        if (m == OCTO_SLICING_SPECIFIED && p) c->pos[b].assign(p, p + (ns - 1));
        c->ns[b] = ns;
    }
    c->opt.positions1 = nullptr;
    c->opt.positions2 = nullptr;
    DevOptions &d = c->dopt;
    d.nx = options->nx; d.ny = options->ny;
    d.method = options->deposit_method;
    d.lum_method = options->lum_deposit_method < 0 ? options->deposit_method : options->lum_deposit_method;
    d.lnx = options->lum_nx > 0 ? options->lum_nx : options->nx;
    d.lny = options->lum_ny > 0 ? options->lum_ny : options->ny;
    d.green_type = options->green_type;
    d.green_cache = options->green_cache;
    d.fourth = options->field_derivative == 4;
    d.quadratic = options->slice_interpolation == 1;
    d.node = options->interaction_grid == OCTO_GRID_NODE;
    d.shared_grid = options->interaction_grid == OCTO_GRID_SOURCE_SLICE;
    d.longitudinal_kick = options->longitudinal_kick;
    d.min_ex = options->min_extent_x;
    d.min_ey = options->min_extent_y;
    d.quantize = options->grid_quantize;
    d.min_ratio = options->green_min_ratio;
    d.growth = options->green_growth;
    d.gaussian = options->gaussian != 0;
    d.neutralize = options->neutralize != 0;
    d.margin = options->margin_sigma;
    d.grid_extent = options->grid_extent;
    d.extent_k = options->grid_extent_sigma;
    d.coupling_tol = options->coupling_tol;
    try {
        CK(cudaSetDevice(device));
        CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
        c->fp32 = options->precision == 1;
        // the Faddeeva coefficients of the Bassetti-Erskine field: the hybrid's add-back and the soft-Gaussian kick
        if (d.gaussian || options->solver == OCTO_SOLVER_SOFT_GAUSSIAN) upload_weideman();
        upload_twiddles(c->tw_x, 2 * options->nx);
        upload_twiddles(c->tw_y, 2 * options->ny);
        if (c->fp32) {
            upload_twiddles(c->twf_x, 2 * options->nx);
            upload_twiddles(c->twf_y, 2 * options->ny);
        }
        c->gstride = (long long)(options->nx + 1) * 2 * options->ny;
        for (int b = 0; b < 2; ++b) {
            int ns = c->ns[b];
            int m = b == 0 ? options->slicing_method1 : options->slicing_method2;
            // the quantile table of :normal_quantile, the positions of :specified (the other methods use neither)
            std::vector<double> q(kMaxSlices + 1, 0.0);
            for (int s = 1; s <= ns - 1; ++s) {
                if (m == OCTO_SLICING_NORMAL_QUANTILE)
                    q[s] = std::sqrt(2.0) * erfinv_host((double)(2 * s) / (double)ns - 1.0);
                else if (m == OCTO_SLICING_SPECIFIED && (size_t)(s - 1) < c->pos[b].size())
                    q[s] = c->pos[b][s - 1];
            }
            c->bw[b].q.ensure(kMaxSlices + 1);
            CK(cudaMemcpy(c->bw[b].q.p, q.data(), sizeof(double) * q.size(), cudaMemcpyHostToDevice));
        }
        // Charge grids up to 227 KB (168 x 168 int64 cells) accumulate in shared memory; larger ones go
        // straight to the plane's grid with global atomics.
        size_t dep = (size_t)options->nx * options->ny * sizeof(long long);
        size_t lum = (size_t)(d.lnx + 1) * (d.lny + 1) * sizeof(long long);
        d.dep_global = dep > kSmemLimit;
        d.lum_global = lum > kSmemLimit;
        // The dynamic shared-memory limit is a per-kernel attribute shared by every context in the
        // process, so it is raised to the opt-in maximum once rather than to this context's sizes (a later
        // context with smaller grids must not cap an earlier one's launches).
        set_smem_limits();
    } catch (CudaFail &e) {
        c->err = e.msg;
        c->opt.nx = 0;
    }
    return c;
}

void octo_destroy(octo_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    for (auto &b : c->bw) b.release();
    c->tw_x.release(); c->tw_y.release(); c->twf_x.release(); c->twf_y.release(); c->tasks.release(); c->planes.release(); c->lumjobs.release();
    c->geom.release(); c->blockmap.release(); c->cache.release(); c->nodes.release(); c->lumgeom.release();
    c->bnd.release(); c->lumb.release(); c->nodebox_s.release(); c->nodebox_f.release(); c->nanflag.release();
    c->nodenan.release(); c->status.release(); c->ghat.release(); c->qgrid.release(); c->lq.release();
    c->spec.release(); c->fields.release(); c->lum_parts.release(); c->lum_partial.release(); c->node_ref.release(); c->stats.release();
    c->partial.release(); c->soa_ptrs.release();
    c->first_lum.release(); c->lum_tick.release(); c->cap_q.release(); c->cap_grid.release();
    c->cnn_flags.release(); c->h_cnn_flags.release(); c->cnn_q.release();
    c->hyb.release(); c->hmom.release(); c->hprof.release(); c->hsum.release(); c->qtot.release();
    c->esum.release(); c->ubox.release(); c->uflag.release(); c->slr.release();
    c->stage.release(); c->h_lum.release(); c->h_status.release(); c->h_noderef.release(); c->h_slices.release();
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->lum_stream) cudaStreamDestroy(c->lum_stream);
    drop_replay(c);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    c->rp_sig.release(); c->rp_fronts.release(); c->rp_ok.release(); c->h_rp_ok.release();
    delete c;
}

int32_t octo_pic_collide(octo_ctx *c, octo_beam *beam1, octo_beam *beam2, const octo_beam_params *p1,
                         const octo_beam_params *p2, int64_t turn, int32_t compute_luminosity, double *luminosity,
                         octo_collide_report *report, void *stream) {
    if (!c) return OCTO_ERR_ARG;
    if (report) { std::memset(report, 0, sizeof(*report)); report->turn = turn; }
    if (c->opt.nx == 0) return fail(c, OCTO_ERR_UNSUPPORTED, c->err.empty() ? "invalid context" : c->err);
    try {
        CollideJob job{c, beam1, beam2, p1, p2, turn, compute_luminosity, report, (cudaStream_t)stream};
        job.begin();
        double lum = NAN;
        bool done = false;
        if (replay_eligible(c) && replay_key_matches(c, job)) {
            // the captured collide behind its guard; the ordinary path if the guard finds another schedule
            auto &R = c->rp;
            const long long sliced = job.launches;
            job.order = R.order;
            job.batches = R.batches;
            job.ran = R.ran;
            job.tasks = R.tasks;
            job.ntasks = R.ntasks;
            job.npairs_total = R.npairs_total;
            job.launches = sliced + 1 + R.body_launches;
            // nothing an earlier (failed) collide left on the luminosity stream may overlap the graph's own
            // luminosity work, as in the ordinary path
            CK(cudaEventRecord(c->ev_join, c->lum_stream));
            CK(cudaStreamWaitEvent(job.st, c->ev_join, 0));
            CK(cudaGraphLaunch(R.exec, job.st));
            CK(cudaStreamSynchronize(job.st));
            if (*c->h_rp_ok.p) {
                R.replays++;
                // this collide's order (the guard found its wavefronts equal to the captured ones); each pair's
                // results sit in the slot of its captured position
                const SliceInfo &S1 = c->h_slices.p[0], &S2 = c->h_slices.p[1];
                job.order = collision_order(S1.center, c->ns[0], S2.center, c->ns[1]);
                job.slot.resize(job.order.size());
                for (size_t q = 0; q < job.order.size(); ++q)
                    job.slot[q] = R.pos_of[(size_t)(job.order[q].i - 1) * c->ns[1] + (job.order[q].j - 1)];
                lum = job.finish();
                done = true;
                if (report) report->replayed = 1;
            } else {
                // the guard found another schedule, or slices the graph has no room for: the ordinary path,
                // after which the next repeat of a schedule is captured afresh
                R.declined++;
                drop_replay(c);
                job.launches = sliced + 1;
                job.order.clear();
                job.slot.clear();
                job.batches.clear();
                job.ran.clear();
                job.tasks.clear();
                job.ntasks = job.npairs_total = 0;
            }
        }
        if (!done) {
            job.run();
            lum = job.finish();
            if (replay_eligible(c)) maybe_build_replay(c, job);
        }
        if (luminosity) *luminosity = lum;
        c->err.clear();
        if (report) report->status = OCTO_OK;
        return OCTO_OK;
    } catch (OctoFail &e) {
        if (report) report->status = e.code;
        return fail(c, e.code, e.msg);
    } catch (CudaFail &e) {
        if (report) report->status = OCTO_ERR_CUDA;
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
}

int32_t octo_pic_autotune(octo_ctx *c, octo_beam *beam1, octo_beam *beam2, const octo_beam_params *p1,
                          const octo_beam_params *p2, int32_t rounds, int32_t *choice, void *stream) {
    if (!c) return OCTO_ERR_ARG;
    if (rounds < 1 || rounds > 16) return fail(c, OCTO_ERR_ARG, "autotune rounds must be 1..16");
    static const int kShapes[4][2] = {{1, 1}, {2, 1}, {1, 2}, {2, 2}};  // (dep_waves, kick_slots)
    const cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best[4];
    for (double &b : best) b = 1e300;
    int32_t rc = OCTO_OK;
    try {
        CK(cudaSetDevice(c->device));
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        // one collide first (Green cache, workspaces), then every shape once per round; ordinary collides
        // only, so no graph capture is timed
        c->in_autotune = 1;
        for (int r = -1; r < rounds && rc == OCTO_OK; ++r) {
            for (int k = 0; k < 4 && rc == OCTO_OK; ++k) {
                if (r < 0 && k > 0) break;
                c->dep_waves = kShapes[k][0];
                c->kick_slots = kShapes[k][1];
                CK(cudaEventRecord(e0, st));
                double lum;
                rc = octo_pic_collide(c, beam1, beam2, p1, p2, -1, 1, &lum, nullptr, stream);
                CK(cudaEventRecord(e1, st));
                CK(cudaEventSynchronize(e1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (r >= 0) best[k] = std::min(best[k], (double)ms);
            }
        }
    } catch (CudaFail &e) {
        rc = fail(c, OCTO_ERR_CUDA, e.msg);
    }
    c->in_autotune = 0;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    int pick = 0;
    for (int k = 1; k < 4; ++k)
        if (best[k] < best[pick]) pick = k;
    if (rc != OCTO_OK) pick = 0;  // a failed collide leaves the default shape
    c->dep_waves = kShapes[pick][0];
    c->kick_slots = kShapes[pick][1];
    if (choice) *choice = pick;
    return rc;
}

int32_t octo_pic_collide_batch(int32_t count, octo_ctx *const *ctxs, octo_beam *const *beam1, octo_beam *const *beam2,
                               const octo_beam_params *const *p1, const octo_beam_params *const *p2, int64_t turn,
                               int32_t compute_luminosity, double *luminosity, octo_collide_report *reports,
                               int32_t *status, void *const *streams) {
    if (count < 0 || (count > 0 && (!ctxs || !beam1 || !beam2 || !p1 || !p2))) return OCTO_ERR_ARG;
    for (int k = 0; k < count; ++k) {
        if (!ctxs[k]) return OCTO_ERR_ARG;
        for (int m = 0; m < k; ++m)
            if (ctxs[m] == ctxs[k]) return fail(ctxs[k], OCTO_ERR_ARG, "a batch needs a distinct context per collide");
    }
    std::vector<CollideJob> jobs;
    std::vector<int32_t> rc(count, OCTO_OK);
    jobs.reserve(count);
    for (int k = 0; k < count; ++k) {
        octo_collide_report *r = reports ? reports + k : nullptr;
        if (r) { std::memset(r, 0, sizeof(*r)); r->turn = turn; }
        jobs.push_back(CollideJob{ctxs[k], beam1[k], beam2[k], p1[k], p2[k], turn, compute_luminosity, r,
                                  streams ? (cudaStream_t)streams[k] : (cudaStream_t)0});
        if (luminosity) luminosity[k] = NAN;
        if (ctxs[k]->opt.nx == 0) rc[k] = fail(ctxs[k], OCTO_ERR_UNSUPPORTED, ctxs[k]->err.empty() ? "invalid context" : ctxs[k]->err);
    }
    // Each stage of each collide runs under its own error handler, so one failing collide leaves the
    // others of the batch to complete.
    auto stage = [&](int k, int which) {
        if (rc[k] != OCTO_OK) return;
        try {
            if (which == 0) jobs[k].begin();
            else if (which == 1) jobs[k].run();
            else {
                const double lum = jobs[k].finish();
                if (luminosity) luminosity[k] = lum;
                jobs[k].c->err.clear();
            }
        } catch (OctoFail &e) {
            rc[k] = fail(jobs[k].c, e.code, e.msg);
        } catch (CudaFail &e) {
            rc[k] = fail(jobs[k].c, OCTO_ERR_CUDA, e.msg);
        }
    };
    for (int which = 0; which < 3; ++which)
        for (int k = 0; k < count; ++k) stage(k, which);
    int32_t first = OCTO_OK;
    for (int k = 0; k < count; ++k) {
        if (reports) reports[k].status = rc[k];
        if (status) status[k] = rc[k];
        if (first == OCTO_OK) first = rc[k];
    }
    return first;
}

int32_t octo_green_cache_stats(octo_ctx *c, int64_t *hits, int64_t *misses, int64_t *rebuilds) {
    if (!c) return OCTO_ERR_ARG;
    DevStatus s{};
    if (c->status.p) {
        if (cudaMemcpy(&s, c->status.p, sizeof s, cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(c, OCTO_ERR_CUDA, "reading the Green-cache counters failed");
    }
    if (hits) *hits = s.hits;
    if (misses) *misses = s.misses;
    if (rebuilds) *rebuilds = s.rebuilds;
    return OCTO_OK;
}

int64_t octo_pair_luminosity_trace(octo_ctx *c, int32_t *pi, int32_t *pj, double *lum, int64_t cap) {
    if (!c) return 0;
    int64_t n = (int64_t)c->trace_lum.size();
    for (int64_t k = 0; k < n && k < cap; ++k) {
        if (pi) pi[k] = c->trace_i[k];
        if (pj) pj[k] = c->trace_j[k];
        if (lum) lum[k] = c->trace_lum[k];
    }
    return n;
}

int32_t octo_linear6d(octo_ctx *c, octo_beam *beam, const double matrix[36], int32_t turns, void *stream) {
    if (!c || !beam || !matrix) return OCTO_ERR_ARG;
    std::string msg;
    int rc = check_beam(beam, msg, -1);
    if (rc != OCTO_OK) return fail(c, rc, msg);
    try {
        CK(cudaSetDevice(c->device));
        Mat6 M;
        for (int k = 0; k < 36; ++k) M.m[k] = matrix[k];
        with_real(beam->dtype == 1, [&](auto r) {
            using R = decltype(r);
            k_linear6d<R><<<(unsigned)((beam->n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
                (R *)beam->x, (R *)beam->px, (R *)beam->y, (R *)beam->py, (R *)beam->z, (R *)beam->pz, beam->n, M, turns);
        });
        CK(cudaGetLastError());
        return OCTO_OK;
    } catch (CudaFail &e) {
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
}

int32_t octo_track_line(octo_ctx *c, octo_beam *beam, const octo_element *elems, int32_t n_elems, int64_t turn,
                        int32_t turns, uint64_t seed, int32_t rng_method, void *stream) {
    if (!c || !beam || (n_elems > 0 && !elems)) return OCTO_ERR_ARG;
    if (n_elems < 0 || n_elems > OCTO_LINE_MAX_ELEMENTS)
        return fail(c, OCTO_ERR_ARG, "a line holds 0.." + std::to_string(OCTO_LINE_MAX_ELEMENTS) + " elements");
    if (turns < 0) return fail(c, OCTO_ERR_ARG, "turns must be non-negative");
    if (turn < 0) return fail(c, OCTO_ERR_ARG, "turn must be non-negative");
    if (rng_method != OCTO_RNG_PHILOX && rng_method != OCTO_RNG_SPLITMIX)
        return fail(c, OCTO_ERR_ARG, "unknown RNG method code; use RNG_PHILOX or RNG_SPLITMIX");
    if (beam->n < 0 || beam->n >= (1LL << 40)) return fail(c, OCTO_ERR_ARG, "beam size out of range");
    if (beam->dtype != 0 && beam->dtype != 1) return fail(c, OCTO_ERR_ARG, "beam dtype must be 0 (float64) or 1 (float32)");
    if (beam->n > 0 && (!beam->x || !beam->px || !beam->y || !beam->py || !beam->z || !beam->pz))
        return fail(c, OCTO_ERR_ARG, "beam coordinate pointer is NULL");
    std::vector<LineOp> ops((size_t)std::max(n_elems, 1));
    for (int k = 0; k < n_elems; ++k) {
        std::string msg;
        const int rc = compile_line_op(elems[k], rng_method, seed, ops[k], msg);
        if (rc != OCTO_OK) return fail(c, rc, "line element " + std::to_string(k + 1) + ": " + msg);
    }
    if (beam->n == 0 || turns == 0 || n_elems == 0) return OCTO_OK;
    cudaStream_t st = (cudaStream_t)stream;
    try {
        CK(cudaSetDevice(c->device));
        const unsigned blocks = (unsigned)((beam->n + 255) / 256);
        // One launch runs every turn when the line fits one program; a longer line runs turn by turn, its
        // programs in element order (the same per-particle sequence).
        const int nprog = (n_elems + kLineOpsPerLaunch - 1) / kLineOpsPerLaunch;
        const int outer = nprog == 1 ? 1 : turns;
        for (int t = 0; t < outer; ++t)
            for (int g = 0; g < nprog; ++g) {
                LineProgram P;
                std::memset(&P, 0, sizeof P);
                P.nops = std::min(kLineOpsPerLaunch, n_elems - g * kLineOpsPerLaunch);
                P.rng = rng_method;
                P.turns = nprog == 1 ? turns : 1;
                P.turn0 = turn + t;
                for (int k = 0; k < P.nops; ++k) P.op[k] = ops[g * kLineOpsPerLaunch + k];
                with_real(beam->dtype == 1, [&](auto r) {
                    using R = decltype(r);
                    launch_pdl(k_track_line<R>, blocks, 256, 0, st, (R *)beam->x, (R *)beam->px, (R *)beam->y,
                               (R *)beam->py, (R *)beam->z, (R *)beam->pz, (long long)beam->n, P);
                });
            }
        CK(cudaGetLastError());
        return OCTO_OK;
    } catch (CudaFail &e) {
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
}

int32_t octo_beam_moments(octo_ctx *c, const octo_beam *beam, const int32_t *powers, int32_t n_moments,
                          int32_t mask_lost, int64_t turn, double *row, void *stream) {
    if (!c || !beam || !row || (n_moments > 0 && !powers)) return OCTO_ERR_ARG;
    if (n_moments < 0 || n_moments > kMomentsMax)
        return fail(c, OCTO_ERR_ARG, "a moment row holds 0.." + std::to_string(kMomentsMax) + " moments");
    if (beam->n < 0 || beam->n >= (1LL << 40)) return fail(c, OCTO_ERR_ARG, "beam size out of range");
    if (beam->dtype != 0 && beam->dtype != 1) return fail(c, OCTO_ERR_ARG, "beam dtype must be 0 (float64) or 1 (float32)");
    if (beam->n > 0 && (!beam->x || !beam->px || !beam->y || !beam->py || !beam->z || !beam->pz))
        return fail(c, OCTO_ERR_ARG, "beam coordinate pointer is NULL");
    MomentHead head{};
    MomentPairRows pairs{};
    std::vector<int> general;  // rows of order >= 3
    unsigned mean_seen = 0, pair_seen = 0;
    for (int k = 0; k < n_moments; ++k) {
        int order = 0, coord = -1, second = -1;
        for (int d = 0; d < 6; ++d) {
            const int p = powers[6 * k + d];
            if (p < 0 || p > 32) return fail(c, OCTO_ERR_ARG, "moment powers must be integers in 0..32");
            order += p;
            if (p && coord < 0) coord = d;
            if (p == 2) second = d;
            else if (p == 1 && coord != d) second = d;
        }
        if (order == 0) return fail(c, OCTO_ERR_ARG, "a moment needs a positive order");
        if (order == 1) {
            if (mean_seen & (1u << coord)) return fail(c, OCTO_ERR_ARG, "a moment row holds each mean once");
            mean_seen |= 1u << coord;
            head.slot[head.n] = (unsigned char)k;
            head.coord[head.n] = (unsigned char)coord;
            ++head.n;
        } else if (order == 2) {
            // (coord, second) with coord <= second; pair index over the upper triangle, row-major
            const int a = coord, b = second;
            const int pidx = a * 6 - a * (a - 1) / 2 + (b - a);
            if (pair_seen & (1u << pidx)) return fail(c, OCTO_ERR_ARG, "a moment row holds each second moment once");
            pair_seen |= 1u << pidx;
            pairs.pair[pairs.n] = (unsigned char)pidx;
            pairs.slot[pairs.n] = (unsigned char)k;
            ++pairs.n;
        } else {
            general.push_back(k);
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    try {
        CK(cudaSetDevice(c->device));
        c->mom_partial.ensure((size_t)kMomentBlocks * kMomentPairs);
        c->mom_means.ensure(16);
        const long long n = beam->n;
        const int mask = mask_lost != 0;
        with_real(beam->dtype == 1, [&](auto r) {
            using R = decltype(r);
            R *b[6] = {(R *)beam->x, (R *)beam->px, (R *)beam->y, (R *)beam->py, (R *)beam->z, (R *)beam->pz};
            const double *means = c->mom_means.p;
            launch_pdl(k_moment_sums<R>, kMomentBlocks, kMomentThreads, 0, st, b[0], b[1], b[2], b[3], b[4], b[5], n,
                       mask, c->mom_partial.p);
            launch_pdl(k_moment_means, 7, kMomentThreads, 0, st, (const double *)c->mom_partial.p, (int)kMomentBlocks,
                       c->mom_means.p);
            launch_pdl(k_moment_divide, 1, 32, 0, st, c->mom_means.p);
            launch_pdl(k_moment_row_head, 1, 32, 0, st, means, (double)turn, head, row);
            if (pairs.n) {
                launch_pdl(k_moment_pairs<R>, kMomentBlocks, kMomentThreads, 0, st, b[0], b[1], b[2], b[3], b[4],
                           b[5], n, mask, means, c->mom_partial.p);
                launch_pdl(k_moment_fold_pairs, pairs.n, kMomentThreads, 0, st, (const double *)c->mom_partial.p,
                           (int)kMomentBlocks, means, pairs, row);
            }
            for (size_t g0 = 0; g0 < general.size(); g0 += kMomentChunk) {
                MomentPowers P{};
                P.n = (int)std::min<size_t>(kMomentChunk, general.size() - g0);
                for (int k = 0; k < P.n; ++k) {
                    for (int d = 0; d < 6; ++d) P.p[k][d] = (unsigned char)powers[6 * general[g0 + k] + d];
                    P.slot[k] = (unsigned char)general[g0 + k];
                }
                launch_pdl(k_moment_general<R>, kMomentBlocks, kMomentThreads, 0, st, b[0], b[1], b[2], b[3], b[4],
                           b[5], n, mask, means, P, c->mom_partial.p);
                launch_pdl(k_moment_fold, P.n, kMomentThreads, 0, st, (const double *)c->mom_partial.p,
                           (int)kMomentBlocks, means, P, row);
            }
        });
        CK(cudaGetLastError());
        return OCTO_OK;
    } catch (CudaFail &e) {
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
}

int32_t octo_beam_gaussian(octo_ctx *c, octo_beam *beam, uint64_t seed, uint64_t rng_id, const double beta[3],
                           const double alpha[3], const double sigma[3], double cutoff, void *stream) {
    if (!c || !beam || !beta || !alpha || !sigma) return OCTO_ERR_ARG;
    std::string msg;
    int rc = check_beam(beam, msg);
    if (rc != OCTO_OK) return fail(c, rc, msg);
    cudaStream_t st = (cudaStream_t)stream;
    try {
        CK(cudaSetDevice(c->device));
        const long long n = beam->n;
        double *comp[6] = {(double *)beam->x, (double *)beam->px, (double *)beam->y, (double *)beam->py,
                           (double *)beam->z, (double *)beam->pz};
        const int nb = 256;
        c->partial.ensure(nb);
        c->stats.ensure(kMaxSlices * 2);
        double *stats = c->stats.p;
        for (int d = 0; d < 6; ++d) {
            k_beam_normals<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(comp[d], n, seed, rng_id, d + 1, cutoff);
            k_partial_sum<<<nb, 256, 0, st>>>(comp[d], n, stats, 0, c->partial.p);
            k_fold_partials<<<1, 1, 0, st>>>(c->partial.p, nb, n, 0, stats);
            k_partial_sum<<<nb, 256, 0, st>>>(comp[d], n, stats, 1, c->partial.p);
            k_fold_partials<<<1, 1, 0, st>>>(c->partial.p, nb, n, 1, stats);
            k_standardize<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(comp[d], n, stats);
        }
        for (int a = 0; a < 3; ++a)
            k_twiss<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(comp[2 * a], comp[2 * a + 1], n, sigma[a], beta[a], alpha[a]);
        CK(cudaGetLastError());
        return OCTO_OK;
    } catch (CudaFail &e) {
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
}

int32_t octo_set_collide_graph(octo_ctx *c, int32_t enable) {
    if (!c) return OCTO_ERR_ARG;
    if (enable != 0 && enable != 1) return fail(c, OCTO_ERR_ARG, "collide graph setting must be 0 or 1");
    try {
        CK(cudaSetDevice(c->device));
        CK(cudaDeviceSynchronize());
    } catch (CudaFail &e) {
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
    drop_replay(c);
    c->rp.enabled = enable;
    c->rp.failures = 0;
    c->rp.last_sig.clear();
    return OCTO_OK;
}

int32_t octo_collide_graph_stats(octo_ctx *c, int64_t out[4]) {
    if (!c || !out) return OCTO_ERR_ARG;
    out[0] = c->rp.builds;
    out[1] = c->rp.replays;
    out[2] = c->rp.declined;
    out[3] = c->rp.failures;
    return OCTO_OK;
}

int32_t octo_set_particle_order(octo_ctx *c, int32_t order) {
    if (!c || (order != 0 && order != 1)) return OCTO_ERR_ARG;
    c->spatial = order;
    return OCTO_OK;
}

int32_t octo_set_field_correction(octo_ctx *c, octo_cnn *net, float out_scale, float tolerance, int32_t edge) {
    if (!c) return OCTO_ERR_ARG;
    if (!net) {
        c->cnn = nullptr;
        return OCTO_OK;
    }
    if (c->opt.solver != OCTO_SOLVER_PIC || c->opt.interaction_grid != OCTO_GRID_SLICE_PAIR ||
        c->opt.slice_interpolation != 0 || c->opt.green_cache != OCTO_CACHE_NONE ||
        c->opt.green_type != OCTO_GREEN_INTEGRATED)
        return fail(c, OCTO_ERR_UNSUPPORTED,
                    "the learned field correction runs on a PIC (or Gaussian-subtracted hybrid) collide with "
                    ":slice_pair grids, linear slice interpolation, the :integrated Green function and "
                    "green_cache = :none (so every field mesh is its source mesh shifted by whole cells)");
    if (net->net.H != c->opt.ny || net->net.W != c->opt.nx)
        return fail(c, OCTO_ERR_ARG, "the network's height x width must equal the solver grid's ny x nx");
    if (net->net.device != c->device) return fail(c, OCTO_ERR_ARG, "the network lives on another device");
    if (!(out_scale > 0.f) || !(tolerance > 0.f) || edge < 0 || 2 * edge >= std::min(c->opt.nx, c->opt.ny))
        return fail(c, OCTO_ERR_ARG, "out_scale and tolerance must be positive and edge below half the grid");
    c->cnn = net;
    c->cnn_scale = out_scale;
    c->cnn_tol = tolerance;
    c->cnn_edge = edge;
    return OCTO_OK;
}

int32_t octo_field_correction_report(octo_ctx *c, int32_t *planes_over_tolerance) {
    if (!c || !planes_over_tolerance) return OCTO_ERR_ARG;
    if (!c->cnn || !c->cnn_flags.p) { *planes_over_tolerance = 0; return OCTO_OK; }
    try {
        CK(cudaSetDevice(c->device));
        c->h_cnn_flags.ensure(1);
        CK(cudaMemcpy(c->h_cnn_flags.p, c->cnn_flags.p, sizeof(int), cudaMemcpyDeviceToHost));
        *planes_over_tolerance = c->h_cnn_flags.p[0];
        return OCTO_OK;
    } catch (CudaFail &e) {
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
}

int32_t octo_capture_charge_plane(octo_ctx *c, int32_t pair_i, int32_t pair_j, int32_t direction, int32_t plane) {
    if (!c) return OCTO_ERR_ARG;
    if (pair_i < 1 || pair_j < 1 || (direction != 1 && direction != 2) || plane < 0 || plane > 2)
        return fail(c, OCTO_ERR_ARG, "capture: pair indices are 1-based, direction 1 or 2, plane 0..2");
    c->cap_armed = 1;
    c->cap_taken = 0;
    c->cap_i = pair_i; c->cap_j = pair_j; c->cap_dir = direction; c->cap_kind = plane;
    return OCTO_OK;
}

int32_t octo_captured_charge_plane(octo_ctx *c, int64_t *grid, double mesh[4], double field_mesh[4],
                                   int32_t *fixed_bits) {
    if (!c || !grid || !mesh || !fixed_bits) return OCTO_ERR_ARG;
    if (!c->cap_armed || !c->cap_taken)
        return fail(c, OCTO_ERR_ARG, "capture: no charge plane was captured (not armed, or the pair did not run)");
    try {
        CK(cudaSetDevice(c->device));
        CK(cudaDeviceSynchronize());
        Grid g[2]{};
        CK(cudaMemcpy(grid, c->cap_q.p, sizeof(long long) * (size_t)c->opt.nx * c->opt.ny, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(g, c->cap_grid.p, 2 * sizeof(Grid), cudaMemcpyDeviceToHost));
        mesh[0] = g[0].x0; mesh[1] = g[0].y0; mesh[2] = g[0].w; mesh[3] = g[0].h;
        if (field_mesh) { field_mesh[0] = g[1].x0; field_mesh[1] = g[1].y0; field_mesh[2] = g[1].w; field_mesh[3] = g[1].h; }
        *fixed_bits = c->cap_bits;
        c->cap_armed = 0;
        c->cap_taken = 0;
        return OCTO_OK;
    } catch (CudaFail &e) {
        return fail(c, OCTO_ERR_CUDA, e.msg);
    }
}

int32_t octo_set_timing_phases(octo_ctx *c, uint32_t mask) {
    if (!c) return OCTO_ERR_ARG;
    c->timing_mask = mask;
    return OCTO_OK;
}

int32_t octo_set_timing(octo_ctx *c, int32_t enable) {
    if (!c) return OCTO_ERR_ARG;
    c->timing = enable ? 1 : 0;
    for (int k = 0; k < OCTO_NPHASES; ++k) { c->phase_ms[k] = 0; c->phase_launches[k] = 0; c->phase_bytes[k] = 0; }
    c->ev_marks.clear();
    c->ev_used = 0;
    return OCTO_OK;
}

int32_t octo_timing_report(octo_ctx *c, double ms[OCTO_NPHASES], int64_t launches[OCTO_NPHASES],
                           double bytes[OCTO_NPHASES]) {
    if (!c) return OCTO_ERR_ARG;
    for (int k = 0; k < OCTO_NPHASES; ++k) {
        if (ms) ms[k] = c->phase_ms[k];
        if (launches) launches[k] = c->phase_launches[k];
        if (bytes) bytes[k] = c->phase_bytes[k];
    }
    return OCTO_OK;
}

}  // extern "C"

namespace {
// Device status word of the tensor-core kernels (set to OCTO_ERR_TIMEOUT by a wait that gave up), one per
// device, allocated on first use.
int *nn_error_flag() {
    static std::mutex mu;
    static int *flag[64] = {nullptr};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (!flag[dev]) CK(cudaMalloc(&flag[dev], sizeof(int)));
    return flag[dev];
}
}  // namespace


// ---------------------------------------------------------------- allocation-free beam construction
// Reduction scratch of octo_beam_gaussian_noalloc: OCTO_NOALLOC_MAX_BLOCKS block partial sums followed
// by the mean and sigma slots.  4096 doubles = 32 KiB, resident on every device that loads the library.
static __device__ __align__(256) double g_noalloc_scratch[OCTO_NOALLOC_MAX_BLOCKS + 2];

namespace {
constexpr int kNoallocMaxDevices = 64;
// Device address of g_noalloc_scratch per device and context (see noalloc_cache.h): looked up with the
// device current, and again whenever the device's current context is not the one it was looked up in.
SymbolAddressCache<kNoallocMaxDevices> g_noalloc_addr;

// cuCtxGetCurrent / cuCtxSetCurrent, resolved through the runtime so the library needs no link against the
// driver library.  Both take and return the driver's context handle as an opaque pointer.
using CtxGetFn = int (*)(void **);
using CtxSetFn = int (*)(void *);
struct DriverCtxFns {
    CtxGetFn get = nullptr;
    CtxSetFn set = nullptr;
};
const DriverCtxFns &driver_ctx_fns() {
    static DriverCtxFns f = [] {
        DriverCtxFns r;
        void *g = nullptr, *s = nullptr;
        cudaDriverEntryPointQueryResult qg{}, qs{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &g, cudaEnableDefault, &qg) == cudaSuccess &&
            qg == cudaDriverEntryPointSuccess && g)
            r.get = (CtxGetFn)g;
        if (cudaGetDriverEntryPoint("cuCtxSetCurrent", &s, cudaEnableDefault, &qs) == cudaSuccess &&
            qs == cudaDriverEntryPointSuccess && s)
            r.set = (CtxSetFn)s;
        return r;
    }();
    return f;
}

// Saves the calling thread's current CUDA context on entry and makes it current again on every return
// path, so a host that tracks its own current device (CUDA.jl, PyTorch) sees it unchanged after the call.
struct CurrentContextGuard {
    void *saved = nullptr;
    int saved_device = -1;
    bool have_ctx = false;
    CurrentContextGuard() {
        const DriverCtxFns &f = driver_ctx_fns();
        if (f.get && f.set && f.get(&saved) == 0) have_ctx = true;
        else if (cudaGetDevice(&saved_device) != cudaSuccess) saved_device = -1;
    }
    ~CurrentContextGuard() {
        if (have_ctx) driver_ctx_fns().set(saved);
        else if (saved_device >= 0) cudaSetDevice(saved_device);
    }
};

void noalloc_message(char *err, int64_t len, const std::string &m) {
    if (!err || len <= 0) return;
    size_t n = std::min<size_t>(m.size(), (size_t)len - 1);
    std::memcpy(err, m.data(), n);
    err[n] = 0;
}
}  // namespace

extern "C" {

int32_t octo_beam_gaussian_noalloc(int32_t device, octo_beam *beam, uint64_t seed, uint64_t rng_id,
                                   const double beta[3], const double alpha[3], const double sigma[3], double cutoff,
                                   void *stream, char *err, int64_t err_len) {
    if (!beam || !beta || !alpha || !sigma) {
        noalloc_message(err, err_len, "beam, beta, alpha and sigma must be non-NULL");
        return OCTO_ERR_ARG;
    }
    std::string msg;
    int rc = check_beam(beam, msg);
    if (rc != OCTO_OK) {
        noalloc_message(err, err_len, msg);
        return rc;
    }
    if (beam->n > (int64_t)OCTO_NOALLOC_MAX_PARTICLES) {
        noalloc_message(err, err_len, "octo_beam_gaussian_noalloc: " + std::to_string(beam->n) +
                                          " particles exceed its fixed scratch limit of " +
                                          std::to_string((long long)OCTO_NOALLOC_MAX_PARTICLES) +
                                          "; use octo_beam_gaussian with a context");
        return OCTO_ERR_ARG;
    }
    if (device < 0 || device >= kNoallocMaxDevices) {
        noalloc_message(err, err_len, "device index out of range");
        return OCTO_ERR_ARG;
    }
    CurrentContextGuard restore_caller_context;
    if (cudaSetDevice(device) != cudaSuccess) {
        noalloc_message(err, err_len, "cudaSetDevice failed");
        return OCTO_ERR_CUDA;
    }
    // the device's current context keys the cached address: a reset device gets a new context, whose
    // module (and scratch array) is looked up again.  cudaSetDevice made the primary context current.
    void *ctx = nullptr;
    if (driver_ctx_fns().get) driver_ctx_fns().get(&ctx);
    cudaError_t lookup_err = cudaSuccess;
    double *scratch = (double *)g_noalloc_addr.lookup(device, ctx, [&]() -> void * {
        void *p = nullptr;
        lookup_err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        return lookup_err == cudaSuccess ? p : nullptr;
    });
    if (!scratch) {
        noalloc_message(err, err_len, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(lookup_err));
        return OCTO_ERR_CUDA;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const long long n = beam->n;
    const int nb = (int)std::max<long long>(1, (n + OCTO_NOALLOC_PARTICLES_PER_BLOCK - 1) / OCTO_NOALLOC_PARTICLES_PER_BLOCK);
    double *partial = scratch;                         // nb entries, every one rewritten each pass
    double *stats = scratch + OCTO_NOALLOC_MAX_BLOCKS;  // mean, sigma: written by the folds before use
    double *comp[6] = {(double *)beam->x, (double *)beam->px, (double *)beam->y, (double *)beam->py,
                       (double *)beam->z, (double *)beam->pz};
    const unsigned grid = (unsigned)((n + 255) / 256);
    for (int d = 0; d < 6; ++d) {
        k_beam_normals<<<grid, 256, 0, st>>>(comp[d], n, seed, rng_id, d + 1, cutoff);
        k_partial_sum<<<nb, 256, 0, st>>>(comp[d], n, stats, 0, partial);
        k_fold_partials<<<1, 1, 0, st>>>(partial, nb, n, 0, stats);
        k_partial_sum<<<nb, 256, 0, st>>>(comp[d], n, stats, 1, partial);
        k_fold_partials<<<1, 1, 0, st>>>(partial, nb, n, 1, stats);
        k_standardize<<<grid, 256, 0, st>>>(comp[d], n, stats);
    }
    for (int a = 0; a < 3; ++a)
        k_twiss<<<grid, 256, 0, st>>>(comp[2 * a], comp[2 * a + 1], n, sigma[a], beta[a], alpha[a]);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        noalloc_message(err, err_len, std::string("kernel launch failed: ") + cudaGetErrorString(e));
        return OCTO_ERR_CUDA;
    }
    return OCTO_OK;
}

octo_cnn *octo_cnn_create(int32_t device, int32_t height, int32_t width, int32_t max_batch, uint64_t seed) {
    if (height < 16 || width < 16 || height % 8 || width % 8 || max_batch < 1) return nullptr;
    if ((long long)max_batch * height * width * 64 >= (1LL << 31)) return nullptr;
    octo_cnn *c = new octo_cnn();
    try {
        c->net.create(device, height, width, max_batch, seed);
        CK(cudaDeviceSynchronize());
    } catch (CudaFail &) {
        c->net.release();
        delete c;
        return nullptr;
    }
    return c;
}

void octo_cnn_destroy(octo_cnn *c) {
    if (!c) return;
    cudaSetDevice(c->net.device);
    cudaDeviceSynchronize();
    c->net.release();
    delete c;
}

int64_t octo_cnn_num_params(const octo_cnn *c) { return c ? c->net.nparams : 0; }

int32_t octo_cnn_get_params(octo_cnn *c, float *params, int64_t n) {
    if (!c || !params || n != c->net.nparams) return OCTO_ERR_ARG;
    try {
        CK(cudaSetDevice(c->net.device));
        CK(cudaDeviceSynchronize());
        CK(cudaMemcpy(params, c->net.master.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
        return OCTO_OK;
    } catch (CudaFail &e) {
        c->err = e.msg;
        return OCTO_ERR_CUDA;
    }
}

int32_t octo_cnn_set_params(octo_cnn *c, const float *params, int64_t n) {
    if (!c || !params || n != c->net.nparams) return OCTO_ERR_ARG;
    try {
        CK(cudaSetDevice(c->net.device));
        CK(cudaDeviceSynchronize());
        CK(cudaMemcpy(c->net.master.p, params, sizeof(float) * n, cudaMemcpyHostToDevice));
        c->net.weights_dirty = true;
        return OCTO_OK;
    } catch (CudaFail &e) {
        c->err = e.msg;
        return OCTO_ERR_CUDA;
    }
}

namespace {
int cnn_status(octo_cnn *c, cudaStream_t st) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, c->net.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (e) {
        CK(cudaMemsetAsync(c->net.err, 0, sizeof(int), st));
        c->err = "a tensor-core wait gave up";
        return OCTO_ERR_TIMEOUT;
    }
    return OCTO_OK;
}
}  // namespace

int32_t octo_cnn_forward(octo_cnn *c, const void *input, int32_t batch, float *output, void *stream) {
    if (!c || !input || !output || batch < 1 || batch > c->net.maxB) return OCTO_ERR_ARG;
    try {
        nn::Cnn &N = c->net;
        CK(cudaSetDevice(N.device));
        cudaStream_t st = (cudaStream_t)stream;
        const long long M0 = N.ml(0, batch);
        CK(cudaMemcpyAsync(N.x0.p, input, sizeof(nn::bf16) * M0 * nn::kCnnIn, cudaMemcpyDeviceToDevice, st));
        N.forward(batch, st, false);
        // channels 0 and 1 of the head
        CK(cudaMemcpy2DAsync(output, 2 * sizeof(float), N.out.p, 8 * sizeof(float), 2 * sizeof(float), (size_t)M0,
                             cudaMemcpyDeviceToDevice, st));
        return cnn_status(c, st);
    } catch (CudaFail &e) {
        c->err = e.msg;
        return OCTO_ERR_CUDA;
    }
}

int32_t octo_cnn_train_step(octo_cnn *c, const void *input, const float *target, const float *mask, int32_t batch,
                            float lr, int32_t update, double *loss, float *grads, void *stream) {
    if (!c || !input || !target || batch < 1 || batch > c->net.maxB) return OCTO_ERR_ARG;
    try {
        nn::Cnn &N = c->net;
        CK(cudaSetDevice(N.device));
        cudaStream_t st = (cudaStream_t)stream;
        const long long M0 = N.ml(0, batch);
        double wt = (double)M0;
        if (mask) {  // the loss is normalised by the total weight
            std::vector<float> hm((size_t)M0);
            CK(cudaMemcpyAsync(hm.data(), mask, sizeof(float) * M0, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            wt = 0.0;
            for (float v : hm) wt += v;
        }
        CK(cudaMemcpyAsync(N.x0.p, input, sizeof(nn::bf16) * M0 * nn::kCnnIn, cudaMemcpyDeviceToDevice, st));
        N.forward(batch, st);
        const int nblk = N.backward(batch, target, mask, wt, st);
        if (loss) {
            CK(cudaMemcpyAsync(N.h_loss.p, N.loss_part.p, sizeof(double) * 2 * nblk, cudaMemcpyDeviceToHost, st));
        }
        if (grads) CK(cudaMemcpyAsync(grads, N.grad.p, sizeof(float) * N.nparams, cudaMemcpyDeviceToHost, st));
        if (update) N.adam(lr, st);
        const int rc = cnn_status(c, st);
        if (loss) {
            double se = 0.0;
            for (int b = 0; b < nblk; ++b) se += N.h_loss.p[2 * b];
            *loss = se / (2.0 * std::max(wt, 1e-300));
        }
        return rc;
    } catch (CudaFail &e) {
        c->err = e.msg;
        return OCTO_ERR_CUDA;
    }
}

int32_t octo_gemm_bf16(int32_t device, const octo_gemm_desc *d, void *stream) {
    if (!d || !d->A || !d->B || (!d->out && !d->out_bf16)) return OCTO_ERR_ARG;
    if (d->M < 1 || d->N < 1 || d->K < 8 || d->K % 8 || d->splits < 1) return OCTO_ERR_ARG;
    if (d->a_mode == 1 && (d->C < 8 || d->C % 8 || d->K != 9 * d->C || d->M % (d->H * d->W))) return OCTO_ERR_ARG;
    if (d->a_mode == 0 && (d->lda % 8 || ((uintptr_t)d->A & 15))) return OCTO_ERR_ARG;
    if (d->ldb % 8 || ((uintptr_t)d->B & 15)) return OCTO_ERR_ARG;
    if (d->out_bf16 && d->splits != 1) return OCTO_ERR_ARG;
    try {
        CK(cudaSetDevice(device));
        nn::GemmArgs g{};
        g.M = d->M; g.N = d->N; g.K = d->K;
        g.A = (const __nv_bfloat16 *)d->A; g.lda = d->lda; g.a_mode = d->a_mode;
        g.H = d->H; g.W = d->W; g.C = d->C;
        g.B = (const __nv_bfloat16 *)d->B; g.ldb = d->ldb;
        g.out = d->out; g.ldc = d->ldc; g.split_stride = (long long)d->M * d->ldc;
        const int kchunks = (d->K + nn::kBK - 1) / nn::kBK;
        g.k_per_split = ((kchunks + d->splits - 1) / d->splits) * nn::kBK;
        g.bias = d->bias; g.relu = d->relu; g.out_bf16 = (__nv_bfloat16 *)d->out_bf16; g.ldo = d->ldo;
        g.error = nn_error_flag();
        cudaStream_t st = (cudaStream_t)stream;
        CK(cudaMemsetAsync(g.error, 0, sizeof(int), st));
        nn::launch_gemm(g, d->splits, st);
        int e = 0;
        CK(cudaMemcpyAsync(&e, g.error, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return e ? OCTO_ERR_TIMEOUT : OCTO_OK;
    } catch (CudaFail &) {
        return OCTO_ERR_CUDA;
    }
}

int32_t octo_last_error(octo_ctx *c, char *buf, int64_t len) {
    if (!c || !buf || len <= 0) return OCTO_ERR_ARG;
    size_t n = std::min<size_t>(c->err.size(), (size_t)len - 1);
    std::memcpy(buf, c->err.data(), n);
    buf[n] = 0;
    return OCTO_OK;
}

}  // extern "C"
