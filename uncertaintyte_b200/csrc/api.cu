// api.cu - C ABI of libuncte.so: validation, workspace planning and the
// orchestration of the covariance pipeline on one CUDA stream.
//
// Replaces computeCovariances (compute.cpp:458-540). Host code; every
// arithmetic step runs in the kernels of assembly.cu / dense.cu / points.cu.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/uncte.h"
#include "internal.h"
#include "pipeline.h"

namespace unc {
thread_local std::string g_last_error;
long long g_launches = 0;
thread_local long long g_thread_launches = 0;

int device_sms() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148;
    }
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
        cudaGetLastError();
        v = 148;
    }
    cache[dev].store(v, std::memory_order_relaxed);
    return v;
}
}  // namespace unc

using namespace unc;

using GraphKey = std::array<unsigned long long, 8>;
struct StageGraph {
    GraphKey key{};
    cudaGraphExec_t exec = nullptr;
    size_t npev = 0;          // profiling events recorded by the stage
    long long launches = 0;   // kernels the stage launches (added to the counter on every replay)
};

struct unc_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    void* mp = nullptr;   // int8 slice planes of the mixed-precision products
    size_t mp_bytes = 0;
    void* jac = nullptr;  // unc_compute_scene: scene inputs, the generated CRS Jacobian, outputs
    size_t jac_bytes = 0;
    // pinned staging ring for copies of ordinary (pageable) host memory
    // (allocated at the first such copy, freed with the context)
    char* stage = nullptr;
    cudaEvent_t stage_ev[16] = {};
    bool stage_used[16] = {};
    cudaEvent_t ev[12] = {};
    int priority = 0;  // of `stream` (0: the default priority)
    int sm_count = 148;  // of `device`
    // grid bound of the tile-task inverse: a server running requests side by side
    // lowers it, so that one request's persistent kernel (its CTAs wait on
    // dependencies in place) leaves SMs to the other requests' kernels
    int task_ctas = 148;  // set to the device's SM count at creation
    // dense-stage graphs: a stage seen twice with the same key is captured and
    // replayed (kStageGraphs most recent kept)
    std::vector<StageGraph> graphs;
    std::vector<GraphKey> seen;
    // profiling of the Taylor-series products
    bool prof = false;
    std::vector<cudaEvent_t> pev;
    long long prof_launches = 0;
    double prof_seconds = 0, prof_flops = 0, prof_int8_ops = 0;
};

namespace unc {
// (declared in internal.h)
void context_set_task_ctas(unc_context* c, int max_ctas) {
    if (c) c->task_ctas = std::max(1, std::min(c->sm_count, max_ctas));
}
}  // namespace unc

namespace {

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
            return e_ == cudaErrorMemoryAllocation ? UNC_ERR_OUT_OF_MEMORY : UNC_ERR_CUDA;        \
        }                                                                                         \
    } while (0)

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace

namespace unc {

// Lay out the workspace; with base == nullptr only the size is computed.
size_t carve(char* base, const Plan& pl, bool host_io, long long nnz, int nrows, Buffers& b) {
    Carver c{base};
    memset(&b, 0, sizeof(b));
    if (host_io) {
        b.rows = c.take<int>((size_t)nrows + 1);
        b.cols = c.take<int>((size_t)nnz);
        b.vals = c.take<double>((size_t)nnz);
        b.cam_out = c.take<double>((size_t)pl.C * 45);
        b.pt_out = c.take<double>((size_t)pl.P * 6);
    }
    SceneDev& s = b.s;
    s.obs_cam = c.take<int>(pl.nobs);
    s.obs_pt = c.take<int>(pl.nobs);
    s.cam_ptr = c.take<int>((size_t)pl.C + 1);
    s.cam_obs = c.take<int>(pl.nobs);
    s.pt_ptr = c.take<int>((size_t)pl.P + 1);
    s.pt_obs = c.take<int>(pl.nobs);
    s.cursor = c.take<int>((size_t)pl.C + pl.P + 1);
    s.scan_tmp = c.take<int>(scan_tmp_ints(std::max(pl.C, pl.P)));
    s.s_cam = c.take<double>((size_t)pl.C * 9);
    s.s_pt = c.take<double>((size_t)pl.P * 3);
    s.Vraw = c.take<double>((size_t)pl.P * 6);
    s.iVs = c.take<double>((size_t)pl.P * 6);
    s.Ws = c.take<double>((size_t)pl.nobs * 27);
    s.Ys = c.take<double>((size_t)pl.nobs * 27);
    s.cam_part = c.take<double>(45 * camera_tile_slots(pl.C, pl.nobs));
    s.Ucam = c.take<double>(81 * (size_t)pl.C);
    s.err = c.take<int>(4);
    b.amax = c.take<unsigned long long>(4);
    b.te = c.take<TeState>(1);
    const size_t nn = (size_t)pl.ld * pl.N;
    b.Z = c.take<double>(nn);
    b.iZ = c.take<double>(nn);
    b.add = c.take<double>(nn);
    b.tmp = c.take<double>(nn);
    b.p4 = c.take<double>(nn);
    b.p8 = c.take<double>(nn);
    b.p12 = c.take<double>(nn);
    b.p16 = c.take<double>(nn);
    b.g = c.take<double>(nn);
    b.dmax = c.take<unsigned long long>(24);
    b.e = c.take<double>(pl.N);
    b.gjws = c.take<double>(chol_small_doubles(pl.N));
    b.dag_state = c.take<int>(spd_task_state_ints(pl.N));
    b.sig = c.take<double>((size_t)pl.C * 81);
    if (pl.svd_schur) {
        const size_t used = (c.off + 255) & ~size_t(255);
        return used + pinv_carve(base ? base + used : nullptr, pl.N, pl.ld, b.pb);
    }
    return c.off + 256;
}

// Grow-only context buffer, allocated in stream order on the call's stream:
// several contexts (one per host thread) can run concurrently on one GPU, and
// a cudaFree would synchronise the whole device under all of them. Every call
// ends with a stream synchronisation, so the old buffer is idle when freed.
int grow_buffer(void** p, size_t* have, size_t need, size_t want, cudaStream_t sm) {
    if (*have >= need) return UNC_OK;
    if (*p) CK(cudaFreeAsync(*p, sm));
    *p = nullptr;
    *have = 0;
    CK(cudaMallocAsync(p, want, sm));
    *have = want;
    return UNC_OK;
}

int ensure_ws(unc_context* ctx, size_t bytes, cudaStream_t sm) {
    return grow_buffer(&ctx->ws, &ctx->ws_bytes, bytes, bytes, sm);
}

// Copies between the caller's host arrays and the device. A copy from page-
// locked (pinned or registered) memory goes to the copy engine directly. A
// copy of ordinary pageable memory of kStageMin bytes or more is staged: host
// threads copy kStageChunk pieces into a pinned ring owned by the context and
// each piece is sent from there as soon as it is in, so that the host copies
// run side by side and overlap the transfers (the driver's own path for
// pageable memory is one host thread through small bounce buffers). Each ring
// slot belongs to one thread during a call and is reused only after the
// transfer recorded on its event has completed.
constexpr int kStageSlots = 16;
constexpr size_t kStageChunk = 4u << 20;
constexpr size_t kStageMin = 8u << 20;

struct HostCopy {
    void* dst;
    const void* src;
    size_t bytes;
};

bool is_pageable(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

int ensure_stage(unc_context* ctx) {
    if (ctx->stage) return UNC_OK;
    CK(cudaHostAlloc((void**)&ctx->stage, kStageSlots * kStageChunk, cudaHostAllocDefault));
    for (int i = 0; i < kStageSlots; ++i) {
        CK(cudaEventCreateWithFlags(&ctx->stage_ev[i], cudaEventDisableTiming));
        ctx->stage_used[i] = false;
    }
    return UNC_OK;
}

// to_device: host -> device (returns once every piece is queued on sm);
// otherwise device -> host (returns once every piece has arrived in host memory).
int copy_host(unc_context* ctx, const std::vector<HostCopy>& jobs, bool to_device, cudaStream_t sm) {
    const cudaMemcpyKind kind = to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    struct Piece {
        char* dst;
        const char* src;
        size_t n;
    };
    std::vector<Piece> pieces;
    for (const HostCopy& j : jobs) {
        if (!j.bytes) continue;
        const void* host = to_device ? j.src : j.dst;
        if (j.bytes < kStageMin || !is_pageable(host)) {
            CK(cudaMemcpyAsync(j.dst, j.src, j.bytes, kind, sm));
            continue;
        }
        for (size_t o = 0; o < j.bytes; o += kStageChunk)
            pieces.push_back({(char*)j.dst + o, (const char*)j.src + o, std::min(kStageChunk, j.bytes - o)});
    }
    if (pieces.empty()) return UNC_OK;
    if (int r = ensure_stage(ctx)) return r;
    const int hw = (int)std::max(2u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min({kStageSlots / 2, (int)pieces.size(), hw / 2}));
    std::vector<cudaError_t> failed(nt, cudaSuccess);
    auto run = [&](int t) {
        cudaError_t& e = failed[t];
        if ((e = cudaSetDevice(ctx->device)) != cudaSuccess) return;
        for (size_t c = t, m = 0; c < pieces.size(); c += nt, ++m) {
            const int slot = t + nt * (int)(m & 1);  // two slots per thread, alternating
            char* buf = ctx->stage + (size_t)slot * kStageChunk;
            if (ctx->stage_used[slot] && (e = cudaEventSynchronize(ctx->stage_ev[slot])) != cudaSuccess) return;
            const Piece& p = pieces[c];
            if (to_device) memcpy(buf, p.src, p.n);
            e = to_device ? cudaMemcpyAsync(p.dst, buf, p.n, kind, sm) : cudaMemcpyAsync(buf, p.src, p.n, kind, sm);
            if (e != cudaSuccess || (e = cudaEventRecord(ctx->stage_ev[slot], sm)) != cudaSuccess) return;
            ctx->stage_used[slot] = true;
            if (!to_device) {
                if ((e = cudaEventSynchronize(ctx->stage_ev[slot])) != cudaSuccess) return;
                memcpy(p.dst, buf, p.n);
            }
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(run, t);
    run(0);
    for (auto& x : th) x.join();
    for (cudaError_t e : failed)
        if (e != cudaSuccess) return fail(UNC_ERR_CUDA, std::string("staged host copy: ") + cudaGetErrorString(e));
    return UNC_OK;
}

int check_options(const unc_options* o, int num_rows, int num_cols) {
    if (!o) return fail(UNC_ERR_INVALID_ARG, "options is NULL");
    if (o->num_cams <= 0 || o->num_points < 0 || num_rows < 0 || (num_rows & 1))
        return fail(UNC_ERR_INVALID_ARG, "invalid sizes (num_cams > 0, num_points >= 0, even num_rows)");
    if (o->cam_params != kCamParams)
        return fail(UNC_ERR_UNSUPPORTED, "only 9 camera parameters are supported");
    if ((long long)num_cols != 9LL * o->num_cams + 3LL * o->num_points)
        return fail(UNC_ERR_INVALID_ARG, "num_cols != 9*num_cams + 3*num_points");
    if (o->algorithm == UNC_SVD_QR_ITERATION || o->algorithm == UNC_SVD_DEVIDE_AND_CONQUER) {
        // dense (9C + 3P)^2 J^T J plus four scratch matrices of that size
        const long long n = 9LL * o->num_cams + 3LL * o->num_points;
        if (n > 46000) return fail(UNC_ERR_TOO_LARGE, "SVD algorithms: 9*num_cams + 3*num_points above 46000");
        if (o->svd_remove_n < -1 || o->svd_remove_n > 31)
            return fail(UNC_ERR_UNSUPPORTED, "svd_remove_n must be -1 (epsilon rule) or 0..31");
        return UNC_OK;
    }
    if (o->algorithm == UNC_SVD_SCHUR) {
        if (9LL * o->num_cams > 46000) return fail(UNC_ERR_TOO_LARGE, "9*num_cams above 46000");
        if (o->svd_remove_n < -1 || o->svd_remove_n > 31)
            return fail(UNC_ERR_UNSUPPORTED, "svd_remove_n must be -1 (epsilon rule) or 0..31");
        return UNC_OK;
    }
    if (o->algorithm != UNC_TAYLOR_EXPANSION) return fail(UNC_ERR_INVALID_ARG, "unknown algorithm");
    if (!o->has_pts2fix) return fail(UNC_ERR_NO_FIXED_POINTS, "TAYLOR_EXPANSION needs three fixed points");
    for (int i = 0; i < 3; ++i)
        if (o->pts2fix[i] < 0 || o->pts2fix[i] >= o->num_points)
            return fail(UNC_ERR_INVALID_ARG, "fixed point id out of range");
    if (o->precision < UNC_PRECISION_FP64 || o->precision > UNC_PRECISION_MIXED3)
        return fail(UNC_ERR_INVALID_ARG, "unknown precision");
    if (9LL * o->num_cams > 46000) return fail(UNC_ERR_TOO_LARGE, "9*num_cams above 46000");
    return UNC_OK;
}

bool is_svd(const unc_options* o) {
    return o->algorithm == UNC_SVD_QR_ITERATION || o->algorithm == UNC_SVD_DEVIDE_AND_CONQUER;
}

double auto_lambda(int N) { return pow(10, -1.2653 * log10((double)N) - 2.9415); }

int32_t factorial_i32(int n) {
    uint32_t f = 1;
    for (int i = 2; i <= n; ++i) f *= (uint32_t)i;
    return (int32_t)f;
}

Plan make_plan(const unc_options* o, int num_rows) {
    Plan pl;
    pl.C = o->num_cams;
    pl.P = o->num_points;
    pl.nobs = num_rows / 2;
    pl.N = 9 * pl.C;
    pl.ld = ld_of(pl.N);
    pl.svd_schur = o->algorithm == UNC_SVD_SCHUR;
    return pl;
}

int sparse_stage(const unc_options* o, const Plan& pl, long long nnz, const int* rows, const int* cols,
                 const double* vals, Buffers& b, int fx[3], cudaEvent_t* ev, cudaStream_t sm) {
    SceneDev& s = b.s;
    s.nnz = (long)nnz;
    s.num_cams = pl.C;
    s.num_points = pl.P;
    s.num_obs = pl.nobs;
    s.rows = rows;
    s.cols = cols;
    s.J = vals;
    fx[0] = o->pts2fix[0];
    fx[1] = o->pts2fix[1];
    fx[2] = o->pts2fix[2];
    std::sort(fx, fx + 2);  // the reference sorts only the first two ids (compute.cpp:285)
    s.has_fix = pl.svd_schur ? 0 : 1;  // the SVD on Z keeps every point
    if (pl.svd_schur) fx[0] = fx[1] = fx[2] = -1;
    for (int i = 0; i < 3; ++i) s.fix[i] = fx[i];
    const int N = pl.N, ld = pl.ld;
    auto mark = [&](int i) -> int {
        if (ev) CK(cudaEventRecord(ev[i], sm));
        return UNC_OK;
    };

    if (int r = mark(0)) return r;
    CK(cudaMemsetAsync(s.err, 0, 16, sm));
    launch_validate_obs(s, sm);
    if (int r = mark(1)) return r;
    launch_build_index(s, sm);
    if (int r = mark(2)) return r;
    // zero the dense work buffers once (padding rows must stay finite for the GEMM loads)
    CK(cudaMemsetAsync(b.iZ, 0, (size_t)((char*)(b.tmp + (size_t)ld * N) - (char*)b.iZ), sm));
    launch_camera_blocks(s, sm);
    launch_point_blocks(s, sm);
    if (int r = mark(3)) return r;
    launch_obs_blocks(s, sm);
    if (int r = mark(4)) return r;
    CK(cudaMemsetAsync(b.Z, 0, sizeof(double) * (size_t)ld * N, sm));
    if (launch_schur_columns(s, b.Z, ld, sm) != UNC_OK)
        return fail(UNC_ERR_TOO_LARGE, "more cameras than the Schur stage supports");
    if (int r = mark(5)) return r;
    return UNC_OK;
}

void output_stage(const Plan& pl, Buffers& b, double* cam_out, double* pt_out, cudaStream_t sm) {
    launch_camera_output(b.iZ, pl.ld, b.s.s_cam, pl.C, cam_out, b.sig, sm);
    if (pl.P > 3) cudaMemsetAsync(pt_out, 0, sizeof(double) * 6 * ((size_t)pl.P - 3), sm);
    launch_point_cov(b.s, b.sig, pt_out, sm);
}

}  // namespace unc

namespace {

constexpr size_t kStageGraphs = 8, kSeenKeys = 16;

void drop_graphs(unc_context* ctx) {
    for (auto& g : ctx->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    ctx->graphs.clear();
    ctx->seen.clear();
}

// Run a fixed launch sequence (the dense stage) on sm. A key seen before is
// captured into a CUDA graph and replayed from then on: several hundred small
// launches cost one graph launch. Keys name the sizes, the options that change
// kernel arguments and every buffer address, so a replay is the same work.
// If capture or instantiation fails, the stage runs directly.
template <class F>
int run_stage(unc_context* ctx, const GraphKey& key, cudaStream_t sm, F&& stage, size_t& npev) {
    for (auto& g : ctx->graphs)
        if (g.key == key) {
            npev = g.npev;
            CK(cudaGraphLaunch(g.exec, sm));
            count_launch((int)g.launches);
            return UNC_OK;
        }
    const bool again = std::find(ctx->seen.begin(), ctx->seen.end(), key) != ctx->seen.end();
    if (!again) {
        if (ctx->seen.size() >= kSeenKeys) ctx->seen.erase(ctx->seen.begin());
        ctx->seen.push_back(key);
        return stage();
    }
    const long long l0 = g_thread_launches;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ok = cudaStreamBeginCapture(sm, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    int rc = UNC_OK;
    if (ok) {
        rc = stage();
        ok = cudaStreamEndCapture(sm, &graph) == cudaSuccess && rc == UNC_OK && graph;
    }
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    const long long launches = g_thread_launches - l0;  // this thread's launches were captured, not run
    __atomic_sub_fetch(&g_launches, launches, __ATOMIC_RELAXED);
    g_thread_launches -= launches;
    if (!ok) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        npev = 0;
        return stage();
    }
    if (ctx->graphs.size() >= kStageGraphs) {
        cudaGraphExecDestroy(ctx->graphs.front().exec);
        ctx->graphs.erase(ctx->graphs.begin());
    }
    ctx->graphs.push_back(StageGraph{key, exec, npev, launches});
    CK(cudaGraphLaunch(exec, sm));
    count_launch((int)launches);
    return UNC_OK;
}


float ev_s(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();  // leave no error behind for the next call's checks
        return 0.0f;
    }
    return ms * 1e-3f;
}

// The pipeline (all device pointers). rows/cols/vals: the Jacobian.
int run_pipeline(unc_context* ctx, const unc_options* o, int num_rows, long long nnz, const int* rows,
                 const int* cols, const double* vals, double* cam_out, double* pt_out, Buffers& b,
                 const Plan& pl, unc_statistic* st, cudaStream_t sm) {
    SceneDev& s = b.s;
    int fx[3];
    const int N = pl.N, ld = pl.ld;
    cudaEvent_t* ev = ctx->ev;
    if (int r = sparse_stage(o, pl, nnz, rows, cols, vals, b, fx, ev, sm)) return r;

    PinvInfo pinfo{};
    if (pl.svd_schur) {
        // pseudo-inverse of the unscaled Z = S Z_s S (s: camera column norms)
        // without its svd_remove_n smallest eigenvalues, then iZ_s = S P S so
        // that the camera output's d_j d_k iZ_s(j, k) is P(j, k)
        launch_unequilibrate(b.Z, N, ld, s.s_cam, nullptr, sm);
        const double eps = o->epsilon < 0 ? 1e-10 : o->epsilon;
        if (int r = pinv_psd(b.Z, N, ld, o->svd_remove_n, eps, b.pb, sm, &pinfo)) return r;
        CK(cudaEventRecord(ev[6], sm));
        launch_unequilibrate(b.Z, N, ld, s.s_cam, b.iZ, sm);
        CK(cudaEventRecord(ev[7], sm));
        launch_camera_output(b.iZ, ld, s.s_cam, pl.C, cam_out, b.sig, sm);
        if (pl.P > 0) CK(cudaMemsetAsync(pt_out, 0, sizeof(double) * 6 * (size_t)pl.P, sm));
        launch_point_cov(s, b.sig, pt_out, sm);
        CK(cudaEventRecord(ev[8], sm));
        int err = 0;
        CK(cudaMemcpyAsync(&err, s.err, sizeof(int), cudaMemcpyDeviceToHost, sm));
        CK(cudaStreamSynchronize(sm));
        CK(cudaGetLastError());
        if (st) {
            st->lambda = 0;
            for (int i = 0; i < 3; ++i) st->fixed_pts[i] = -1;
            st->te_iterations = pinfo.iterations;  // subspace iterations
            st->time_create_j = ev_s(ev[0], ev[1]);
            st->time_fix_j = ev_s(ev[1], ev[2]);
            st->time_norm_j = ev_s(ev[2], ev[3]);
            st->time_multiply_jj = ev_s(ev[3], ev[4]);
            st->time_compose_z = ev_s(ev[4], ev[5]);
            st->time_inv_z = ev_s(ev[5], ev[6]);
            st->time_pts_unc = ev_s(ev[7], ev[8]);
            st->time_all = ev_s(ev[0], ev[8]);
        }
        if (err & ERRBIT_LAYOUT)
            return fail(UNC_ERR_LAYOUT, "Jacobian rows are not in the 2 x (9 camera + 3 point) observation layout");
        if (err & (ERRBIT_SINGULAR | ERRBIT_NONFINITE))
            return fail(UNC_ERR_SINGULAR, "singular point block or non-finite value");
        return UNC_OK;
    }

    double lambda = o->lambda;
    if (lambda == -1) lambda = auto_lambda(N);  // compute.cpp:124-125

    // Every power X^(i+1) is symmetric: only the lower-triangle tiles of each
    // product are computed (half the flops), then mirrored for the next product.
    // FP64 mode: DMMA products. Mixed modes: int8-sliced tcgen05 products of
    // the FP64 operands (X sliced once, each new operand sliced per product).
    const bool mixed = o->precision != UNC_PRECISION_FP64;
    const bool powers = o->taylor_eval != UNC_TAYLOR_SEQUENTIAL;
    const int slices = o->precision == UNC_PRECISION_MIXED4 ? 4 : (o->precision == UNC_PRECISION_MIXED3 ? 3 : 5);
    // slice buffers: X, the A operand of the moment, and (powers) X^4, X^8, X^12, X^16
    constexpr int kX = 0, kA = 1, k4 = 2, k8 = 3, k12 = 4, k16 = 5;
    const int nbuf = powers ? 6 : 2;
    MixedOperand opa[6], opb[6];  // each buffer as the A (128-row boxes) and as the B operand
    MixedOperand opa_k[6][6], opb_k[6][6];  // [buffer][k]: its first k slices
    size_t mp_need = 0;
    if (mixed) {  // host-side preparation: buffers and tensor maps
        const size_t sb = (mixed_slice_bytes(N, slices) + 255) & ~size_t(255);
        const size_t eb = (sizeof(int) * ((size_t)N + 64) + 255) & ~size_t(255);
        mp_need = nbuf * (sb + eb) + 256;
        if (int r = grow_buffer(&ctx->mp, &ctx->mp_bytes, mp_need, mp_need, sm)) return r;
        char* w = (char*)ctx->mp;
        for (int q = 0; q < nbuf; ++q) {
            int8_t* buf = reinterpret_cast<int8_t*>(w + q * sb);
            int* ex = reinterpret_cast<int*>(w + nbuf * sb + q * eb);
            if (!mixed_plan(opa[q], buf, ex, N, slices, false) || !mixed_plan(opb[q], buf, ex, N, slices, true))
                return fail(UNC_ERR_CUDA, "tensor-map encoding failed");
        }
        // the same buffers with fewer slices (power_product_slices)
        for (int q = 0; q < nbuf; ++q)
            for (int k = 2; k < slices; ++k) {
                bool ok_a = false, ok_b = false;
                opa_k[q][k] = mixed_fewer_slices(opa[q], k, false, &ok_a);
                opb_k[q][k] = mixed_fewer_slices(opb[q], k, true, &ok_b);
                if (!ok_a || !ok_b) return fail(UNC_ERR_CUDA, "tensor-map encoding failed");
            }
        for (int q = 0; q < nbuf; ++q) {
            opa_k[q][slices] = opa[q];
            opb_k[q][slices] = opb[q];
        }
    }
    const double* X = b.Z;
    size_t npev = 0;
    auto prof_mark = [&]() -> int {
        if (!ctx->prof) return UNC_OK;
        if (npev == ctx->pev.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            ctx->pev.push_back(e);
        }
        CK(cudaEventRecord(ctx->pev[npev++], sm));
        return UNC_OK;
    };
    // the profiled region is the product kernel alone (slicing excluded)
    // Each product writes its lower triangle and, transposed, the upper one
    // (the powers are symmetric). In mixed mode the Taylor update iZ += k P of
    // the power being sliced rides along in the slicing kernel.
    auto product = [&](const double* P, double* out, const int* skip) -> int {
        if (mixed) {
            if (P != X) mixed_slice(P, ld, opa[kA], sm, skip, b.iZ, b.te);
            if (int r = prof_mark()) return r;
            mixed_gemm(P == X ? opa[kX] : opa[kA], opb[kX], out, ld, b.amax, true, s.err, sm, skip, true);
        } else {
            if (int r = prof_mark()) return r;
            gemm_f64_mode(N, N, N, 1.0, P, ld, X, ld, 0.0, out, ld, b.amax, GEMM_LOWER | GEMM_MIRROR, sm, nullptr,
                          0, skip);
        }
        return prof_mark();
    };
    // blocked powers: out (+)= A B, A and B powers of X (symmetric, commuting)
    // given as FP64 matrices and, in mixed mode, as slice buffers ia / ib;
    // q: the product's index in power_product_slices
    auto power_product = [&](int q, const double* A, int ia, const double* B, int ib, double* out, bool acc,
                             const int* skip) -> int {
        if (int r = prof_mark()) return r;
        if (mixed) {
            const int k = power_product_slices(q, slices);
            mixed_gemm(opa_k[ia][k], opb_k[ib][k], out, ld, nullptr, true, s.err, sm, skip, true, acc);
        } else
            gemm_f64_mode(N, N, N, 1.0, A, ld, B, ld, acc ? 1.0 : 0.0, out, ld, nullptr, GEMM_LOWER | GEMM_MIRROR,
                          sm, nullptr, 0, skip);
        return prof_mark();
    };
    auto slice = [&](const double* A, int q, const int* skip) {
        if (mixed) mixed_slice(A, ld, opa[q], sm, skip);
    };
    // The dense stage, a fixed launch sequence for given sizes and buffers:
    // equilibration, the SPD inverse (SDM::inv, ScaledDenseMatrix.cpp:232-279)
    // and the Taylor expansion (compute.cpp:141-160),
    //   iZ = X + sum lambda^i/(i-1)! X^(i+1).
    // The stop rule runs on the device (k_te_decide): all 19 iterations are
    // launched and, once the rule fires, the remaining kernels return at once;
    // k = lambda^i / factorial(i-1) is evaluated here (32-bit factorial wrap).
    // moderate sizes: the tile-task inverse (one persistent kernel); larger: the recursive form
    const bool tasks = spd_tasks_apply(N);
    // mixed modes, recursive inverse: its last product T^T T on the int8 path, in the
    // first two slice buffers (free until the Taylor stage) and the first exponent array
    const size_t slice_region = mixed ? (size_t)nbuf * ((mixed_slice_bytes(N, slices) + 255) & ~size_t(255)) : 0;
    const bool gram = mixed && !tasks && mixed_gram_bytes(N) <= slice_region;
    int* gram_exps = mixed ? opa[kX].exps : nullptr;
    if (tasks)
        if (int r = spd_tasks_prepare(N)) return fail(r, "tile-task inverse: cannot upload the task list");
    auto inverse_stage = [&]() -> int {
        launch_shift_equilibrate(b.Z, N, ld, lambda, b.e, s.err, sm);
        if (tasks) {
            if (int r = chol_inverse_tasks(b.Z, N, ld, b.iZ, b.add, b.dag_state, s.err, sm, ctx->task_ctas))
                return r;
            launch_unequilibrate_from(b.add, b.Z, N, ld, b.e, b.iZ, sm);  // X in Z, iZ = X
        } else if (gram) {
            // mixed: T = L^{-1} in FP64 (its products feed the pivots), A^{-1} = T^T T
            // from int8 slices of T on the tensor cores
            chol_lower_inverse(b.Z, N, ld, b.iZ, b.add, b.tmp, s.err, sm);
            CK(cudaMemsetAsync(ctx->mp, 0, mixed_gram_bytes(N), sm));  // slice padding must be zero
            if (!mixed_gram_lower_tri(b.iZ, N, ld, reinterpret_cast<int8_t*>(ctx->mp), gram_exps, b.Z, ld, s.err, sm))
                return fail(UNC_ERR_CUDA, "tensor-map encoding failed");
            launch_unequilibrate(b.Z, N, ld, b.e, b.iZ, sm);  // X in Z, iZ = X
        } else {
            chol_inverse(b.Z, N, ld, b.iZ, b.add, b.tmp, b.gjws, s.err, sm);
            launch_unequilibrate(b.Z, N, ld, b.e, b.iZ, sm);  // X in Z, iZ = X
        }
        return UNC_OK;
    };
    auto taylor_stage = [&]() -> int {
        double* add = b.add;
        double* tmp = b.tmp;
        if (mixed) {
            CK(cudaMemsetAsync(ctx->mp, 0, mp_need, sm));  // slice padding must be zero
            mixed_slice(X, ld, opa[kX], sm);
        }
        launch_te_init(b.te, sm);
        const int* skip = &b.te->done;
        CK(cudaMemsetAsync(b.amax, 0, 8, sm));
        if (int r = product(X, add, nullptr)) return r;
        for (int i = 1; i < 20; ++i) {  // the reference's order: one product per iteration
            const double k = pow(lambda, i) / factorial_i32(i - 1);
            launch_te_decide(b.te, b.amax, k, sm);
            if (!mixed) launch_axpy_te(b.iZ, add, b.te, N, ld, sm);
            CK(cudaMemsetAsync(b.amax, 0, 8, sm));
            if (int r = product(add, tmp, skip)) return r;
            std::swap(add, tmp);
        }
        return UNC_OK;
    };
    // The blocked-power evaluation (powers.cu): X^2, X^3, X^4, X^8, X^12 and
    // X^16 (skipped on the device unless the rule passes iteration 15); the
    // stop rule from their diagonal maxima; iZ = G_0 + sum_q X^(4q) G_q, the
    // products on the camera blocks only, with the blocks whose coefficients
    // are all zero skipped on the device.
    PowerSet ps{};
    ps.M[0] = b.Z;
    ps.M[1] = b.add;
    ps.M[2] = b.tmp;
    ps.M[3] = b.p4;
    ps.M[4] = b.p8;
    ps.M[5] = b.p12;
    ps.M[6] = b.p16;
    ps.iZ = b.iZ;
    ps.G = b.g;
    ps.n = N;
    ps.ld = ld;
    ps.dmax = b.dmax;
    ps.te = b.te;
    TaylorCoefs kc{};
    for (int i = 1; i < 20; ++i) kc.k[i - 1] = pow(lambda, i) / factorial_i32(i - 1);
    auto powers_stage = [&]() -> int {
        const int* sk = b.te->skip;
        if (ld != N)  // padding rows of the extra power buffers must stay finite for the product loads
            for (double* m : {b.p4, b.p8, b.p12, b.p16, b.g})
                CK(cudaMemset2DAsync(m + N, sizeof(double) * (size_t)ld, 0, sizeof(double) * (size_t)(ld - N), N, sm));
        if (mixed) {
            CK(cudaMemsetAsync(ctx->mp, 0, mp_need, sm));  // slice padding must be zero
            slice(X, kX, nullptr);
        }
        launch_te_init(b.te, sm);
        CK(cudaMemsetAsync(b.dmax, 0, sizeof(unsigned long long) * 24, sm));
        if (int r = power_product(0, X, kX, X, kX, b.add, false, nullptr)) return r;  // X^2
        slice(b.add, kA, nullptr);
        if (int r = power_product(1, b.add, kA, X, kX, b.tmp, false, nullptr)) return r;  // X^3
        slice(b.tmp, kA, nullptr);
        if (int r = power_product(2, b.tmp, kA, X, kX, b.p4, false, nullptr)) return r;  // X^4
        slice(b.p4, k4, nullptr);
        if (int r = power_product(3, b.p4, k4, b.p4, k4, b.p8, false, nullptr)) return r;  // X^8
        slice(b.p8, k8, nullptr);
        if (int r = power_product(4, b.p8, k8, b.p4, k4, b.p12, false, nullptr)) return r;  // X^12
        slice(b.p12, k12, nullptr);
        launch_power_diag(ps, 2, 16, nullptr, sm);
        launch_power_decide(b.te, b.dmax, kc, 1, 15, sm);
        if (int r = power_product(5, b.p8, k8, b.p8, k8, b.p16, false, sk)) return r;  // X^16
        slice(b.p16, k16, sk);
        launch_power_diag(ps, 17, 20, sk, sm);
        launch_power_decide(b.te, b.dmax, kc, 16, 19, sm);
        launch_power_combine(ps, 0, b.iZ, nullptr, sm);  // iZ = G_0
        // iZ += X^(4q) G_q on the camera blocks, the only part of iZ that is read after
        launch_taylor_blocks(ps, sm);
        return UNC_OK;
    };
    while (ctx->prof && ctx->pev.size() < 2 * 20 + 2) {  // events exist before any capture
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        ctx->pev.push_back(e);
    }
    {
        unsigned long long lam_bits;
        memcpy(&lam_bits, &lambda, 8);
        // events are recorded between the graphs (elapsed times of events
        // recorded inside a graph are not available); per-product profiling
        // runs the stages directly
        GraphKey key = {1ULL, (unsigned long long)N, (unsigned long long)ld, lam_bits,
                        (unsigned long long)(uintptr_t)b.Z, (unsigned long long)(uintptr_t)b.gjws,
                        (unsigned long long)(uintptr_t)s.err, 0ULL};
        size_t none = 0;
        if (int r = ctx->prof ? inverse_stage() : run_stage(ctx, key, sm, inverse_stage, none)) return r;
        CK(cudaEventRecord(ev[6], sm));
        key[0] = powers ? 3ULL : 2ULL;
        key[7] = ((unsigned long long)o->precision << 56) ^ (unsigned long long)(uintptr_t)ctx->mp;
        if (powers) {
            if (int r = ctx->prof ? powers_stage() : run_stage(ctx, key, sm, powers_stage, npev)) return r;
        } else {
            if (int r = ctx->prof ? taylor_stage() : run_stage(ctx, key, sm, taylor_stage, npev)) return r;
        }
        CK(cudaEventRecord(ev[7], sm));
    }

    output_stage(pl, b, cam_out, pt_out, sm);
    CK(cudaEventRecord(ev[8], sm));

    int err = 0;
    TeState te{};
    CK(cudaMemcpyAsync(&err, s.err, sizeof(int), cudaMemcpyDeviceToHost, sm));
    CK(cudaMemcpyAsync(&te, b.te, sizeof(TeState), cudaMemcpyDeviceToHost, sm));
    CK(cudaStreamSynchronize(sm));
    CK(cudaGetLastError());
    const int iters = te.iters;
    // products actually computed. Sequential: the first one and one per
    // performed iteration. Powers: X^2..X^12 (5), X^16 unless skipped, one per
    // non-zero block.
    std::vector<bool> ran(npev / 2, false);
    for (size_t q = 0; q < ran.size(); ++q)
        ran[q] = powers ? (q < 5 || (q == 5 && !te.skip[0]) || (q > 5 && q < 10 && !te.skip[q - 5]))
                        : q < (size_t)iters + 1;
    for (size_t q = 0; q < ran.size(); ++q) {
        if (!ran[q]) continue;
        ctx->prof_seconds += ev_s(ctx->pev[2 * q], ctx->pev[2 * q + 1]);
        ctx->prof_launches += 1;
        ctx->prof_flops += (double)N * N * (N + 1);  // symmetric product: lower half of 2 N^3
        if (mixed) ctx->prof_int8_ops += mixed_issued_ops(N, powers ? power_product_slices((int)q, slices) : slices);
    }
    if (st) {
        st->lambda = lambda;
        for (int i = 0; i < 3; ++i) st->fixed_pts[i] = fx[i];
        st->te_iterations = iters;
        for (int i = 0; i < iters && i < 20; ++i) st->cycle_change[i] = te.change[i];
        st->time_create_j = ev_s(ev[0], ev[1]);
        st->time_fix_j = ev_s(ev[1], ev[2]);
        st->time_norm_j = ev_s(ev[2], ev[3]);
        st->time_multiply_jj = ev_s(ev[3], ev[4]);
        st->time_split_jj = 0;
        st->time_inv_v = 0;
        st->time_compose_z = ev_s(ev[4], ev[5]);
        st->time_inv_z = ev_s(ev[5], ev[6]);
        st->time_te = ev_s(ev[6], ev[7]);
        st->time_pts_unc = ev_s(ev[7], ev[8]);
        st->time_all = ev_s(ev[0], ev[8]);
    }
    if (err & ERRBIT_LAYOUT)
        return fail(UNC_ERR_LAYOUT, "Jacobian rows are not in the 2 x (9 camera + 3 point) observation layout");
    if (err & (ERRBIT_SINGULAR | ERRBIT_NONFINITE))
        return fail(UNC_ERR_SINGULAR, "non-positive pivot or non-finite value while inverting Z + lambda*I");
    if (err & ERRBIT_TIMEOUT)
        return fail(UNC_ERR_CUDA, "a bounded device wait ran out (tensor-core pipeline or tile-task inverse)");
    if (err & ERRBIT_SCHUR_CAP)
        return fail(UNC_ERR_TOO_LARGE, "an observation shares its point with more observations than the Schur stage holds");
    if (te.bad) return fail(UNC_ERR_SINGULAR, "non-finite Taylor-series power");
    return UNC_OK;
}

// SDM::inv on the GPU (unc_dense_inverse_device). poll_limit / skip_task are
// passed to the tile-task form (n <= 3584): 0 / -1 for the regular schedule.
int dense_inverse(double* d_A, int n, int lda, void* stream, long long poll_limit, int skip_task) {
    g_last_error.clear();
    if (!d_A || n <= 0 || lda < n || (lda & 1)) return fail(UNC_ERR_INVALID_ARG, "bad matrix arguments");
    cudaStream_t sm = (cudaStream_t)stream;
    const size_t mat = (size_t)lda * n;
    // n <= 3584: the tile-task inverse (one persistent kernel), else the recursive form
    const bool tasks = spd_tasks_apply(n);
    if (tasks)
        if (int r = spd_tasks_prepare(n)) return fail(r, "tile-task inverse: cannot upload the task list");
    const size_t small_d = std::max(chol_small_doubles(n), (spd_task_state_ints(n) + 1) / 2);
    const size_t wsd = 3 * mat + small_d + (size_t)n + 64;
    double* ws = nullptr;
    CK(cudaMalloc(&ws, wsd * sizeof(double) + 256));
    double *T = ws, *W = ws + mat, *Tt = ws + 2 * mat, *small = ws + 3 * mat;
    double* e = small + small_d;
    int* err = reinterpret_cast<int*>(ws + wsd);
    int h_err = 0;
    cudaError_t ce = cudaMemsetAsync(ws, 0, wsd * sizeof(double) + 256, sm);
    if (ce == cudaSuccess) {
        launch_shift_equilibrate(d_A, n, lda, 0.0, e, err, sm);
        if (tasks) {
            if (chol_inverse_tasks(d_A, n, lda, T, W, reinterpret_cast<int*>(small), err, sm, device_sms(),
                                   poll_limit, skip_task) != UNC_OK)
                ce = cudaErrorUnknown;
            launch_unequilibrate_from(W, d_A, n, lda, e, nullptr, sm);
        } else {
            chol_inverse(d_A, n, lda, T, W, Tt, small, err, sm);
            launch_unequilibrate(d_A, n, lda, e, nullptr, sm);
        }
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, sm);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(sm);
    cudaFree(ws);
    if (ce != cudaSuccess) return fail(UNC_ERR_CUDA, cudaGetErrorString(ce));
    if (h_err & ERRBIT_TIMEOUT) return fail(UNC_ERR_CUDA, "a bounded device wait of the tile-task inverse ran out");
    if (h_err & (ERRBIT_SINGULAR | ERRBIT_NONFINITE)) return fail(UNC_ERR_SINGULAR, "matrix is not positive definite");
    return UNC_OK;
}

}  // namespace

extern "C" {

void unc_options_init(unc_options* o, int num_cams, int cam_params, int num_points, int num_obs) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->algorithm = UNC_TAYLOR_EXPANSION;
    o->epsilon = 1e-10;
    o->lambda = -1;
    o->num_cams = num_cams;
    o->cam_params = cam_params;
    o->num_points = num_points;
    o->num_obs = num_obs;
    o->svd_remove_n = -1;
    o->max_iter_te = -1;
    o->precision = UNC_PRECISION_FP64;
}

int unc_context_create(int device, unc_context** out) {
    if (!out) return fail(UNC_ERR_INVALID_ARG, "ctx is NULL");
    *out = nullptr;
    unc_context* c = new unc_context();
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) {  // kernel attributes now, never inside a stream capture
        c->sm_count = device_sms();
        c->task_ctas = c->sm_count;
        prepare_assembly_kernels();
        prepare_dense_kernels();
        prepare_mixed_kernels();
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    }
    for (int i = 0; i < 12 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
    if (e != cudaSuccess) {
        g_last_error = std::string("context creation: ") + cudaGetErrorString(e);
        delete c;
        return UNC_ERR_CUDA;
    }
    *out = c;
    return UNC_OK;
}

int unc_context_set_profiling(unc_context* c, int enable) {
    if (!c) return fail(UNC_ERR_INVALID_ARG, "ctx is NULL");
    c->prof = enable != 0;
    return UNC_OK;
}

int unc_context_profile(unc_context* c, long long* launches, double* seconds, double* flops, int reset) {
    if (!c) return fail(UNC_ERR_INVALID_ARG, "ctx is NULL");
    if (launches) *launches = c->prof_launches;
    if (seconds) *seconds = c->prof_seconds;
    if (flops) *flops = c->prof_flops;
    if (reset) {
        c->prof_launches = 0;
        c->prof_seconds = 0;
        c->prof_flops = 0;
        c->prof_int8_ops = 0;
    }
    return UNC_OK;
}

int unc_context_profile_int8(unc_context* c, double* int8_ops) {
    if (!c || !int8_ops) return fail(UNC_ERR_INVALID_ARG, "ctx or int8_ops is NULL");
    *int8_ops = c->prof_int8_ops;
    return UNC_OK;
}

int unc_context_destroy(unc_context* c) {
    if (!c) return UNC_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    unc_context_release(c);
    for (cudaEvent_t e : c->pev) cudaEventDestroy(e);
    for (int i = 0; i < 12; ++i)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (int i = 0; i < kStageSlots; ++i)
        if (c->stage_ev[i]) cudaEventDestroy(c->stage_ev[i]);
    if (c->stage) cudaFreeHost(c->stage);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return UNC_OK;
}

int unc_context_release(unc_context* c) {
    if (!c) return fail(UNC_ERR_INVALID_ARG, "ctx is NULL");
    cudaSetDevice(c->device);
    drop_graphs(c);  // they name the buffers freed below
    void** bufs[3] = {&c->ws, &c->mp, &c->jac};
    size_t* sizes[3] = {&c->ws_bytes, &c->mp_bytes, &c->jac_bytes};
    for (int i = 0; i < 3; ++i) {
        if (*bufs[i]) cudaFreeAsync(*bufs[i], c->stream);
        *bufs[i] = nullptr;
        *sizes[i] = 0;
    }
    CK(cudaStreamSynchronize(c->stream));
    return UNC_OK;
}

int unc_context_set_priority(unc_context* c, int high) {
    if (!c) return fail(UNC_ERR_INVALID_ARG, "ctx is NULL");
    int least = 0, greatest = 0;
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int want = high ? greatest : least;
    if (want == c->priority) return UNC_OK;
    cudaStream_t s = nullptr;
    CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, want));
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    c->stream = s;
    c->priority = want;
    return UNC_OK;
}

long long unc_context_device_bytes(const unc_context* c) {
    if (!c) return -1;
    return (long long)(c->ws_bytes + c->mp_bytes + c->jac_bytes);
}

long long unc_request_bytes(const unc_options* o, int num_rows, int num_cols, const int* rows, const int* cols) {
    if (!o || num_rows < 0 || !rows || !cols) return -1;
    if (check_options(o, num_rows, num_cols) != UNC_OK) return -1;
    const long long nnz = rows[num_rows];
    const int nobs = num_rows / 2;
    if (is_svd(o)) return (long long)svd_workspace_bytes(o->num_cams, o->num_points, nobs, true, nnz, num_rows);
    Plan pl = make_plan(o, num_rows);
    Buffers b;
    long long bytes = (long long)carve(nullptr, pl, true, nnz, num_rows, b);
    if (o->precision != UNC_PRECISION_FP64) {  // slice buffers: 6 (blocked powers) or 2 (sequential)
        const int slices = o->precision == UNC_PRECISION_MIXED4 ? 4 : (o->precision == UNC_PRECISION_MIXED3 ? 3 : 5);
        const long long nbuf = o->taylor_eval == UNC_TAYLOR_SEQUENTIAL ? 2 : 6;
        bytes += nbuf * ((long long)((mixed_slice_bytes(pl.N, slices) + 255) & ~size_t(255)) +
                         (long long)((4 * ((size_t)pl.N + 64) + 255) & ~size_t(255))) + 256;
    }
    return bytes;
}

long long unc_workspace_bytes(const unc_options* o, int num_rows, int num_cols) {
    if (!o || num_rows < 0) return -1;
    (void)num_cols;
    Plan pl = make_plan(o, num_rows);
    Buffers b;
    return (long long)carve(nullptr, pl, false, 0, num_rows, b);
}

int unc_compute_device(unc_context* ctx, const unc_options* o, int num_rows, int num_cols,
                       const int* d_rows, const int* d_cols, const double* d_values,
                       double* d_cam_unc, double* d_pt_unc, unc_statistic* st, void* stream) {
    g_last_error.clear();
    if (!ctx) return fail(UNC_ERR_INVALID_ARG, "unc_compute_device needs a context");
    int rc = check_options(o, num_rows, num_cols);
    if (rc) return rc;
    if (!d_rows || !d_cols || !d_values || !d_cam_unc || !d_pt_unc)
        return fail(UNC_ERR_INVALID_ARG, "null device pointer");
    if (((uintptr_t)d_cols & 15) || ((uintptr_t)d_values & 15))
        return fail(UNC_ERR_INVALID_ARG, "cols/values must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t sm = stream ? (cudaStream_t)stream : ctx->stream;
    if (is_svd(o)) {
        const size_t bytes = svd_workspace_bytes(o->num_cams, o->num_points, num_rows / 2, false, 0, num_rows);
        rc = ensure_ws(ctx, bytes, sm);
        if (rc) return rc;
        if (st) {
            memset(st, 0, sizeof(*st));
            st->device_bytes = (long long)bytes;
        }
        return svd_pipeline((char*)ctx->ws, o, num_rows, 24LL * (num_rows / 2), d_rows, d_cols, d_values,
                            d_cam_unc, d_pt_unc, false, st, ctx->ev, sm);
    }
    Plan pl = make_plan(o, num_rows);
    Buffers b;
    size_t bytes = carve(nullptr, pl, false, 0, num_rows, b);
    rc = ensure_ws(ctx, bytes, sm);
    if (rc) return rc;
    carve((char*)ctx->ws, pl, false, 0, num_rows, b);
    if (st) {
        memset(st, 0, sizeof(*st));
        st->device_bytes = (long long)bytes;
    }
    // the arrays are trusted to hold the reference layout's 24 entries per observation
    return run_pipeline(ctx, o, num_rows, 24LL * pl.nobs, d_rows, d_cols, d_values, d_cam_unc, d_pt_unc,
                        b, pl, st, sm);
}

int unc_compute(unc_context* ctx, const unc_options* o, int num_rows, int num_cols, const int* rows,
                const int* cols, const double* values, double* cam_unc, double* pt_unc,
                unc_statistic* st) {
    g_last_error.clear();
    int rc = check_options(o, num_rows, num_cols);
    if (rc) return rc;
    if (!rows || !cols || !values || !cam_unc || !pt_unc) return fail(UNC_ERR_INVALID_ARG, "null pointer");
    unc_context* own = nullptr;
    if (!ctx) {
        rc = unc_context_create(0, &own);
        if (rc) return rc;
        ctx = own;
    }
    struct Guard {
        unc_context* c;
        ~Guard() { unc_context_destroy(c); }
    } guard{own};
    const long long nnz = rows[num_rows];
    if (nnz < 0 || rows[0] != 0) return fail(UNC_ERR_INVALID_ARG, "rowptr must start at 0 and end at nnz >= 0");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t sm = ctx->stream;
    if (is_svd(o)) {
        const size_t bytes = svd_workspace_bytes(o->num_cams, o->num_points, num_rows / 2, true, nnz, num_rows);
        rc = ensure_ws(ctx, bytes, sm);
        if (rc) return rc;
        if (st) {
            memset(st, 0, sizeof(*st));
            st->device_bytes = (long long)bytes;
        }
        return svd_pipeline((char*)ctx->ws, o, num_rows, nnz, rows, cols, values, cam_unc, pt_unc, true, st,
                            ctx->ev, sm);
    }
    Plan pl = make_plan(o, num_rows);
    Buffers b;
    size_t bytes = carve(nullptr, pl, true, nnz, num_rows, b);
    rc = ensure_ws(ctx, bytes, sm);
    if (rc) return rc;
    carve((char*)ctx->ws, pl, true, nnz, num_rows, b);
    if (st) {
        memset(st, 0, sizeof(*st));
        st->device_bytes = (long long)bytes;
    }
    rc = copy_host(ctx,
                   {{b.rows, rows, sizeof(int) * ((size_t)num_rows + 1)},
                    {b.cols, cols, sizeof(int) * (size_t)nnz},
                    {b.vals, values, sizeof(double) * (size_t)nnz}},
                   true, sm);
    if (rc) return rc;
    rc = run_pipeline(ctx, o, num_rows, nnz, b.rows, b.cols, b.vals, b.cam_out, b.pt_out, b, pl, st, sm);
    if (rc) return rc;
    // Points: slots [0, 6(P-3)) are written (zeroed or computed); of the last
    // three points only the non-fixed ones are written (compute.cpp:511,526).
    // The SVD on Z fixes no point: every slot is written.
    size_t head = pl.svd_schur ? (size_t)pl.P : (pl.P > 3 ? (size_t)(pl.P - 3) : 0);
    rc = copy_host(ctx,
                   {{cam_unc, b.cam_out, sizeof(double) * 45 * (size_t)pl.C},
                    {pt_unc, b.pt_out, sizeof(double) * 6 * head}},
                   false, sm);
    if (rc) return rc;
    for (int p = (int)head; p < pl.P; ++p) {
        if (p == b.s.fix[0] || p == b.s.fix[1] || p == b.s.fix[2]) continue;
        CK(cudaMemcpyAsync(pt_unc + 6L * p, b.pt_out + 6L * p, sizeof(double) * 6, cudaMemcpyDeviceToHost, sm));
    }
    CK(cudaStreamSynchronize(sm));
    return UNC_OK;
}

int unc_compute_scene(unc_context* ctx, const unc_options* o, const double* cams, const double* points,
                      const int* obs_cam, const int* obs_pt, double* cam_unc, double* pt_unc, unc_statistic* st) {
    g_last_error.clear();
    if (!o) return fail(UNC_ERR_INVALID_ARG, "options is NULL");
    const int C = o->num_cams, P = o->num_points, nobs = o->num_obs;
    const int num_rows = 2 * nobs, num_cols = 9 * C + 3 * P;
    int rc = check_options(o, num_rows, num_cols);
    if (rc) return rc;
    if (!cams || (P && !points) || (nobs && (!obs_cam || !obs_pt)) || !cam_unc || !pt_unc)
        return fail(UNC_ERR_INVALID_ARG, "null pointer");
    unc_context* own = nullptr;
    if (!ctx) {
        rc = unc_context_create(0, &own);
        if (rc) return rc;
        ctx = own;
    }
    struct Guard {
        unc_context* c;
        ~Guard() { unc_context_destroy(c); }
    } guard{own};
    CK(cudaSetDevice(ctx->device));
    cudaStream_t sm = ctx->stream;
    Carver c{nullptr};
    auto lay = [&](Carver& k, double*& dc, double*& dp, int*& oc, int*& op, int*& rows, int*& cols, double*& vals,
                   double*& co, double*& po, int*& err) {
        dc = k.take<double>(9 * (size_t)C);
        dp = k.take<double>(3 * (size_t)P);
        oc = k.take<int>(nobs);
        op = k.take<int>(nobs);
        rows = k.take<int>(2 * (size_t)nobs + 1);
        cols = k.take<int>(24 * (size_t)nobs);
        vals = k.take<double>(24 * (size_t)nobs);
        co = k.take<double>(45 * (size_t)C);
        po = k.take<double>(6 * (size_t)P);
        err = k.take<int>(4);
    };
    double *dc, *dp, *dv, *co, *po;
    int *oc, *op, *drows, *dcols, *derr;
    lay(c, dc, dp, oc, op, drows, dcols, dv, co, po, derr);
    const size_t bytes = c.off + 256;
    if (int r = grow_buffer(&ctx->jac, &ctx->jac_bytes, bytes, bytes, sm)) return r;
    Carver k{(char*)ctx->jac};
    lay(k, dc, dp, oc, op, drows, dcols, dv, co, po, derr);
    rc = copy_host(ctx,
                   {{dc, cams, sizeof(double) * 9 * (size_t)C},
                    {dp, points, sizeof(double) * 3 * (size_t)P},
                    {oc, obs_cam, sizeof(int) * (size_t)nobs},
                    {op, obs_pt, sizeof(int) * (size_t)nobs}},
                   true, sm);
    if (rc) return rc;
    CK(cudaMemsetAsync(derr, 0, sizeof(int), sm));
    if (launch_scene_jacobian(C, P, nobs, dc, dp, oc, op, drows, dcols, dv, derr, sm) != UNC_OK)
        return fail(UNC_ERR_CUDA, "scene Jacobian launch failed");
    int h_err = 0;
    CK(cudaMemcpyAsync(&h_err, derr, sizeof(int), cudaMemcpyDeviceToHost, sm));
    CK(cudaStreamSynchronize(sm));
    if (h_err & ERRBIT_LAYOUT) return fail(UNC_ERR_INVALID_ARG, "camera or point id out of range");
    rc = unc_compute_device(ctx, o, num_rows, num_cols, drows, dcols, dv, co, po, st, sm);
    if (rc) return rc;
    const bool no_fix = is_svd(o) || o->algorithm == UNC_SVD_SCHUR;
    // the fixed points' slots past 6 (P - 3) are left as the caller had them (compute.cpp:511,526)
    const size_t head = no_fix ? (size_t)P : (P > 3 ? (size_t)(P - 3) : 0);
    rc = copy_host(ctx,
                   {{cam_unc, co, sizeof(double) * 45 * (size_t)C},
                    {pt_unc, po, sizeof(double) * 6 * head}},
                   false, sm);
    if (rc) return rc;
    if (!no_fix) {
        int fx[3] = {o->pts2fix[0], o->pts2fix[1], o->pts2fix[2]};
        std::sort(fx, fx + 2);
        for (int q = (int)head; q < P; ++q) {
            if (q == fx[0] || q == fx[1] || q == fx[2]) continue;
            CK(cudaMemcpyAsync(pt_unc + 6L * q, po + 6L * q, sizeof(double) * 6, cudaMemcpyDeviceToHost, sm));
        }
    }
    CK(cudaStreamSynchronize(sm));
    return UNC_OK;
}

int unc_dense_inverse_device(double* d_A, int n, int lda, void* stream) {
    return dense_inverse(d_A, n, lda, stream, 0, -1);
}

int unc_spd_inverse_tasks_bounded(double* d_A, int n, int lda, long long poll_limit, int skip_task, void* stream) {
    g_last_error.clear();
    if (!spd_tasks_apply(n)) return fail(UNC_ERR_INVALID_ARG, "the tile-task inverse takes n in 1..3584");
    if (poll_limit < 1 || poll_limit > (1LL << 22)) return fail(UNC_ERR_INVALID_ARG, "poll_limit must be in 1..2^22");
    return dense_inverse(d_A, n, lda, stream, poll_limit, skip_task);
}

int unc_jtj_crs(int num_rows, int num_cols, const int* rows, const int* cols, const double* values,
                int num_cams, int cam_params, long long* nnz_out, int* out_rows, int* out_cols,
                double* out_vals) {
    g_last_error.clear();
    if (!rows || !cols || !values || !nnz_out || num_rows < 0 || (num_rows & 1) || num_cams <= 0)
        return fail(UNC_ERR_INVALID_ARG, "bad arguments");
    if (cam_params != kCamParams) return fail(UNC_ERR_UNSUPPORTED, "only 9 camera parameters are supported");
    const int C = num_cams, cam_off = 9 * C;
    if (num_cols < cam_off || (num_cols - cam_off) % 3) return fail(UNC_ERR_INVALID_ARG, "bad num_cols");
    const int P = (num_cols - cam_off) / 3;
    const int nobs = num_rows / 2;
    const long long nnz = rows[num_rows];
    if (rows[0] != 0) return fail(UNC_ERR_INVALID_ARG, "rowptr must start at 0");
    for (int i = 0; i < num_rows; ++i)
        if (rows[i + 1] < rows[i] || rows[i + 1] > nnz) return fail(UNC_ERR_INVALID_ARG, "rowptr not monotone");
    // device buffers
    int *d_rows = nullptr, *d_cols = nullptr;
    double *d_vals = nullptr, *d_J = nullptr, *d_U = nullptr, *d_W = nullptr;
    SceneDev s{};
    s.num_cams = C;
    s.num_points = P;
    s.num_obs = nobs;
    std::vector<void*> owned;
    auto dal = [&](void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess) owned.push_back(*p);
        return e;
    };
    struct Free {
        std::vector<void*>& v;
        ~Free() {
            for (void* p : v) cudaFree(p);
        }
    } fr{owned};
    cudaStream_t sm = nullptr;
    CK(dal((void**)&d_rows, sizeof(int) * ((size_t)num_rows + 1)));
    CK(dal((void**)&d_cols, sizeof(int) * (size_t)nnz));
    CK(dal((void**)&d_vals, sizeof(double) * (size_t)nnz));
    CK(dal((void**)&d_J, sizeof(double) * 24 * (size_t)nobs));
    CK(dal((void**)&s.obs_cam, sizeof(int) * (size_t)nobs));
    CK(dal((void**)&s.obs_pt, sizeof(int) * (size_t)nobs));
    CK(dal((void**)&s.cam_ptr, sizeof(int) * ((size_t)C + 1)));
    CK(dal((void**)&s.cam_obs, sizeof(int) * (size_t)nobs));
    CK(dal((void**)&s.pt_ptr, sizeof(int) * ((size_t)P + 1)));
    CK(dal((void**)&s.pt_obs, sizeof(int) * (size_t)nobs));
    CK(dal((void**)&s.cursor, sizeof(int) * ((size_t)C + P + 1)));
    CK(dal((void**)&s.scan_tmp, sizeof(int) * scan_tmp_ints(std::max(C, P))));
    CK(dal((void**)&s.s_pt, sizeof(double) * 3 * (size_t)P));
    CK(dal((void**)&s.Vraw, sizeof(double) * 6 * (size_t)P));
    CK(dal((void**)&s.iVs, sizeof(double) * 6 * (size_t)P));
    CK(dal((void**)&s.err, sizeof(int) * 4));
    CK(dal((void**)&d_U, sizeof(double) * 81 * (size_t)C));
    CK(dal((void**)&d_W, sizeof(double) * 27 * (size_t)nobs));
    s.J = d_J;
    CK(cudaMemcpy(d_rows, rows, sizeof(int) * ((size_t)num_rows + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_cols, cols, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_vals, values, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice));
    CK(cudaMemset(s.err, 0, 16));
    launch_repack_generic(nobs, cam_off, d_rows, d_cols, d_vals, d_J, s.obs_cam, s.obs_pt, s.err, sm);
    launch_build_index(s, sm);
    launch_point_blocks(s, sm);
    launch_unscaled_blocks(s, d_U, d_W, sm);
    CK(cudaDeviceSynchronize());
    int err = 0;
    CK(cudaMemcpy(&err, s.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err & ERRBIT_LAYOUT) return fail(UNC_ERR_LAYOUT, "rows must have 12 (camera + point) or 9 (camera) entries");
    std::vector<double> U(81 * (size_t)C), W(27 * (size_t)nobs), V(6 * (size_t)P);
    std::vector<int> ocam(nobs), opt(nobs);
    CK(cudaMemcpy(U.data(), d_U, sizeof(double) * U.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(W.data(), d_W, sizeof(double) * W.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(V.data(), s.Vraw, sizeof(double) * V.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ocam.data(), s.obs_cam, sizeof(int) * nobs, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(opt.data(), s.obs_pt, sizeof(int) * nobs, cudaMemcpyDeviceToHost));
    // Pattern of J^T J from the block structure: camera rows hold their own
    // 9x9 block then one 3-wide block per observed point; point rows hold one
    // 9-wide block per observing camera then their own 3x3 block.
    std::vector<char> cam_seen(C, 0);
    std::vector<std::vector<std::pair<int, int>>> cam_pts(C), pt_cams(P);  // (other id, obs)
    for (int o = 0; o < nobs; ++o) {
        if (ocam[o] < 0) continue;
        cam_seen[ocam[o]] = 1;
        if (opt[o] >= 0) {
            cam_pts[ocam[o]].push_back({opt[o], o});
            pt_cams[opt[o]].push_back({ocam[o], o});
        }
    }
    for (auto& v : cam_pts) std::sort(v.begin(), v.end());
    for (auto& v : pt_cams) std::sort(v.begin(), v.end());
    std::vector<int> orow(num_cols + 1, 0), ocol;
    std::vector<double> oval;
    for (int c = 0; c < C; ++c)
        for (int j = 0; j < 9; ++j) {
            if (cam_seen[c])
                for (int k = 0; k < 9; ++k) {
                    ocol.push_back(9 * c + k);
                    oval.push_back(U[81L * c + 9 * j + k]);
                }
            auto& lst = cam_pts[c];
            for (size_t a = 0; a < lst.size();) {
                size_t e = a;
                double sum[3] = {0, 0, 0};
                while (e < lst.size() && lst[e].first == lst[a].first) {
                    for (int k = 0; k < 3; ++k) sum[k] += W[27L * lst[e].second + 3 * j + k];
                    ++e;
                }
                for (int k = 0; k < 3; ++k) {
                    ocol.push_back(cam_off + 3 * lst[a].first + k);
                    oval.push_back(sum[k]);
                }
                a = e;
            }
            orow[9 * c + j + 1] = (int)ocol.size();
        }
    for (int p = 0; p < P; ++p)
        for (int k = 0; k < 3; ++k) {
            auto& lst = pt_cams[p];
            for (size_t a = 0; a < lst.size();) {
                size_t e = a;
                double sum[9] = {0};
                while (e < lst.size() && lst[e].first == lst[a].first) {
                    for (int j = 0; j < 9; ++j) sum[j] += W[27L * lst[e].second + 3 * j + k];
                    ++e;
                }
                for (int j = 0; j < 9; ++j) {
                    ocol.push_back(9 * lst[a].first + j);
                    oval.push_back(sum[j]);
                }
                a = e;
            }
            if (!lst.empty()) {
                const double* v = V.data() + 6L * p;
                const double full[3][3] = {{v[0], v[1], v[2]}, {v[1], v[3], v[4]}, {v[2], v[4], v[5]}};
                for (int q = 0; q < 3; ++q) {
                    ocol.push_back(cam_off + 3 * p + q);
                    oval.push_back(full[k][q]);
                }
            }
            orow[cam_off + 3 * p + k + 1] = (int)ocol.size();
        }
    *nnz_out = (long long)ocol.size();
    if (out_cols) {
        if (!out_rows || !out_vals) return fail(UNC_ERR_INVALID_ARG, "null output arrays");
        std::copy(orow.begin(), orow.end(), out_rows);
        std::copy(ocol.begin(), ocol.end(), out_cols);
        std::copy(oval.begin(), oval.end(), out_vals);
    }
    return UNC_OK;
}

int unc_gemm_f64_device(int M, int N, int K, double alpha, const double* d_A, int lda, const double* d_B,
                        int ldb, double beta, double* d_C, int ldc, void* stream) {
    g_last_error.clear();
    if (M < 0 || N < 0 || K < 0 || !d_A || !d_B || !d_C || (lda & 1) || (ldb & 1) || lda < M || ldb < K ||
        ldc < M || ((uintptr_t)d_A & 15) || ((uintptr_t)d_B & 15))
        return fail(UNC_ERR_INVALID_ARG, "bad GEMM arguments");
    gemm_f64(M, N, K, alpha, d_A, lda, d_B, ldb, beta, d_C, ldc, nullptr, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return UNC_OK;
}

int unc_gemm_mixed_device(int n, const double* d_P, const double* d_X, int ld, double* d_C, int slices,
                          void* stream) {
    g_last_error.clear();
    if (n <= 0 || !d_P || !d_X || !d_C || ld < n || slices < 3 || slices > 5)
        return fail(UNC_ERR_INVALID_ARG, "bad mixed GEMM arguments");
    cudaStream_t sm = (cudaStream_t)stream;
    const size_t sb = mixed_slice_bytes(n, slices);
    char* ws = nullptr;
    const size_t exp_off = 2 * ((sb + 255) & ~size_t(255));
    CK(cudaMalloc(&ws, exp_off + 2 * sizeof(int) * ((size_t)n + 64) + 256));
    int8_t* bufP = reinterpret_cast<int8_t*>(ws);
    int8_t* bufX = reinterpret_cast<int8_t*>(ws + (exp_off / 2));
    int* eP = reinterpret_cast<int*>(ws + exp_off);
    int* eX = eP + n + 64;
    int* err = eX + n + 64;
    MixedOperand a, b;
    if (!mixed_plan(a, bufP, eP, n, slices, false) || !mixed_plan(b, bufX, eX, n, slices, true)) {
        cudaFree(ws);
        return fail(UNC_ERR_CUDA, "tensor-map encoding failed");
    }
    int h_err = 0;
    cudaError_t ce = cudaMemsetAsync(ws, 0, exp_off + 2 * sizeof(int) * ((size_t)n + 64) + 256, sm);
    if (ce == cudaSuccess) {
        mixed_slice(d_P, ld, a, sm);
        mixed_slice(d_X, ld, b, sm);
        mixed_gemm(a, b, d_C, ld, nullptr, false, err, sm);
        ce = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, sm);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(sm);
    cudaFree(ws);
    if (ce != cudaSuccess) return fail(UNC_ERR_CUDA, cudaGetErrorString(ce));
    if (h_err & ERRBIT_TIMEOUT) return fail(UNC_ERR_CUDA, "tensor-core pipeline wait timed out");
    return UNC_OK;
}

int unc_gram_lower_mixed_device(int n, const double* d_T, int ld, double* d_A, void* stream) {
    g_last_error.clear();
    if (n <= 0 || !d_T || !d_A || ld < n) return fail(UNC_ERR_INVALID_ARG, "bad mixed Gram arguments");
    cudaStream_t sm = (cudaStream_t)stream;
    const size_t sb = mixed_gram_bytes(n);
    const size_t total = sb + sizeof(int) * ((size_t)n + 64) + 256;
    char* ws = nullptr;
    CK(cudaMalloc(&ws, total));
    int* ex = reinterpret_cast<int*>(ws + sb);
    int* err = ex + n + 64;
    int h_err = 0;
    cudaError_t ce = cudaMemsetAsync(ws, 0, total, sm);
    if (ce == cudaSuccess && !mixed_gram_lower_tri(d_T, n, ld, reinterpret_cast<int8_t*>(ws), ex, d_A, ld, err, sm)) {
        cudaStreamSynchronize(sm);
        cudaFree(ws);
        return fail(UNC_ERR_CUDA, "tensor-map encoding failed");
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, sm);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(sm);
    cudaFree(ws);
    if (ce != cudaSuccess) return fail(UNC_ERR_CUDA, cudaGetErrorString(ce));
    if (h_err & ERRBIT_TIMEOUT) return fail(UNC_ERR_CUDA, "tensor-core pipeline wait timed out");
    return UNC_OK;
}

const char* unc_status_string(int s) {
    switch (s) {
        case UNC_OK: return "UNC_OK";
        case UNC_ERR_INVALID_ARG: return "UNC_ERR_INVALID_ARG";
        case UNC_ERR_LAYOUT: return "UNC_ERR_LAYOUT";
        case UNC_ERR_NO_FIXED_POINTS: return "UNC_ERR_NO_FIXED_POINTS";
        case UNC_ERR_CUDA: return "UNC_ERR_CUDA";
        case UNC_ERR_OUT_OF_MEMORY: return "UNC_ERR_OUT_OF_MEMORY";
        case UNC_ERR_SINGULAR: return "UNC_ERR_SINGULAR";
        case UNC_ERR_UNSUPPORTED: return "UNC_ERR_UNSUPPORTED";
        case UNC_ERR_TOO_LARGE: return "UNC_ERR_TOO_LARGE";
        case UNC_ERR_TIMEOUT: return "UNC_ERR_TIMEOUT";
        default: return "UNC_ERR_UNKNOWN";
    }
}

const char* unc_last_error(void) { return g_last_error.c_str(); }

long long unc_kernel_launches(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

}  // extern "C"
