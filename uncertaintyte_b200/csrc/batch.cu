// batch.cu - many reconstructions solved together: one grouped launch
// sequence over a batch of scenes (host code).
//
// The reference computes one reconstruction per call (computeCovariances,
// compute.cpp:458-540) and is not re-entrant; this is the batched form of that
// call, with no counterpart there. Per batch:
//
//   * inputs of all scenes packed into one pinned staging area by host
//     threads, each piece sent to the device as soon as it is packed; outputs
//     come back in one transfer and are unpacked by host threads;
//   * the sparse stages (validation, J^T J blocks, Schur complement) of every
//     scene as parallel branches of one launch sequence;
//   * the dense stage grouped across scenes: one persistent tile-task kernel
//     runs the SPD inverses of all scenes from one interleaved work list, and
//     every step of the blocked-power Taylor evaluation (powers.cu: slicing,
//     int8 tensor-core products, diagonal maxima, stop rule, coefficient
//     blocks) is one launch over the tiles / rows / columns of all scenes;
//   * the camera and point outputs again as parallel branches.
//
// The sequence for a given batch shape (sizes, fixed points, lambda, buffer
// addresses) is captured in a CUDA graph the second time the shape is seen and
// replayed from then on. The product's tile width (64 or 96 for 5 slices)
// comes from a cost model of the group's tiles on the SMs; the products'
// per-element arithmetic does not depend on it.
// Every grouped kernel performs, per element, exactly the arithmetic of its
// per-scene counterpart, so each scene's result is bitwise the one
// unc_compute gives for it alone.
//
// Scenes the grouped path does not cover (the SVD algorithms, the FP64
// precision, the sequential Taylor evaluation, N = 9 cameras above 3584) are
// computed one after another with unc_compute in the same call.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>
#include <vector>

#include "../../include/uncte.h"
#include "pipeline.h"

using namespace unc;

namespace {

#define BCK(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
            return e_ == cudaErrorMemoryAllocation ? UNC_ERR_OUT_OF_MEMORY : UNC_ERR_CUDA;        \
        }                                                                                         \
    } while (0)

int bfail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

constexpr int kBranches = 8;      // parallel streams for the per-scene stages
constexpr int kGraphs = 4;        // batch-shape graphs kept
constexpr int kTaylorIters = 19;  // Taylor iterations at most (compute.cpp:145)

struct Scene {
    int idx;  // position in the caller's arrays
    unc_options opt;
    Plan pl;
    long long nnz;
    int fx[3];
    double lambda;
    Buffers b;
    int* in_rows;
    int* in_cols;
    double* in_vals;
    double* out_cam;
    double* out_pt;
    size_t in_off[3], out_off[2];  // byte offsets in the staging areas
    int8_t* buf[6];  // slices of X, of the A operand of the moment, of X^4, X^8, X^12, X^16
    int* ex[6];      // their row exponents
};

struct Layout {
    size_t in_bytes = 0, out_bytes = 0, total = 0;
    // device regions (offsets)
    size_t mixed_off = 0, mixed_bytes = 0;
    size_t zero_off = 0, zero_bytes = 0;  // dag states + control words
    size_t amax_off = 0, amax_bytes = 0;
    size_t stat_off = 0, stat_bytes = 0;  // error words + Taylor states
    size_t desc_off = 0, desc_bytes = 0;  // descriptors uploaded from the host
};

struct Graph {
    std::vector<unsigned long long> key;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
};

}  // namespace

struct unc_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t branch[kBranches] = {};
    cudaEvent_t fork = nullptr, join[kBranches] = {}, ev[4] = {};
    void* ws = nullptr;
    size_t ws_bytes = 0;
    void* host = nullptr;  // pinned staging: inputs, outputs, descriptors, status words
    size_t host_bytes = 0;
    // outgrown staging areas, freed with the batch: cudaFreeHost waits for the
    // whole device (every other stream's work), so a serving worker never calls
    // it while other requests compute; the sizes grow by half at least, so the
    // retired areas hold at most twice the current one
    std::vector<void*> host_retired;
    std::vector<Graph> graphs;
    std::vector<std::vector<unsigned long long>> seen;
    unc_context* single = nullptr;                  // scenes outside the grouped path
    double t_h2d = 0, t_dev = 0, t_d2h = 0;
    int grouped = 0, tile_n = 0;
    int force_nt = 0;  // unc_batch_set_tile_width: 0 = cost model
};

namespace {

struct Copy {
    void* dst;
    const void* src;
    size_t bytes;
};

// Host-side copies with several threads (the staging area is pinned; the
// caller's arrays are ordinary host memory).
void parallel_copy(const std::vector<Copy>& jobs) {
    const int nt = (int)std::min<size_t>(16, std::max<size_t>(1, std::thread::hardware_concurrency()));
    size_t total = 0;
    for (auto& j : jobs) total += j.bytes;
    if (total < (64u << 20) || nt == 1) {
        for (auto& j : jobs) memcpy(j.dst, j.src, j.bytes);
        return;
    }
    // split every copy into pieces of at most 8 MB and deal them out
    struct Piece {
        char* d;
        const char* s;
        size_t n;
    };
    std::vector<Piece> pieces;
    for (auto& j : jobs)
        for (size_t o = 0; o < j.bytes; o += (8u << 20))
            pieces.push_back({(char*)j.dst + o, (const char*)j.src + o, std::min<size_t>(8u << 20, j.bytes - o)});
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (size_t p = t; p < pieces.size(); p += nt) memcpy(pieces[p].d, pieces[p].s, pieces[p].n);
        });
    for (auto& x : th) x.join();
}

// The inputs into the pinned staging area and on to the device: the staging
// area mirrors the device region byte for byte (dev = stage_base -> dev_base),
// so every thread sends each 8 MB piece as soon as it has copied it, and the
// host copies overlap the transfers. Small totals: host copies, then one
// transfer of the whole region.
cudaError_t parallel_copy_to_device(const std::vector<Copy>& jobs, const char* stage_base, char* dev_base,
                                    size_t region_bytes, int device, cudaStream_t sm) {
    const int nt = (int)std::min<size_t>(16, std::max<size_t>(1, std::thread::hardware_concurrency()));
    size_t total = 0;
    for (auto& j : jobs) total += j.bytes;
    if (total < (64u << 20) || nt == 1) {
        parallel_copy(jobs);
        return cudaMemcpyAsync(dev_base, stage_base, region_bytes, cudaMemcpyHostToDevice, sm);
    }
    struct Piece {
        char* d;
        const char* s;
        size_t n;
    };
    std::vector<Piece> pieces;
    for (auto& j : jobs)
        for (size_t o = 0; o < j.bytes; o += (8u << 20))
            pieces.push_back({(char*)j.dst + o, (const char*)j.src + o, std::min<size_t>(8u << 20, j.bytes - o)});
    std::vector<cudaError_t> err(nt, cudaSuccess);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            if ((err[t] = cudaSetDevice(device)) != cudaSuccess) return;
            for (size_t p = t; p < pieces.size(); p += nt) {
                memcpy(pieces[p].d, pieces[p].s, pieces[p].n);
                err[t] = cudaMemcpyAsync(dev_base + (pieces[p].d - stage_base), pieces[p].d, pieces[p].n,
                                         cudaMemcpyHostToDevice, sm);
                if (err[t] != cudaSuccess) return;
            }
        });
    for (auto& x : th) x.join();
    for (cudaError_t e : err)
        if (e != cudaSuccess) return e;
    return cudaSuccess;
}

int slices_of(int precision) {
    return precision == UNC_PRECISION_MIXED4 ? 4 : (precision == UNC_PRECISION_MIXED3 ? 3 : 5);
}

// per scene: X (A, B), A operand (A), X^4 (A, B), X^8 (A, B), X^12 (B), X^16 (B), and X^4, X^8, X^12, X^16
// as B operands of 128-column tiles (the products with fewer slices than the group's)
constexpr int kMaps = 13;
// descriptor sets (the last four of each are laid out but not launched: the
// block terms X^(4q) G_q are formed on the camera blocks, launch_taylor_blocks)
constexpr int kSliceSets = 11;  // X, X^2, X^3, X^4, X^8, X^12, X^16, G_1..G_4
constexpr int kGemmSets = 10;   // X^2, X^3, X^4, X^8, X^12, X^16, X^4 G_1 .. X^16 G_4

// Device addresses of the descriptor region, in lay_out's order.
struct Desc {
    SpdTaskMatrix* mats;
    int4* tasks;
    CUtensorMap* maps;
    DenseJob* dense;
    long* blk_rows;
    long* blk_elems;
    long* blk_cols;
    MixedSliceJob* slice;  // kSliceSets sets of n jobs
    int* row_start;
    MixedGemmJob* gemm;    // kGemmSets sets of n jobs
    int4* tiles;
    PowerSet* powers;
    double* kpow;          // 19 coefficients per scene
};

// With measure: advance that carver (sizes only); else lay out at base.
Desc desc_at(char* base, size_t n, size_t ntasks, size_t ntiles, Carver* measure) {
    Carver own{base};
    Carver& c = measure ? *measure : own;
    Desc d;
    d.mats = c.take<SpdTaskMatrix>(n);
    d.tasks = c.take<int4>(ntasks);
    d.maps = c.take<CUtensorMap>(kMaps * n);
    d.dense = c.take<DenseJob>(n);
    d.blk_rows = c.take<long>(n + 1);
    d.blk_elems = c.take<long>(n + 1);
    d.blk_cols = c.take<long>(n + 1);
    d.slice = c.take<MixedSliceJob>(kSliceSets * n);
    d.row_start = c.take<int>(n + 1);
    d.gemm = c.take<MixedGemmJob>(kGemmSets * n);
    d.tiles = c.take<int4>(ntiles);
    d.powers = c.take<PowerSet>(n);
    d.kpow = c.take<double>(19 * n);
    return d;
}

// Lay out the device workspace of a group for tile width nt (base == nullptr:
// sizes only). Fills the per-scene pointers.
void lay_out(char* base, std::vector<Scene>& sc, int slices, int nt, Layout& L, size_t ntasks, size_t ntiles) {
    Carver c{base};
    const size_t in0 = c.off;
    for (auto& s : sc) {
        s.in_rows = c.take<int>((size_t)s.pl.nobs * 2 + 1);
        s.in_off[0] = (char*)s.in_rows - base;
        s.in_cols = c.take<int>((size_t)s.nnz);
        s.in_off[1] = (char*)s.in_cols - base;
        s.in_vals = c.take<double>((size_t)s.nnz);
        s.in_off[2] = (char*)s.in_vals - base;
    }
    c.off = (c.off + 255) & ~size_t(255);
    L.in_bytes = c.off - in0;
    const size_t out0 = c.off;
    for (auto& s : sc) {
        s.out_cam = c.take<double>((size_t)s.pl.C * 45);
        s.out_off[0] = (char*)s.out_cam - base;
        s.out_pt = c.take<double>((size_t)s.pl.P * 6);
        s.out_off[1] = (char*)s.out_pt - base;
    }
    c.off = (c.off + 255) & ~size_t(255);
    L.out_bytes = c.off - out0;
    for (auto& s : sc) {
        const size_t need = carve(nullptr, s.pl, false, 0, s.pl.nobs * 2, s.b);
        char* at = c.take<char>(need);
        carve(base ? at : nullptr, s.pl, false, 0, s.pl.nobs * 2, s.b);
    }
    c.off = (c.off + 255) & ~size_t(255);
    L.mixed_off = c.off;
    for (auto& s : sc) {
        const size_t sb = mixed_slice_bytes_nt(s.pl.N, slices, nt);
        for (int q = 0; q < 6; ++q) s.buf[q] = c.take<int8_t>(sb);
        for (int q = 0; q < 6; ++q) s.ex[q] = c.take<int>((size_t)s.pl.N + 64);
    }
    c.off = (c.off + 255) & ~size_t(255);
    L.mixed_bytes = c.off - L.mixed_off;
    // zero at the start of the dense stage: tile-task counters of every scene,
    // the powers' diagonal maxima, control words (last)
    L.zero_off = c.off;
    for (auto& s : sc) s.b.dag_state = c.take<int>(spd_task_state_ints(s.pl.N));
    for (auto& s : sc) s.b.dmax = c.take<unsigned long long>(24);
    c.take<int>(4);
    c.off = (c.off + 255) & ~size_t(255);
    L.zero_bytes = c.off - L.zero_off;
    L.amax_off = c.off;
    for (auto& s : sc) s.b.amax = c.take<unsigned long long>(4);
    c.off = (c.off + 255) & ~size_t(255);
    L.amax_bytes = c.off - L.amax_off;
    // status words read back at the end: error words, then Taylor states
    L.stat_off = c.off;
    int* errs = c.take<int>(4 * sc.size());
    TeState* te = c.take<TeState>(sc.size());
    c.off = (c.off + 255) & ~size_t(255);
    L.stat_bytes = c.off - L.stat_off;
    for (size_t i = 0; i < sc.size(); ++i) {
        sc[i].b.s.err = base ? errs + 4 * i : nullptr;
        sc[i].b.te = base ? te + i : nullptr;
    }
    // descriptors (host-filled, one upload)
    L.desc_off = c.off;
    desc_at(nullptr, sc.size(), ntasks, ntiles, &c);
    c.off = (c.off + 255) & ~size_t(255);
    L.desc_bytes = c.off - L.desc_off;
    L.total = c.off + 256;
}

struct GroupRun {
    std::vector<Scene> sc;
    int slices = 5, nt = 96;
    Layout L;
    size_t ntasks = 0, ntiles = 0;
    size_t ntiles_nt = 0, ntiles_128 = 0;  // tiles of width nt, then (nt != 128) of width 128
    long nblk_rows = 0, nblk_elems = 0, nblk_cols = 0;
    int total_rows = 0;
    Desc dd{};  // device descriptors
    char* dbase = nullptr;
    char* hbase = nullptr;  // staging: [IN | OUT | descriptors | status]
    size_t h_in = 0, h_out = 0, h_desc = 0, h_stat = 0;
};

// The launch sequence of a group on b->stream (captured or direct).
int launch_group(unc_batch* b, GroupRun& g) {
    cudaStream_t sm = b->stream;
    const int n = (int)g.sc.size();
    BCK(cudaEventRecord(b->fork, sm));
    for (int k = 0; k < kBranches; ++k) BCK(cudaStreamWaitEvent(b->branch[k], b->fork, 0));
    for (int i = 0; i < n; ++i) {
        Scene& s = g.sc[i];
        cudaStream_t br = b->branch[i % kBranches];
        int fx[3];
        if (int r = sparse_stage(&s.opt, s.pl, s.nnz, s.in_rows, s.in_cols, s.in_vals, s.b, fx, nullptr, br))
            return r;
        const int N = s.pl.N, ld = s.pl.ld;
        if (ld != N)  // padding rows of the extra power buffers must stay finite for the product loads
            for (double* m : {s.b.p4, s.b.p8, s.b.p12, s.b.p16, s.b.g})
                BCK(cudaMemset2DAsync(m + N, sizeof(double) * (size_t)ld, 0, sizeof(double) * (size_t)(ld - N), N,
                                      br));
    }
    for (int k = 0; k < kBranches; ++k) {
        BCK(cudaEventRecord(b->join[k], b->branch[k]));
        BCK(cudaStreamWaitEvent(sm, b->join[k], 0));
    }
    // the dense stage, grouped (compute.cpp:121-166)
    BCK(cudaMemsetAsync(g.dbase + g.L.mixed_off, 0, g.L.mixed_bytes, sm));  // slice padding must be zero
    BCK(cudaMemsetAsync(g.dbase + g.L.zero_off, 0, g.L.zero_bytes, sm));
    launch_shift_equilibrate_grouped(g.dd.dense, n, g.dd.blk_rows, g.nblk_rows, g.dd.blk_elems, g.nblk_elems, sm);
    int* ctl = reinterpret_cast<int*>(g.dbase + g.L.zero_off + g.L.zero_bytes - 256);
    if (int r = chol_inverse_tasks_grouped(g.dd.mats, g.dd.tasks, (int)g.ntasks, ctl, sm, device_sms())) return r;
    launch_unequilibrate_grouped(g.dd.dense, n, g.dd.blk_elems, g.nblk_elems, sm);  // X in Z, iZ = X
    // the Taylor series from blocked powers (powers.cu), every step over all scenes
    auto slice = [&](int set) {
        mixed_slice_grouped(g.dd.slice + (size_t)set * n, n, g.dd.row_start, g.total_rows, sm);
    };
    auto gemm = [&](int set) {  // product `set` with its slices (power_product_slices)
        const int k = power_product_slices(set, g.slices);
        if (k == g.slices || g.nt == 128)
            mixed_gemm_grouped(k, g.nt, g.dd.gemm + (size_t)set * n, g.dd.tiles, (int)g.ntiles_nt, sm);
        else
            mixed_gemm_grouped(k, 128, g.dd.gemm + (size_t)set * n, g.dd.tiles + g.ntiles_nt, (int)g.ntiles_128,
                               sm);
    };
    slice(0);  // X
    launch_te_init_grouped(g.dd.dense, n, sm);
    gemm(0);  // X^2
    slice(1);
    gemm(1);  // X^3
    slice(2);
    gemm(2);  // X^4
    slice(3);
    gemm(3);  // X^8
    slice(4);
    gemm(4);  // X^12
    slice(5);
    launch_power_diag_grouped(g.dd.powers, n, g.dd.blk_cols, g.nblk_cols, 2, 16, false, sm);
    launch_power_decide_grouped(g.dd.powers, n, g.dd.kpow, 1, 15, sm);
    gemm(5);  // X^16 (skipped per scene)
    slice(6);
    launch_power_diag_grouped(g.dd.powers, n, g.dd.blk_cols, g.nblk_cols, 17, 20, true, sm);
    launch_power_decide_grouped(g.dd.powers, n, g.dd.kpow, 16, 19, sm);
    launch_power_combine_grouped(g.dd.powers, n, g.dd.blk_elems, g.nblk_elems, 0, sm);  // iZ = G_0
    // iZ += X^(4q) G_q on the camera blocks (the per-scene path's device function)
    launch_taylor_blocks_grouped(g.dd.powers, n, g.dd.blk_cols, g.nblk_cols, sm);
    // outputs (compute.cpp:168-183, 370-455)
    BCK(cudaEventRecord(b->fork, sm));
    for (int k = 0; k < kBranches; ++k) BCK(cudaStreamWaitEvent(b->branch[k], b->fork, 0));
    for (int i = 0; i < n; ++i) output_stage(g.sc[i].pl, g.sc[i].b, g.sc[i].out_cam, g.sc[i].out_pt,
                                             b->branch[i % kBranches]);
    for (int k = 0; k < kBranches; ++k) {
        BCK(cudaEventRecord(b->join[k], b->branch[k]));
        BCK(cudaStreamWaitEvent(sm, b->join[k], 0));
    }
    return UNC_OK;
}

// Prepare a group for tile width nt: layout, buffers, descriptors uploaded.
int prepare_group(unc_batch* b, GroupRun& g, int nt) {
    g.nt = nt;
    const int n = (int)g.sc.size();
    std::vector<int> ns(n);
    for (int i = 0; i < n; ++i) ns[i] = g.sc[i].pl.N;
    const std::vector<int4> tasks = spd_tasks_grouped_list(ns);
    g.ntasks = tasks.size();
    // product tiles, larger K first (longer tiles start early)
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return ns[a] > ns[c]; });
    std::vector<int4> tiles;
    for (int i : order) mixed_lower_tiles(i, ns[i], nt, tiles);
    g.ntiles_nt = tiles.size();
    if (nt != 128)
        for (int i : order) mixed_lower_tiles(i, ns[i], 128, tiles);
    g.ntiles_128 = tiles.size() - g.ntiles_nt;
    g.ntiles = tiles.size();
    lay_out(nullptr, g.sc, g.slices, nt, g.L, g.ntasks, g.ntiles);
    cudaStream_t sm = b->stream;
    if (b->ws_bytes < g.L.total) {
        if (b->ws) BCK(cudaFreeAsync(b->ws, sm));
        b->ws = nullptr;
        b->ws_bytes = 0;
        BCK(cudaMallocAsync(&b->ws, g.L.total, sm));
        b->ws_bytes = g.L.total;
        for (auto& gr : b->graphs) cudaGraphExecDestroy(gr.exec);  // they name the old addresses
        b->graphs.clear();
    }
    g.dbase = (char*)b->ws;
    lay_out(g.dbase, g.sc, g.slices, nt, g.L, g.ntasks, g.ntiles);
    // pinned staging: [IN | OUT | descriptors | status]
    g.h_in = 0;
    g.h_out = g.L.in_bytes;
    g.h_desc = g.h_out + g.L.out_bytes;
    g.h_stat = g.h_desc + g.L.desc_bytes;
    const size_t hneed = g.h_stat + g.L.stat_bytes + 256;
    if (b->host_bytes < hneed) {
        // grown by half again at least; the old area is retired (freed with the batch)
        const size_t want = std::max(hneed, b->host_bytes + b->host_bytes / 2);
        BCK(cudaStreamSynchronize(sm));
        if (b->host) b->host_retired.push_back(b->host);
        b->host = nullptr;
        b->host_bytes = 0;
        BCK(cudaMallocHost(&b->host, want));
        b->host_bytes = want;
    }
    g.hbase = (char*)b->host;
    // descriptors
    g.dd = desc_at(g.dbase + g.L.desc_off, n, g.ntasks, g.ntiles, nullptr);
    BCK(cudaStreamSynchronize(sm));  // the staging area is reused
    char* hd = g.hbase + g.h_desc;
    const Desc hdd = desc_at(hd, n, g.ntasks, g.ntiles, nullptr);
    memset(hd, 0, g.L.desc_bytes);
    long br = 0, be = 0, bc = 0;
    int rs = 0;
    for (int i = 0; i < n; ++i) {
        Scene& s = g.sc[i];
        const int N = s.pl.N;
        const long ld = s.pl.ld;
        const int nt64 = (N + 63) / 64;
        hdd.mats[i] = SpdTaskMatrix{s.b.Z, s.b.iZ, s.b.add, ld, N, nt64 * (nt64 + 1) / 2, s.b.dag_state, s.b.s.err};
        // tensor maps: X (A, B), A operand (A), X^4 (A, B), X^8 (A, B), X^12 (B), X^16 (B); then
        // X^4, X^8, X^12, X^16 as B operands with 128-row boxes (same buffers and plane stride)
        const int mbuf[kMaps] = {0, 0, 1, 2, 2, 3, 3, 4, 5, 2, 3, 4, 5};
        const bool mb[kMaps] = {false, true, false, false, true, false, true, true, true, true, true, true, true};
        MixedOperand op[kMaps];
        for (int m = 0; m < kMaps; ++m) {
            bool ok = mixed_plan_nt(op[m], s.buf[mbuf[m]], s.ex[mbuf[m]], N, g.slices, mb[m], nt);
            if (ok && m >= 9) op[m] = mixed_fewer_slices(op[m], 2, true, &ok);  // 128-row boxes
            if (!ok) return bfail(UNC_ERR_CUDA, "tensor-map encoding failed");
            hdd.maps[kMaps * i + m] = op[m].map;
        }
        const int rows = op[0].rows, kp = op[0].kp;
        hdd.dense[i] = DenseJob{s.b.Z, s.b.iZ, s.b.add, s.b.e, ld, N, s.lambda, s.b.s.err, s.b.te, s.b.amax};
        hdd.blk_rows[i] = br;
        hdd.blk_elems[i] = be;
        hdd.blk_cols[i] = bc;
        br += (N + 255) / 256;
        be += ((long)N * N + 255) / 256;
        bc += N;
        hdd.row_start[i] = rs;
        rs += N;
        // slicing sets (powers.cu's order): X, X^2, X^3, X^4, X^8, X^12, X^16, G_1..G_4
        const int* sk = s.b.te->skip;
        struct SliceDef {
            const double* src;
            int buf;
            const int* skip;
        };
        const SliceDef sd[kSliceSets] = {{s.b.Z, 0, nullptr},  {s.b.add, 1, nullptr}, {s.b.tmp, 1, nullptr},
                                         {s.b.p4, 2, nullptr}, {s.b.p8, 3, nullptr},  {s.b.p12, 4, nullptr},
                                         {s.b.p16, 5, sk},     {s.b.g, 1, sk + 1},    {s.b.g, 1, sk + 2},
                                         {s.b.g, 1, sk + 3},   {s.b.g, 1, sk + 4}};
        for (int q = 0; q < kSliceSets; ++q)
            hdd.slice[(size_t)q * n + i] = MixedSliceJob{sd[q].src, ld, N, g.slices, s.buf[sd[q].buf], rows, kp,
                                                         s.ex[sd[q].buf], nullptr, nullptr, sd[q].skip};
        // products: A map, B map, A / B exponent buffers, output, accumulate, skip
        const CUtensorMap* dm = g.dd.maps + kMaps * i;
        struct GemmDef {
            int a, b, b128, ea, eb;  // b128: the B map with 128-row boxes (-1: always full slices)
            double* C;
            int acc;
            const int* skip;
        };
        const GemmDef gd[kGemmSets] = {
            {0, 1, -1, 0, 0, s.b.add, 0, nullptr}, {2, 1, -1, 1, 0, s.b.tmp, 0, nullptr},
            {2, 1, -1, 1, 0, s.b.p4, 0, nullptr},  {3, 4, 9, 2, 2, s.b.p8, 0, nullptr},
            {5, 4, 9, 3, 2, s.b.p12, 0, nullptr},  {5, 6, 10, 3, 3, s.b.p16, 0, sk},
            {2, 4, 9, 1, 2, s.b.iZ, 1, sk + 1},    {2, 6, 10, 1, 3, s.b.iZ, 1, sk + 2},
            {2, 7, 11, 1, 4, s.b.iZ, 1, sk + 3},   {2, 8, 12, 1, 5, s.b.iZ, 1, sk + 4}};
        for (int q = 0; q < kGemmSets; ++q) {
            const bool narrow = power_product_slices(q, g.slices) != g.slices && nt != 128;
            const int bm = narrow ? gd[q].b128 : gd[q].b;
            if (bm < 0) return bfail(UNC_ERR_UNSUPPORTED, "slice schedule and map table disagree");
            hdd.gemm[(size_t)q * n + i] = MixedGemmJob{dm + gd[q].a,   dm + bm,        N,          kp, rows, rows,
                                                       s.ex[gd[q].ea], s.ex[gd[q].eb], gd[q].C,    ld, nullptr,
                                                       s.b.s.err,      gd[q].skip,     gd[q].acc};
        }
        PowerSet ps{};
        ps.M[0] = s.b.Z;
        ps.M[1] = s.b.add;
        ps.M[2] = s.b.tmp;
        ps.M[3] = s.b.p4;
        ps.M[4] = s.b.p8;
        ps.M[5] = s.b.p12;
        ps.M[6] = s.b.p16;
        ps.iZ = s.b.iZ;
        ps.G = s.b.g;
        ps.n = N;
        ps.ld = ld;
        ps.dmax = s.b.dmax;
        ps.te = s.b.te;
        hdd.powers[i] = ps;
        for (int it = 1; it <= kTaylorIters; ++it)
            hdd.kpow[19L * i + it - 1] = pow(s.lambda, it) / factorial_i32(it - 1);
    }
    hdd.blk_rows[n] = br;
    hdd.blk_elems[n] = be;
    hdd.blk_cols[n] = bc;
    hdd.row_start[n] = rs;
    g.nblk_rows = br;
    g.nblk_elems = be;
    g.nblk_cols = bc;
    g.total_rows = rs;
    memcpy(hdd.tasks, tasks.data(), sizeof(int4) * tasks.size());
    memcpy(hdd.tiles, tiles.data(), sizeof(int4) * tiles.size());
    BCK(cudaMemcpyAsync(g.dbase + g.L.desc_off, hd, g.L.desc_bytes, cudaMemcpyHostToDevice, sm));
    return UNC_OK;
}

std::vector<unsigned long long> shape_key(const unc_batch* b, const GroupRun& g) {
    std::vector<unsigned long long> k = {(unsigned long long)(uintptr_t)b->ws, (unsigned long long)g.sc.size(),
                                         (unsigned long long)g.slices, (unsigned long long)g.nt};
    for (const Scene& s : g.sc) {
        unsigned long long lam;
        memcpy(&lam, &s.lambda, 8);
        k.insert(k.end(), {(unsigned long long)s.pl.C, (unsigned long long)s.pl.P, (unsigned long long)s.pl.nobs,
                           (unsigned long long)s.nnz,
                           (unsigned long long)(unsigned)s.fx[0] << 32 | (unsigned)s.fx[1],
                           (unsigned long long)(unsigned)s.fx[2], lam});
    }
    return k;
}

// Run the device part of a group: from the graph of its shape when there is
// one, else directly (and capture it when the shape was seen before).
int run_device(unc_batch* b, GroupRun& g) {
    const auto key = shape_key(b, g);
    for (auto& gr : b->graphs)
        if (gr.key == key) {
            BCK(cudaGraphLaunch(gr.exec, b->stream));
            count_launch((int)gr.launches);
            return UNC_OK;
        }
    const bool again = std::find(b->seen.begin(), b->seen.end(), key) != b->seen.end();
    if (!again) {
        if (b->seen.size() >= 16) b->seen.erase(b->seen.begin());
        b->seen.push_back(key);
        return launch_group(b, g);
    }
    const long long l0 = g_thread_launches;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ok = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    int rc = UNC_OK;
    if (ok) {
        rc = launch_group(b, g);
        ok = cudaStreamEndCapture(b->stream, &graph) == cudaSuccess && rc == UNC_OK && graph;
    }
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    const long long launches = g_thread_launches - l0;  // captured, not run
    __atomic_sub_fetch(&g_launches, launches, __ATOMIC_RELAXED);
    g_thread_launches -= launches;
    if (!ok) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return launch_group(b, g);
    }
    if (b->graphs.size() >= (size_t)kGraphs) {
        cudaGraphExecDestroy(b->graphs.front().exec);
        b->graphs.erase(b->graphs.begin());
    }
    b->graphs.push_back(Graph{key, exec, launches});
    BCK(cudaGraphLaunch(exec, b->stream));
    count_launch((int)launches);
    return UNC_OK;
}

int run_group(unc_batch* b, GroupRun& g, const int* const* rows, const int* const* cols,
              const double* const* values, double* const* cam_unc, double* const* pt_unc, int* status,
              unc_statistic* stats) {
    cudaStream_t sm = b->stream;
    // tile width by the cost model over all the group's tiles (deterministic:
    // no timed trial runs, so a serving worker never solves a pack twice)
    std::vector<int> ns;
    for (const Scene& s : g.sc) ns.push_back(s.pl.N);
    const int nt = g.slices == 5 && b->force_nt ? b->force_nt : mixed_group_tile_n(g.slices, ns);
    if (int r = prepare_group(b, g, nt)) return r;
    // inputs: packed into the staging area and sent on piece by piece
    BCK(cudaEventRecord(b->ev[0], sm));
    {
        std::vector<Copy> cp;
        for (const Scene& s : g.sc) {
            cp.push_back({g.hbase + g.h_in + s.in_off[0], rows[s.idx], sizeof(int) * ((size_t)s.pl.nobs * 2 + 1)});
            cp.push_back({g.hbase + g.h_in + s.in_off[1], cols[s.idx], sizeof(int) * (size_t)s.nnz});
            cp.push_back({g.hbase + g.h_in + s.in_off[2], values[s.idx], sizeof(double) * (size_t)s.nnz});
        }
        BCK(parallel_copy_to_device(cp, g.hbase + g.h_in, g.dbase, g.L.in_bytes, b->device, sm));
    }
    BCK(cudaEventRecord(b->ev[1], sm));
    if (int r = run_device(b, g)) return r;
    BCK(cudaEventRecord(b->ev[2], sm));
    BCK(cudaMemcpyAsync(g.hbase + g.h_out, g.dbase + g.L.in_bytes, g.L.out_bytes, cudaMemcpyDeviceToHost, sm));
    BCK(cudaMemcpyAsync(g.hbase + g.h_stat, g.dbase + g.L.stat_off, g.L.stat_bytes, cudaMemcpyDeviceToHost, sm));
    BCK(cudaEventRecord(b->ev[3], sm));
    BCK(cudaStreamSynchronize(sm));
    BCK(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
    b->t_h2d += ms * 1e-3;
    cudaEventElapsedTime(&ms, b->ev[1], b->ev[2]);
    b->t_dev += ms * 1e-3;
    cudaEventElapsedTime(&ms, b->ev[2], b->ev[3]);
    b->t_d2h += ms * 1e-3;
    b->grouped += (int)g.sc.size();
    b->tile_n = g.nt;
    // outputs: the reference's zeroing rule as in unc_compute (fixed points past
    // 6 (P - 3) keep the caller's values)
    std::vector<Copy> cp;
    const int* errs = reinterpret_cast<const int*>(g.hbase + g.h_stat);
    const TeState* tes = reinterpret_cast<const TeState*>(g.hbase + g.h_stat + ((4 * g.sc.size() * sizeof(int) + 255) & ~size_t(255)));
    for (size_t i = 0; i < g.sc.size(); ++i) {
        const Scene& s = g.sc[i];
        const int err = errs[4 * i];
        const TeState& te = tes[i];
        int rc = UNC_OK;
        if (err & ERRBIT_LAYOUT) rc = UNC_ERR_LAYOUT;
        else if (err & (ERRBIT_SINGULAR | ERRBIT_NONFINITE)) rc = UNC_ERR_SINGULAR;
        else if (err & ERRBIT_TIMEOUT) rc = UNC_ERR_CUDA;
        else if (err & ERRBIT_SCHUR_CAP) rc = UNC_ERR_TOO_LARGE;
        else if (te.bad) rc = UNC_ERR_SINGULAR;
        status[s.idx] = rc;
        if (stats) {
            unc_statistic& st = stats[s.idx];
            memset(&st, 0, sizeof(st));
            st.lambda = s.lambda;
            for (int k = 0; k < 3; ++k) st.fixed_pts[k] = s.fx[k];
            st.te_iterations = te.iters;
            for (int k = 0; k < te.iters && k < 20; ++k) st.cycle_change[k] = te.change[k];
            st.time_all = b->t_h2d + b->t_dev + b->t_d2h;  // the batch's, shared by its scenes
            st.device_bytes = (long long)(g.L.total / g.sc.size());
        }
        if (rc != UNC_OK) continue;
        cp.push_back({cam_unc[s.idx], g.hbase + g.h_out + (s.out_off[0] - g.L.in_bytes),
                      sizeof(double) * 45 * (size_t)s.pl.C});
        const size_t head = s.pl.P > 3 ? (size_t)(s.pl.P - 3) : 0;
        const char* hp = g.hbase + g.h_out + (s.out_off[1] - g.L.in_bytes);
        if (head) cp.push_back({pt_unc[s.idx], hp, sizeof(double) * 6 * head});
        for (int p = (int)head; p < s.pl.P; ++p) {
            if (p == s.fx[0] || p == s.fx[1] || p == s.fx[2]) continue;
            cp.push_back({pt_unc[s.idx] + 6L * p, hp + sizeof(double) * 6 * (size_t)p, sizeof(double) * 6});
        }
    }
    parallel_copy(cp);
    return UNC_OK;
}

}  // namespace

extern "C" {

int unc_batch_create(int device, unc_batch** out) {
    if (!out) return bfail(UNC_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    unc_batch* b = new unc_batch();
    b->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) {
        prepare_assembly_kernels();
        prepare_dense_kernels();
        prepare_mixed_kernels();
        prepare_task_kernels();
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    }
    for (int k = 0; k < kBranches && e == cudaSuccess; ++k) e = cudaStreamCreateWithFlags(&b->branch[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int k = 0; k < kBranches && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming);
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = cudaEventCreate(&b->ev[k]);
    if (e != cudaSuccess) {
        g_last_error = std::string("unc_batch_create: ") + cudaGetErrorString(e);
        unc_batch_destroy(b);
        return UNC_ERR_CUDA;
    }
    *out = b;
    return UNC_OK;
}

int unc_batch_destroy(unc_batch* b) {
    if (!b) return UNC_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& g : b->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (b->ws) cudaFree(b->ws);
    if (b->host) cudaFreeHost(b->host);
    for (void* h : b->host_retired) cudaFreeHost(h);
    if (b->single) unc_context_destroy(b->single);
    for (int k = 0; k < 4; ++k)
        if (b->ev[k]) cudaEventDestroy(b->ev[k]);
    for (int k = 0; k < kBranches; ++k) {
        if (b->join[k]) cudaEventDestroy(b->join[k]);
        if (b->branch[k]) cudaStreamDestroy(b->branch[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return UNC_OK;
}

int unc_batch_compute(unc_batch* b, int num_scenes, const unc_options* opts, const int* num_rows,
                      const int* num_cols, const int* const* rows, const int* const* cols,
                      const double* const* values, double* const* cam_unc, double* const* pt_unc, int* status,
                      unc_statistic* stats) {
    g_last_error.clear();
    if (!b || num_scenes < 0 || (num_scenes > 0 && (!opts || !num_rows || !num_cols || !rows || !cols || !values ||
                                                    !cam_unc || !pt_unc || !status)))
        return bfail(UNC_ERR_INVALID_ARG, "unc_batch_compute: null argument");
    BCK(cudaSetDevice(b->device));
    b->t_h2d = b->t_dev = b->t_d2h = 0;
    b->grouped = 0;
    std::map<int, GroupRun> groups;  // by slice count
    std::vector<int> single;
    for (int i = 0; i < num_scenes; ++i) {
        const unc_options* o = opts + i;
        status[i] = check_options(o, num_rows[i], num_cols[i]);
        if (status[i] != UNC_OK) continue;
        if (!rows[i] || !cols[i] || !values[i] || !cam_unc[i] || !pt_unc[i]) {
            status[i] = UNC_ERR_INVALID_ARG;
            continue;
        }
        const long long nnz = rows[i][num_rows[i]];
        if (nnz < 0 || rows[i][0] != 0 || nnz != 24LL * (num_rows[i] / 2)) {  // the layout the grouped path stages
            single.push_back(i);
            continue;
        }
        if (o->algorithm != UNC_TAYLOR_EXPANSION || o->precision == UNC_PRECISION_FP64 ||
            o->taylor_eval == UNC_TAYLOR_SEQUENTIAL || !spd_tasks_apply(9 * o->num_cams)) {
            single.push_back(i);
            continue;
        }
        Scene s{};
        s.idx = i;
        s.opt = *o;
        s.pl = make_plan(o, num_rows[i]);
        s.nnz = nnz;
        s.fx[0] = o->pts2fix[0];
        s.fx[1] = o->pts2fix[1];
        s.fx[2] = o->pts2fix[2];
        std::sort(s.fx, s.fx + 2);  // the reference sorts only the first two ids (compute.cpp:285)
        s.lambda = o->lambda == -1 ? auto_lambda(s.pl.N) : o->lambda;  // compute.cpp:124-125
        GroupRun& g = groups[slices_of(o->precision)];
        g.slices = slices_of(o->precision);
        g.sc.push_back(s);
    }
    for (auto& kv : groups) {
        if (int r = run_group(b, kv.second, rows, cols, values, cam_unc, pt_unc, status, stats)) return r;
    }
    for (int i : single) {
        if (!b->single) {
            if (int r = unc_context_create(b->device, &b->single)) return r;
        }
        status[i] = unc_compute(b->single, opts + i, num_rows[i], num_cols[i], rows[i], cols[i], values[i],
                                cam_unc[i], pt_unc[i], stats ? stats + i : nullptr);
    }
    return UNC_OK;
}

long long unc_batch_device_bytes(const unc_batch* b) {
    if (!b) return -1;
    return (long long)b->ws_bytes + (b->single ? unc_context_device_bytes(b->single) : 0);
}

int unc_batch_release(unc_batch* b) {
    if (!b) return bfail(UNC_ERR_INVALID_ARG, "batch is NULL");
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->stream));
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
    b->graphs.clear();
    b->seen.clear();
    // stream-ordered free: a cudaFree would wait for every other stream's work
    // (a serving process releases idle workspaces while others compute)
    if (b->ws) BCK(cudaFreeAsync(b->ws, b->stream));
    b->ws = nullptr;
    b->ws_bytes = 0;
    BCK(cudaStreamSynchronize(b->stream));
    if (b->single) unc_context_release(b->single);
    return UNC_OK;
}

int unc_batch_set_tile_width(unc_batch* b, int tile_n) {
    if (!b) return bfail(UNC_ERR_INVALID_ARG, "batch is NULL");
    if (tile_n != 0 && tile_n != 64 && tile_n != 96)
        return bfail(UNC_ERR_INVALID_ARG, "tile_n must be 0 (cost model), 64 or 96");
    b->force_nt = tile_n;
    return UNC_OK;
}

int unc_batch_last_timing(const unc_batch* b, double* h2d_s, double* device_s, double* d2h_s, int* grouped_scenes,
                          int* tile_n) {
    if (!b) return bfail(UNC_ERR_INVALID_ARG, "batch is NULL");
    if (h2d_s) *h2d_s = b->t_h2d;
    if (device_s) *device_s = b->t_dev;
    if (d2h_s) *d2h_s = b->t_d2h;
    if (grouped_scenes) *grouped_scenes = b->grouped;
    if (tile_n) *tile_n = b->tile_n;
    return UNC_OK;
}

}  // extern "C"
