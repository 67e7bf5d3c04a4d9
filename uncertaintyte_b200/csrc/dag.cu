// dag.cu - SPD inverse A^{-1} = L^{-T} L^{-1} as a graph of 64 x 64 tile tasks
// run by one persistent kernel (sm_100a), for the moderate sizes where the
// recursive form (dense.cu) is bound by its ~200 dependent launches.
//
// Tiles (i, j), j <= i, of the lower triangle; nt = ceil(n / 64). Tasks:
//   POTRF(k)      T(k,k) = chol(A(k,k))^{-1}                  (the 64 x 64 leaf)
//   TRSM(i,k)     L(i,k) = A(i,k) T(k,k)^T                    (in place in A)
//   UPDATE(i,j,k) A(i,j) -= L(i,k) L(j,k)^T                   (k < j <= i)
//   TACC(i,j,m)   W(i,j) += L(i,m) T(m,j)                     (j <= m < i, in the T(i,j) slot)
//   TFIN(i,j)     T(i,j) = -T(i,i) W(i,j)                     (block forward substitution)
//   PACC(i,j,k)   O(i,j) += T(k,i)^T T(k,j)                   (k >= i >= j; the last term also
//                                                             writes the transposed tile)
// POTRF(k) also applies the last update of its tile (from panel k-1) before
// factoring and computes TRSM(k+1,k) after it, so the dependent chain from one
// diagonal tile to the next is one task. The host lists the tasks in a
// topological order that puts each diagonal factorisation right after the
// tasks it waits for (look-ahead).
// CTAs claim tasks from a global cursor in list order, wait (thread 0, with an
// iteration limit) on per-tile counters, run the task with all 512 threads
// and publish its counter. Every dependency of a claimed task was claimed
// earlier by a running CTA that waits only on still earlier tasks, so the
// schedule completes with any number of resident CTAs; updates of one tile
// are applied in a fixed order, so the result is bitwise repeatable. Tile data
// written by other CTAs is read through L2 only (ld.global.cg).
//
// Counters (ints, zeroed before the launch): cursor, abort flag, then per
// lower tile: ver (updates applied to A), lrdy (L final / T(k,k) ready),
// tacc (W accumulations), trdy (T final), pacc (O accumulations).
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "chol_leaf.cuh"
#include "internal.h"

namespace unc {
namespace {

constexpr int TB = NB;                   // tile size (the leaf size)
constexpr int DAG_THREADS = LEAF_THREADS;
constexpr int TLD = TB + 4;              // shared tile stride: fragment reads conflict-free in both orientations
constexpr size_t TILE_SMEM = sizeof(double) * 2 * TB * TLD;
constexpr size_t DAG_SMEM = TILE_SMEM + LEAF_SMEM;  // two operand tiles, then the leaf's block
constexpr long kDagSpin = 1L << 22;      // polls of one dependency before the kernel gives up
constexpr int kMaxTilesN = 56;           // tasks are used up to n = 56 * 64

enum : int { K_POTRF = 0, K_TRSM = 1, K_UPDATE = 2, K_TACC = 3, K_TFIN = 4, K_PACC = 5 };

__device__ __forceinline__ int tri(int i, int j) { return i * (i + 1) / 2 + j; }

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// thread 0 only: wait until *flag >= v (or the abort flag is raised / the
// limit of `spin` polls runs out)
__device__ bool wait_ge(const int* flag, int v, const int* abort, long spin) {
    for (long it = 0; it < spin; ++it) {
        if (ld_acquire(flag) >= v) return true;
        if (ld_acquire(abort)) return false;
        __nanosleep(32);
    }
    return false;
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Tile X (column-major, leading dimension ld; rows < vr and columns < vc
// valid, the rest read as zero) into shared memory as sm[c * TLD + r].
__device__ __forceinline__ void load_tile(double* sm, const double* X, long ld, int vr, int vc, int tid) {
#pragma unroll
    for (int u = 0; u < TB * TB / 2 / DAG_THREADS; ++u) {
        const int q = tid + u * DAG_THREADS;
        const int c = q >> 5, r2 = (q & 31) * 2;
        double2 v = make_double2(0.0, 0.0);
        if (c < vc && r2 < vr) v = __ldcg(reinterpret_cast<const double2*>(X + r2 + (long)c * ld));
        if (r2 + 1 >= vr) v.y = 0.0;
        *reinterpret_cast<double2*>(sm + c * TLD + r2) = v;
    }
}

// acc += op(A) op(B) over k in [kb, ke) (multiples of 4) for this warp's 16 x 16
// block (rows wm.., columns wn..). op(A)(m, k) = kTA ? A(k, m) : A(m, k),
// op(B)(k, n) = kTB ? B(n, k) : B(k, n), tiles as left by load_tile.
template <bool kTA, bool kTB>
__device__ __forceinline__ void tile_mma(const double* As, const double* Bs, int wm, int wn, int g, int t, int kb,
                                         int ke, double (&acc)[2][2][2]) {
    for (int kk = kb; kk < ke; kk += 4) {
        double a[2], b[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int m = wm + 8 * i + g, k = kk + t;
            a[i] = kTA ? As[m * TLD + k] : As[k * TLD + m];
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int n = wn + 8 * j + g, k = kk + t;
            b[j] = kTB ? Bs[k * TLD + n] : Bs[n * TLD + k];
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
}

// X(r, c) = alpha acc + (accumulate ? X(r, c) : 0) for r < vr, c < vc; with
// Xm, also Xm(c, r) = the same value (the transposed tile).
__device__ __forceinline__ void store_tile(double* X, long ld, int vr, int vc, const double (&acc)[2][2][2],
                                           double alpha, bool accumulate, double* Xm, int wm, int wn, int g,
                                           int t) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = wm + 8 * i + g, c = wn + 8 * j + 2 * t + h;
                if (r < vr && c < vc) {
                    double v = alpha * acc[i][j][h];
                    if (accumulate) v += __ldcg(X + r + (long)c * ld);
                    X[r + (long)c * ld] = v;
                    if (Xm) Xm[c + (long)r * ld] = v;
                }
            }
}

// One tile task (type, i, j, k) of the n x n matrix whose tiles A, T, O and
// counters (`state`, laid out as described at the top) are given, run by all
// DAG_THREADS threads of the block; thread 0 waits for its dependencies first.
// Returns false when a wait gave up (ERRBIT_TIMEOUT and the abort flag are
// set): the caller stops taking tasks.
__device__ __forceinline__ bool run_task(double* A, double* T, double* O, int n, long ld, int* state, int ntri,
                                         int* err, int* abort, long spin, int type, int i, int j, int k, double* sm,
                                         int& s_ok) {
    int* const ver = state + 4;
    int* const lrdy = ver + ntri;
    int* const tacc = lrdy + ntri;
    int* const trdy = tacc + ntri;
    int* const pacc = trdy + ntri;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t4 = lane & 3;
    const int wm = (warp & 3) * 16, wn = (warp >> 2) * 16;
    double* As = sm;
    double* Bs = sm + TB * TLD;
    auto ext = [n](int b) { return min(TB, n - TB * b); };
    auto kext = [n](int b) { return (min(TB, n - TB * b) + 3) & ~3; };  // K extent of a partial tile, DMMA steps
    auto tile = [ld](double* M, int i, int j) { return M + (long)TB * i + (long)TB * j * ld; };
    if (tid == 0) {
        bool ok = true;
        switch (type) {
            case K_POTRF:  // its last update (from panel k-1) is applied inside the task
                ok = k == 0 || (wait_ge(ver + tri(k, k), k - 1, abort, spin) &&
                                wait_ge(lrdy + tri(k, k - 1), 1, abort, spin));
                break;
            case K_TRSM:
                ok = wait_ge(ver + tri(i, k), k, abort, spin) && wait_ge(lrdy + tri(k, k), 1, abort, spin);
                break;
            case K_UPDATE:
                ok = wait_ge(ver + tri(i, j), k, abort, spin) && wait_ge(lrdy + tri(i, k), 1, abort, spin) &&
                     wait_ge(lrdy + tri(j, k), 1, abort, spin);
                break;
            case K_TACC:
                ok = wait_ge(tacc + tri(i, j), k - j, abort, spin) && wait_ge(lrdy + tri(i, k), 1, abort, spin) &&
                     wait_ge(trdy + tri(k, j), 1, abort, spin);
                break;
            case K_TFIN:
                ok = wait_ge(tacc + tri(i, j), i - j, abort, spin) && wait_ge(trdy + tri(i, i), 1, abort, spin);
                break;
            default:  // K_PACC
                ok = wait_ge(pacc + tri(i, j), k - i, abort, spin) && wait_ge(trdy + tri(k, i), 1, abort, spin) &&
                     wait_ge(trdy + tri(k, j), 1, abort, spin);
                break;
        }
        if (!ok) {
            atomicOr(err, ERRBIT_TIMEOUT);
            atomicExch(abort, 1);
        }
        s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return false;
    if (type == K_POTRF) {
        // A(k,k) -= L(k,k-1) L(k,k-1)^T applied to the leaf's block (both tiles loaded
        // together), the leaf, T(k,k) published, then L(k+1,k) = A(k+1,k) T(k,k)^T with
        // T(k,k) still in shared memory
        double* lsm = sm + 2 * TB * TLD;
        chol_leaf_load(A, ld, TB * k, ext(k), lsm);
        if (k > 0) {
            double acc[2][2][2] = {};
            load_tile(As, tile(A, k, k - 1), ld, ext(k), ext(k - 1), tid);
            __syncthreads();
            if (wn <= wm) tile_mma<false, true>(As, As, wm, wn, g, t4, 0, TB, acc);  // lower blocks only
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int r = wm + 8 * a + g, c = wn + 8 * b + 2 * t4 + h;
                        if (c <= r) lsm[r * LEAF_LD + c] -= acc[a][b][h];
                    }
        }
        __syncthreads();
        chol_leaf_factor(TB * k, ext(k), T, ld, err, lsm);
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch(lrdy + tri(k, k), 1);
            atomicExch(trdy + tri(k, k), 1);
        }
        if (k + 1 >= (n + TB - 1) / TB) return true;
        if (tid == 0) {
            const bool ok = wait_ge(ver + tri(k + 1, k), k, abort, spin);
            if (!ok) {
                atomicOr(err, ERRBIT_TIMEOUT);
                atomicExch(abort, 1);
            }
            s_ok = ok;
        }
        const double* Tl = lsm + NB * LEAF_LD;  // T(r, c) at Tl[r * LEAF_LD + c], lower triangle valid
        for (int e = tid; e < TB * TB; e += DAG_THREADS) {
            const int r = e & (TB - 1), c = e >> 6;
            Bs[c * TLD + r] = r >= c ? Tl[r * LEAF_LD + c] : 0.0;
        }
        __syncthreads();
        if (!s_ok) return false;
        load_tile(As, tile(A, k + 1, k), ld, ext(k + 1), ext(k), tid);
        __syncthreads();
        double acc[2][2][2] = {};
        tile_mma<false, true>(As, Bs, wm, wn, g, t4, 0, wn + 16, acc);
        store_tile(tile(A, k + 1, k), ld, ext(k + 1), ext(k), acc, 1.0, false, nullptr, wm, wn, g, t4);
    } else {
        double acc[2][2][2] = {};
        switch (type) {
            case K_TRSM:  // L(i,k) = A(i,k) T(k,k)^T; T(k,k) lower: terms k' <= n only
                load_tile(As, tile(A, i, k), ld, ext(i), ext(k), tid);
                load_tile(Bs, tile(T, k, k), ld, ext(k), ext(k), tid);
                __syncthreads();
                tile_mma<false, true>(As, Bs, wm, wn, g, t4, 0, min(wn + 16, kext(k)), acc);
                __syncthreads();
                store_tile(tile(A, i, k), ld, ext(i), ext(k), acc, 1.0, false, nullptr, wm, wn, g, t4);
                break;
            case K_UPDATE:  // A(i,j) -= L(i,k) L(j,k)^T
                load_tile(As, tile(A, i, k), ld, ext(i), ext(k), tid);
                load_tile(Bs, tile(A, j, k), ld, ext(j), ext(k), tid);
                __syncthreads();
                tile_mma<false, true>(As, Bs, wm, wn, g, t4, 0, kext(k), acc);
                store_tile(tile(A, i, j), ld, ext(i), ext(j), acc, -1.0, true, nullptr, wm, wn, g, t4);
                break;
            case K_TACC:  // W(i,j) += L(i,k) T(k,j); T(j,j) lower: terms k' >= n only
                load_tile(As, tile(A, i, k), ld, ext(i), ext(k), tid);
                load_tile(Bs, tile(T, k, j), ld, ext(k), ext(j), tid);
                __syncthreads();
                tile_mma<false, false>(As, Bs, wm, wn, g, t4, k == j ? wn : 0, kext(k), acc);
                store_tile(tile(T, i, j), ld, ext(i), ext(j), acc, 1.0, k > j, nullptr, wm, wn, g, t4);
                break;
            case K_TFIN:  // T(i,j) = -T(i,i) W(i,j); T(i,i) lower: terms k' <= m only
                load_tile(As, tile(T, i, i), ld, ext(i), ext(i), tid);
                load_tile(Bs, tile(T, i, j), ld, ext(i), ext(j), tid);
                __syncthreads();
                tile_mma<false, false>(As, Bs, wm, wn, g, t4, 0, min(wm + 16, kext(i)), acc);
                __syncthreads();
                store_tile(tile(T, i, j), ld, ext(i), ext(j), acc, -1.0, false, nullptr, wm, wn, g, t4);
                break;
            default: {  // K_PACC: O(i,j) += T(k,i)^T T(k,j); diagonal T tiles lower
                load_tile(As, tile(T, k, i), ld, ext(k), ext(i), tid);
                load_tile(Bs, tile(T, k, j), ld, ext(k), ext(j), tid);
                __syncthreads();
                int kb = 0;
                if (k == i) kb = wm;
                if (k == j) kb = max(kb, wn);
                tile_mma<true, false>(As, Bs, wm, wn, g, t4, kb, kext(k), acc);
                const bool last = k == (n + TB - 1) / TB - 1;
                store_tile(tile(O, i, j), ld, ext(i), ext(j), acc, 1.0, k > i,
                           (last && i > j) ? tile(O, j, i) : nullptr, wm, wn, g, t4);
                break;
            }
        }
    }
    // release: the barrier orders every thread's tile writes before thread 0's
    // gpu-scope fence, which orders them before the counter
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        switch (type) {
            case K_POTRF: atomicExch(lrdy + tri(k + 1, k), 1); break;  // the fused L(k+1,k)
            case K_TRSM: atomicExch(lrdy + tri(i, k), 1); break;
            case K_UPDATE: atomicAdd(ver + tri(i, j), 1); break;
            case K_TACC: atomicAdd(tacc + tri(i, j), 1); break;
            case K_TFIN: atomicExch(trdy + tri(i, j), 1); break;
            default: atomicAdd(pacc + tri(i, j), 1); break;
        }
    }
    return true;
}

__global__ void __launch_bounds__(DAG_THREADS, 1)
    k_spd_inverse_tasks(double* A, double* T, double* O, int n, long ld, const int4* __restrict__ tasks, int ntasks,
                        int* state, int ntri, int* err, long spin) {
    extern __shared__ __align__(16) double sm[];
    __shared__ int s_task, s_ok;
    int* const cursor = state;
    int* const abort = state + 1;
    while (true) {
        if (threadIdx.x == 0) s_task = atomicAdd(cursor, 1);
        __syncthreads();
        const int task = s_task;
        if (task >= ntasks) break;
        const int4 tk = tasks[task];
        if (!run_task(A, T, O, n, ld, state, ntri, err, abort, spin, tk.x, tk.y, tk.z, tk.w, sm, s_ok)) break;
    }
}

// The same schedule over the tile tasks of many matrices (a batch of
// reconstructions) in one persistent launch: task.x = type + 8 * matrix, the
// matrices' descriptors in `mats`, their counters at mats[m].state, one cursor
// and one abort flag (ctl[0], ctl[1]) for the whole list. The list interleaves
// the matrices' own topological orders, so every dependency of a task is still
// earlier in the list and the launch completes with any number of resident
// CTAs; each task does exactly the arithmetic of the single-matrix kernel, so
// the results are bitwise those of one launch per matrix.
__global__ void __launch_bounds__(DAG_THREADS, 1)
    k_spd_inverse_tasks_grouped(const SpdTaskMatrix* __restrict__ mats, const int4* __restrict__ tasks, int ntasks,
                                int* ctl, long spin) {
    extern __shared__ __align__(16) double sm[];
    __shared__ int s_task, s_ok;
    while (true) {
        if (threadIdx.x == 0) s_task = atomicAdd(ctl, 1);
        __syncthreads();
        const int task = s_task;
        if (task >= ntasks) break;
        const int4 tk = tasks[task];
        const SpdTaskMatrix& m = mats[tk.x >> 3];
        if (!run_task(m.A, m.T, m.O, m.n, m.ld, m.state, m.ntri, m.err, ctl + 1, spin, tk.x & 7, tk.y, tk.z, tk.w, sm,
                      s_ok))
            break;
    }
}

// The task list of nt x nt tiles in the order described above.
std::vector<int4> build_tasks(int nt) {
    std::vector<int4> v;
    auto add = [&v](int ty, int i, int j, int k) { v.push_back(make_int4(ty, i, j, k)); };
    // POTRF(k) also applies UPDATE(k,k,k-1) first and computes TRSM(k+1,k) last
    add(K_POTRF, 0, 0, 0);
    for (int i = 2; i < nt; ++i) add(K_TRSM, i, 0, 0);
    for (int s = 0; s < nt; ++s) {
        if (s + 1 < nt) {
            if (s + 2 < nt) add(K_UPDATE, s + 2, s + 1, s);  // the input of the fused TRSM(s+2,s+1)
            add(K_POTRF, s + 1, s + 1, s + 1);
            for (int i = s + 3; i < nt; ++i) {
                add(K_UPDATE, i, s + 1, s);
                add(K_TRSM, i, s + 1, s + 1);
            }
            for (int j = s + 2; j < nt; ++j)
                for (int i = j; i < nt; ++i) add(K_UPDATE, i, j, s);
        }
        if (s >= 1)
            for (int r = s; r < nt; ++r)
                for (int c = 0; c < s; ++c) add(K_TACC, r, c, s - 1);
        for (int c = 0; c < s; ++c) add(K_TFIN, s, c, 0);
        for (int r = 0; r <= s; ++r)
            for (int c = 0; c <= r; ++c) add(K_PACC, r, c, s);
    }
    return v;
}

struct TaskLists {
    std::mutex mu;
    std::map<std::pair<int, int>, std::pair<int4*, int>> lists;  // (device, nt) -> device copy
    std::map<int, cudaStream_t> upload;                          // device -> upload stream
};
TaskLists& task_lists() {
    static TaskLists* t = new TaskLists;  // lives until exit, like the device buffers it holds
    return *t;
}

}  // namespace

bool spd_tasks_apply(int n) { return n > 0 && (n + TB - 1) / TB <= kMaxTilesN; }

size_t spd_task_state_ints(int n) {
    const size_t nt = (size_t)(n + TB - 1) / TB;
    return 4 + 5 * nt * (nt + 1) / 2;
}

int spd_tasks_prepare(int n) {
    if (!spd_tasks_apply(n)) return UNC_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return UNC_ERR_CUDA;
    const int nt = (n + TB - 1) / TB;
    TaskLists& tl = task_lists();
    std::lock_guard<std::mutex> lock(tl.mu);
    if (tl.lists.count({dev, nt})) return UNC_OK;
    const std::vector<int4> h = build_tasks(nt);
    // upload on a private non-blocking stream: a copy on the legacy default
    // stream would wait for every other stream's work (a serving process runs
    // several requests at once)
    auto it = tl.upload.find(dev);
    if (it == tl.upload.end()) {
        cudaStream_t us = nullptr;
        if (cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking) != cudaSuccess) return UNC_ERR_CUDA;
        it = tl.upload.emplace(dev, us).first;
    }
    cudaStream_t us = it->second;
    int4* d = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(int4) * h.size(), us) != cudaSuccess)
        return UNC_ERR_OUT_OF_MEMORY;
    if (cudaMemcpyAsync(d, h.data(), sizeof(int4) * h.size(), cudaMemcpyHostToDevice, us) != cudaSuccess ||
        cudaStreamSynchronize(us) != cudaSuccess) {
        cudaFreeAsync(d, us);
        return UNC_ERR_CUDA;
    }
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_spd_inverse_tasks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)DAG_SMEM) == cudaSuccess;
    });
    tl.lists[{dev, nt}] = {d, (int)h.size()};
    return UNC_OK;
}

int chol_inverse_tasks(double* A, int n, int lda, double* T, double* O, int* state, int* err, cudaStream_t st,
                       int max_ctas, long long poll_limit, int skip_task) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return UNC_ERR_CUDA;
    const int nt = (n + TB - 1) / TB;
    std::pair<int4*, int> list{nullptr, 0};
    {
        TaskLists& tl = task_lists();
        std::lock_guard<std::mutex> lock(tl.mu);
        auto it = tl.lists.find({dev, nt});
        if (it == tl.lists.end()) return UNC_ERR_INVALID_ARG;  // spd_tasks_prepare first (outside any capture)
        list = it->second;
    }
    const int ntri = nt * (nt + 1) / 2;
    if (cudaMemsetAsync(state, 0, sizeof(int) * spd_task_state_ints(n), st) != cudaSuccess) return UNC_ERR_CUDA;
    const long spin = poll_limit > 0 ? (long)std::min<long long>(poll_limit, kDagSpin) : kDagSpin;
    int4* own = nullptr;  // a schedule with one task left out (tests of the bounded waits)
    if (skip_task >= 0 && skip_task < list.second) {
        std::vector<int4> h = build_tasks(nt);
        h.erase(h.begin() + skip_task);
        if (cudaMallocAsync(reinterpret_cast<void**>(&own), sizeof(int4) * h.size(), st) != cudaSuccess)
            return UNC_ERR_OUT_OF_MEMORY;
        if (cudaMemcpyAsync(own, h.data(), sizeof(int4) * h.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaFreeAsync(own, st);
            return UNC_ERR_CUDA;
        }
        list = {own, (int)h.size()};
    }
    const int grid = std::max(1, std::min(std::min(device_sms(), max_ctas), list.second));
    k_spd_inverse_tasks<<<grid, DAG_THREADS, DAG_SMEM, st>>>(A, T, O, n, lda, list.first, list.second, state, ntri,
                                                             err, spin);
    count_launch();
    if (own && cudaFreeAsync(own, st) != cudaSuccess) return UNC_ERR_CUDA;
    return UNC_OK;
}

std::vector<int4> spd_tasks_grouped_list(const std::vector<int>& ns) {
    struct Item {
        double key;
        int m, q;
        int4 t;
    };
    std::vector<Item> items;
    for (int m = 0; m < (int)ns.size(); ++m) {
        const std::vector<int4> v = build_tasks((ns[m] + TB - 1) / TB);
        for (int q = 0; q < (int)v.size(); ++q) {
            int4 t = v[q];
            t.x += 8 * m;
            items.push_back({(q + 1.0) / (double)v.size(), m, q, t});
        }
    }
    // stable in (key, matrix, position): a matrix's own order is kept
    std::sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
        if (a.key != b.key) return a.key < b.key;
        if (a.m != b.m) return a.m < b.m;
        return a.q < b.q;
    });
    std::vector<int4> out(items.size());
    for (size_t i = 0; i < items.size(); ++i) out[i] = items[i].t;
    return out;
}

void prepare_task_kernels() {
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_spd_inverse_tasks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)DAG_SMEM) == cudaSuccess &&
               cudaFuncSetAttribute(k_spd_inverse_tasks_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)DAG_SMEM) == cudaSuccess;
    });
}

int chol_inverse_tasks_grouped(const SpdTaskMatrix* d_mats, const int4* d_tasks, int ntasks, int* ctl,
                               cudaStream_t st, int max_ctas, long long poll_limit) {
    if (ntasks <= 0) return UNC_OK;
    prepare_task_kernels();
    const long spin = poll_limit > 0 ? (long)std::min<long long>(poll_limit, kDagSpin) : kDagSpin;
    const int grid = std::max(1, std::min(std::min(device_sms(), max_ctas), ntasks));
    k_spd_inverse_tasks_grouped<<<grid, DAG_THREADS, DAG_SMEM, st>>>(d_mats, d_tasks, ntasks, ctl, spin);
    count_launch();
    return UNC_OK;
}

}  // namespace unc

// The task order of the tile-task inverse for an n x n matrix, for tools that
// check or draw the schedule: returns the number of tasks; with out != NULL and
// capacity >= that number, out receives 4 ints per task (kind 0..5 = POTRF,
// TRSM, UPDATE, TACC, TFIN, PACC; then i, j, k as in the kernel). Host only.
extern "C" int unc_spd_task_list(int n, int* out, int capacity) {
    unc::g_last_error.clear();
    if (!unc::spd_tasks_apply(n)) {
        unc::g_last_error = "unc_spd_task_list: n must be in 1..3584";
        return UNC_ERR_INVALID_ARG;
    }
    const std::vector<int4> v = unc::build_tasks((n + unc::NB - 1) / unc::NB);
    if (out && capacity >= (int)v.size())
        for (size_t q = 0; q < v.size(); ++q) {
            out[4 * q] = v[q].x;
            out[4 * q + 1] = v[q].y;
            out[4 * q + 2] = v[q].z;
            out[4 * q + 3] = v[q].w;
        }
    return (int)v.size();
}
