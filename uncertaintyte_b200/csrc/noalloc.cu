// noalloc.cu - the SPD dense inverse without any device allocation.
//
// Some callers cannot let a library allocate device memory: applications whose
// device memory is entirely reserved by their own pool allocator (a cudaMalloc
// would fail or fragment their pool), and latency-critical loops where
// cudaMalloc / cudaFree would synchronize the device and add stalls. For them
// unc_dense_inverse_noalloc runs the same kernels as unc_dense_inverse_device
// with its scratch in a file-scope __device__ array of fixed size.
//
// Limits and sharing rules:
//   * n <= kNoAllocMaxN and lda <= kNoAllocMaxN (512): larger sizes are
//     rejected with UNC_ERR_TOO_LARGE.
//   * The array (about 6.3 MB) is part of every device this library is loaded
//     on, until the process exits.
//   * Every call on a device shares the one array and it keeps the previous
//     call's contents; the entry point clears what must start at zero. Calls
//     that overlap on the GPU (different streams or threads, not ordered with
//     respect to each other) race on the array and give wrong results.
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture. The lookup is repeated after a device reset
//     (the CUDA context changed), so the library may outlive a reset.
#include <mutex>

#include "../../include/uncte.h"
#include "internal.h"

namespace unc {
namespace {

constexpr int kNoAllocMaxN = 512;                                    // largest n and lda
constexpr size_t kMat = (size_t)kNoAllocMaxN * kNoAllocMaxN;        // one n x lda matrix
constexpr size_t kSmall = (size_t)64 * 64 + 64;                      // >= chol_small_doubles(n)
constexpr size_t kEq = (size_t)kNoAllocMaxN + 64;                    // equilibration scales
constexpr size_t kScratchDoubles = 3 * kMat + kSmall + kEq + 8;      // + the error word

// The scratch: host code may only use its name to look up the device address.
__device__ __align__(256) double g_inverse_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
// Per device: the array's device address and the CUDA context it was looked
// up in. A device reset (cudaDeviceReset, or a primary-context reset by other
// code in the process) unloads the module; the next context loads it again,
// possibly at another address, so the lookup is repeated when the current
// context is not the one recorded.
double* g_scratch_addr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};
std::mutex g_scratch_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
    static const CtxGetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<CtxGetCurrentFn>(p);
        cudaGetLastError();
        return (CtxGetCurrentFn) nullptr;
    }();
    return fn;
}

int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_last_error = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return UNC_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        g_last_error = "device index above the supported range";
        return UNC_ERR_UNSUPPORTED;
    }
    CtxGetCurrentFn get = ctx_get_current();
    if (!get) {
        g_last_error = "cuCtxGetCurrent is unavailable";
        return UNC_ERR_CUDA;
    }
    // before the runtime has set up the device no context is current yet; the
    // symbol lookup below does that set-up
    CUcontext ctx = nullptr;
    if (get(&ctx) != CUDA_SUCCESS) ctx = nullptr;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev] || !ctx || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_inverse_scratch);
        if (e != cudaSuccess || !p) {
            g_last_error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return UNC_ERR_CUDA;
        }
        if (get(&ctx) != CUDA_SUCCESS || !ctx) {
            g_last_error = "no current CUDA context after the symbol lookup";
            return UNC_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double*>(p);
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_addr[dev];
    return UNC_OK;
}

}  // namespace
}  // namespace unc

using namespace unc;

extern "C" int unc_dense_inverse_noalloc(double* d_A, int n, int lda, void* stream) {
    g_last_error.clear();
    if (!d_A || n <= 0 || lda < n || (lda & 1)) {
        g_last_error = "bad matrix arguments";
        return UNC_ERR_INVALID_ARG;
    }
    if (n > kNoAllocMaxN || lda > kNoAllocMaxN) {
        g_last_error = "unc_dense_inverse_noalloc: n and lda must be at most 512 (static scratch size)";
        return UNC_ERR_TOO_LARGE;
    }
    if (chol_small_doubles(n) > kSmall) {
        g_last_error = "static scratch too small for the panel buffers";
        return UNC_ERR_TOO_LARGE;
    }
    double* ws = nullptr;
    int rc = scratch_for_current_device(&ws);
    if (rc != UNC_OK) return rc;
    cudaStream_t sm = (cudaStream_t)stream;
    const size_t mat = (size_t)lda * n;  // <= kMat
    double* T = ws;
    double* W = ws + kMat;
    double* Tt = ws + 2 * kMat;
    double* small = ws + 3 * kMat;
    double* e = small + kSmall;
    int* err = reinterpret_cast<int*>(e + kEq);
    // the previous call's contents stay in the array: clear what must start at
    // zero (T above its diagonal blocks, the padding rows, the error word)
    cudaError_t ce = cudaMemsetAsync(T, 0, sizeof(double) * mat, sm);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(W, 0, sizeof(double) * mat, sm);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(Tt, 0, sizeof(double) * mat, sm);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(small, 0, sizeof(double) * (kSmall + kEq + 8), sm);
    int h_err = 0;
    if (ce == cudaSuccess) {
        launch_shift_equilibrate(d_A, n, lda, 0.0, e, err, sm);
        chol_inverse(d_A, n, lda, T, W, Tt, small, err, sm);
        launch_unequilibrate(d_A, n, lda, e, nullptr, sm);
        ce = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, sm);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(sm);
    if (ce != cudaSuccess) {
        g_last_error = cudaGetErrorString(ce);
        return UNC_ERR_CUDA;
    }
    if (h_err & (ERRBIT_SINGULAR | ERRBIT_NONFINITE)) {
        g_last_error = "matrix is not positive definite";
        return UNC_ERR_SINGULAR;
    }
    return UNC_OK;
}
