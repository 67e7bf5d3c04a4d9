// accessors.cu - batched eigen-decompositions of the covariance blocks behind
// the Uncertainty accessors (uncertainty.cpp:74-183: eigenvalues of every
// camera and point block, sorted descending, and eigenvectors of the point
// blocks and of the camera-centre 3 x 3 sub-blocks). The reference runs one
// Eigen::EigenSolver per block on the host; here one warp owns one block.
//
// Input: packed upper triangles (row-major, i <= j) of src x src blocks
// (45 values for src = 9, 6 for src = 3); the sub-block [off, off + dim) of each
// is decomposed. Output: dim eigenvalues per block in descending order and the
// matching unit eigenvectors, column c of block b at vectors[b*dim*dim + c*dim].
// Method: cyclic Jacobi rotations (Golub & Van Loan, symmetric Schur 2 x 2),
// off-diagonal entries below 1e-17 sqrt(|a_pp a_qq|) left alone; eigenvector
// signs are arbitrary (as with the reference's EigenSolver).
#include "../../include/uncte.h"
#include "internal.h"

namespace unc {
namespace {

constexpr int kMaxDim = 9;
constexpr int kWarpsPerCta = 4;

__global__ void __launch_bounds__(32 * kWarpsPerCta)
    k_block_eigen(const double* __restrict__ packed, int nblk, int src, int off, int dim, double* vals,
                  double* vecs) {
    __shared__ double As[kWarpsPerCta][kMaxDim][kMaxDim + 1], Vs[kWarpsPerCta][kMaxDim][kMaxDim + 1];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int blk = blockIdx.x * kWarpsPerCta + w;
    if (blk >= nblk) return;  // whole warps leave together
    double(*A)[kMaxDim + 1] = As[w];
    double(*V)[kMaxDim + 1] = Vs[w];
    const int per = src * (src + 1) / 2;
    const double* in = packed + (long)blk * per;
    if (l < dim) {
        const int i = off + l;
        for (int c = 0; c < dim; ++c) {
            const int j = off + c;
            const int a = i < j ? i : j, b = i < j ? j : i;  // upper-triangle index of (a, b)
            A[l][c] = in[a * src - a * (a - 1) / 2 + (b - a)];
            V[l][c] = (l == c) ? 1.0 : 0.0;
        }
    }
    __syncwarp();
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off2 = 0.0, dg = 0.0;
        if (l < dim) {
            for (int c = 0; c < l; ++c) off2 += A[l][c] * A[l][c];
            dg = A[l][l] * A[l][l];
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            off2 += __shfl_xor_sync(0xffffffffu, off2, d);
            dg += __shfl_xor_sync(0xffffffffu, dg, d);
        }
        if (off2 <= 1e-30 * dg) break;
        for (int p = 0; p < dim - 1; ++p)
            for (int q = p + 1; q < dim; ++q) {
                const double apq = A[p][q], app = A[p][p], aqq = A[q][q];
                if (apq == 0.0 || fabs(apq) <= 1e-17 * sqrt(fabs(app * aqq))) continue;
                const double th = (aqq - app) / (2.0 * apq);
                const double t = fabs(th) > 1e100 ? 0.5 / th
                                                  : (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                __syncwarp();
                if (l < dim) {
                    const double x = A[l][p], y = A[l][q];
                    A[l][p] = c * x - s * y;
                    A[l][q] = s * x + c * y;
                    const double vx = V[l][p], vy = V[l][q];
                    V[l][p] = c * vx - s * vy;
                    V[l][q] = s * vx + c * vy;
                }
                __syncwarp();
                if (l < dim) {
                    const double x = A[p][l], y = A[q][l];
                    A[p][l] = c * x - s * y;
                    A[q][l] = s * x + c * y;
                }
                __syncwarp();
            }
    }
    if (l < dim) {  // descending order, ties by index
        const double ev = A[l][l];
        int rank = 0;
        for (int i = 0; i < dim; ++i) {
            const double u = A[i][i];
            rank += (u > ev) || (u == ev && i < l);
        }
        vals[(long)blk * dim + rank] = ev;
        double* out = vecs ? vecs + (long)blk * dim * dim + (long)rank * dim : nullptr;
        if (out)
            for (int r = 0; r < dim; ++r) out[r] = V[r][l];
    }
}

}  // namespace
}  // namespace unc

using namespace unc;

extern "C" int unc_block_eigen_device(const double* d_packed, int num_blocks, int block_params, int sub_offset,
                                      int sub_dim, double* d_values, double* d_vectors, void* stream) {
    g_last_error.clear();
    if (num_blocks < 0 || block_params < 1 || block_params > kMaxDim || sub_offset < 0 || sub_dim < 1 ||
        sub_offset + sub_dim > block_params || (num_blocks && (!d_packed || !d_values))) {
        g_last_error = "unc_block_eigen_device: bad arguments (block_params <= 9, sub-block inside the block)";
        return UNC_ERR_INVALID_ARG;
    }
    if (num_blocks == 0) return UNC_OK;
    cudaStream_t sm = (cudaStream_t)stream;
    k_block_eigen<<<(num_blocks + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0, sm>>>(
        d_packed, num_blocks, block_params, sub_offset, sub_dim, d_values, d_vectors);
    count_launch();
    cudaError_t e = cudaStreamSynchronize(sm);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_error = std::string("unc_block_eigen_device: ") + cudaGetErrorString(e);
        return UNC_ERR_CUDA;
    }
    return UNC_OK;
}

extern "C" int unc_block_eigen(const double* packed, int num_blocks, int block_params, int sub_offset, int sub_dim,
                               double* values, double* vectors) {
    g_last_error.clear();
    if (num_blocks < 0 || block_params < 1 || block_params > kMaxDim || sub_offset < 0 || sub_dim < 1 ||
        sub_offset + sub_dim > block_params || (num_blocks && (!packed || !values))) {
        g_last_error = "unc_block_eigen: bad arguments (block_params <= 9, sub-block inside the block)";
        return UNC_ERR_INVALID_ARG;
    }
    if (num_blocks == 0) return UNC_OK;
    const size_t nin = (size_t)num_blocks * block_params * (block_params + 1) / 2;
    const size_t nv = (size_t)num_blocks * sub_dim, nvec = vectors ? nv * sub_dim : 0;
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(double) * (nin + nv + nvec));
    if (e != cudaSuccess) {
        g_last_error = std::string("unc_block_eigen: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? UNC_ERR_OUT_OF_MEMORY : UNC_ERR_CUDA;
    }
    e = cudaMemcpy(d, packed, sizeof(double) * nin, cudaMemcpyHostToDevice);
    int rc = UNC_OK;
    if (e == cudaSuccess)
        rc = unc_block_eigen_device(d, num_blocks, block_params, sub_offset, sub_dim, d + nin,
                                    vectors ? d + nin + nv : nullptr, nullptr);
    if (e == cudaSuccess && rc == UNC_OK) e = cudaMemcpy(values, d + nin, sizeof(double) * nv, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && rc == UNC_OK && vectors)
        e = cudaMemcpy(vectors, d + nin + nv, sizeof(double) * nvec, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (rc != UNC_OK) return rc;
    if (e != cudaSuccess) {
        g_last_error = std::string("unc_block_eigen: ") + cudaGetErrorString(e);
        return UNC_ERR_CUDA;
    }
    return UNC_OK;
}
