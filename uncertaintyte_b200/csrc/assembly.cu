// assembly.cu - sparse-Jacobian ingest, J^T J block assembly, point 3x3
// inverses and the camera Schur-complement scatter (sm_100a).
//
// Replaces, for the TAYLOR_EXPANSION path of uncertaintyTE:
//   fixPts                       compute.cpp:283-368
//   SSM::scaleMat(RIGHT)         ScaledSparseMatrix.cpp:334-358, compute.cpp:77-82
//   J^T J + splitTo3Blocks       compute.cpp:86-96, ScaledSparseMatrix.cpp:238-299,517-539
//   inv3x3blockSymmDiag          ScaledSparseMatrix.cpp:210-230
//   Z = U - W iV W^T (dense)     compute.cpp:108-112
//
// Device layout: the Jacobian values are used in place. With the reference's
// layout (every row 12 entries) observation o occupies values[24o, 24o+24):
// [row0: 9 camera, 3 point | row1: 9 camera, 3 point], a 192-byte record
// read with 128-bit loads. Fixed-point observations are masked (obs_pt = -1)
// instead of compacted; the reference deletes those rows (compute.cpp:337-366).
#include "internal.h"

namespace unc {

// ------------------------------------------------------------------------
// validation / ids
// ------------------------------------------------------------------------
__global__ void k_validate_obs(int num_obs, int num_cams, int num_points, int3 fix, int has_fix,
                               long nnz, const int* __restrict__ rows, const int* __restrict__ cols,
                               int* __restrict__ obs_cam, int* __restrict__ obs_pt, int* err) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= num_obs) return;
    const long base = 24L * o;
    bool bad = rows[2 * o] != base || rows[2 * o + 1] != base + 12 || rows[2 * o + 2] != base + 24 ||
               base + 24 > nnz;
    int cam = -1, pt = -1;
    if (!bad) {
        const int4* c4 = reinterpret_cast<const int4*>(cols + base);
        int c[24];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            int4 v = c4[q];
            c[4 * q] = v.x;
            c[4 * q + 1] = v.y;
            c[4 * q + 2] = v.z;
            c[4 * q + 3] = v.w;
        }
        cam = c[0] / kCamParams;
        const int cam_off = kCamParams * num_cams;
        pt = (c[9] - cam_off) / 3;
        bad |= c[0] < 0 || cam >= num_cams || c[9] < cam_off || pt >= num_points;
#pragma unroll
        for (int j = 0; j < 9; ++j) bad |= (c[j] != cam * 9 + j) | (c[12 + j] != cam * 9 + j);
#pragma unroll
        for (int j = 0; j < 3; ++j)
            bad |= (c[9 + j] != cam_off + 3 * pt + j) | (c[21 + j] != cam_off + 3 * pt + j);
    }
    if (bad) {
        atomicOr(err, ERRBIT_LAYOUT);
        cam = pt = -1;
    } else if (has_fix && (pt == fix.x || pt == fix.y || pt == fix.z)) {
        cam = pt = -1;  // all rows of a fixed point are deleted (compute.cpp:337-366)
    }
    obs_cam[o] = cam;
    obs_pt[o] = pt;
}

void launch_validate_obs(const SceneDev& s, cudaStream_t st) {
    if (s.num_obs == 0) return;
    int3 fix = make_int3(s.fix[0], s.fix[1], s.fix[2]);
    k_validate_obs<<<(s.num_obs + 255) / 256, 256, 0, st>>>(s.num_obs, s.num_cams, s.num_points,
                                                            fix, s.has_fix, s.nnz, s.rows, s.cols,
                                                            s.obs_cam, s.obs_pt, s.err);
    count_launch();
}

// Generic repack for J^T J export: rows of 12 (camera + point) or 9 (camera
// only) entries; writes the 24-value observation record with zero point part.
__global__ void k_repack_generic(int num_obs, int cam_off, const int* __restrict__ rows,
                                 const int* __restrict__ cols, const double* __restrict__ vals,
                                 double* __restrict__ J, int* obs_cam, int* obs_pt, int* err) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= num_obs) return;
    int r0 = rows[2 * o], r1 = rows[2 * o + 1], r2 = rows[2 * o + 2];
    int n0 = r1 - r0, n1 = r2 - r1;
    bool bad = n0 != n1 || (n0 != 12 && n0 != 9);
    int cam = -1, pt = -1;
    double* out = J + 24L * o;
    if (!bad) {
        cam = cols[r0] / kCamParams;
        for (int j = 0; j < 9; ++j) {
            bad |= cols[r0 + j] != cam * 9 + j || cols[r1 + j] != cam * 9 + j;
            out[j] = vals[r0 + j];
            out[12 + j] = vals[r1 + j];
        }
        if (n0 == 12) {
            pt = (cols[r0 + 9] - cam_off) / 3;
            for (int j = 0; j < 3; ++j) {
                bad |= cols[r0 + 9 + j] != cam_off + 3 * pt + j || cols[r1 + 9 + j] != cam_off + 3 * pt + j;
                out[9 + j] = vals[r0 + 9 + j];
                out[21 + j] = vals[r1 + 9 + j];
            }
        } else {
            for (int j = 0; j < 3; ++j) out[9 + j] = out[21 + j] = 0.0;
        }
    }
    if (bad) {
        atomicOr(err, ERRBIT_LAYOUT);
        cam = pt = -1;
    }
    obs_cam[o] = cam;
    obs_pt[o] = pt;
}

void launch_repack_generic(int num_obs, int cam_off, const int* rows, const int* cols,
                           const double* vals, double* J, int* obs_cam, int* obs_pt, int* err,
                           cudaStream_t st) {
    if (num_obs == 0) return;
    k_repack_generic<<<(num_obs + 255) / 256, 256, 0, st>>>(num_obs, cam_off, rows, cols, vals, J,
                                                            obs_cam, obs_pt, err);
    count_launch();
}

// ------------------------------------------------------------------------
// exclusive scan (n + 1 outputs, out[n] = total)
// ------------------------------------------------------------------------
constexpr int kScanBlock = 1024;

__global__ void k_scan_block(const int* __restrict__ in, int* __restrict__ out, int n,
                             int* __restrict__ block_sums) {
    __shared__ int warp_sums[32];
    int i = blockIdx.x * kScanBlock + threadIdx.x;
    int v = i < n ? in[i] : 0;
    // inclusive warp scan
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = warp_sums[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    int incl = x + (w > 0 ? warp_sums[w - 1] : 0);
    if (i < n) out[i] = incl - v;
    if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = incl;
}

__global__ void k_scan_add(int* out, int n, const int* __restrict__ block_offsets) {
    int i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n && blockIdx.x > 0) out[i] += block_offsets[blockIdx.x];
}

__global__ void k_scan_total(const int* in, int* out, int n) {
    out[n] = (n > 0 ? out[n - 1] + in[n - 1] : 0);
}

size_t scan_tmp_ints(int n) {
    size_t total = 0;
    int m = n;
    while (true) {
        int nb = (m + kScanBlock - 1) / kScanBlock;
        total += 2 * ((size_t)nb + 1);  // block sums + their scan, per level
        if (nb <= 1) break;
        m = nb;
    }
    return total + 8;
}

void exclusive_scan(const int* in, int* out, int n, int* tmp, cudaStream_t st) {
    if (n <= 0) {
        cudaMemsetAsync(out, 0, sizeof(int), st);
        return;
    }
    int nb = (n + kScanBlock - 1) / kScanBlock;
    int* sums = tmp;
    k_scan_block<<<nb, kScanBlock, 0, st>>>(in, out, n, sums);
    count_launch();
    if (nb > 1) {
        int* offs = tmp + nb + 1;
        exclusive_scan(sums, offs, nb, offs + nb + 1, st);
        k_scan_add<<<nb, kScanBlock, 0, st>>>(out, n, offs);
        count_launch();
    }
    k_scan_total<<<1, 1, 0, st>>>(in, out, n);
    count_launch();
}

// ------------------------------------------------------------------------
// observation index by camera and by point (counting sort + segment sort)
// ------------------------------------------------------------------------
__global__ void k_count_keys(int num_obs, const int* __restrict__ obs_cam,
                             const int* __restrict__ obs_pt, int* cam_cnt, int* pt_cnt) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= num_obs) return;
    int c = obs_cam[o], p = obs_pt[o];
    if (c >= 0) atomicAdd(cam_cnt + c, 1);
    if (p >= 0) atomicAdd(pt_cnt + p, 1);
}

__global__ void k_scatter_keys(int num_obs, const int* __restrict__ obs_cam,
                               const int* __restrict__ obs_pt, int* cam_cur, int* pt_cur,
                               int* cam_obs, int* pt_obs) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= num_obs) return;
    int c = obs_cam[o], p = obs_pt[o];
    if (c >= 0) cam_obs[atomicAdd(cam_cur + c, 1)] = o;
    if (p >= 0) pt_obs[atomicAdd(pt_cur + p, 1)] = o;
}

// One warp per segment; rank sort through shared memory (segments <= 1024).
constexpr int kWarpSortCap = 1024;
__global__ void k_sort_segments_warp(int nseg, const int* __restrict__ ptr, int* data, int* err) {
    __shared__ int sh[4][kWarpSortCap];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int seg = blockIdx.x * 4 + w;
    if (seg >= nseg) return;
    int b = ptr[seg], n = ptr[seg + 1] - b;
    if (n <= 1) return;
    if (n > kWarpSortCap) {
        if (lane == 0) atomicOr(err, ERRBIT_SORT_CAP);
        return;
    }
    int* s = sh[w];
    for (int i = lane; i < n; i += 32) s[i] = data[b + i];
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
        int v = s[i], r = 0;
        for (int j = 0; j < n; ++j) r += s[j] < v;
        data[b + r] = v;
    }
}

// One block per segment; bitonic sort in shared memory (segments <= 8192).
constexpr int kBlockSortCap = 8192;
__global__ void k_sort_segments_block(const int* __restrict__ ptr, int* data, int* err) {
    __shared__ int s[kBlockSortCap];
    int seg = blockIdx.x;
    int b = ptr[seg], n = ptr[seg + 1] - b;
    if (n <= 1) return;
    if (n > kBlockSortCap) {
        if (threadIdx.x == 0) atomicOr(err, ERRBIT_SORT_CAP);
        return;
    }
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = threadIdx.x; i < m; i += blockDim.x) s[i] = i < n ? data[b + i] : 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                int l = i ^ j;
                if (l > i) {
                    bool up = (i & k) == 0;
                    int a = s[i], c = s[l];
                    if ((a > c) == up) {
                        s[i] = c;
                        s[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) data[b + i] = s[i];
}

void launch_build_index(SceneDev& s, cudaStream_t st) {
    const int C = s.num_cams, P = s.num_points, n = s.num_obs;
    int* cam_cnt = s.cursor;       // C
    int* pt_cnt = s.cursor + C;    // P
    cudaMemsetAsync(s.cursor, 0, sizeof(int) * ((size_t)C + P), st);
    if (n > 0) {
        k_count_keys<<<(n + 255) / 256, 256, 0, st>>>(n, s.obs_cam, s.obs_pt, cam_cnt, pt_cnt);
        count_launch();
    }
    exclusive_scan(cam_cnt, s.cam_ptr, C, s.scan_tmp, st);
    exclusive_scan(pt_cnt, s.pt_ptr, P, s.scan_tmp, st);
    cudaMemcpyAsync(cam_cnt, s.cam_ptr, sizeof(int) * C, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(pt_cnt, s.pt_ptr, sizeof(int) * P, cudaMemcpyDeviceToDevice, st);
    if (n > 0) {
        k_scatter_keys<<<(n + 255) / 256, 256, 0, st>>>(n, s.obs_cam, s.obs_pt, cam_cnt, pt_cnt,
                                                        s.cam_obs, s.pt_obs);
        count_launch();
    }
    if (C > 0) {
        k_sort_segments_block<<<C, 512, 0, st>>>(s.cam_ptr, s.cam_obs, s.err);
        count_launch();
    }
    if (P > 0) {
        k_sort_segments_warp<<<(P + 3) / 4, 128, 0, st>>>(P, s.pt_ptr, s.pt_obs, s.err);
        count_launch();
    }
}

// ------------------------------------------------------------------------
// J^T J blocks
// ------------------------------------------------------------------------
// upper-triangle index of (j,k), j <= k < 9, row-major: t = j*9 - j*(j-1)/2 + (k-j)
__host__ __device__ constexpr int ut9(int j, int k) { return j * 9 - (j * (j - 1)) / 2 + (k - j); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

// Load the 18 camera values of observation o (row0 c0..c8, row1 c0..c8) with
// 128-bit loads from the 24-double record.
__device__ __forceinline__ void load_cam_rows(const double* __restrict__ J, int o, double r0[9],
                                              double r1[9]) {
    const double2* q = reinterpret_cast<const double2*>(J + 24L * o);
    double2 a0 = __ldg(q + 0), a1 = __ldg(q + 1), a2 = __ldg(q + 2), a3 = __ldg(q + 3),
            a4 = __ldg(q + 4);
    double2 b0 = __ldg(q + 6), b1 = __ldg(q + 7), b2 = __ldg(q + 8), b3 = __ldg(q + 9),
            b4 = __ldg(q + 10);
    r0[0] = a0.x; r0[1] = a0.y; r0[2] = a1.x; r0[3] = a1.y; r0[4] = a2.x;
    r0[5] = a2.y; r0[6] = a3.x; r0[7] = a3.y; r0[8] = a4.x;
    r1[0] = b0.x; r1[1] = b0.y; r1[2] = b1.x; r1[3] = b1.y; r1[4] = b2.x;
    r1[5] = b2.y; r1[6] = b3.x; r1[7] = b3.y; r1[8] = b4.x;
}

__device__ __forceinline__ void load_pt_rows(const double* __restrict__ J, int o, double p0[3],
                                             double p1[3]) {
    const double* r = J + 24L * o;
    double2 a = __ldg(reinterpret_cast<const double2*>(r + 8));   // c8, p0
    double2 b = __ldg(reinterpret_cast<const double2*>(r + 10));  // p1, p2
    double2 c = __ldg(reinterpret_cast<const double2*>(r + 20));  // c8', p0'
    double2 d = __ldg(reinterpret_cast<const double2*>(r + 22));  // p1', p2'
    p0[0] = a.y; p0[1] = b.x; p0[2] = b.y;
    p1[0] = c.y; p1[1] = d.x; p1[2] = d.y;
}

// ------------------------------------------------------------------------
// per-camera observation tiles
// ------------------------------------------------------------------------
// The observations of camera c, cam_obs[cam_ptr[c], cam_ptr[c+1]), are cut
// into tiles of kObsTile. Camera c owns the tile slots [base(c), base(c+1))
// with base(c) = c + cam_ptr[c] / kObsTile: never fewer than its tiles, since
// ceil((B - A) / T) <= floor(B / T) - floor(A / T) + 1. Slots past a camera's
// last tile are empty. The slot count base(C) is bounded on the host by
// C + num_obs / kObsTile, so the grids need no read-back; a CTA finds its
// camera by binary search over cam_ptr. Per-tile partial sums are combined per
// camera in slot order: a fixed summation order, bitwise repeatable.
constexpr int kObsTile = 256;
constexpr int kTileGroups = 5;  // 45 upper-triangle elements x 5 groups = 225 of the 256 threads

size_t camera_tile_slots(int num_cams, int num_obs) { return (size_t)num_cams + num_obs / kObsTile + 1; }

__device__ __forceinline__ int tile_base(const int* __restrict__ cam_ptr, int c) {
    return c + cam_ptr[c] / kObsTile;
}

struct ObsTile {
    int cam, begin, end;
};

__device__ __forceinline__ bool find_tile(const int* __restrict__ cam_ptr, int num_cams, int k, ObsTile& t) {
    if (k >= tile_base(cam_ptr, num_cams)) return false;
    int lo = 0, hi = num_cams;  // tile_base(lo) <= k < tile_base(hi)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tile_base(cam_ptr, mid) <= k)
            lo = mid;
        else
            hi = mid;
    }
    t.cam = lo;
    t.end = cam_ptr[lo + 1];
    t.begin = min(cam_ptr[lo] + (k - tile_base(cam_ptr, lo)) * kObsTile, t.end);
    t.end = min(t.begin + kObsTile, t.end);
    return true;
}

// (j, k), j <= k, of upper-triangle element el (inverse of ut9)
__device__ __forceinline__ void ut9_inv(int el, int& j, int& k) {
    j = 0;
    while (j < 8 && ut9(j + 1, j + 1) <= el) ++j;
    k = j + (el - ut9(j, j));
}

// U = sum_o Jc_o^T Jc_o per tile: the tile's 18 camera values per observation
// are staged in shared memory (odd row stride: conflict-free), then thread
// (el, g) sums element el over the tile's observations g, g + 5, ...
constexpr int kGramStride = 19;
__global__ void __launch_bounds__(kObsTile) k_camera_gram_tiles(int num_cams, const double* __restrict__ J,
                                                                const int* __restrict__ cam_ptr,
                                                                const int* __restrict__ cam_obs,
                                                                double* __restrict__ part) {
    __shared__ double sj[kObsTile * kGramStride];
    __shared__ double red[kTileGroups][45];
    ObsTile tile;
    if (!find_tile(cam_ptr, num_cams, blockIdx.x, tile)) return;
    const int n = tile.end - tile.begin, t = threadIdx.x;
    if (t < n) {
        double r0[9], r1[9];
        load_cam_rows(J, cam_obs[tile.begin + t], r0, r1);
        double* row = sj + t * kGramStride;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            row[j] = r0[j];
            row[9 + j] = r1[j];
        }
    }
    __syncthreads();
    if (t < 45 * kTileGroups) {
        const int el = t % 45, g = t / 45;
        int j, k;
        ut9_inv(el, j, k);
        double acc = 0.0;
        for (int i = g; i < n; i += kTileGroups) {
            const double* row = sj + i * kGramStride;
            acc += row[j] * row[k] + row[9 + j] * row[9 + k];
        }
        red[g][el] = acc;
    }
    __syncthreads();
    if (t < 45) {
        double v = red[0][t];
#pragma unroll
        for (int g = 1; g < kTileGroups; ++g) v += red[g][t];
        part[45L * blockIdx.x + t] = v;
    }
}

// One warp per camera: U = sum of the camera's tile partials, column norms
// s = sqrt(diag U), scaled block U/(s s) written as a full 9 x 9 block
// (column-major, 81 per camera). J <- J diag(1/s) skips s == 0
// (ScaledSparseMatrix.cpp:352-356).
__global__ void __launch_bounds__(128) k_camera_gram_reduce(int num_cams, const int* __restrict__ cam_ptr,
                                                            const double* __restrict__ part,
                                                            double* __restrict__ s_cam, double* __restrict__ U) {
    __shared__ double sh[4][45];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cam = blockIdx.x * 4 + w;
    if (cam >= num_cams) return;
    const int k0 = tile_base(cam_ptr, cam), k1 = tile_base(cam_ptr, cam + 1);
    double a0 = 0.0, a1 = 0.0;
    for (int k = k0; k < k1; ++k) {
        a0 += part[45L * k + lane];
        if (lane < 13) a1 += part[45L * k + 32 + lane];
    }
    double* u = sh[w];
    u[lane] = a0;
    if (lane < 13) u[32 + lane] = a1;
    __syncwarp();
    if (lane < 9 && s_cam) s_cam[9L * cam + lane] = sqrt(u[ut9(lane, lane)]);
    for (int el = lane; el < 45; el += 32) {
        int j, k;
        ut9_inv(el, j, k);
        const double sj = sqrt(u[ut9(j, j)]), sk = sqrt(u[ut9(k, k)]);
        double v = u[el];
        if (sj != 0) v *= 1.0 / sj;
        if (sk != 0) v *= 1.0 / sk;
        U[81L * cam + j + 9 * k] = v;
        U[81L * cam + k + 9 * j] = v;
    }
}

size_t camera_tile_part_doubles(int num_cams, int num_obs) { return 45 * camera_tile_slots(num_cams, num_obs); }

void launch_camera_blocks(const SceneDev& s, cudaStream_t st) {
    if (s.num_cams == 0) return;
    const unsigned slots = (unsigned)camera_tile_slots(s.num_cams, s.num_obs);
    k_camera_gram_tiles<<<slots, kObsTile, 0, st>>>(s.num_cams, s.J, s.cam_ptr, s.cam_obs, s.cam_part);
    k_camera_gram_reduce<<<(s.num_cams + 3) / 4, 128, 0, st>>>(s.num_cams, s.cam_ptr, s.cam_part, s.s_cam,
                                                                s.Ucam);
    count_launch(2);
}

// One thread per point: V_p = sum Jp^T Jp (unscaled), s = sqrt(diag), scaled
// inverse with the reference's closed-form adjugate (ScaledSparseMatrix.cpp:219-228).
__global__ void k_point_blocks(int num_points, const double* __restrict__ J,
                               const int* __restrict__ pt_ptr, const int* __restrict__ pt_obs,
                               double* __restrict__ s_pt, double* __restrict__ Vraw,
                               double* __restrict__ iVs) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= num_points) return;
    double v00 = 0, v01 = 0, v02 = 0, v11 = 0, v12 = 0, v22 = 0;
    for (int i = pt_ptr[p]; i < pt_ptr[p + 1]; ++i) {
        double a[3], b[3];
        load_pt_rows(J, pt_obs[i], a, b);
        v00 += a[0] * a[0] + b[0] * b[0];
        v01 += a[0] * a[1] + b[0] * b[1];
        v02 += a[0] * a[2] + b[0] * b[2];
        v11 += a[1] * a[1] + b[1] * b[1];
        v12 += a[1] * a[2] + b[1] * b[2];
        v22 += a[2] * a[2] + b[2] * b[2];
    }
    double* V = Vraw + 6L * p;
    V[0] = v00; V[1] = v01; V[2] = v02; V[3] = v11; V[4] = v12; V[5] = v22;
    double s0 = sqrt(v00), s1 = sqrt(v11), s2 = sqrt(v22);
    s_pt[3L * p] = s0;
    s_pt[3L * p + 1] = s1;
    s_pt[3L * p + 2] = s2;
    double i0 = s0 != 0 ? 1.0 / s0 : 1.0, i1 = s1 != 0 ? 1.0 / s1 : 1.0, i2 = s2 != 0 ? 1.0 / s2 : 1.0;
    // scaled block entries a b c / . e f / . . k
    double a = v00 * i0 * i0, b = v01 * i0 * i1, c = v02 * i0 * i2;
    double e = v11 * i1 * i1, f = v12 * i1 * i2, k = v22 * i2 * i2;
    double* o = iVs + 6L * p;
    if (pt_ptr[p + 1] == pt_ptr[p]) {  // unobserved or fixed point: unused
        o[0] = o[1] = o[2] = o[3] = o[4] = o[5] = 0.0;
        return;
    }
    double div = a * e * k - a * f * f - b * b * k + 2 * b * c * f - c * c * e;
    o[0] = (e * k - f * f) / div;
    o[1] = (-b * k + c * f) / div;
    o[2] = (b * f - c * e) / div;
    o[3] = (a * k - c * c) / div;
    o[4] = (-a * f + b * c) / div;
    o[5] = (a * e - b * b) / div;
}

void launch_point_blocks(const SceneDev& s, cudaStream_t st) {
    if (s.num_points == 0) return;
    k_point_blocks<<<(s.num_points + 127) / 128, 128, 0, st>>>(s.num_points, s.J, s.pt_ptr,
                                                               s.pt_obs, s.s_pt, s.Vraw, s.iVs);
    count_launch();
}

// W_o = Jc^T Jp scaled by the column norms and Y_o = W_o iV_p (the
// camera-point block of Y = W * iV, compute.cpp:108), one camera tile per CTA.
// One thread per observation computes its two 9 x 3 blocks into shared memory
// (odd record stride 27: conflict-free); the block then writes them out as
// 216-byte records, consecutive threads on consecutive elements.
constexpr size_t kObsTileSmem = 2ul * kObsTile * 27 * sizeof(double);  // 110,592 bytes

__global__ void __launch_bounds__(kObsTile) k_camera_obs_tiles(
    int num_cams, const double* __restrict__ J, const int* __restrict__ cam_ptr, const int* __restrict__ cam_obs,
    const int* __restrict__ obs_pt, const double* __restrict__ s_cam, const double* __restrict__ s_pt,
    const double* __restrict__ iVs, double* __restrict__ Ws, double* __restrict__ Ys) {
    extern __shared__ double smem[];
    double* sw = smem;                   // [kObsTile][27] W_o
    double* sy = smem + kObsTile * 27;   // [kObsTile][27] Y_o
    __shared__ int so[kObsTile];
    __shared__ double isc[9];
    ObsTile tile;
    if (!find_tile(cam_ptr, num_cams, blockIdx.x, tile)) return;
    const int n = tile.end - tile.begin, t = threadIdx.x;
    if (t < 9) {
        const double v = s_cam[9L * tile.cam + t];
        isc[t] = v != 0 ? 1.0 / v : 1.0;
    }
    __syncthreads();
    if (t < n) {
        const int o = cam_obs[tile.begin + t];
        const int p = obs_pt[o];
        so[t] = o;
        double r0[9], r1[9], a[3], b[3];
        load_cam_rows(J, o, r0, r1);
        load_pt_rows(J, o, a, b);
        double sp[3], is[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double v = s_pt[3L * p + k];
            sp[k] = v != 0 ? 1.0 / v : 1.0;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) is[k] = iVs[6L * p + k];
        const double iv[3][3] = {{is[0], is[1], is[2]}, {is[1], is[3], is[4]}, {is[2], is[4], is[5]}};
        double* W = sw + 27 * t;
        double* Y = sy + 27 * t;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            const double sc = isc[j];
            double w[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) w[k] = (r0[j] * a[k] + r1[j] * b[k]) * sc * sp[k];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                W[3 * j + k] = w[k];
                Y[3 * j + k] = w[0] * iv[0][k] + w[1] * iv[1][k] + w[2] * iv[2][k];
            }
        }
    }
    __syncthreads();
    // write-out over the flattened (record, element) index: consecutive threads take consecutive
    // elements of a record and then the next record, so every store instruction covers 256 bytes
    for (int idx = t; idx < n * 27; idx += kObsTile) {
        const int i = idx / 27, e = idx - 27 * i;
        const long o = so[i];
        Ws[27 * o + e] = sw[idx];
        Ys[27 * o + e] = sy[idx];
    }
}

void launch_obs_blocks(const SceneDev& s, cudaStream_t st) {
    if (s.num_cams == 0) return;
    prepare_assembly_kernels();
    const unsigned slots = (unsigned)camera_tile_slots(s.num_cams, s.num_obs);
    k_camera_obs_tiles<<<slots, kObsTile, kObsTileSmem, st>>>(s.num_cams, s.J, s.cam_ptr, s.cam_obs, s.obs_pt,
                                                              s.s_cam, s.s_pt, s.iVs, s.Ws, s.Ys);
    count_launch();
}

void prepare_assembly_kernels() {
    prepare_schur_columns();
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_camera_obs_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kObsTileSmem) == cudaSuccess &&
               cudaFuncSetAttribute(k_camera_obs_tiles, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared) == cudaSuccess;
    });
}

// Unscaled blocks for the J^T J export: U (9x9 per camera, column-major
// inside a (9C x 9C) dense buffer is too large, so U is written per camera as
// 81 values) and W_o per observation (27 values, row-major 9x3).
__global__ void __launch_bounds__(128) k_camera_blocks_raw(int num_cams, const double* __restrict__ J,
                                                           const int* __restrict__ cam_ptr,
                                                           const int* __restrict__ cam_obs,
                                                           double* __restrict__ U) {
    int cam = blockIdx.x * 4 + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (cam >= num_cams) return;
    double acc[45];
#pragma unroll
    for (int t = 0; t < 45; ++t) acc[t] = 0.0;
    for (int i = cam_ptr[cam] + lane; i < cam_ptr[cam + 1]; i += 32) {
        double r0[9], r1[9];
        load_cam_rows(J, cam_obs[i], r0, r1);
#pragma unroll
        for (int j = 0; j < 9; ++j)
#pragma unroll
            for (int k = j; k < 9; ++k) acc[ut9(j, k)] += r0[j] * r0[k] + r1[j] * r1[k];
    }
#pragma unroll
    for (int t = 0; t < 45; ++t) acc[t] = warp_sum(acc[t]);
#pragma unroll
    for (int j = 0; j < 9; ++j)
#pragma unroll
        for (int k = j; k < 9; ++k)
            if (lane == ut9(j, k) || lane + 32 == ut9(j, k)) {
                U[81L * cam + 9 * j + k] = acc[ut9(j, k)];
                U[81L * cam + 9 * k + j] = acc[ut9(j, k)];
            }
}

__global__ void k_obs_blocks_raw(int num_obs, const double* __restrict__ J,
                                 const int* __restrict__ obs_cam, const int* __restrict__ obs_pt,
                                 double* __restrict__ W) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= num_obs) return;
    if (obs_cam[o] < 0 || obs_pt[o] < 0) return;
    double r0[9], r1[9], a[3], b[3];
    load_cam_rows(J, o, r0, r1);
    load_pt_rows(J, o, a, b);
#pragma unroll
    for (int j = 0; j < 9; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) W[27L * o + 3 * j + k] = r0[j] * a[k] + r1[j] * b[k];
}

void launch_unscaled_blocks(const SceneDev& s, double* U, double* W, cudaStream_t st) {
    if (s.num_cams > 0) {
        k_camera_blocks_raw<<<(s.num_cams + 3) / 4, 128, 0, st>>>(s.num_cams, s.J, s.cam_ptr,
                                                                  s.cam_obs, U);
        count_launch();
    }
    if (s.num_obs > 0) {
        k_obs_blocks_raw<<<(s.num_obs + 127) / 128, 128, 0, st>>>(s.num_obs, s.J, s.obs_cam,
                                                                  s.obs_pt, W);
        count_launch();
    }
}

}  // namespace unc
