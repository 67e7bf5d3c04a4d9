// schur.cu - the camera Schur complement Z = U - W V^-1 W^T (compute.cpp:108-118;
// Y = W V^-1 is formed per observation by the observation tiles), one camera
// column per CTA, without a global pair list.
//
// Z(ca, cb) = U(ca, cb) - sum over the points p seen by both cameras of
// Y_o W_o'^T, o the observation of p by camera ca and o' by cb (9 x 3 records,
// Y_o = W_o V_p^-1). The CTA of camera cb forms the blocks ca <= cb of column
// cb and writes each one twice, in place (upper triangle) and transposed
// (Z(cb, ca)), so Z comes out exactly symmetric and needs no mirror pass:
//  1. the observations o' of cb (its index list) are taken in chunks; the
//     observation lists of their points are copied into shared memory (the
//     partners; those of cameras <= cb, o' itself included, count), one list
//     slot per thread, so the lookups run in parallel;
//  2. the partner cameras get slots (ascending camera); a bit mask per slot
//     marks the chunk's observations with a partner in that camera, so the
//     set bits walk the terms of one block in a fixed order;
//  3. one warp per slot sums its block in registers, ten terms per step and
//     three lanes per term (each a band of three rows of the 9 x 9 block); the
//     partial sums are added in a fixed order and the block is stored
//     (subtracted from U on the diagonal, read back and updated for the second
//     and later chunks).
// No floating-point atomics, no device-to-host round trip: the result is
// bitwise repeatable and the stage can be captured in a graph. A camera that
// observes a point more than once gives more than one term per (slot,
// observation); those extra terms are added by further passes.
#include "internal.h"

namespace unc {
namespace {

constexpr int kSzThreads = 384;       // 12 warps
constexpr int kSzWarps = kSzThreads / 32;
constexpr int kSzChunk = 2048;        // owner observations per chunk, at most
constexpr int kSzParts = 16384;       // partner list slots per chunk, at most
constexpr int kSzMaskWords = 16384;   // run-mask words (also the list-slot owners and the camera scan)
constexpr int kSzGroups = 10;         // terms per step of sz_block10 (three lanes each)
constexpr int kSzSegCap = 512;        // run entries staged per warp at a time
constexpr unsigned short kNoSlot = 0xFFFF;

static_assert(kSzMaskWords >= kSchurMaxCams, "the camera scan reuses the mask words");
static_assert(kSzMaskWords * 2 >= kSzParts, "the list-slot owners (16-bit) reuse the mask words");
static_assert(kSzWarps * kSzSegCap >= kSzChunk, "the point-list starts reuse the run buffers");
static_assert(kSzParts <= 65536 && kSzChunk <= 65536, "run entries pack a list slot and an observation in 16 bits each");
static_assert(kSchurMaxCams < kNoSlot, "slot ids are 16-bit");

struct SzShared {
    int* off;             // [kSzChunk + 1] partner-entry offsets of the chunk's observations
    int* own;             // [kSzChunk] the chunk's observations (owner side)
    int* part_o;          // [kSzParts] partner observations
    unsigned short* part_c;  // [kSzParts] partner cameras
    unsigned* mask;       // [kSzMaskWords] slot x word run masks; camera scan buffer before
    unsigned short* slot_of;      // [C] slot of a camera, kNoSlot when none
    unsigned short* cam_of_slot;  // [C]
    int* tmp;             // [kSzWarps + 4] scan scratch and broadcast words
    unsigned* runbuf;     // [kSzWarps][kSzSegCap] staged run entries, one buffer per warp
    int* sb;              // [kSzChunk] start of each observation's point list (aliases runbuf)
    unsigned short* seg;  // [kSzParts] observation of each list slot (aliases mask)
};

__device__ __forceinline__ SzShared sz_layout(char* base, int C) {
    SzShared s;
    s.mask = reinterpret_cast<unsigned*>(base);
    s.off = reinterpret_cast<int*>(s.mask + kSzMaskWords);
    s.own = s.off + kSzChunk + 1;
    s.part_o = s.own + kSzChunk;
    s.tmp = s.part_o + kSzParts;
    s.runbuf = reinterpret_cast<unsigned*>(s.tmp + kSzWarps + 4);
    s.sb = reinterpret_cast<int*>(s.runbuf);
    s.seg = reinterpret_cast<unsigned short*>(s.mask);
    s.part_c = reinterpret_cast<unsigned short*>(s.runbuf + kSzWarps * kSzSegCap);
    s.slot_of = s.part_c + kSzParts;
    s.cam_of_slot = s.slot_of + C;
    return s;
}

// In-place exclusive scan of a[0, n) over the block; returns the total.
__device__ int sz_scan(int* a, int n, int* tmp) {
    const int per = (n + kSzThreads - 1) / kSzThreads;
    const int b = min(n, (int)threadIdx.x * per), e = min(n, b + per);
    int s = 0;
    for (int i = b; i < e; ++i) s += a[i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = s;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) tmp[w] = x;
    __syncthreads();
    if (w == 0) {
        int v = lane < kSzWarps ? tmp[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v += y;
        }
        if (lane < kSzWarps) tmp[lane] = v;
    }
    __syncthreads();
    int base = (w ? tmp[w - 1] : 0) + x - s;
    for (int i = b; i < e; ++i) {
        const int v = a[i];
        a[i] = base;
        base += v;
    }
    const int total = tmp[kSzWarps - 1];
    __syncthreads();
    return total;
}

// One block, ten terms per step: lanes 3g .. 3g+2 (g = 0..9) take the g-th
// term of the step, lane band r3 = lane % 3 owns rows 3 r3 .. 3 r3 + 2 of the
// 9 x 9 block and all nine columns. A lane loads its three rows of both
// records (P = Y_o, partner; O = W_o', owner) and receives the other two
// bands of O from its group's lanes by shuffles; its columns are kept in
// rotated band order (band (r3 + k) mod 3 in slot k), so the accumulator
// indices are compile-time. The run (the observations marked for this slot,
// in index order, each with its partner entry) is staged in a per-warp
// buffer, segment by segment; the records of the next step are loaded while
// the current one is summed. The ten partial sums are added in a fixed tree
// order (g + 1, g + 2, g + 4, g + 8). Warp-level.
__device__ void sz_block10(const SzShared& sh, unsigned* buf, int s, int ca, int cb, int W, int u, bool store,
                           const double* __restrict__ Ws, const double* __restrict__ Ys,
                           const double* __restrict__ U, double* Z, long ldz) {
    const int lane = threadIdx.x & 31;
    const int g = lane / 3;          // term group 0..9 (10: lanes 30, 31, idle)
    const int r3 = lane - 3 * g;     // row band
    const bool act = g < kSzGroups;
    const unsigned* mk = sh.mask + (size_t)s * W;
    double acc[3][3][3];  // [row a][band slot k][row of the band bb]
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int b = 0; b < 3; ++b) acc[a][k][b] = 0.0;
    auto fetch = [&](int e, int nseg, double (&p)[9], double (&q)[9]) {
        unsigned v = 0xFFFFFFFFu;
        if (act && e < nseg) v = buf[e];
        const bool ok = v != 0xFFFFFFFFu;
        const int o = ok ? sh.part_o[v & 0xFFFFu] : 0, o2 = ok ? sh.own[v >> 16] : 0;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            p[k] = ok ? __ldg(Ys + 27L * o + 9 * r3 + k) : 0.0;
            q[k] = ok ? __ldg(Ws + 27L * o2 + 9 * r3 + k) : 0.0;
        }
    };
    auto sum_step = [&](const double (&p)[9], const double (&q)[9]) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double ob[9];
            const int src = 3 * g + (r3 + k) % 3;
#pragma unroll
            for (int i = 0; i < 9; ++i) ob[i] = k == 0 ? q[i] : __shfl_sync(0xffffffffu, q[i], src);
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    double v = acc[a][k][b];
                    v = fma(p[3 * a + 0], ob[3 * b + 0], v);
                    v = fma(p[3 * a + 1], ob[3 * b + 1], v);
                    v = fma(p[3 * a + 2], ob[3 * b + 2], v);
                    acc[a][k][b] = v;
                }
        }
    };
    for (int wi = 0; wi < W;) {
        // stage a segment of the run: the marked observations j in order (32
        // mask words per step, a prefix scan of their bit counts gives every
        // lane its place), then each entry's partner list slot t, one entry
        // per lane; entry = t | j << 16
        int nseg = 0;
        while (wi < W && nseg <= kSzSegCap - 32) {
            const int nw = min(32, W - wi);
            const unsigned word = lane < nw ? mk[wi + lane] : 0u;
            const int c = __popc(word);
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += y;
            }
            // whole words that fit (a prefix of the lanes: incl grows with the lane)
            const int take = __popc(__ballot_sync(0xffffffffu, lane < nw && nseg + incl <= kSzSegCap));
            if (lane < take) {
                int pos = nseg + incl - c;
                for (unsigned bb = word; bb; bb &= bb - 1u) buf[pos++] = 32u * (unsigned)(wi + lane) + (__ffs(bb) - 1);
            }
            nseg += __shfl_sync(0xffffffffu, incl, take - 1);
            wi += take;
        }
        __syncwarp();
        for (int e = lane; e < nseg; e += 32) {
            const int j = (int)buf[e];
            const int t1 = sh.off[j + 1];
            int t = sh.off[j], c = 0;
            for (; t < t1; ++t)
                if (sh.part_c[t] == ca && c++ == u) break;
            buf[e] = t < t1 ? ((unsigned)t | ((unsigned)j << 16)) : 0xFFFFFFFFu;
        }
        __syncwarp();
        double pa[9], qa[9], pb[9], qb[9];
        fetch(g, nseg, pa, qa);
        for (int base = 0; base < nseg; base += 2 * kSzGroups) {
            fetch(base + kSzGroups + g, nseg, pb, qb);
            sum_step(pa, qa);
            fetch(base + 2 * kSzGroups + g, nseg, pa, qa);
            if (base + kSzGroups < nseg) sum_step(pb, qb);
        }
        __syncwarp();  // the buffer is refilled next
    }
    // the ten partial sums into group 0, in a fixed tree order
#pragma unroll
    for (int d = 1; d < 16; d <<= 1) {
        const bool take = (g % (2 * d)) == 0 && g + d < kSzGroups;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const double v = __shfl_sync(0xffffffffu, acc[a][k][b], lane + 3 * d);
                    if (take) acc[a][k][b] += v;
                }
    }
    if (g != 0) return;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int r = 3 * r3 + a, q = 3 * ((r3 + k) % 3) + b;
                const double t = acc[a][k][b];
                if (ca < cb) {
                    const long row = 9L * ca + r, col = 9L * cb + q;
                    double* up = Z + row + col * ldz;
                    const double v = store ? -t : *up - t;
                    *up = v;
                    Z[col + row * ldz] = v;
                } else if (r <= q) {  // the diagonal block: U minus the terms, kept symmetric
                    const long row = 9L * cb + r, col = 9L * cb + q;
                    double* up = Z + row + col * ldz;
                    const double v = (store ? U[81L * cb + r + 9 * q] : *up) - t;
                    *up = v;
                    Z[col + row * ldz] = v;
                }
            }
}

// The terms of the partners of rank u (their camera's (u+1)-th observation of
// the point in the owner observation's list) into the run masks; true when
// some partner has a higher rank (another pass is needed). Block-level.
__device__ bool sz_masks(const SzShared& sh, int cb, int len, int K, int W, int u) {
    for (int k = threadIdx.x; k < K * W; k += kSzThreads) sh.mask[k] = 0u;
    __syncthreads();
    int more = 0;
    for (int j = threadIdx.x; j < len; j += kSzThreads) {
        const int t0 = sh.off[j], t1 = sh.off[j + 1];
        for (int t = t0; t < t1; ++t) {
            const unsigned short c = sh.part_c[t];
            if (c > cb) continue;
            if (u == 0) {  // first occurrences: a second one finds its bit set
                const unsigned bit = 1u << (j & 31);
                const unsigned old = atomicOr(sh.mask + (size_t)sh.slot_of[c] * W + (j >> 5), bit);
                more |= (old & bit) != 0u;
            } else {
                int r = 0;
                for (int q = t0; q < t; ++q) r += sh.part_c[q] == c;
                if (r == u) atomicOr(sh.mask + (size_t)sh.slot_of[c] * W + (j >> 5), 1u << (j & 31));
                more |= r > u;
            }
        }
    }
    return __syncthreads_or(more) != 0;
}

__global__ void __launch_bounds__(kSzThreads, 1)
    k_schur_columns(int C, const int* __restrict__ cam_ptr, const int* __restrict__ cam_obs,
                    const int* __restrict__ obs_pt, const int* __restrict__ pt_ptr, const int* __restrict__ pt_obs,
                    const int* __restrict__ obs_cam, const double* __restrict__ Ws, const double* __restrict__ Ys,
                    const double* __restrict__ U, double* Z, long ldz, int* err) {
    extern __shared__ __align__(16) char sz_smem[];
    const SzShared sh = sz_layout(sz_smem, C);
    const int cb = C - 1 - (int)blockIdx.x;  // the most partners (cameras <= cb) first
    const int base = cam_ptr[cb], n = cam_ptr[cb + 1] - base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (n == 0) {  // no observations: the diagonal block is U alone
        if (tid < 81) Z[9L * cb + tid % 9 + (9L * cb + tid / 9) * ldz] = U[81L * cb + tid];
        return;
    }
    for (int c = tid; c <= cb; c += kSzThreads) sh.slot_of[c] = kNoSlot;
    __syncthreads();
    for (int j0 = 0; j0 < n;) {
        const int jn = min(n, j0 + kSzChunk) - j0;
        // the chunk's observations and the observation lists of their points
        // (four observations per thread in flight: each step is a dependent load)
        for (int j = tid; j < jn; j += 4 * kSzThreads) {
            int o[4], p[4], pb[4], pe[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) o[q] = j + q * kSzThreads < jn ? cam_obs[base + j0 + j + q * kSzThreads] : -1;
#pragma unroll
            for (int q = 0; q < 4; ++q) p[q] = o[q] >= 0 ? obs_pt[o[q]] : 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                pb[q] = o[q] >= 0 ? pt_ptr[p[q]] : 0;
                pe[q] = o[q] >= 0 ? pt_ptr[p[q] + 1] : 0;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (o[q] >= 0) {
                    sh.own[j + q * kSzThreads] = o[q];
                    sh.sb[j + q * kSzThreads] = pb[q];
                    sh.off[j + q * kSzThreads] = pe[q] - pb[q];
                }
        }
        __syncthreads();
        const int total = sz_scan(sh.off, jn, sh.tmp);
        if (tid == 0) {
            sh.off[jn] = total;
            int lo = 0, hi = jn;  // the longest prefix whose lists fit
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sh.off[mid] <= kSzParts) lo = mid; else hi = mid - 1;
            }
            sh.tmp[kSzWarps] = lo;
        }
        __syncthreads();
        int len = sh.tmp[kSzWarps];
        if (len == 0) {  // one point with more observations than the list holds
            if (tid == 0) atomicOr(err, ERRBIT_SCHUR_CAP);
            return;
        }
        // every list slot: its observation (then its partner and camera, in parallel)
        for (int j = tid; j < len; j += kSzThreads)
            for (int i = sh.off[j]; i < sh.off[j + 1]; ++i) sh.seg[i] = (unsigned short)j;
        __syncthreads();
        const int E = sh.off[len];
        for (int i = tid; i < E; i += 8 * kSzThreads) {  // eight list slots per thread in flight
            int o[8], c[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = i + q * kSzThreads;
                int j = 0;
                if (k < E) j = sh.seg[k];
                o[q] = k < E ? pt_obs[sh.sb[j] + (k - sh.off[j])] : 0;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) c[q] = i + q * kSzThreads < E ? obs_cam[o[q]] : 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = i + q * kSzThreads;
                if (k < E) {
                    sh.part_o[k] = o[q];
                    sh.part_c[k] = (unsigned short)c[q];
                    if (c[q] <= cb) sh.slot_of[c[q]] = 0;
                }
            }
        }
        __syncthreads();
        int K = 0, W = 0;
        for (;;) {
            int* scan = reinterpret_cast<int*>(sh.mask);
            for (int c = tid; c <= cb; c += kSzThreads) scan[c] = sh.slot_of[c] != kNoSlot;
            __syncthreads();
            K = sz_scan(scan, cb + 1, sh.tmp);
            W = (len + 31) >> 5;
            if (K * W <= kSzMaskWords) break;
            // too many slots for the masks: the first half of the chunk, its cameras again
            for (int c = tid; c <= cb; c += kSzThreads) sh.slot_of[c] = kNoSlot;
            len = (len + 1) >> 1;
            __syncthreads();
            for (int i = tid; i < sh.off[len]; i += kSzThreads)
                if (sh.part_c[i] <= cb) sh.slot_of[sh.part_c[i]] = 0;
            __syncthreads();
        }
        {
            const int* scan = reinterpret_cast<const int*>(sh.mask);
            for (int c = tid; c <= cb; c += kSzThreads)
                if (sh.slot_of[c] != kNoSlot) {
                    const int s = scan[c];
                    sh.slot_of[c] = (unsigned short)s;
                    sh.cam_of_slot[s] = (unsigned short)c;
                }
        }
        __syncthreads();
        for (int u = 0;; ++u) {
            const bool more = sz_masks(sh, cb, len, K, W, u);
            if (tid == 0) sh.tmp[kSzWarps + 1] = 0;  // slot cursor: warps take slots as they finish
            __syncthreads();
            for (;;) {
                int s = 0;
                if (lane == 0) s = atomicAdd(sh.tmp + kSzWarps + 1, 1);
                s = __shfl_sync(0xffffffffu, s, 0);
                if (s >= K) break;
                sz_block10(sh, sh.runbuf + warp * kSzSegCap, s, sh.cam_of_slot[s], cb, W, u, j0 == 0 && u == 0,
                           Ws, Ys, U, Z, ldz);
            }
            __syncthreads();
            if (!more) break;
        }
        for (int s = tid; s < K; s += kSzThreads) sh.slot_of[sh.cam_of_slot[s]] = kNoSlot;
        __syncthreads();
        j0 += len;
    }
}

}  // namespace

size_t schur_columns_smem(int C) {
    return (size_t)kSzMaskWords * 4 + (size_t)(kSzChunk + 1) * 4 + (size_t)kSzChunk * 4 + (size_t)kSzParts * 4 +
           (size_t)(kSzWarps + 4) * 4 + (size_t)kSzWarps * kSzSegCap * 4 + (size_t)kSzParts * 2 +
           2 * (size_t)C * 2 + 16;
}

void prepare_schur_columns() {
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_schur_columns, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)schur_columns_smem(kSchurMaxCams)) == cudaSuccess;
    });
}

int launch_schur_columns(const SceneDev& s, double* Z, int ldz, cudaStream_t st) {
    const int C = s.num_cams;
    if (C == 0) return UNC_OK;
    if (C > kSchurMaxCams) return UNC_ERR_TOO_LARGE;
    const size_t smem = schur_columns_smem(C);
    prepare_schur_columns();
    k_schur_columns<<<C, kSzThreads, smem, st>>>(C, s.cam_ptr, s.cam_obs, s.obs_pt, s.pt_ptr, s.pt_obs, s.obs_cam,
                                                 s.Ws, s.Ys, s.Ucam, Z, ldz, s.err);
    count_launch();
    return UNC_OK;
}

}  // namespace unc
