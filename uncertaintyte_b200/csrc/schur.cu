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
//     and later chunks). The self terms Y_o' W_o'^T of the diagonal block (one
//     per observation of cb, as many as all other terms of a typical block
//     together) are summed first by all warps over contiguous ranges and added
//     in warp order.
// Scenes with few cameras split every column over several CTAs (camera ca's
// block to CTA (cb - ca) mod parts, in every chunk), so that the grid covers
// the SMs.
// No floating-point atomics, no device-to-host round trip: the result is
// bitwise repeatable and the stage can be captured in a graph. A camera that
// observes a point more than once gives more than one term per (slot,
// observation); those extra terms are added by further passes.
#include "internal.h"

namespace unc {
namespace {

constexpr int kSzThreads = 256;       // 8 warps (registers for three steps of records in flight)
constexpr int kSzWarps = kSzThreads / 32;
constexpr int kSzChunk = 2048;        // owner observations per chunk, at most
constexpr int kSzParts = 12288;       // partner list slots per chunk, at most
constexpr int kSzMaskWords = 11776;   // run-mask words (also the list-slot owners and the camera scan)
constexpr int kSzGroups = 10;         // terms per step of sz_block10 (three lanes each)
constexpr int kSzSegCap = 512;        // run entries staged per warp at a time
constexpr unsigned short kNoSlot = 0xFFFF;
constexpr unsigned short kSelf = 0xFFFE;  // list-slot camera of the owner observation itself

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
    double* self;         // [81] the chunk's self terms of the diagonal block (column-major)
    double* red;          // [kSzWarps][81 + 81 * kSzGroups] per-warp block sums and group partials
    unsigned* runbuf;     // [kSzWarps][kSzSegCap] staged run entries, one buffer per warp
    int* sb;              // [kSzChunk] start of each observation's point list (aliases runbuf)
    unsigned short* seg;  // [kSzParts] observation of each list slot (aliases mask)
};

// Shared-memory layout (byte offsets; every array starts 16-byte aligned).
struct SzOffsets {
    size_t mask, off, own, part_o, tmp, self, red, runbuf, part_c, slot_of, cam_of_slot, total;
};
__host__ __device__ constexpr size_t sz_align(size_t x) { return (x + 15) & ~size_t(15); }
__host__ __device__ inline SzOffsets sz_offsets(int C) {
    SzOffsets o{};
    o.mask = 0;
    o.off = sz_align(o.mask + sizeof(unsigned) * kSzMaskWords);
    o.own = sz_align(o.off + sizeof(int) * (kSzChunk + 1));
    o.part_o = sz_align(o.own + sizeof(int) * kSzChunk);
    o.tmp = sz_align(o.part_o + sizeof(int) * kSzParts);
    o.self = sz_align(o.tmp + sizeof(int) * (kSzWarps + 4));
    o.red = sz_align(o.self + sizeof(double) * 81);
    o.runbuf = sz_align(o.red + sizeof(double) * kSzWarps * 81 * (1 + kSzGroups));
    o.part_c = sz_align(o.runbuf + sizeof(unsigned) * kSzWarps * kSzSegCap);
    o.slot_of = sz_align(o.part_c + sizeof(unsigned short) * kSzParts);
    o.cam_of_slot = sz_align(o.slot_of + sizeof(unsigned short) * (size_t)C);
    o.total = sz_align(o.cam_of_slot + sizeof(unsigned short) * (size_t)C);
    return o;
}

__device__ __forceinline__ SzShared sz_layout(char* base, int C) {
    const SzOffsets o = sz_offsets(C);
    SzShared s;
    s.mask = reinterpret_cast<unsigned*>(base + o.mask);
    s.off = reinterpret_cast<int*>(base + o.off);
    s.own = reinterpret_cast<int*>(base + o.own);
    s.part_o = reinterpret_cast<int*>(base + o.part_o);
    s.tmp = reinterpret_cast<int*>(base + o.tmp);
    s.self = reinterpret_cast<double*>(base + o.self);
    s.red = reinterpret_cast<double*>(base + o.red);
    s.runbuf = reinterpret_cast<unsigned*>(base + o.runbuf);
    s.part_c = reinterpret_cast<unsigned short*>(base + o.part_c);
    s.slot_of = reinterpret_cast<unsigned short*>(base + o.slot_of);
    s.cam_of_slot = reinterpret_cast<unsigned short*>(base + o.cam_of_slot);
    s.sb = reinterpret_cast<int*>(s.runbuf);
    s.seg = reinterpret_cast<unsigned short*>(s.mask);
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

// Ten terms per step: lanes 3g .. 3g+2 (g = 0..9) take the g-th term of a
// step, lane band r3 = lane % 3 owns rows 3 r3 .. 3 r3 + 2 of the 9 x 9 block
// and all nine columns. A lane loads its three rows of both records (P = Y_o,
// partner; O = W_o', owner) and receives the other two bands of O from its
// group's lanes by shuffles; its columns are kept in rotated band order (band
// (r3 + k) mod 3 in slot k), so the accumulator indices are compile-time. The
// records of the next two steps are in flight while a step is summed.
struct SzSteps {
    int lane, g, r3;
    bool act;
    double acc[3][3][3];  // [row a][band slot k][row of the band bb]

    __device__ explicit SzSteps(int lane_) : lane(lane_), g(lane_ / 3), r3(lane_ - 3 * (lane_ / 3)) {
        act = g < kSzGroups;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int b = 0; b < 3; ++b) acc[a][k][b] = 0.0;
    }
    __device__ void load(int o, int o2, bool ok, const double* __restrict__ Ws, const double* __restrict__ Ys,
                         double (&p)[9], double (&q)[9]) const {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            p[k] = ok ? __ldg(Ys + 27L * o + 9 * r3 + k) : 0.0;
            q[k] = ok ? __ldg(Ws + 27L * o2 + 9 * r3 + k) : 0.0;
        }
    }
    __device__ void sum(const double (&p)[9], const double (&q)[9]) {
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
    }
    // steps over entries 0 .. n-1; fetch(e, p, q) loads entry e (or zeros past n)
    template <class F>
    __device__ void run(int n, F&& fetch) {
        double p0[9], q0[9], p1[9], q1[9], p2[9], q2[9];
        fetch(g, p0, q0);
        fetch(kSzGroups + g, p1, q1);
        for (int base = 0; base < n; base += 3 * kSzGroups) {
            fetch(base + 2 * kSzGroups + g, p2, q2);
            sum(p0, q0);
            if (base + kSzGroups >= n) break;
            fetch(base + 3 * kSzGroups + g, p0, q0);
            sum(p1, q1);
            if (base + 2 * kSzGroups >= n) break;
            fetch(base + 4 * kSzGroups + g, p1, q1);
            sum(p2, q2);
        }
    }
    // the ten partial blocks added in group order into red[0..80] (column-major
    // element r + 9 q), through the warp's buffer red[81 .. 81 + 810)
    __device__ void reduce(double* red) const {
        double* part = red + 81;
        if (act) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int b = 0; b < 3; ++b)
                        part[81 * g + (3 * r3 + a) + 9 * (3 * ((r3 + k) % 3) + b)] = acc[a][k][b];
        }
        __syncwarp();
        for (int e = lane; e < 81; e += 32) {
            double v = part[e];
#pragma unroll
            for (int q = 1; q < kSzGroups; ++q) v += part[81 * q + e];
            red[e] = v;
        }
        __syncwarp();
    }
};

// One block: the terms of slot s (camera ca <= cb) over the chunk, pass u (the
// (u+1)-th partner of camera ca of each marked observation), then the block
// stored in both triangles (the diagonal: U minus the terms and the self
// terms). The run is staged in the warp's buffer segment by segment.
// Warp-level.
__device__ void sz_block10(const SzShared& sh, unsigned* buf, double* red, int s, int ca, int cb, int W, int u,
                           bool store, const double* __restrict__ Ws, const double* __restrict__ Ys,
                           const double* __restrict__ U, double* Z, long ldz) {
    const int lane = threadIdx.x & 31;
    const unsigned* mk = sh.mask + (size_t)s * W;
    SzSteps st(lane);
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
        st.run(nseg, [&](int e, double (&p)[9], double (&q)[9]) {
            unsigned v = 0xFFFFFFFFu;
            if (st.act && e < nseg) v = buf[e];
            const bool ok = v != 0xFFFFFFFFu;
            st.load(ok ? sh.part_o[v & 0xFFFFu] : 0, ok ? sh.own[v >> 16] : 0, ok, Ws, Ys, p, q);
        });
        __syncwarp();  // the buffer is refilled next
    }
    st.reduce(red);
    for (int e = lane; e < 81; e += 32) {
        const int r = e % 9, q = e / 9;
        const double t = ca == cb && u == 0 ? red[e] + sh.self[e] : red[e];
        if (ca < cb) {
            const long row = 9L * ca + r, col = 9L * cb + q;
            double* up = Z + row + col * ldz;
            const double v = store ? -t : *up - t;
            *up = v;
            Z[col + row * ldz] = v;
        } else if (r <= q) {  // the diagonal block: U minus the terms, kept symmetric
            const long row = 9L * cb + r, col = 9L * cb + q;
            double* up = Z + row + col * ldz;
            const double v = (store ? U[81L * cb + e] : *up) - t;
            *up = v;
            Z[col + row * ldz] = v;
        }
    }
    __syncwarp();  // red is reused by the next block
}

// The self terms sum_o' Y_o' W_o'^T of the chunk's observations into sh.self:
// warp w sums observations [w len / warps, (w+1) len / warps) ten per step,
// its partial goes to scratch[w] (81 doubles), and the partials are added in
// warp order. Block-level.
__device__ void sz_self(const SzShared& sh, int len, double* scratch, double* red, const double* __restrict__ Ws,
                        const double* __restrict__ Ys) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j0 = (int)((long)warp * len / kSzWarps), j1 = (int)((long)(warp + 1) * len / kSzWarps);
    SzSteps st(lane);
    st.run(j1 - j0, [&](int e, double (&p)[9], double (&q)[9]) {
        const bool ok = st.act && e < j1 - j0;
        const int o = ok ? sh.own[j0 + e] : 0;
        st.load(o, o, ok, Ws, Ys, p, q);
    });
    st.reduce(red);
    for (int e = lane; e < 81; e += 32) scratch[81 * warp + e] = red[e];
    __syncthreads();
    if (threadIdx.x < 81) {
        double v = scratch[threadIdx.x];
        for (int w = 1; w < kSzWarps; ++w) v += scratch[81 * w + threadIdx.x];
        sh.self[threadIdx.x] = v;
    }
    __syncthreads();
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
                    const double* __restrict__ U, double* Z, long ldz, int* err, int parts) {
    extern __shared__ __align__(16) char sz_smem[];
    const SzShared sh = sz_layout(sz_smem, C);
    const int cb = C - 1 - (int)(blockIdx.x / parts);  // the most partners (cameras <= cb) first
    const int part = (int)(blockIdx.x % parts);        // this CTA's share of the column's slots
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
                    const bool self = o[q] == sh.own[sh.seg[k]];
                    sh.part_o[k] = o[q];
                    sh.part_c[k] = self ? kSelf : (unsigned short)c[q];
                    if (!self && c[q] <= cb) sh.slot_of[c[q]] = 0;
                }
            }
        }
        if (tid == 0) sh.slot_of[cb] = 0;  // the diagonal block always has a slot (its self terms)
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
            if (tid == 0) sh.slot_of[cb] = 0;
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
        if (part == 0)  // before the masks (its scratch is their words)
            sz_self(sh, len, reinterpret_cast<double*>(sh.mask), sh.red + warp * 81 * (1 + kSzGroups), Ws, Ys);
        for (int u = 0;; ++u) {
            const bool more = sz_masks(sh, cb, len, K, W, u);
            if (tid == 0) sh.tmp[kSzWarps + 1] = 0;  // slot cursor: warps take slots as they finish
            __syncthreads();
            for (;;) {  // this CTA's blocks: cameras ca with (cb - ca) mod parts == part, the same in
                        // every chunk (slot numbers are not), so no block is updated by two CTAs
                int q = 0;
                if (lane == 0) q = atomicAdd(sh.tmp + kSzWarps + 1, 1);
                q = __shfl_sync(0xffffffffu, q, 0);
                const int s = K - 1 - q;
                if (s < 0) break;
                if ((cb - sh.cam_of_slot[s]) % parts != part) continue;
                sz_block10(sh, sh.runbuf + warp * kSzSegCap, sh.red + warp * 81 * (1 + kSzGroups), s,
                           sh.cam_of_slot[s], cb, W, u, j0 == 0 && u == 0,
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

size_t schur_columns_smem(int C) { return sz_offsets(C).total; }

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
    // few cameras: split every column so that the grid covers about two waves of SMs
    const int parts = std::max(1, std::min(8, (2 * device_sms() + C - 1) / C));
    k_schur_columns<<<C * parts, kSzThreads, smem, st>>>(C, s.cam_ptr, s.cam_obs, s.obs_pt, s.pt_ptr, s.pt_obs, s.obs_cam,
                                                 s.Ws, s.Ys, s.Ucam, Z, ldz, s.err, parts);
    count_launch();
    return UNC_OK;
}

}  // namespace unc
