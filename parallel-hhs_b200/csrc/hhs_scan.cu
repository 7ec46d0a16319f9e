// hhs_scan.cu -- standalone exact exclusive scan and the fast/slow index split.
#include <atomic>
#include <cstdlib>
#include <cstring>

#include "hhs_scan.cuh"
#include "hhs_kernels.h"
#include "hhs_tma.cuh"

namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 16;  // 4096 values (16 KiB) per tile
using ScanT = TileScan<kScanBlock, kScanItems, 1>;
// workspace sizes are quoted for the smallest tile any scan launch shape uses
constexpr int kScanMinTile = 2048;

// Exclusive scan of int32 values. VEC: 16-byte aligned input/output, so full chunks
// move with one 128-bit streaming load/store per lane.
// SELF_RESET: the last CTA resets the workspace header for the next call (used where the
// workspace is reused without a memset); the standalone calls memset it instead.
template <bool VEC, bool SELF_RESET>
__global__ void __launch_bounds__(kScanBlock, 6)
    k_scan_exclusive_i32(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                         long long n, ScanHeader* hdr, unsigned long long* status,
                         int num_tiles) {
    __shared__ int s_tile;
    __shared__ unsigned s_epoch, s_prefix, s_limit;
    __shared__ unsigned s_warp[ScanT::WARPS];
    __shared__ int s_last;
    scan_begin(hdr, &s_tile, &s_epoch, &s_limit);
    const int tile = s_tile;
    const unsigned epoch = s_epoch;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long tbase = (long long)tile * ScanT::TILE;

    unsigned v[kScanItems], cb[ScanT::CHUNKS];
#pragma unroll
    for (int c = 0; c < ScanT::CHUNKS; c++) {
        const long long e = tbase + ScanT::offset(warp, c, lane);
        if (VEC && e + 4 <= n) {
            const int4 q = __ldcs(reinterpret_cast<const int4*>(in + e));
            v[4 * c] = q.x; v[4 * c + 1] = q.y; v[4 * c + 2] = q.z; v[4 * c + 3] = q.w;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) v[4 * c + k] = (e + k < n) ? (unsigned)in[e + k] : 0u;
        }
    }
    ScanT::scan(v, cb, status, tile, epoch, &hdr->error, s_warp, &s_prefix, s_limit);
#pragma unroll
    for (int c = 0; c < ScanT::CHUNKS; c++) {
        const long long e = tbase + ScanT::offset(warp, c, lane);
        const unsigned p0 = cb[c], p1 = p0 + v[4 * c], p2 = p1 + v[4 * c + 1],
                       p3 = p2 + v[4 * c + 2];
        if (VEC && e + 4 <= n) {
            __stcs(reinterpret_cast<int4*>(out + e), make_int4((int)p0, (int)p1, (int)p2, (int)p3));
        } else {
            const unsigned pp[4] = {p0, p1, p2, p3};
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (e + k < n) out[e + k] = (int)pp[k];
        }
    }
    if (SELF_RESET && scan_finish_is_last(hdr, num_tiles, &s_last)) scan_reset(hdr, epoch);
}

// Large inputs (n >= 2^22). The single pass is held back by how fast the inclusive
// prefixes propagate through hundreds of resident tiles, so large inputs are scanned in
// two steps over contiguous chunks of whole tiles, one chunk per CTA: sum the chunk,
// then scan it from the sum of the chunks before it.
//  - Two-kernel form: a chunk-sum kernel and a chunk-scan kernel over the whole input,
//    12 bytes of DRAM traffic per value. The default for the scan from 2^22 values up to
//    the streamed pass below (4.25 TB/s at 2^28, where the streamed pass reaches 5.0), and
//    for unaligned inputs.
//  - Wave form: one cooperative launch walks the input in waves of 2^24 values (64 MB,
//    half of L2). Per wave every CTA sums its chunk, the grid meets at a counting
//    barrier, and every CTA scans its chunk while most of it is still in L2. Each CTA
//    adds up all of the wave's chunk sums itself, so the running total passes from wave
//    to wave without another barrier. The default for stream compaction of n >= 2^24
//    (3.27 against 2.88 TB/s at 2^28); for the scan it measured no faster (4.15 TB/s),
//    and below 2^24 the cooperative launch and the header clear cost more than the
//    re-read saves. Launch-shape variants 11-13 run the scan in waves of 2^22, 2^23 and
//    2^24 values.
constexpr int kChunkCtasPerSm = 4;
constexpr long long kTwoPassMinN = 1LL << 22;
constexpr long long kWaveValues = 1LL << 24;  // 64 MB of int32 per wave
constexpr long long kWaveMinN = 1LL << 24;    // compaction: the wave form from here on
constexpr unsigned long long kWaveBarrierTimeoutNs = 10ull * 1000000000ull;

// Block-wide sum of in[b, e) (FLAGS: the number of nonzero values), returned to every
// thread. b is a multiple of 4.
template <bool VEC, bool FLAGS>
__device__ unsigned block_chunk_sum(const int32_t* __restrict__ in, long long b, long long e,
                                    unsigned* s_red) {
    unsigned a0 = 0u, a1 = 0u, a2 = 0u, a3 = 0u;
    if (VEC) {
        // four 16-byte loads in flight per thread
        const long long nv = (e - b) / 4;
        const int4* v = reinterpret_cast<const int4*>(in + b);
        auto add = [&](const int4 q) {
            if (FLAGS) {
                a0 += q.x != 0; a1 += q.y != 0; a2 += q.z != 0; a3 += q.w != 0;
            } else {
                a0 += (unsigned)q.x; a1 += (unsigned)q.y; a2 += (unsigned)q.z; a3 += (unsigned)q.w;
            }
        };
        long long k = threadIdx.x;
        for (; k + 3 * kScanBlock < nv; k += 4 * kScanBlock) {
            const int4 q0 = __ldg(v + k), q1 = __ldg(v + k + kScanBlock),
                       q2 = __ldg(v + k + 2 * kScanBlock), q3 = __ldg(v + k + 3 * kScanBlock);
            add(q0); add(q1); add(q2); add(q3);
        }
        for (; k < nv; k += kScanBlock) add(__ldg(v + k));
        for (long long t = b + nv * 4 + threadIdx.x; t < e; t += kScanBlock)
            a0 += FLAGS ? (unsigned)(in[t] != 0) : (unsigned)in[t];
    } else {
        for (long long t = b + threadIdx.x; t < e; t += kScanBlock)
            a0 += FLAGS ? (unsigned)(in[t] != 0) : (unsigned)in[t];
    }
    const unsigned t = (unsigned)warp_sum((int)(a0 + a1 + a2 + a3));
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = t;
    __syncthreads();
    unsigned sum = 0u;
#pragma unroll
    for (int w = 0; w < kScanBlock / 32; w++) sum += s_red[w];
    __syncthreads();  // s_red may be reused
    return sum;
}

// Scans in[b, e) tile by tile starting from `offset` and returns the running total at e.
// out may be null with FLAGS; FLAGS: idx_out[scan] = index of each nonzero value.
template <bool VEC, bool FLAGS>
__device__ unsigned block_chunk_scan(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                                     long long b, long long e, unsigned offset,
                                     int32_t* __restrict__ idx_out, unsigned* s_warp,
                                     unsigned* s_total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long tbase = b; tbase < e; tbase += ScanT::TILE) {
        unsigned v[kScanItems], cbase[ScanT::CHUNKS];
#pragma unroll
        for (int c = 0; c < ScanT::CHUNKS; c++) {
            const long long el = tbase + ScanT::offset(warp, c, lane);
            if (VEC && el + 4 <= e) {
                const int4 q = __ldcs(reinterpret_cast<const int4*>(in + el));
                v[4 * c] = q.x; v[4 * c + 1] = q.y; v[4 * c + 2] = q.z; v[4 * c + 3] = q.w;
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) v[4 * c + k] = (el + k < e) ? (unsigned)in[el + k] : 0u;
            }
            if (FLAGS) {
#pragma unroll
                for (int k = 0; k < 4; k++) v[4 * c + k] = v[4 * c + k] != 0u;
            }
        }
        unsigned run = 0u;
#pragma unroll
        for (int c = 0; c < ScanT::CHUNKS; c++) {
            const unsigned sc = v[4 * c] + v[4 * c + 1] + v[4 * c + 2] + v[4 * c + 3];
            const unsigned inc = (unsigned)warp_incl_scan((int)sc, lane);
            cbase[c] = run + inc - sc;
            run += (unsigned)__shfl_sync(HHS_FULL_MASK, (int)inc, 31);
        }
        if (lane == 0) s_warp[warp] = run;
        __syncthreads();
        if (warp == 0) {
            const unsigned wt = lane < ScanT::WARPS ? s_warp[lane] : 0u;
            const unsigned wi = (unsigned)warp_incl_scan((int)wt, lane);
            if (lane < ScanT::WARPS) s_warp[lane] = wi - wt;
            if (lane == 31) *s_total = wi;
        }
        __syncthreads();
        const unsigned wbase = offset + s_warp[warp];
#pragma unroll
        for (int c = 0; c < ScanT::CHUNKS; c++) {
            const long long el = tbase + ScanT::offset(warp, c, lane);
            const unsigned p0 = wbase + cbase[c], p1 = p0 + v[4 * c], p2 = p1 + v[4 * c + 1],
                           p3 = p2 + v[4 * c + 2];
            if (!FLAGS || out) {
                if (VEC && el + 4 <= e) {
                    __stcs(reinterpret_cast<int4*>(out + el),
                           make_int4((int)p0, (int)p1, (int)p2, (int)p3));
                } else {
                    const unsigned pp[4] = {p0, p1, p2, p3};
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (el + k < e) out[el + k] = (int)pp[k];
                }
            }
            if (FLAGS) {
                const unsigned pp[4] = {p0, p1, p2, p3};
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (v[4 * c + k]) idx_out[pp[k]] = (int)(el + k);
            }
        }
        offset += *s_total;
        __syncthreads();
    }
    return offset;
}

// ---- two-kernel form
template <bool VEC, bool FLAGS>
__global__ void __launch_bounds__(kScanBlock)
    k_chunk_reduce(const int32_t* __restrict__ in, long long n, long long chunk,
                   unsigned* __restrict__ agg, unsigned* __restrict__ clear_word) {
    __shared__ unsigned s_red[kScanBlock / 32];
    if (clear_word && blockIdx.x == 0 && threadIdx.x == 0) *clear_word = 0u;
    const long long b = (long long)blockIdx.x * chunk;
    const unsigned sum = block_chunk_sum<VEC, FLAGS>(in, b, min(n, b + chunk), s_red);
    if (threadIdx.x == 0) agg[blockIdx.x] = sum;
}

// the last chunk writes the total to *count (FLAGS)
template <bool VEC, bool FLAGS>
__global__ void __launch_bounds__(kScanBlock)
    k_chunk_scan(const int32_t* __restrict__ in, int32_t* __restrict__ out, long long n,
                 long long chunk, const unsigned* __restrict__ agg,
                 int32_t* __restrict__ idx_out, int32_t* __restrict__ count) {
    __shared__ unsigned s_warp[ScanT::WARPS], s_red[ScanT::WARPS];
    __shared__ unsigned s_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // offset of this chunk: the sum of the chunks before it
    unsigned part = 0u;
    for (int c = threadIdx.x; c < (int)blockIdx.x; c += kScanBlock) part += agg[c];
    part = (unsigned)warp_sum((int)part);
    if (lane == 0) s_red[warp] = part;
    __syncthreads();
    unsigned offset = 0u;
#pragma unroll
    for (int w = 0; w < ScanT::WARPS; w++) offset += s_red[w];
    const long long b = (long long)blockIdx.x * chunk;
    const long long e = min(n, b + chunk);
    offset = block_chunk_scan<VEC, FLAGS>(in, out, b, e, offset, idx_out, s_warp, &s_total);
    if (FLAGS && count && e == n && threadIdx.x == 0) *count = (int)offset;
}

// ---- wave form
// Grid barrier of the wave kernel: arrivals are release reductions on a counter that
// the host clears before the launch; the k-th barrier waits for k x grid arrivals.
// Thread 0 polls with acquire loads and gives up after timeout_ns, or as soon as another
// CTA has recorded an error, recording HHS_ERRBIT_BARRIER_TIMEOUT.
__device__ __forceinline__ bool wave_barrier(unsigned* count, unsigned target, unsigned* err,
                                             unsigned* s_ok, unsigned long long timeout_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned ok = 1u;
        red_add_release_u32(count, 1u);
        unsigned polls = 0;
        unsigned long long t0 = 0;
        while (ld_acquire_u32(count) < target) {
            if (++polls < 128) continue;
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (t0 == 0) t0 = t;
            if (*reinterpret_cast<volatile unsigned*>(err) != 0u) { ok = 0u; break; }
            if (t - t0 > timeout_ns) {
                atomicOr(err, HHS_ERRBIT_BARRIER_TIMEOUT);
                ok = 0u;
                break;
            }
            __nanosleep(64);
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0u;
}

// Cooperative launch, every CTA resident. Wave k covers [k*wave, (k+1)*wave) with
// wave = chunk x gridDim.x; CTA c owns [k*wave + c*chunk, ... + chunk) of it. agg holds
// two sets of gridDim.x chunk sums, used by alternate waves (a CTA can be at most one
// barrier ahead, so it never overwrites a set another CTA is still reading).
// missing: arrivals each barrier waits for beyond the grid's own (0; 1 makes every
// barrier wait for a CTA that does not exist: the failure-detection self-test).
template <bool VEC, bool FLAGS>
__global__ void __launch_bounds__(kScanBlock)
    k_wave_scan(const int32_t* __restrict__ in, int32_t* __restrict__ out, long long n,
                long long chunk, unsigned* __restrict__ agg, ScanHeader* hdr,
                int32_t* __restrict__ idx_out, int32_t* __restrict__ count,
                unsigned missing, unsigned long long timeout_ns) {
    __shared__ unsigned s_warp[ScanT::WARPS], s_red[ScanT::WARPS], s_red2[ScanT::WARPS];
    __shared__ unsigned s_total, s_ok;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long wave = chunk * gridDim.x;
    unsigned carry = 0u;
    int k = 0;
    for (long long wb = 0; wb < n; wb += wave, k++) {
        const long long b = wb + (long long)blockIdx.x * chunk;
        const long long e = min(n, b + chunk);
        unsigned* A = agg + (size_t)(k & 1) * gridDim.x;
        const unsigned sum = b < e ? block_chunk_sum<VEC, FLAGS>(in, b, e, s_red) : 0u;
        if (threadIdx.x == 0) A[blockIdx.x] = sum;
        if (!wave_barrier(&hdr->wave_count, (unsigned)(k + 1) * (gridDim.x + missing),
                          &hdr->error, &s_ok, timeout_ns))
            return;
        // the chunks before this one, and the whole wave (loads that bypass L1: the sets
        // are rewritten every other wave)
        unsigned before = 0u, all = 0u;
        for (int c = threadIdx.x; c < (int)gridDim.x; c += kScanBlock) {
            const unsigned a = __ldcg(A + c);
            all += a;
            if (c < (int)blockIdx.x) before += a;
        }
        before = (unsigned)warp_sum((int)before);
        all = (unsigned)warp_sum((int)all);
        if (lane == 0) { s_red[warp] = before; s_red2[warp] = all; }
        __syncthreads();
        unsigned off = carry;
        unsigned tot = 0u;
#pragma unroll
        for (int w = 0; w < ScanT::WARPS; w++) { off += s_red[w]; tot += s_red2[w]; }
        __syncthreads();
        if (b < e) block_chunk_scan<VEC, FLAGS>(in, out, b, e, off, idx_out, s_warp, &s_total);
        carry += tot;
    }
    if (FLAGS && count && blockIdx.x == 0 && threadIdx.x == 0) *count = (int)carry;
}

// chunks of whole tiles for the two-kernel form; returns the chunk count
int chunk_plan(long long n, long long* chunk) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    const long long tiles = (n + ScanT::TILE - 1) / ScanT::TILE;
    const long long want = (long long)sms * kChunkCtasPerSm;
    const long long per = (tiles + want - 1) / want;
    *chunk = per * ScanT::TILE;
    return (int)((n + *chunk - 1) / *chunk);
}

// The two-kernel form over the whole input. agg: the workspace's status words; the
// header's error word is cleared by the first kernel.
template <bool VEC, bool FLAGS>
void launch_two_pass(const int32_t* in, int32_t* out, long long n, ScanHeader* hdr,
                     unsigned* agg, int32_t* idx_out, int32_t* count, cudaStream_t s) {
    long long chunk = 0;
    const int nc = chunk_plan(n, &chunk);
    k_chunk_reduce<VEC, FLAGS><<<nc, kScanBlock, 0, s>>>(in, n, chunk, agg, &hdr->error);
    k_chunk_scan<VEC, FLAGS><<<nc, kScanBlock, 0, s>>>(in, out, n, chunk, agg, idx_out, count);
}

// Resident CTAs of the wave kernel on the current device (0: cannot run).
template <bool VEC, bool FLAGS>
int wave_grid() {
    static int grid[64] = {0};
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (!done[dev]) {
        int sms = 0, per = 0, coop = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_wave_scan<VEC, FLAGS>,
                                                          kScanBlock, 0) != cudaSuccess)
            per = 0;
        per = per < kChunkCtasPerSm ? per : kChunkCtasPerSm;
        grid[dev] = (coop && per > 0 && sms > 0) ? per * sms : 0;
        done[dev] = true;
    }
    return grid[dev];
}

// The large-input scan: the wave form with waves of `wave_values` values, or the
// two-kernel form (wave_values = 0, or when the wave kernel cannot be launched with
// every CTA resident).
template <bool VEC, bool FLAGS>
hhs_status launch_large(const int32_t* in, int32_t* out, long long n, ScanHeader* hdr,
                        unsigned* agg, size_t agg_words, int32_t* idx_out, int32_t* count,
                        cudaStream_t s, long long wave_values, unsigned missing = 0u,
                        unsigned long long timeout_ns = kWaveBarrierTimeoutNs) {
    const int grid = wave_grid<VEC, FLAGS>();
    if (missing && (grid <= 0 || (size_t)2 * grid > agg_words)) return HHS_ERR_INVALID_ARG;
    if (grid <= 0 || wave_values <= 0 || (size_t)2 * grid > agg_words) {
        launch_two_pass<VEC, FLAGS>(in, out, n, hdr, agg, idx_out, count, s);
        HHS_LAUNCH_CHECK();
        return HHS_OK;
    }
    const long long tiles = (wave_values + ScanT::TILE - 1) / ScanT::TILE;
    long long chunk = (tiles + grid - 1) / grid * ScanT::TILE;
    // the header (error word, barrier counter) starts at zero
    HHS_CUDA_TRY(cudaMemsetAsync(hdr, 0, sizeof(ScanHeader), s));
    void* args[] = {(void*)&in,     (void*)&out,   (void*)&n,       (void*)&chunk,
                    (void*)&agg,    (void*)&hdr,   (void*)&idx_out, (void*)&count,
                    (void*)&missing, (void*)&timeout_ns};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_wave_scan<VEC, FLAGS>,
                                                      dim3(grid), dim3(kScanBlock), args, 0, s);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        if (missing) return hhs_from_cuda(e);
        launch_two_pass<VEC, FLAGS>(in, out, n, hdr, agg, idx_out, count, s);
    }
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

// Launch-shape variants of the standalone scan (tile = BLOCK x ITEMS values, look-back
// windows of 32 x LB tiles, at least MINB resident CTAs per SM), selected by
// scan_variant(); the default shape is variant 0.
template <int BLOCK, int ITEMS, int LB, int MINB, bool VEC>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_scan_v(const int32_t* __restrict__ in, int32_t* __restrict__ out, long long n,
             ScanHeader* hdr, unsigned long long* status, int num_tiles) {
    using T = TileScan<BLOCK, ITEMS, LB>;
    __shared__ int s_tile;
    __shared__ unsigned s_epoch, s_prefix, s_limit;
    __shared__ unsigned s_warp[T::WARPS];
    scan_begin(hdr, &s_tile, &s_epoch, &s_limit);
    const int tile = s_tile;
    const unsigned epoch = s_epoch;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long tbase = (long long)tile * T::TILE;
    unsigned v[ITEMS], cb[T::CHUNKS];
#pragma unroll
    for (int c = 0; c < T::CHUNKS; c++) {
        const long long e = tbase + T::offset(warp, c, lane);
        if (VEC && e + 4 <= n) {
            const int4 q = __ldcs(reinterpret_cast<const int4*>(in + e));
            v[4 * c] = q.x; v[4 * c + 1] = q.y; v[4 * c + 2] = q.z; v[4 * c + 3] = q.w;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) v[4 * c + k] = (e + k < n) ? (unsigned)in[e + k] : 0u;
        }
    }
    T::scan(v, cb, status, tile, epoch, &hdr->error, s_warp, &s_prefix, s_limit);
#pragma unroll
    for (int c = 0; c < T::CHUNKS; c++) {
        const long long e = tbase + T::offset(warp, c, lane);
        const unsigned p0 = cb[c], p1 = p0 + v[4 * c], p2 = p1 + v[4 * c + 1],
                       p3 = p2 + v[4 * c + 2];
        if (VEC && e + 4 <= n) {
            __stcs(reinterpret_cast<int4*>(out + e), make_int4((int)p0, (int)p1, (int)p2, (int)p3));
        } else {
            const unsigned pp[4] = {p0, p1, p2, p3};
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (e + k < n) out[e + k] = (int)pp[k];
        }
    }
}

template <int BLOCK, int ITEMS, int LB, int MINB>
void launch_scan_v(const int32_t* in, int32_t* out, long long n, void* ws, bool vec,
                   cudaStream_t s) {
    constexpr int TILE = BLOCK * ITEMS;
    const int tiles = (int)((n + TILE - 1) / TILE);
    auto* hdr = static_cast<ScanHeader*>(ws);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(ws) +
                                                         sizeof(ScanHeader));
    if (vec) k_scan_v<BLOCK, ITEMS, LB, MINB, true><<<tiles, BLOCK, 0, s>>>(in, out, n, hdr, status, tiles);
    else k_scan_v<BLOCK, ITEMS, LB, MINB, false><<<tiles, BLOCK, 0, s>>>(in, out, n, hdr, status, tiles);
}

int scan_variant() {
    static int v = [] {
        const char* e = std::getenv("HHS_SCAN_VARIANT");
        return e ? std::atoi(e) : 0;
    }();
    return v;
}

// ---- streamed single pass
// One cooperative launch of persistent CTAs (every CTA resident). CTA b owns chunks
// b, b + G, b + 2G, ... (G CTAs, chunks of BLOCK x VPT values), so round r is the chunks
// [rG, rG + G). A chunk's exclusive prefix is the running total of the rounds before it
// plus the aggregates of the chunks before it in its round. Every CTA publishes the
// aggregate of its chunk two rounds ahead, as soon as that chunk is in shared memory, and
// warp 0 reads all aggregates of the next round while the other warps store the current
// one: their sum over the chunks before its own is its prefix within the round, and their
// sum over the round carries the running total, which every CTA keeps itself. No chain
// of inclusive prefixes runs through the grid (with a decoupled look-back over chunks of
// this size, that chain of L2 round trips held the same data path to 1.9 TB/s), and a CTA
// waits only when another is more than a round behind.
// Data: a CTA keeps STAGES chunks in flight. When its threads have read a chunk out of
// shared memory, thread 0 bulk-copies (cp.async.bulk, completing on an mbarrier) the
// chunk STAGES rounds ahead into the freed buffer. Values are scanned in registers and
// stored from registers with 16-byte streaming stores; input and output must be 16-byte
// aligned. The bulk copy of the last chunk stops at a multiple of 4 values; the last
// n mod 4 values are read with plain loads. Status words (one per chunk) carry the
// call's epoch and the chunk's aggregate.

// Internal status of launch_stream: the device cannot take the cooperative launch.
constexpr hhs_status kStreamUnavailable = static_cast<hhs_status>(-1);

template <int BLOCK, int VPT, int STAGES>
struct StreamShape {
    static constexpr int CHUNK = BLOCK * VPT;  // values per chunk
    static constexpr size_t SMEM = (size_t)STAGES * CHUNK * sizeof(int32_t);
    static_assert(CHUNK % 4 == 0 && CHUNK * 4 < (1 << 20), "chunk bytes within one phase");
    static_assert(BLOCK % 32 == 0 && BLOCK + 32 <= 1024 && VPT % 4 == 0, "launch shape");
    static_assert(STAGES >= 3, "aggregates are published two rounds ahead");
};

// values of the chunk starting at `base` that its bulk copy delivers (a multiple of 4)
__device__ __forceinline__ long long stream_bulk_values(long long base, long long n,
                                                        int chunk) {
    const long long r = n - base;
    return (r < chunk ? r : (long long)chunk) & ~3LL;
}

// FLAGS: scan (flag != 0), store the scan to `out` when it is not null, the index of every
// nonzero flag to idx_out[scan], and the number of them to *count (by the CTA that holds
// the last chunk). Requires gridDim.x <= num_chunks.
template <int BLOCK, int VPT, int STAGES, int MINB, bool FLAGS>
__global__ void __launch_bounds__(BLOCK + 32, MINB)
    k_scan_stream(const int32_t* __restrict__ in, int32_t* __restrict__ out, long long n,
                  ScanHeader* hdr, unsigned long long* status, int num_chunks,
                  int32_t* __restrict__ idx_out, int32_t* __restrict__ count) {
    constexpr int CHUNK = StreamShape<BLOCK, VPT, STAGES>::CHUNK;
    constexpr int WARPS = BLOCK / 32, GROUPS = VPT / 4;
    extern __shared__ __align__(128) int4 s_buf[];  // STAGES x CHUNK/4
    __shared__ __align__(8) uint64_t s_bar[STAGES];
    // parity-indexed by round: a warp can be one round ahead of the slowest
    __shared__ unsigned s_warp[2][WARPS], s_red[2][WARPS], s_prefix[2];
    __shared__ unsigned s_epoch, s_limit;
    __shared__ int s_issued;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int G = (int)gridDim.x, b = (int)blockIdx.x;
    const int rounds = (num_chunks - b + G - 1) / G;  // chunks of this CTA
    auto chunk_of = [&](int r) { return (long long)b + (long long)r * G; };

    const bool coord = warp == WARPS;  // the coordinator warp (holds no values)
    // coordinator lane 0: start the copy of round r's chunk into its buffer
    auto issue = [&](int r) {
        if (r >= rounds) return;
        const int slot = r % STAGES;
        const long long base = chunk_of(r) * CHUNK;
        const unsigned bytes = (unsigned)(stream_bulk_values(base, n, CHUNK) * 4);
        mbar_arrive_expect_tx(&s_bar[slot], bytes);
        if (bytes) bulk_load(s_buf + (size_t)slot * (CHUNK / 4), in + base, bytes, &s_bar[slot]);
        s_issued = r + 1;
    };
    // every thread: round r's copy has landed (false: it did not within the poll limit)
    auto wait_round = [&](int r) {
        return mbar_wait(&s_bar[r % STAGES], (unsigned)(r / STAGES) & 1u, &hdr->error);
    };
    // this thread's group g (4 consecutive values) of round r's chunk; 0 past n
    auto group = [&](int r, int g, unsigned (&q)[4]) {
        const long long base = chunk_of(r) * CHUNK;
        const long long bulk_end = base + stream_bulk_values(base, n, CHUNK);
        const int o = warp * (32 * VPT) + g * 128 + lane * 4;
        const long long e = base + o;
        const int4 w = s_buf[(size_t)(r % STAGES) * (CHUNK / 4) + (o >> 2)];
        q[0] = (unsigned)w.x; q[1] = (unsigned)w.y; q[2] = (unsigned)w.z; q[3] = (unsigned)w.w;
        if (e + 4 > bulk_end) {  // the last chunk's tail
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (e + k >= bulk_end) q[k] = e + k < n ? (unsigned)__ldg(in + e + k) : 0u;
        }
        if (FLAGS) {
#pragma unroll
            for (int k = 0; k < 4; k++) q[k] = q[k] != 0u;
        }
    };
    // this thread's share of the aggregate of round r's chunk, summed over the warp
    auto warp_aggregate = [&](int r) {
        unsigned t = 0u;
#pragma unroll
        for (int g = 0; g < GROUPS; g++) {
            unsigned q[4];
            group(r, g, q);
            t += q[0] + q[1] + q[2] + q[3];
        }
        return (unsigned)warp_sum((int)t);
    };

    // coordinator: the aggregates of round r's chunks, summed over those before this CTA's
    // chunk and over all of them (batches of 8 words per lane, loads of a batch in flight
    // together; a word that stays unpublished past the poll limit records a timeout)
    auto poll_round = [&](int r, unsigned epoch, unsigned limit, unsigned& before,
                          unsigned& all) {
        const long long r0 = (long long)r * G;
        const int cnt = (int)min((long long)G, (long long)num_chunks - r0);
        before = 0u;
        all = 0u;
        for (int k0 = 0; k0 < cnt; k0 += 8 * 32) {
            unsigned long long sw[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int k = k0 + i * 32 + lane;
                sw[i] = k < cnt ? ld_relaxed_u64(&status[r0 + k]) : 0ull;
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int k = k0 + i * 32 + lane;
                if (k >= cnt) continue;
                for (unsigned spins = 0;
                     (unsigned)(sw[i] >> 34) != epoch || ((sw[i] >> 32) & 3u) == 0u; spins++) {
                    if (spins >= limit) {
                        atomicOr(&hdr->error, HHS_ERRBIT_LOOKBACK_TIMEOUT);
                        sw[i] = 0ull;
                        break;
                    }
                    if (spins > 64) __nanosleep(64);
                    sw[i] = ld_relaxed_u64(&status[r0 + k]);
                }
                all += (unsigned)sw[i];
                before += k < b ? (unsigned)sw[i] : 0u;
            }
        }
        before = (unsigned)warp_sum((int)before);
        all = (unsigned)warp_sum((int)all);
    };
    // coordinator: publish the aggregate of round r's chunk from the data warps' shares
    auto publish = [&](int r, const unsigned* red, unsigned epoch) {
        const unsigned a = (unsigned)warp_sum((int)(lane < WARPS ? red[lane] : 0u));
        if (lane == 0) st_relaxed_u64(&status[chunk_of(r)], scan_pack(epoch, 1u, a));
    };

    if (coord && lane == 0) {
        s_epoch = scan_next_epoch(hdr);
        const unsigned lim = *reinterpret_cast<volatile const unsigned*>(&hdr->spin_limit);
        s_limit = lim ? lim : HHS_SPIN_LIMIT;
        s_issued = 0;
#pragma unroll
        for (int k = 0; k < STAGES; k++) mbar_init(&s_bar[k], 1u);
        fence_barrier_init();
#pragma unroll 1
        for (int r = 0; r < STAGES; r++) issue(r);
    }
    __syncthreads();
    const unsigned epoch = s_epoch, limit = s_limit;
    // Aggregates are published two rounds ahead, and the coordinator reads round r + 1's
    // while the data warps store round r and read round r + 1: the prefix of a round is
    // known when the round starts, and the L2 round trips of the coordinator overlap the
    // data warps' work.
    int waited = 0;       // rounds whose copies every data thread has seen land
    unsigned carry = 0u;  // coordinator: the total of the rounds read so far
    {
        bool ok = true;
        if (!coord) {
            ok = wait_round(0);
            unsigned t = warp_aggregate(0);
            if (lane == 0) s_red[0][warp] = t;
            if (rounds > 1) {
                ok = wait_round(1) && ok;
                t = warp_aggregate(1);
                if (lane == 0) s_red[1][warp] = t;
            }
        }
        if (__syncthreads_and(ok)) {
            waited = rounds > 1 ? 2 : 1;
            if (coord) {
                publish(0, s_red[0], epoch);
                if (rounds > 1) publish(1, s_red[1], epoch);
                unsigned before, all;
                poll_round(0, epoch, limit, before, all);
                if (lane == 0) s_prefix[0] = before;
                if (FLAGS && count && lane == 0 && chunk_of(0) == num_chunks - 1)
                    *count = (int)all;
                carry = all;
            }
        }
        __syncthreads();
    }
    for (int r = 0; r < rounds && waited > r; r++) {
        const int p = r & 1;  // also the parity of round r + 2
        const bool has2 = r + 2 < rounds;
        bool ok = true;
        unsigned v[VPT], cb[GROUPS];
        if (!coord) {
            // the aggregate of the chunk two rounds ahead
            if (has2) {
                ok = wait_round(r + 2);
                const unsigned t = warp_aggregate(r + 2);
                if (lane == 0) s_red[p][warp] = t;
            }
            // this chunk: values, scans within each 128-value group and over the warp
            unsigned run = 0u;
#pragma unroll
            for (int g = 0; g < GROUPS; g++) {
                unsigned q[4];
                group(r, g, q);
                v[4 * g] = q[0]; v[4 * g + 1] = q[1]; v[4 * g + 2] = q[2]; v[4 * g + 3] = q[3];
                const unsigned sg = q[0] + q[1] + q[2] + q[3];
                const unsigned inc = (unsigned)warp_incl_scan((int)sg, lane);
                cb[g] = run + inc - sg;
                run += (unsigned)__shfl_sync(HHS_FULL_MASK, (int)inc, 31);
            }
            if (lane == 0) s_warp[p][warp] = run;
        }
        // every data thread has read this chunk's buffer and agrees whether the copy landed
        if (!__syncthreads_and(ok)) break;
        if (has2) waited = r + 3;
        if (coord) {
            if (lane == 0) issue(r + STAGES);
            if (has2) publish(r + 2, s_red[p], epoch);
            const unsigned wt = lane < WARPS ? s_warp[p][lane] : 0u;
            const unsigned wi = (unsigned)warp_incl_scan((int)wt, lane);
            if (lane < WARPS) s_warp[p][lane] = wi - wt;
        }
        __syncthreads();
        if (coord) {
            if (r + 1 < rounds) {
                unsigned before, all;
                poll_round(r + 1, epoch, limit, before, all);
                if (lane == 0) s_prefix[p ^ 1] = carry + before;
                if (FLAGS && count && lane == 0 && chunk_of(r + 1) == num_chunks - 1)
                    *count = (int)(carry + all);
                carry += all;
            }
            continue;
        }
        const unsigned wbase = s_prefix[p] + s_warp[p][warp];
        const long long base = chunk_of(r) * CHUNK;
#pragma unroll
        for (int g = 0; g < GROUPS; g++) {
            const long long e = base + warp * (32 * VPT) + g * 128 + lane * 4;
            const unsigned p0 = wbase + cb[g], p1 = p0 + v[4 * g], p2 = p1 + v[4 * g + 1],
                           p3 = p2 + v[4 * g + 2];
            if (!FLAGS || out) {
                if (e + 4 <= n) {
                    __stcs(reinterpret_cast<int4*>(out + e),
                           make_int4((int)p0, (int)p1, (int)p2, (int)p3));
                } else {
                    if (e < n) out[e] = (int)p0;
                    if (e + 1 < n) out[e + 1] = (int)p1;
                    if (e + 2 < n) out[e + 2] = (int)p2;
                }
            }
            if (FLAGS) {
                if (v[4 * g]) idx_out[p0] = (int)e;
                if (v[4 * g + 1]) idx_out[p1] = (int)(e + 1);
                if (v[4 * g + 2]) idx_out[p2] = (int)(e + 2);
                if (v[4 * g + 3]) idx_out[p3] = (int)(e + 3);
            }
        }
    }
    // A copy that did not land in time ended the loop early: wait once more (bounded) for
    // the copies this CTA still has in flight before its shared memory goes away. On the
    // normal exit every issued copy has been waited for.
    __syncthreads();
    if (coord && lane == 0) {
        for (int j = waited; j < s_issued; j++)
            if (!wait_round(j)) break;
    }
}

// One streamed scan: clears the header and the status words it uses, then launches as
// many persistent CTAs as are resident on the device at once (at most one per chunk) as
// one cooperative launch. Returns kStreamUnavailable, with nothing queued after the
// header clear, when the device cannot take the cooperative launch; the caller then uses
// the tiled scan.
template <int BLOCK, int VPT, int STAGES, int MINB, bool FLAGS>
hhs_status launch_stream(const int32_t* in, int32_t* out, long long n, void* ws,
                         size_t ws_bytes, int32_t* idx_out, int32_t* count, cudaStream_t s) {
    using Shape = StreamShape<BLOCK, VPT, STAGES>;
    auto* kern = k_scan_stream<BLOCK, VPT, STAGES, MINB, FLAGS>;
    const long long chunks = (n + Shape::CHUNK - 1) / Shape::CHUNK;
    const size_t used = sizeof(ScanHeader) + (size_t)chunks * sizeof(unsigned long long);
    if (used > ws_bytes || chunks > 0x7fffffffLL) return HHS_ERR_INVALID_ARG;
    static int resident[64] = {0};  // per device: CTAs resident at once (-1: none)
    int dev = 0;
    HHS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return kStreamUnavailable;
    if (resident[dev] == 0) {
        int sms = 0, per = 0, coop = 0;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Shape::SMEM) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, BLOCK + 32, Shape::SMEM) !=
                cudaSuccess) {
            (void)cudaGetLastError();
            per = 0;
        }
        resident[dev] = (coop && per > 0 && sms > 0) ? sms * per : -1;
    }
    if (resident[dev] < 0) return kStreamUnavailable;
    const int grid = (int)(chunks < resident[dev] ? chunks : resident[dev]);
    HHS_CUDA_TRY(cudaMemsetAsync(ws, 0, used, s));
    auto* hdr = static_cast<ScanHeader*>(ws);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(ws) +
                                                         sizeof(ScanHeader));
    int nch = (int)chunks;
    void* args[] = {(void*)&in,  (void*)&out,    (void*)&n,       (void*)&hdr,
                    (void*)&status, (void*)&nch, (void*)&idx_out, (void*)&count};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void*)kern, dim3(grid),
                                                      dim3(BLOCK + 32), args, Shape::SMEM, s);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return kStreamUnavailable;
    }
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

// Launch shapes of the streamed scan (threads, values per thread, stages, CTAs per SM).
// Shape 0 is the default; HHS_SCAN_VARIANT 20 + k selects shape k at every size.
constexpr int kStreamShapes = 5;
// The streamed form is the default scan of aligned inputs of at least kStreamMinN values
// (below that the pipeline's fill and drain cost more than the look-back form saves), in
// shape kStreamDefaultShape: at 2^28 values 5.0 TB/s against 4.25 for the two-kernel
// form, at 2^26 4.35 against 3.87; at 2^24 2.8 against 3.3.
constexpr long long kStreamMinN = 1LL << 25;
constexpr int kStreamDefaultShape = 3;
template <bool FLAGS>
hhs_status launch_stream_shape(int shape, const int32_t* in, int32_t* out, long long n,
                               void* ws, size_t ws_bytes, int32_t* idx_out, int32_t* count,
                               cudaStream_t s) {
    switch (shape) {
        case 1:  // 72 KiB chunks, 3 stages
            return launch_stream<512, 36, 3, 1, FLAGS>(in, out, n, ws, ws_bytes, idx_out, count, s);
        case 2:  // 50 KiB chunks, 4 stages, 640 data threads
            return launch_stream<640, 20, 4, 1, FLAGS>(in, out, n, ws, ws_bytes, idx_out, count, s);
        case 3:  // 48 KiB chunks, 4 stages, 768 data threads
            return launch_stream<768, 16, 4, 1, FLAGS>(in, out, n, ws, ws_bytes, idx_out, count, s);
        case 4:  // 48 KiB chunks, 4 stages
            return launch_stream<512, 24, 4, 1, FLAGS>(in, out, n, ws, ws_bytes, idx_out, count, s);
        default:  // 64 KiB chunks, 3 stages, 512 data threads and a coordinator warp
            return launch_stream<512, 32, 3, 1, FLAGS>(in, out, n, ws, ws_bytes, idx_out, count, s);
    }
}

// Stream compaction of int32 flags: the indices of the nonzero flags, in order, go to
// idx_out[scan]; the exclusive scan of (flag != 0) optionally goes to scan_out; the last
// CTA writes the number of selected elements to *count.
template <bool VEC, bool SELF_RESET>
__global__ void __launch_bounds__(kScanBlock, 6)
    k_compact_flags(const int32_t* __restrict__ flags, int32_t* __restrict__ scan_out,
                    int32_t* __restrict__ idx_out, int32_t* __restrict__ count, long long n,
                    ScanHeader* hdr, unsigned long long* status, int num_tiles) {
    __shared__ int s_tile;
    __shared__ unsigned s_epoch, s_prefix, s_limit;
    __shared__ unsigned s_warp[ScanT::WARPS];
    __shared__ int s_last;
    scan_begin(hdr, &s_tile, &s_epoch, &s_limit);
    const int tile = s_tile;
    const unsigned epoch = s_epoch;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long tbase = (long long)tile * ScanT::TILE;
    unsigned v[kScanItems], cb[ScanT::CHUNKS];
#pragma unroll
    for (int c = 0; c < ScanT::CHUNKS; c++) {
        const long long e = tbase + ScanT::offset(warp, c, lane);
        if (VEC && e + 4 <= n) {
            const int4 q = __ldcs(reinterpret_cast<const int4*>(flags + e));
            v[4 * c] = q.x != 0; v[4 * c + 1] = q.y != 0;
            v[4 * c + 2] = q.z != 0; v[4 * c + 3] = q.w != 0;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) v[4 * c + k] = (e + k < n) ? (flags[e + k] != 0) : 0u;
        }
    }
    ScanT::scan(v, cb, status, tile, epoch, &hdr->error, s_warp, &s_prefix, s_limit);
#pragma unroll
    for (int c = 0; c < ScanT::CHUNKS; c++) {
        const long long e = tbase + ScanT::offset(warp, c, lane);
        unsigned pp[4];
        pp[0] = cb[c];
#pragma unroll
        for (int k = 1; k < 4; k++) pp[k] = pp[k - 1] + v[4 * c + k - 1];
        if (scan_out) {
            if (VEC && e + 4 <= n) {
                __stcs(reinterpret_cast<int4*>(scan_out + e),
                       make_int4((int)pp[0], (int)pp[1], (int)pp[2], (int)pp[3]));
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (e + k < n) scan_out[e + k] = (int)pp[k];
            }
        }
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (v[4 * c + k]) idx_out[pp[k]] = (int)(e + k);
    }
    // the tile holding the last element knows the total
    if (tile == num_tiles - 1 && threadIdx.x == 0)
        *count = (int)(unsigned)(ld_relaxed_u64(&status[num_tiles - 1]) & 0xffffffffull);
    if (SELF_RESET && scan_finish_is_last(hdr, num_tiles, &s_last)) scan_reset(hdr, epoch);
}

constexpr int kSplitBlock = 256;
constexpr int kSplitItems = 8;  // 2048 particles per tile
using SplitT = TileScan<kSplitBlock, kSplitItems>;

// Fast/slow split of a list of particle indices (identity when list_in == nullptr):
// pred = ts[g] <= pivot (src/split.cuh:114-116); fast g -> fast_out[scan],
// slow g -> slow_out[i - scan] (src/split.cuh:335-357). The last CTA applies the
// N_fast == 1 fold (lone fast particle appended as slow_out[n-1]) and writes the
// partition counts; with leaf_time set it also adds dt there when N_fast == 0
// (globals->simtime, src/hold.cuh:106-114).
__global__ void __launch_bounds__(kSplitBlock)
    k_split_list(const int32_t* __restrict__ list_in, int n, const double* __restrict__ ts,
                 double pivot, int32_t* __restrict__ fast_out, int32_t* __restrict__ slow_out,
                 int32_t* __restrict__ pred_out, int32_t* __restrict__ scan_out,
                 hhs_partition* counts, double* leaf_time, double dt, hhs_stats* stats,
                 int level, int calc_ts, ScanHeader* hdr, unsigned long long* status,
                 int num_tiles) {
    __shared__ int s_tile;
    __shared__ unsigned s_epoch, s_prefix, s_limit;
    __shared__ unsigned s_warp[SplitT::WARPS];
    __shared__ int s_last;
    scan_begin(hdr, &s_tile, &s_epoch, &s_limit);
    const int tile = s_tile;
    const unsigned epoch = s_epoch;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long tbase = (long long)tile * SplitT::TILE;

    unsigned v[kSplitItems], cb[SplitT::CHUNKS];
    int g[kSplitItems];
#pragma unroll
    for (int c = 0; c < SplitT::CHUNKS; c++) {
        const long long e = tbase + SplitT::offset(warp, c, lane);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const long long i = e + k;
            if (i < n) {
                const int gi = list_in ? list_in[i] : (int)i;
                g[4 * c + k] = gi;
                v[4 * c + k] = ts[gi] <= pivot ? 1u : 0u;
            } else {
                g[4 * c + k] = -1;
                v[4 * c + k] = 0u;
            }
        }
    }
    SplitT::scan(v, cb, status, tile, epoch, &hdr->error, s_warp, &s_prefix, s_limit);
#pragma unroll
    for (int c = 0; c < SplitT::CHUNKS; c++) {
        const long long e = tbase + SplitT::offset(warp, c, lane);
        unsigned p = cb[c];
#pragma unroll
        for (int k = 0; k < 4; k++, p += v[4 * c + k - 1]) {
            const long long i = e + k;
            if (i < n) {
                if (v[4 * c + k]) fast_out[p] = g[4 * c + k];
                else slow_out[i - p] = g[4 * c + k];
                if (pred_out) pred_out[i] = (int)v[4 * c + k];
                if (scan_out) scan_out[i] = (int)p;
            }
        }
    }
    if (scan_finish_is_last(hdr, num_tiles, &s_last)) {
        if (threadIdx.x == 0) {
            const unsigned long long s =
                ld_relaxed_u64(&status[num_tiles - 1]);  // inclusive total of the last tile
            int nf = (int)(unsigned)s;
            if (nf == 1) {
                slow_out[n - 1] = fast_out[0];
                nf = 0;
            }
            counts->n_fast = nf;
            counts->n_slow = n - nf;
            if (leaf_time && nf == 0) *leaf_time += dt;
            if (stats) {
                const double ns = (double)(n - nf), nfd = (double)nf;
                stats->nodes += 1;
                if (level > stats->max_level) stats->max_level = level;
                stats->kick_pairs += ns * (ns - 1.0) + 2.0 * ns * nfd;
                if (calc_ts) stats->ts_pairs += (double)n * (double)(n - 1);
            }
        }
        scan_reset(hdr, epoch);
    }
}

}  // namespace

size_t scan_workspace_bytes(long long n, int tile) {
    const long long tiles = (n + tile - 1) / tile;
    return sizeof(ScanHeader) + (size_t)(tiles > 0 ? tiles : 1) * sizeof(unsigned long long);
}

size_t split_workspace_bytes(int n) { return scan_workspace_bytes(n, SplitT::TILE); }

hhs_status launch_split_list(const int32_t* list_in, int n, const double* ts, double pivot,
                             int32_t* fast_out, int32_t* slow_out, int32_t* pred_out,
                             int32_t* scan_out, hhs_partition* counts, double* leaf_time,
                             double dt, hhs_stats* stats, int level, int calc_ts, void* ws,
                             cudaStream_t stream) {
    if (n <= 0) return HHS_ERR_INVALID_ARG;
    const int tiles = (n + SplitT::TILE - 1) / SplitT::TILE;
    auto* hdr = static_cast<ScanHeader*>(ws);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(ws) +
                                                         sizeof(ScanHeader));
    k_split_list<<<tiles, kSplitBlock, 0, stream>>>(list_in, n, ts, pivot, fast_out, slow_out,
                                                    pred_out, scan_out, counts, leaf_time, dt,
                                                    stats, level, calc_ts, hdr, status, tiles);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

unsigned* scan_workspace_error_word(void* ws) { return &static_cast<ScanHeader*>(ws)->error; }

extern "C" size_t hhs_scan_workspace_size(int64_t n) {
    return scan_workspace_bytes(n, kScanMinTile);
}

extern "C" hhs_status hhs_scan_exclusive_i32(const int32_t* d_in, int32_t* d_out, int64_t n,
                                             void* d_workspace, size_t workspace_bytes,
                                             void* stream) {
    if (n < 0 || (n > 0 && (!d_in || !d_out || !d_workspace))) return HHS_ERR_INVALID_ARG;
    if (n == 0) return HHS_OK;
    if (n > (int64_t)0x7fffffff) return HHS_ERR_INVALID_ARG;
    if (workspace_bytes < hhs_scan_workspace_size(n)) return HHS_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_workspace) & 7u) != 0) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int tiles = (int)((n + ScanT::TILE - 1) / ScanT::TILE);
    const size_t used = scan_workspace_bytes(n, kScanMinTile);
    const int variant = scan_variant();
    auto* hdr = static_cast<ScanHeader*>(d_workspace);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(d_workspace) +
                                                         sizeof(ScanHeader));
    const bool vec = ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) &
                      15u) == 0;
    const bool stream_variant = variant >= 20 && variant < 20 + kStreamShapes;
    if (vec && (stream_variant || (variant == 0 && n >= kStreamMinN))) {
        const int shape = stream_variant ? variant - 20 : kStreamDefaultShape;
        const hhs_status st = launch_stream_shape<false>(shape, d_in, d_out, n, d_workspace,
                                                         workspace_bytes, nullptr, nullptr, s);
        if (st != kStreamUnavailable) return st;
    }
    if ((variant == 0 || (variant >= 11 && variant <= 13)) && n >= kTwoPassMinN) {
        // the chunk sums are written before they are read: only the header is cleared.
        // Default: the two-kernel form; variants 11-13: waves of 2^22, 2^23, 2^24 values.
        const long long wave = variant == 11   ? (1LL << 22)
                               : variant == 12 ? (1LL << 23)
                               : variant == 13 ? kWaveValues
                                               : 0;
        auto* agg = reinterpret_cast<unsigned*>(status);
        const size_t words = (used - sizeof(ScanHeader)) / sizeof(unsigned);
        return vec ? launch_large<true, false>(d_in, d_out, n, hdr, agg, words, nullptr, nullptr,
                                               s, wave)
                   : launch_large<false, false>(d_in, d_out, n, hdr, agg, words, nullptr,
                                                nullptr, s, wave);
    }
    HHS_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, used, s));
    switch (variant) {
        case 1: launch_scan_v<256, 8, 1, 1>(d_in, d_out, n, d_workspace, vec, s); break;
        case 2: launch_scan_v<128, 16, 1, 1>(d_in, d_out, n, d_workspace, vec, s); break;
        case 3: launch_scan_v<256, 16, 1, 6>(d_in, d_out, n, d_workspace, vec, s); break;
        case 4: launch_scan_v<512, 16, 1, 1>(d_in, d_out, n, d_workspace, vec, s); break;
        case 5: launch_scan_v<256, 32, 1, 1>(d_in, d_out, n, d_workspace, vec, s); break;
        case 6: launch_scan_v<256, 8, 1, 8>(d_in, d_out, n, d_workspace, vec, s); break;
        case 7: launch_scan_v<256, 16, 2, 6>(d_in, d_out, n, d_workspace, vec, s); break;
        case 8: launch_scan_v<256, 16, 4, 6>(d_in, d_out, n, d_workspace, vec, s); break;
        case 9: launch_scan_v<256, 16, 8, 6>(d_in, d_out, n, d_workspace, vec, s); break;
        case 10: launch_scan_v<256, 32, 4, 3>(d_in, d_out, n, d_workspace, vec, s); break;
        default:
            if (vec)
                k_scan_exclusive_i32<true, false><<<tiles, kScanBlock, 0, s>>>(d_in, d_out, n,
                                                                               hdr, status, tiles);
            else
                k_scan_exclusive_i32<false, false><<<tiles, kScanBlock, 0, s>>>(d_in, d_out, n,
                                                                                hdr, status, tiles);
    }
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

extern "C" hhs_status hhs_compact_flags_i32(const int32_t* d_flags, int32_t* d_scan,
                                            int32_t* d_idx, int32_t* d_count, int64_t n,
                                            void* d_workspace, size_t workspace_bytes,
                                            void* stream) {
    if (n < 0 || (n > 0 && (!d_flags || !d_idx || !d_count || !d_workspace)))
        return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        HHS_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(int32_t), s));
        return HHS_OK;
    }
    if (n > (int64_t)0x7fffffff) return HHS_ERR_INVALID_ARG;
    if (workspace_bytes < hhs_scan_workspace_size(n)) return HHS_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_workspace) & 7u) != 0) return HHS_ERR_INVALID_ARG;
    const int tiles = (int)((n + ScanT::TILE - 1) / ScanT::TILE);
    auto* hdr = static_cast<ScanHeader*>(d_workspace);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(d_workspace) +
                                                         sizeof(ScanHeader));
    const bool vec = ((reinterpret_cast<uintptr_t>(d_flags) |
                       reinterpret_cast<uintptr_t>(d_scan)) & 15u) == 0;
    const int variant = scan_variant();
    if (vec && variant >= 20 && variant < 20 + kStreamShapes) {
        const hhs_status st = launch_stream_shape<true>(variant - 20, d_flags, d_scan, n,
                                                        d_workspace, workspace_bytes, d_idx,
                                                        d_count, s);
        if (st != kStreamUnavailable) return st;
    }
    if (n >= kTwoPassMinN) {
        auto* agg = reinterpret_cast<unsigned*>(status);
        const size_t words =
            (scan_workspace_bytes(n, kScanMinTile) - sizeof(ScanHeader)) / sizeof(unsigned);
        const long long wave = n >= kWaveMinN ? kWaveValues : 0;
        return vec ? launch_large<true, true>(d_flags, d_scan, n, hdr, agg, words, d_idx,
                                              d_count, s, wave)
                   : launch_large<false, true>(d_flags, d_scan, n, hdr, agg, words, d_idx,
                                               d_count, s, wave);
    }
    HHS_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, scan_workspace_bytes(n, ScanT::TILE), s));
    if (vec)
        k_compact_flags<true, false><<<tiles, kScanBlock, 0, s>>>(d_flags, d_scan, d_idx,
                                                                  d_count, n, hdr, status, tiles);
    else
        k_compact_flags<false, false><<<tiles, kScanBlock, 0, s>>>(d_flags, d_scan, d_idx,
                                                                   d_count, n, hdr, status, tiles);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

// ------------------------------------------------------------------ allocation-free scan
// The same single-pass scan for callers that may not allocate device memory: its
// workspace is this file-scope device array (128.3 KiB, present on every device that
// loads the library until the process exits), so inputs are limited to
// kStaticScanTiles tiles of ScanT::TILE values (2^26 = 67,108,864 values).
constexpr int kStaticScanTiles = 16384;
constexpr size_t kStaticScanBytes =
    sizeof(ScanHeader) + sizeof(unsigned long long) * (size_t)kStaticScanTiles;
constexpr long long kStaticScanMaxN = (long long)kStaticScanTiles * ScanT::TILE;
static_assert(kStaticScanMaxN == HHS_SCAN_NOALLOC_MAX_N, "limit stated in hhs.h");
static __device__ __align__(256) unsigned char g_static_scan_ws[kStaticScanBytes];

namespace {
// Device address of g_static_scan_ws per device, looked up once with that device current
// (in host code the array's name is only a host-side stand-in, not a device address).
constexpr int kMaxDevices = 64;
std::atomic<void*> g_static_ws_addr[kMaxDevices];

hhs_status static_scan_workspace(void** out) {
    int dev = 0;
    HHS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return HHS_ERR_CUDA;
    void* p = g_static_ws_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scan_ws);
        if (e != cudaSuccess || !p) return hhs_from_cuda(e == cudaSuccess ? cudaErrorUnknown : e);
        g_static_ws_addr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return HHS_OK;
}
}  // namespace

extern "C" hhs_status hhs_scan_exclusive_i32_noalloc(const int32_t* d_in, int32_t* d_out,
                                                     int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!d_in || !d_out))) return HHS_ERR_INVALID_ARG;
    if (n == 0) return HHS_OK;
    if (n > kStaticScanMaxN) return HHS_ERR_CAPACITY;
    void* ws = nullptr;
    hhs_status st = static_scan_workspace(&ws);
    if (st != HHS_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int tiles = (int)((n + ScanT::TILE - 1) / ScanT::TILE);
    auto* hdr = static_cast<ScanHeader*>(ws);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(ws) +
                                                         sizeof(ScanHeader));
    const bool vec = ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) &
                      15u) == 0;
    // The forms of the allocating scan, each within the array: the streamed form (status
    // words of its chunks), the two-kernel form (chunk sums), the single pass (a status
    // word per tile). Each clears the part of the array it uses, which still holds the
    // previous call's contents.
    if (vec && n >= kStreamMinN) {
        st = launch_stream_shape<false>(kStreamDefaultShape, d_in, d_out, n, ws, kStaticScanBytes,
                                        nullptr, nullptr, s);
        if (st != kStreamUnavailable) return st;
    }
    if (n >= kTwoPassMinN) {
        HHS_CUDA_TRY(cudaMemsetAsync(ws, 0, sizeof(ScanHeader), s));
        auto* agg = reinterpret_cast<unsigned*>(status);
        const size_t words = (kStaticScanBytes - sizeof(ScanHeader)) / sizeof(unsigned);
        return vec ? launch_large<true, false>(d_in, d_out, n, hdr, agg, words, nullptr, nullptr,
                                               s, 0)
                   : launch_large<false, false>(d_in, d_out, n, hdr, agg, words, nullptr,
                                                nullptr, s, 0);
    }
    HHS_CUDA_TRY(cudaMemsetAsync(ws, 0, scan_workspace_bytes(n, ScanT::TILE), s));
    if (vec)
        k_scan_exclusive_i32<true, false><<<tiles, kScanBlock, 0, s>>>(d_in, d_out, n, hdr,
                                                                       status, tiles);
    else
        k_scan_exclusive_i32<false, false><<<tiles, kScanBlock, 0, s>>>(d_in, d_out, n, hdr,
                                                                        status, tiles);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}

// Status of the last allocation-free scan on the current device: the error word of the
// static array's header (set by a look-back wait that gave up), read after synchronising
// the stream. Each hhs_scan_exclusive_i32_noalloc call clears the word before it runs.
extern "C" hhs_status hhs_scan_noalloc_status(void* stream) {
    void* ws = nullptr;
    hhs_status st = static_scan_workspace(&ws);
    if (st != HHS_OK) return st;
    return hhs_scan_workspace_status(ws, stream);
}

// Bounded-wait self-test of the allocation-free scan: the same stalled-predecessor run
// as hhs_scan_selftest_stalled_predecessor, on the static array. Its status comes back
// through hhs_scan_noalloc_status (HHS_ERR_TIMEOUT when the waits ran out as designed).
extern "C" hhs_status hhs_scan_noalloc_selftest_stalled_predecessor(const int32_t* d_in,
                                                                    int32_t* d_out, int64_t n,
                                                                    uint32_t max_polls,
                                                                    void* stream) {
    if (n < 2 * (int64_t)ScanT::TILE || n > kStaticScanMaxN || !d_in || !d_out ||
        max_polls == 0 || max_polls > HHS_SPIN_LIMIT)
        return HHS_ERR_INVALID_ARG;
    void* ws = nullptr;
    hhs_status st = static_scan_workspace(&ws);
    if (st != HHS_OK) return st;
    return hhs_scan_selftest_stalled_predecessor(d_in, d_out, n, ws, kStaticScanBytes, max_polls,
                                                 stream);
}

extern "C" hhs_status hhs_scan_workspace_status(const void* d_workspace, void* stream) {
    if (!d_workspace) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HHS_CUDA_TRY(cudaStreamSynchronize(s));
    unsigned err = 0;
    HHS_CUDA_TRY(cudaMemcpy(&err, &static_cast<const ScanHeader*>(d_workspace)->error,
                            sizeof(err), cudaMemcpyDeviceToHost));
    if (err & (HHS_ERRBIT_LOOKBACK_TIMEOUT | HHS_ERRBIT_BARRIER_TIMEOUT)) return HHS_ERR_TIMEOUT;
    return err ? HHS_ERR_DEVICE_FAULT_FLAG : HHS_OK;
}

// ------------------------------------------------------------------ bounded-wait self-test
// Runs the scan of hhs_scan_exclusive_i32 with tile 0 left out (the tile counter starts at
// 1), so every look-back waits on a predecessor that never publishes. Each wait gives up
// after max_polls polls, records HHS_ERRBIT_LOOKBACK_TIMEOUT in the workspace header and
// lets its CTA finish; the call synchronises the stream and returns the workspace status,
// HHS_ERR_TIMEOUT when the waits ran out as designed. The output is not a valid scan.
extern "C" hhs_status hhs_scan_selftest_stalled_predecessor(const int32_t* d_in, int32_t* d_out,
                                                             int64_t n, void* d_workspace,
                                                             size_t workspace_bytes,
                                                             uint32_t max_polls, void* stream) {
    if (n < 2 * (int64_t)ScanT::TILE || n > (int64_t)0x7fffffff || !d_in || !d_out ||
        !d_workspace || max_polls == 0 || max_polls > HHS_SPIN_LIMIT)
        return HHS_ERR_INVALID_ARG;
    if (workspace_bytes < hhs_scan_workspace_size(n)) return HHS_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_workspace) & 7u) != 0) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int tiles = (int)((n + ScanT::TILE - 1) / ScanT::TILE);
    HHS_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, scan_workspace_bytes(n, kScanMinTile), s));
    ScanHeader h;
    std::memset(&h, 0, sizeof(h));
    h.tile_counter = 1u;
    h.spin_limit = max_polls;
    HHS_CUDA_TRY(cudaMemcpyAsync(d_workspace, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    auto* hdr = static_cast<ScanHeader*>(d_workspace);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(d_workspace) +
                                                         sizeof(ScanHeader));
    k_scan_exclusive_i32<false, false><<<tiles - 1, kScanBlock, 0, s>>>(d_in, d_out, n, hdr,
                                                                       status, tiles);
    HHS_LAUNCH_CHECK();
    return hhs_scan_workspace_status(d_workspace, stream);
}

// Runs the wave-form scan with every grid barrier waiting for one CTA more than the grid
// has, so each wait runs out: every CTA gives up after timeout_us, records
// HHS_ERRBIT_BARRIER_TIMEOUT in the workspace header and returns. d_out is left
// unspecified. Synchronises the stream and returns the workspace status.
extern "C" hhs_status hhs_scan_selftest_wave_barrier(const int32_t* d_in, int32_t* d_out,
                                                     int64_t n, void* d_workspace,
                                                     size_t workspace_bytes,
                                                     uint32_t timeout_us, void* stream) {
    if (!d_in || !d_out || !d_workspace || n < kTwoPassMinN || n > (int64_t)0x7fffffff ||
        timeout_us == 0 || timeout_us > 10000000u)
        return HHS_ERR_INVALID_ARG;
    if (workspace_bytes < hhs_scan_workspace_size(n)) return HHS_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_workspace) & 7u) != 0) return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto* hdr = static_cast<ScanHeader*>(d_workspace);
    auto* agg = reinterpret_cast<unsigned*>(static_cast<char*>(d_workspace) + sizeof(ScanHeader));
    const size_t words =
        (scan_workspace_bytes(n, kScanMinTile) - sizeof(ScanHeader)) / sizeof(unsigned);
    const bool vec = ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) &
                      15u) == 0;
    const unsigned long long ns = (unsigned long long)timeout_us * 1000ull;
    const hhs_status st =
        vec ? launch_large<true, false>(d_in, d_out, n, hdr, agg, words, nullptr, nullptr, s,
                                        kWaveValues, 1u, ns)
            : launch_large<false, false>(d_in, d_out, n, hdr, agg, words, nullptr, nullptr, s,
                                         kWaveValues, 1u, ns);
    if (st != HHS_OK) return st;
    return hhs_scan_workspace_status(d_workspace, stream);
}

// ------------------------------------------------------------------ CPU-order split
// The permutation left behind by the in-place two-pointer partition of the HHS CPU
// integrators (cpu_split, src/cpu_scan.h:20-50), computed in closed form from one exclusive
// scan of the fast flags (ts <= pivot). With n_fast fast particles, the k-th slow entry of
// [0, n_fast) counted from the left is exchanged with the k-th fast entry of [n_fast, n)
// counted from the right, and every other entry stays in place: exactly the exchanges the
// two cursors make before they meet.
namespace {

constexpr int kOrderBlock = 256;

__global__ void k_cpu_order_flags(const double* __restrict__ ts, int n, double pivot,
                                  int32_t* __restrict__ flags) {
    const int i = blockIdx.x * kOrderBlock + threadIdx.x;
    if (i < n) flags[i] = ts[i] <= pivot ? 1 : 0;
}

__device__ __forceinline__ int cpu_order_nfast(const int32_t* flags, const int32_t* excl, int n) {
    return excl[n - 1] + flags[n - 1];
}

// identity order; rank of each misplaced entry; the counts
__global__ void k_cpu_order_ranks(const int32_t* __restrict__ flags,
                                  const int32_t* __restrict__ excl, int n,
                                  int32_t* __restrict__ order, int32_t* __restrict__ pos_slow,
                                  int32_t* __restrict__ pos_fast, hhs_partition* counts) {
    const int nf = cpu_order_nfast(flags, excl, n);
    const int i = blockIdx.x * kOrderBlock + threadIdx.x;
    if (i == 0) {
        counts->n_fast = nf;
        counts->n_slow = n - nf;
    }
    if (i >= n) return;
    order[i] = i;
    const int f = flags[i], e = excl[i];
    if (i < nf && !f) pos_slow[i - e] = i;          // slow entries before it: i - e
    if (i >= nf && f) pos_fast[nf - e - 1] = i;     // fast entries after it
}

__global__ void k_cpu_order_swap(const int32_t* __restrict__ flags,
                                 const int32_t* __restrict__ excl, int n,
                                 const int32_t* __restrict__ pos_slow,
                                 const int32_t* __restrict__ pos_fast,
                                 int32_t* __restrict__ order) {
    const int nf = cpu_order_nfast(flags, excl, n);
    const int m = nf < n ? nf - excl[nf] : 0;  // slow entries inside [0, n_fast)
    const int k = blockIdx.x * kOrderBlock + threadIdx.x;
    if (k >= m) return;
    const int a = pos_slow[k], b = pos_fast[k];
    order[a] = b;
    order[b] = a;
}

size_t cpu_order_offset(long long n, int part) {
    const size_t arr = ((size_t)n * sizeof(int32_t) + 255) & ~(size_t)255;
    return ((scan_workspace_bytes(n, kScanMinTile) + 255) & ~(size_t)255) + arr * (size_t)part;
}

}  // namespace

extern "C" size_t hhs_split_cpu_order_workspace_size(int64_t n) {
    return n <= 0 ? 0 : cpu_order_offset(n, 4);
}

extern "C" hhs_status hhs_split_cpu_order(const double* d_ts, int32_t n, double pivot,
                                          int32_t* d_order, hhs_partition* d_counts,
                                          void* d_workspace, size_t workspace_bytes,
                                          void* stream) {
    if (n < 0 || !d_counts || (n > 0 && (!d_ts || !d_order || !d_workspace)))
        return HHS_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        HHS_CUDA_TRY(cudaMemsetAsync(d_counts, 0, sizeof(hhs_partition), s));
        return HHS_OK;
    }
    if (workspace_bytes < hhs_split_cpu_order_workspace_size(n)) return HHS_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_workspace) & 255u) != 0) return HHS_ERR_INVALID_ARG;
    char* base = static_cast<char*>(d_workspace);
    auto* flags = reinterpret_cast<int32_t*>(base + cpu_order_offset(n, 0));
    auto* excl = reinterpret_cast<int32_t*>(base + cpu_order_offset(n, 1));
    auto* pos_slow = reinterpret_cast<int32_t*>(base + cpu_order_offset(n, 2));
    auto* pos_fast = reinterpret_cast<int32_t*>(base + cpu_order_offset(n, 3));
    const int grid = (n + kOrderBlock - 1) / kOrderBlock;
    k_cpu_order_flags<<<grid, kOrderBlock, 0, s>>>(d_ts, n, pivot, flags);
    HHS_LAUNCH_CHECK();
    hhs_status st = hhs_scan_exclusive_i32(flags, excl, n, d_workspace,
                                           scan_workspace_bytes(n, kScanMinTile), stream);
    if (st != HHS_OK) return st;
    k_cpu_order_ranks<<<grid, kOrderBlock, 0, s>>>(flags, excl, n, d_order, pos_slow, pos_fast,
                                                   d_counts);
    HHS_LAUNCH_CHECK();
    k_cpu_order_swap<<<grid, kOrderBlock, 0, s>>>(flags, excl, n, pos_slow, pos_fast, d_order);
    HHS_LAUNCH_CHECK();
    return HHS_OK;
}
