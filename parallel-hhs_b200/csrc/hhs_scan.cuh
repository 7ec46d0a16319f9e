// hhs_scan.cuh -- single-pass exclusive scan (decoupled look-back) used by the
// standalone int32 scan and by the fast/slow split.
//
// The reference computes the same exact exclusive prefix sum with a multi-level
// Blelloch tree scan: per-block up/down-sweep in shared memory, block sums scanned
// recursively, and "add" kernels that fix up block offsets and the remainder
// (src/split.cuh:64-102,131-302,372-394,438-565; 3-6 launches and two cudaMalloc /
// cudaFree pairs per call). Here one launch does it: each CTA scans its tile in
// registers with warp shuffles, then obtains its exclusive prefix by the
// decoupled look-back of Merrill & Garland (2016, "Single-pass Parallel Prefix Scan
// with Decoupled Look-back"), and the last CTA to finish resets the workspace so
// the next call needs no memset.
#pragma once
#include "hhs_common.cuh"

// Workspace: a 256-byte header followed by one 64-bit status word per tile.
struct ScanHeader {
    unsigned tile_counter;  // dynamic tile index (tiles start in index order)
    unsigned done_counter;  // CTAs that finished; the last one resets the header
    unsigned epoch;         // status words of other epochs read as "not ready"
    unsigned error;         // HHS_ERRBIT_* set by timed-out waits
    unsigned spin_limit;    // look-back polls before giving up (0: HHS_SPIN_LIMIT)
    unsigned wave_count;    // grid-barrier arrivals of the wave-form scan
    unsigned pad[58];
};
static_assert(sizeof(ScanHeader) == 256, "scan header must stay 256 bytes");

// status word: [63:34] epoch, [33:32] flag (0 none, 1 aggregate, 2 inclusive), [31:0] value
__device__ __forceinline__ unsigned long long scan_pack(unsigned epoch, unsigned flag,
                                                        unsigned value) {
    return ((unsigned long long)epoch << 34) | ((unsigned long long)flag << 32) | value;
}

__device__ __forceinline__ unsigned scan_next_epoch(const ScanHeader* h) {
    unsigned e = (*(volatile const unsigned*)&h->epoch + 1u) & 0x3fffffffu;
    return e ? e : 1u;
}

// Called by one full warp. Publishes this tile's aggregate, walks predecessors in
// windows of 32*PER_LANE (each lane reads PER_LANE consecutive predecessors), and
// publishes the inclusive prefix. Returns the exclusive prefix. Wider windows let the
// inclusive prefixes propagate further per round trip to L2.
template <int PER_LANE>
__device__ __forceinline__ unsigned scan_lookback_w(unsigned long long* status, int tile,
                                                    unsigned aggregate, unsigned epoch,
                                                    unsigned* err, unsigned limit) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_relaxed_u64(&status[0], scan_pack(epoch, 2u, aggregate));
        return 0u;
    }
    if (lane == 0) st_relaxed_u64(&status[tile], scan_pack(epoch, 1u, aggregate));
    unsigned excl = 0u;
    int pred = tile - 1;
    unsigned spins = 0;
    while (true) {
        unsigned val[PER_LANE], flag[PER_LANE];
        while (true) {
#pragma unroll
            for (int k = 0; k < PER_LANE; k++) {
                const int idx = pred - (lane * PER_LANE + k);
                if (idx >= 0) {
                    const unsigned long long s = ld_relaxed_u64(&status[idx]);
                    flag[k] = ((unsigned)(s >> 34) == epoch) ? (unsigned)(s >> 32) & 3u : 0u;
                    val[k] = (unsigned)s;
                } else {
                    flag[k] = 2u;  // virtual tile -1: inclusive prefix 0
                    val[k] = 0u;
                }
            }
            // only the predecessors up to the nearest inclusive prefix matter: they must
            // all have published (aggregate or inclusive); those beyond it need not have
            int lane_p = PER_LANE;  // this lane's first inclusive entry
            bool gap_before_p = false, gap_any = false;
#pragma unroll
            for (int k = PER_LANE - 1; k >= 0; k--)
                if (flag[k] == 2u) lane_p = k;
#pragma unroll
            for (int k = 0; k < PER_LANE; k++) {
                gap_any = gap_any || flag[k] == 0u;
                gap_before_p = gap_before_p || (flag[k] == 0u && k < lane_p);
            }
            const unsigned with_p = __ballot_sync(HHS_FULL_MASK, lane_p < PER_LANE);
            const int first_p = with_p ? __ffs(with_p) - 1 : 32;
            const bool gap = lane < first_p ? gap_any : (lane == first_p ? gap_before_p : false);
            if (!__any_sync(HHS_FULL_MASK, gap)) break;
            if (++spins > limit) {
                if (lane == 0) atomicOr(err, HHS_ERRBIT_LOOKBACK_TIMEOUT);
#pragma unroll
                for (int k = 0; k < PER_LANE; k++)
                    if (flag[k] == 0u) { flag[k] = 2u; val[k] = 0u; }
                break;
            }
            if (spins > 64) __nanosleep(64);  // poll tightly first, then back off
        }
        // within this lane: values up to and including its first inclusive prefix
        int firstp = PER_LANE;
#pragma unroll
        for (int k = PER_LANE - 1; k >= 0; k--)
            if (flag[k] == 2u) firstp = k;
        unsigned mine = 0u;
#pragma unroll
        for (int k = 0; k < PER_LANE; k++)
            if (k <= firstp) mine += val[k];
        const unsigned pm = __ballot_sync(HHS_FULL_MASK, firstp < PER_LANE);
        if (pm) {
            const int first = __ffs(pm) - 1;
            excl += (unsigned)warp_sum((int)(lane <= first ? mine : 0u));
            break;
        }
        excl += (unsigned)warp_sum((int)mine);
        pred -= 32 * PER_LANE;
    }
    if (lane == 0) st_relaxed_u64(&status[tile], scan_pack(epoch, 2u, excl + aggregate));
    return excl;
}


// Tile layout shared by the scan kernels: BLOCK threads x ITEMS values; value k of
// chunk c of lane l in warp w sits at tile offset w*32*ITEMS + c*128 + l*4 + k, so a
// warp's chunk is 128 consecutive values (one 16-byte load per lane).
template <int BLOCK, int ITEMS, int LOOKBACK = 1>
struct TileScan {
    static constexpr int TILE = BLOCK * ITEMS;
    static constexpr int CHUNKS = ITEMS / 4;
    static constexpr int WARPS = BLOCK / 32;
    static_assert(ITEMS % 4 == 0, "ITEMS must be a multiple of 4");

    __device__ static __forceinline__ long long offset(int warp, int c, int lane) {
        return (long long)warp * (32 * ITEMS) + c * 128 + lane * 4;
    }

    // v: this thread's values. On return cbase[c] holds the exclusive prefix (within the
    // whole input, tile prefix from the look-back included) of the first value of chunk c;
    // the prefixes of the other values follow by adding v in order.
    __device__ static __forceinline__ void scan(const unsigned (&v)[ITEMS],
                                                unsigned (&cbase)[CHUNKS],
                                                unsigned long long* status, int tile,
                                                unsigned epoch, unsigned* err,
                                                unsigned* s_warp, unsigned* s_prefix,
                                                unsigned limit) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        unsigned run = 0u;
#pragma unroll
        for (int c = 0; c < CHUNKS; c++) {
            const unsigned s = v[4 * c] + v[4 * c + 1] + v[4 * c + 2] + v[4 * c + 3];
            const unsigned inc = (unsigned)warp_incl_scan((int)s, lane);
            cbase[c] = run + inc - s;
            run += (unsigned)__shfl_sync(HHS_FULL_MASK, (int)inc, 31);
        }
        if (lane == 0) s_warp[warp] = run;
        __syncthreads();
        if (warp == 0) {
            const unsigned wt = (lane < WARPS) ? s_warp[lane] : 0u;
            const unsigned wi = (unsigned)warp_incl_scan((int)wt, lane);
            const unsigned total = (unsigned)__shfl_sync(HHS_FULL_MASK, (int)wi, 31);
            const unsigned prefix =
                scan_lookback_w<LOOKBACK>(status, tile, total, epoch, err, limit);
            if (lane < WARPS) s_warp[lane] = wi - wt;
            if (lane == 0) *s_prefix = prefix;
        }
        __syncthreads();
        const unsigned base = *s_prefix + s_warp[warp];
#pragma unroll
        for (int c = 0; c < CHUNKS; c++) cbase[c] += base;
    }
};

// Fetches this CTA's tile index, the call's epoch and the look-back poll limit
// (thread 0), broadcast to all.
__device__ __forceinline__ void scan_begin(ScanHeader* hdr, int* s_tile, unsigned* s_epoch,
                                           unsigned* s_limit) {
    if (threadIdx.x == 0) {
        *s_tile = (int)atomicAdd(&hdr->tile_counter, 1u);
        *s_epoch = scan_next_epoch(hdr);
        const unsigned lim = *reinterpret_cast<volatile const unsigned*>(&hdr->spin_limit);
        *s_limit = lim ? lim : HHS_SPIN_LIMIT;
    }
    __syncthreads();
}

// Marks this CTA done; returns true (in every thread) for the last CTA to finish,
// whose view of all other CTAs' global writes is then complete.
__device__ __forceinline__ bool scan_finish_is_last(ScanHeader* hdr, int num_tiles,
                                                    int* s_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned prev = atomicAdd(&hdr->done_counter, 1u);
        *s_flag = (prev == (unsigned)num_tiles - 1u);
    }
    __syncthreads();
    const bool last = *s_flag != 0;
    if (last) __threadfence();
    return last;
}

// Resets the header for the next call (last CTA only, after its final reads).
__device__ __forceinline__ void scan_reset(ScanHeader* hdr, unsigned epoch) {
    if (threadIdx.x == 0) {
        hdr->tile_counter = 0u;
        hdr->done_counter = 0u;
        hdr->epoch = epoch;
    }
}
