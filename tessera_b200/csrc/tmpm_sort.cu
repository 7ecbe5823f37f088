// tmpm_sort.cu -- stable LSD radix sort of (u32 key, u32 value) pairs.
//
// Used to bring particles into block order (Morton key of their 4^3 block).
// Each 8-bit pass is three kernels:
//   k_hist    per-tile digit histogram (tile = 4096 keys), digit-major layout
//   k_scan    per-digit exclusive scan over tiles + digit totals
//   k_scatter stable scatter: each warp ranks 32 keys at a time with
//             __match_any_sync, so equal digits keep their input order.

#include "tmpm_internal.h"

namespace tmpm {

namespace {

constexpr int kSortThreads = 256;
constexpr int kItemsPerThread = 16;
constexpr int kTile = kSortThreads * kItemsPerThread;  // 4096
constexpr int kWarps = kSortThreads / 32;
constexpr int kWarpItems = kTile / kWarps;  // 512 contiguous keys per warp

__global__ void __launch_bounds__(kSortThreads) k_hist(const uint32_t *__restrict__ keys, int n, int shift,
                                                       uint32_t *hist, int tiles) {
    __shared__ uint32_t counts[256];
    counts[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kTile;
#pragma unroll 4
    for (int j = 0; j < kItemsPerThread; ++j) {
        int idx = base + j * kSortThreads + threadIdx.x;
        if (idx < n) atomicAdd(&counts[(keys[idx] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    hist[static_cast<size_t>(threadIdx.x) * tiles + blockIdx.x] = counts[threadIdx.x];
}

// One CTA per digit: exclusive scan of hist[d][0..tiles) in place; totals[d] = sum.
__global__ void __launch_bounds__(kSortThreads) k_scan(uint32_t *hist, int tiles, uint32_t *totals) {
    __shared__ uint32_t warp_sums[kWarps];
    __shared__ uint32_t carry;
    uint32_t *row = hist + static_cast<size_t>(blockIdx.x) * tiles;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int start = 0; start < tiles; start += kSortThreads) {
        int idx = start + threadIdx.x;
        uint32_t v = idx < tiles ? row[idx] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += t;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        uint32_t warp_prefix = 0, chunk_total = 0;
        for (int w = 0; w < kWarps; ++w) {
            if (w < warp) warp_prefix += warp_sums[w];
            chunk_total += warp_sums[w];
        }
        uint32_t c = carry;
        if (idx < tiles) row[idx] = c + warp_prefix + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry = c + chunk_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(kSortThreads) k_scatter(const uint32_t *__restrict__ keys_in,
                                                          const uint32_t *__restrict__ vals_in, uint32_t *keys_out,
                                                          uint32_t *vals_out, int n, int shift,
                                                          const uint32_t *__restrict__ hist, int tiles,
                                                          const uint32_t *__restrict__ totals) {
    __shared__ uint32_t digit_base[256];
    __shared__ uint32_t wcount[kWarps][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // exclusive scan of the 256 digit totals (each CTA redoes this small scan)
    {
        uint32_t v = totals[threadIdx.x];
        uint32_t incl = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += t;
        }
        __shared__ uint32_t sums[kWarps];
        if (lane == 31) sums[warp] = incl;
        __syncthreads();
        uint32_t pre = 0;
        for (int w = 0; w < warp; ++w) pre += sums[w];
        digit_base[threadIdx.x] = pre + incl - v + hist[static_cast<size_t>(threadIdx.x) * tiles + blockIdx.x];
        for (int w = 0; w < kWarps; ++w) wcount[w][threadIdx.x] = 0;
    }
    __syncthreads();

    const int base = blockIdx.x * kTile + warp * kWarpItems;
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t k_reg[kItemsPerThread], v_reg[kItemsPerThread], r_reg[kItemsPerThread];
#pragma unroll
    for (int r = 0; r < kItemsPerThread; ++r) {
        int idx = base + r * 32 + lane;
        bool ok = idx < n;
        uint32_t key = ok ? keys_in[idx] : 0u;
        uint32_t digit = ok ? ((key >> shift) & 0xFFu) : 256u;
        unsigned peers = __match_any_sync(0xffffffffu, digit);
        uint32_t before = 0;
        if (ok) before = wcount[warp][digit];
        __syncwarp();
        int leader = __ffs(peers) - 1;
        if (ok && lane == leader) wcount[warp][digit] = before + __popc(peers);
        __syncwarp();
        k_reg[r] = key;
        v_reg[r] = ok ? vals_in[idx] : 0u;
        r_reg[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    // exclusive scan over warps, per digit
    {
        uint32_t run = 0;
        for (int w = 0; w < kWarps; ++w) {
            uint32_t c = wcount[w][threadIdx.x];
            wcount[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kItemsPerThread; ++r) {
        int idx = base + r * 32 + lane;
        if (idx >= n) continue;
        uint32_t digit = (k_reg[r] >> shift) & 0xFFu;
        uint32_t pos = digit_base[digit] + wcount[warp][digit] + r_reg[r];
        keys_out[pos] = k_reg[r];
        vals_out[pos] = v_reg[r];
    }
}

}  // namespace

int radix_sort_pairs(SortBuffers &sb, int n, int bits, cudaStream_t stream) {
    if (n <= 0) return 0;
    const int tiles = (n + kTile - 1) / kTile;
    int cur = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        k_hist<<<tiles, kSortThreads, 0, stream>>>(sb.keys[cur], n, shift, sb.hist, tiles);
        k_scan<<<256, kSortThreads, 0, stream>>>(sb.hist, tiles, sb.totals);
        k_scatter<<<tiles, kSortThreads, 0, stream>>>(sb.keys[cur], sb.vals[cur], sb.keys[cur ^ 1], sb.vals[cur ^ 1], n,
                                                      shift, sb.hist, tiles, sb.totals);
        cur ^= 1;
    }
    return cur;
}

}  // namespace tmpm
