// sort.cu -- COO -> CSR on the GPU: one-sweep LSD radix sort of packed
// (row<<32|col) keys with a 32-bit payload, plus the row_ptr count-and-scan.
//
// Replaces the reference's per-4-bit-digit pass loop
// (iterative/BiCGSTAB/spmv.cpp:62-228; coo_csr.metal:17-193).  Same result:
// a stable sort by (row, col) in which duplicate keys keep their input order,
// then CSR.  Different machinery, built for B200:
//   * keys are compacted to bits(n_rows-1)+bits(n_cols-1) bits and sorted with
//     8-bit digits (C1: 4 passes instead of the reference's 10);
//   * one histogram kernel computes every pass's digit counts and the row
//     counts in a single read of the keys;
//   * each pass is a single kernel: warp-ballot ranking into per-warp
//     histograms, a decoupled look-back across tiles (bounded spin), a local
//     shuffle through shared memory and a coalesced scatter;
//   * the first pass reads the packed keys directly and the last pass writes
//     col_ind (low bits) instead of keys, so no separate compress kernel;
//   * row_ptr is an exclusive scan of the row counts, so empty rows need no
//     fixer pass.
#include <atomic>
#include "common.cuh"
#include "internal.hpp"

namespace mps {
namespace {

constexpr int kSortNT = 256;
constexpr int kItems = 16;
constexpr int kTile = kSortNT * kItems;   // 4096 keys per tile
constexpr int kWarps = kSortNT / 32;

struct KeyShape {
    unsigned long long row_mask, col_mask;
    int col_bits;
    uint32_t n_rows, n_cols;
};

__device__ __forceinline__ unsigned long long compact_key(unsigned long long k, const KeyShape& ks) {
    unsigned long long r = (k >> 32) & ks.row_mask;
    unsigned long long c = k & ks.col_mask;
    return (r << ks.col_bits) | c;
}

// ---- pass 0: digit histograms of every pass + row counts + range check ----
__global__ void __launch_bounds__(kSortNT)
sort_histogram(const unsigned long long* __restrict__ keys, uint64_t nnz, KeyShape ks, int passes,
               unsigned* __restrict__ hist, unsigned* __restrict__ row_cnt, unsigned* err) {
    __shared__ unsigned sh[8 * 256];
    for (int i = threadIdx.x; i < passes * 256; i += kSortNT) sh[i] = 0;
    __syncthreads();
    bool bad = false;
    for (uint64_t i = (uint64_t)blockIdx.x * kSortNT + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * kSortNT) {
        unsigned long long k = __ldcs(keys + i);
        uint32_t row = (uint32_t)(k >> 32), col = (uint32_t)k;
        if (row < ks.n_rows && col < ks.n_cols) {
            atomicAdd(row_cnt + row, 1u);
        } else {
            bad = true;
        }
        unsigned long long ck = compact_key(k, ks);
        for (int p = 0; p < passes; ++p) atomicAdd(&sh[p * 256 + ((ck >> (8 * p)) & 255u)], 1u);
    }
    if (bad) atomicOr(err, kErrRange);
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kSortNT) {
        unsigned c = sh[i];
        if (c) atomicAdd(hist + i, c);
    }
}

// Exclusive scan of each pass's 256 digit counts (one CTA).
__global__ void __launch_bounds__(256)
sort_digit_bases(const unsigned* __restrict__ hist, unsigned* __restrict__ base, int passes) {
    __shared__ unsigned wsum[8];
    for (int p = 0; p < passes; ++p) {
        unsigned v = hist[p * 256 + threadIdx.x];
        unsigned inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned t = __shfl_up_sync(kFull, inc, o);
            if (lane_id() >= (unsigned)o) inc += t;
        }
        if (lane_id() == 31) wsum[threadIdx.x >> 5] = inc;
        __syncthreads();
        unsigned off = 0;
        for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) off += wsum[w];
        base[p * 256 + threadIdx.x] = off + inc - v;
        __syncthreads();
    }
}

// Block-wide exclusive scan over 256 threads (one value each).
__device__ __forceinline__ unsigned block_excl_scan_256(unsigned v, unsigned* wsum) {
    unsigned inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned t = __shfl_up_sync(kFull, inc, o);
        if (lane_id() >= (unsigned)o) inc += t;
    }
    if (lane_id() == 31) wsum[threadIdx.x >> 5] = inc;
    __syncthreads();
    unsigned off = 0;
    for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) off += wsum[w];
    __syncthreads();
    return off + inc - v;
}

// Look-back status word: epoch (bits 34+, the pass number + 1) | flag (bits
// 32-33: 1 aggregate, 2 inclusive prefix) | count.  A word counts only in the
// pass whose epoch it carries, so the array is zeroed once per sort, not once
// per pass.
constexpr unsigned long long kFlagAgg = 1ull << 32;
constexpr unsigned long long kFlagPrefix = 2ull << 32;
constexpr int kEpochShift = 34;

struct SortSmem {
    unsigned long long keys[kTile];
    unsigned vals[kTile];
    unsigned whist[kWarps][256];
    unsigned dstart[256];
    unsigned gbase[256];
    unsigned wsum[8];
    unsigned tile;
};

// One LSD pass.  FIRST: input keys are packed (row<<32|col) and are compacted
// on load.  LAST: the output is col_ind (low col_bits of the compact key).
template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(kSortNT, 3)
sort_onesweep(const unsigned long long* __restrict__ kin, const unsigned* __restrict__ vin,
              unsigned long long* __restrict__ kout, int32_t* __restrict__ col_out,
              unsigned* __restrict__ vout, uint64_t nnz, KeyShape ks, int shift,
              const unsigned* __restrict__ digit_base, unsigned long long* status,
              unsigned* tile_counter, unsigned* err, unsigned spin_limit, unsigned silent_tile,
              unsigned epoch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem& S = *reinterpret_cast<SortSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;

    if (tid == 0) S.tile = atomicAdd(tile_counter, 1u);
    for (int i = lane; i < 256; i += 32) S.whist[w][i] = 0;
    __syncthreads();
    const unsigned tile = S.tile;
    const uint64_t tile_base = (uint64_t)tile * kTile;
    const uint64_t warp_base = tile_base + (uint64_t)w * (kItems * 32);
    const uint64_t left = nnz - tile_base;
    const int tile_items = left < (uint64_t)kTile ? (int)left : kTile;

    unsigned long long key[kItems];
    unsigned val[kItems];
    unsigned rank[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        uint64_t idx = warp_base + (uint64_t)j * 32 + lane;
        if (idx < nnz) {
            unsigned long long k = __ldcs(kin + idx);
            key[j] = FIRST ? compact_key(k, ks) : k;
            val[j] = __ldcs(vin + idx);
        } else {
            key[j] = 0;
            val[j] = 0;
        }
    }
    // Warp-level stable ranking by 8-bit digit: peers = lanes with the same
    // digit (8 ballots), the lowest peer updates the warp histogram.
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        uint64_t idx = warp_base + (uint64_t)j * 32 + lane;
        const bool valid = idx < nnz;
        const unsigned d = (unsigned)(key[j] >> shift) & 255u;
        unsigned peers = __ballot_sync(kFull, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const bool bit = (d >> b) & 1u;
            const unsigned bal = __ballot_sync(kFull, bit);
            peers &= bit ? bal : ~bal;
        }
        const int leader = valid ? __ffs(peers) - 1 : lane;
        unsigned before = 0;
        if (valid && lane == leader) {
            before = S.whist[w][d];
            S.whist[w][d] = before + __popc(peers);
        }
        before = __shfl_sync(kFull, before, leader);
        rank[j] = before + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    // Per digit (thread = digit): warp-exclusive offsets and the tile count.
    unsigned total = 0;
#pragma unroll
    for (int ww = 0; ww < kWarps; ++ww) {
        unsigned c = S.whist[ww][tid];
        S.whist[ww][tid] = total;
        total += c;
    }
    // Decoupled look-back for digit `tid` across earlier tiles.  Each wait is
    // bounded (spin_limit polls): on a timeout the error word is set and the
    // tile publishes what it has, so no later tile waits on it in turn.
    // silent_tile (only ever set by the timeout test hook) names a tile that
    // publishes nothing, so that the waits of the tiles after it run out.
    unsigned long long* st = status + (size_t)tile * 256 + tid;
    const bool publish = tile != silent_tile;
    const unsigned long long ep = (unsigned long long)epoch << kEpochShift;
    unsigned excl = 0;
    if (tile == 0) {
        if (publish) st_relaxed_u64(st, ep | kFlagPrefix | total);
    } else {
        if (publish) st_relaxed_u64(st, ep | kFlagAgg | total);
        long look = (long)tile - 1;
        unsigned spins = 0;
        while (look >= 0) {
            unsigned long long s = ld_relaxed_u64(status + (size_t)look * 256 + tid);
            const unsigned flag = (s >> kEpochShift) == epoch ? (unsigned)(s >> 32) & 3u : 0u;
            if (flag == 0) {
                if (++spins > spin_limit) {
                    atomicOr(err, kErrTimeout);
                    break;
                }
                if (spins > 32) __nanosleep(64);
                continue;
            }
            excl += (unsigned)s;
            if (flag == 2) break;
            --look;
        }
        if (publish) st_relaxed_u64(st, ep | kFlagPrefix | (unsigned long long)(excl + total));
    }
    const unsigned dstart = block_excl_scan_256(total, S.wsum);
    S.dstart[tid] = dstart;
    S.gbase[tid] = digit_base[tid] + excl;
    __syncthreads();
    // Local shuffle into digit order.
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        uint64_t idx = warp_base + (uint64_t)j * 32 + lane;
        if (idx < nnz) {
            const unsigned d = (unsigned)(key[j] >> shift) & 255u;
            const unsigned lp = S.dstart[d] + S.whist[w][d] + rank[j];
            S.keys[lp] = key[j];
            S.vals[lp] = val[j];
        }
    }
    __syncthreads();
    // Coalesced scatter: runs of equal digits land on consecutive addresses.
    for (int i = tid; i < tile_items; i += kSortNT) {
        const unsigned long long k = S.keys[i];
        const unsigned d = (unsigned)(k >> shift) & 255u;
        const size_t g = (size_t)S.gbase[d] + (unsigned)(i - S.dstart[d]);
        if (LAST)
            col_out[g] = (int32_t)(uint32_t)(k & ks.col_mask);
        else
            kout[g] = k;
        vout[g] = S.vals[i];
    }
}

// ---- exclusive scan of the row counts into row_ptr --------------------------
constexpr int kScanNT = 256, kScanItems = 8, kScanTile = kScanNT * kScanItems;

__global__ void __launch_bounds__(kScanNT)
scan_reduce(const unsigned* __restrict__ in, uint64_t n, unsigned* __restrict__ bsum) {
    __shared__ unsigned sh[kScanNT / 32];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    unsigned s = 0;
    for (int j = 0; j < kScanItems; ++j) {
        uint64_t i = base + (uint64_t)j * kScanNT + threadIdx.x;
        if (i < n) s += in[i];
    }
    s = block_sum<kScanNT>(s, sh);
    if (threadIdx.x == 0) bsum[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) scan_bsums(unsigned* bsum, int nb) {
    __shared__ unsigned wsum[8];
    __shared__ unsigned carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 256) {
        int i = base + threadIdx.x;
        unsigned v = i < nb ? bsum[i] : 0;
        unsigned e = block_excl_scan_256(v, wsum);
        unsigned c = carry;
        __syncthreads();
        if (i < nb) bsum[i] = c + e;
        if (threadIdx.x == 255) carry = c + e + v;
        __syncthreads();
    }
}

// out[i] = sum_{j<i} in[j] for i in [0, n]; in[n] is taken as 0.
__global__ void __launch_bounds__(kScanNT)
scan_apply(const unsigned* __restrict__ in, uint64_t n, const unsigned* __restrict__ bsum,
           int32_t* __restrict__ out) {
    __shared__ unsigned wsum[8];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    unsigned v[kScanItems];
    unsigned s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        uint64_t i = base + j;
        v[j] = i < n ? in[i] : 0u;
        s += v[j];
    }
    unsigned e = block_excl_scan_256(s, wsum) + bsum[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        uint64_t i = base + j;
        if (i <= n) out[i] = (int32_t)e;
        e += v[j];
    }
}

int bit_width(uint32_t v) { return v ? 32 - __builtin_clz(v) : 0; }

}  // namespace

cudaError_t exclusive_scan_rows(const unsigned* counts, uint64_t n, int32_t* out, unsigned* bsum,
                                cudaStream_t s) {
    const uint64_t total = n + 1;
    const int nb = (int)((total + kScanTile - 1) / kScanTile);
    scan_reduce<<<nb, kScanNT, 0, s>>>(counts, n, bsum);
    scan_bsums<<<1, 256, 0, s>>>(bsum, nb);
    scan_apply<<<nb, kScanNT, 0, s>>>(counts, n, bsum, out);
    return cudaGetLastError();
}

cudaError_t sort_to_csr(const uint64_t* keys, const uint32_t* payload, uint64_t nnz,
                        uint32_t n_rows, uint32_t n_cols, int32_t* row_ptr, int32_t* col_out,
                        uint32_t* payload_out, unsigned* d_err, cudaStream_t s,
                        unsigned spin_limit, unsigned silent_tile) {
    if (spin_limit == 0) spin_limit = kSpinLimit;
    const int rb = bit_width(n_rows ? n_rows - 1 : 0), cb = bit_width(n_cols ? n_cols - 1 : 0);
    const int bits = rb + cb;
    const int passes = bits > 0 ? (bits + 7) / 8 : 1;
    KeyShape ks;
    ks.row_mask = rb ? ((1ull << rb) - 1) : 0;
    ks.col_mask = cb ? ((1ull << cb) - 1) : 0;
    ks.col_bits = cb;
    ks.n_rows = n_rows;
    ks.n_cols = n_cols;

    const uint64_t ntiles = nnz ? (nnz + kTile - 1) / kTile : 0;
    const int nb_scan = (int)((n_rows + 1 + kScanTile - 1) / kScanTile);
    // Temporary layout (one allocation).
    size_t off = 0;
    auto carve = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    const size_t o_hist = carve(8 * 256 * 4), o_base = carve(8 * 256 * 4), o_ctr = carve(8 * 4);
    const size_t o_rows = carve((size_t)n_rows * 4), o_bsum = carve((size_t)nb_scan * 4);
    const size_t o_status = carve(ntiles * 256 * 8);
    const size_t o_k0 = carve(nnz * 8), o_k1 = carve(nnz * 8), o_v0 = carve(nnz * 4),
                 o_v1 = carve(nnz * 4);
    unsigned char* tmp = nullptr;
    cudaError_t e = stream_alloc(&tmp, off, s);
    if (e != cudaSuccess) return e;
    unsigned* hist = (unsigned*)(tmp + o_hist);
    unsigned* base = (unsigned*)(tmp + o_base);
    unsigned* ctr = (unsigned*)(tmp + o_ctr);
    unsigned* rows = (unsigned*)(tmp + o_rows);
    unsigned* bsum = (unsigned*)(tmp + o_bsum);
    unsigned long long* status = (unsigned long long*)(tmp + o_status);
    unsigned long long* kb[2] = {(unsigned long long*)(tmp + o_k0), (unsigned long long*)(tmp + o_k1)};
    unsigned* vb[2] = {(unsigned*)(tmp + o_v0), (unsigned*)(tmp + o_v1)};

    // hist, base, ctr and the row counts are contiguous from offset 0.
    e = cudaMemsetAsync(tmp, 0, o_bsum, s);
    if (e != cudaSuccess) goto out;
    if (nnz) {
        int grid = num_sms() * 8;
        uint64_t need = (nnz + kSortNT - 1) / kSortNT;
        if ((uint64_t)grid > need) grid = (int)need;
        sort_histogram<<<grid, kSortNT, 0, s>>>((const unsigned long long*)keys, nnz, ks, passes,
                                                hist, rows, d_err);
        sort_digit_bases<<<1, 256, 0, s>>>(hist, base, passes);
        const size_t smem = sizeof(SortSmem);
        // the shared-memory opt-in is a per-device function attribute
        static std::atomic<unsigned long long> attr_done{0};
        int dev = 0;
        cudaGetDevice(&dev);
        const unsigned long long bit = dev >= 0 && dev < 64 ? 1ull << dev : 0ull;
        if (!bit || !(attr_done.load() & bit)) {
            // three CTAs per SM (80 registers, 3 x 59 KB): the largest
            // shared-memory carve-out
            auto opt_in = [&](const void* k) {
                cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared);
            };
            opt_in(reinterpret_cast<const void*>(sort_onesweep<true, true>));
            opt_in(reinterpret_cast<const void*>(sort_onesweep<true, false>));
            opt_in(reinterpret_cast<const void*>(sort_onesweep<false, true>));
            opt_in(reinterpret_cast<const void*>(sort_onesweep<false, false>));
            attr_done.fetch_or(bit);
        }
        const unsigned long long* kin = (const unsigned long long*)keys;
        const unsigned* vin = payload;
        e = cudaMemsetAsync(status, 0, ntiles * 256 * 8, s);   // epoch 0: no pass's
        if (e != cudaSuccess) goto out;
        for (int p = 0; p < passes; ++p) {
            const bool first = p == 0, last = p == passes - 1;
            unsigned long long* ko = kb[p & 1];
            unsigned* vo = last ? payload_out : vb[p & 1];
            const unsigned* db = base + p * 256;
            const int sh = 8 * p;
            if (first && last)
                sort_onesweep<true, true><<<(unsigned)ntiles, kSortNT, smem, s>>>(
                    kin, vin, ko, col_out, vo, nnz, ks, sh, db, status, ctr + p, d_err, spin_limit, silent_tile,
                    (unsigned)(p + 1));
            else if (first)
                sort_onesweep<true, false><<<(unsigned)ntiles, kSortNT, smem, s>>>(
                    kin, vin, ko, col_out, vo, nnz, ks, sh, db, status, ctr + p, d_err, spin_limit, silent_tile,
                    (unsigned)(p + 1));
            else if (last)
                sort_onesweep<false, true><<<(unsigned)ntiles, kSortNT, smem, s>>>(
                    kin, vin, ko, col_out, vo, nnz, ks, sh, db, status, ctr + p, d_err, spin_limit, silent_tile,
                    (unsigned)(p + 1));
            else
                sort_onesweep<false, false><<<(unsigned)ntiles, kSortNT, smem, s>>>(
                    kin, vin, ko, col_out, vo, nnz, ks, sh, db, status, ctr + p, d_err, spin_limit, silent_tile,
                    (unsigned)(p + 1));
            kin = ko;
            vin = vo;
        }
    }
    e = exclusive_scan_rows(rows, n_rows, row_ptr, bsum, s);
out:
    cudaError_t e2 = cudaFreeAsync(tmp, s);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

}  // namespace mps
