// Near-field kernels: block application (every matvec) and, at setup, the
// near-field entries and radiation patterns.  Included once, by kernels.cu.
#pragma once

#include "common.hpp"
#include "device.cuh"
#include "zmath.cuh"
#include "bulk_copy.cuh"

namespace mlfma {
namespace {

// ------------------------------------------------------------ apply
// y = Z x for the near field (Leaf::evalPairSols, evalNearNonNborSols and
// evalSelfSols, src/fmm/leaf.cpp:318-383; C k is applied when the result is
// written out).  The reference stores each block once and applies it as Z and
// Z^T.
//
// Symmetric form (one right-hand side): every stored block is read once, in
// tiles (NearTile in plan.hpp), and gives both its row sums (Z x, to the
// block's rows) and its column sums (Z^T x, to its columns), as the reference
// applies each block (Leaf::evalPairSols, src/fmm/leaf.cpp:329-354; a self
// block strict-lower packed, Leaf::evalSelfSols, leaf.cpp:361-380).
//
// Persistent thread blocks, warp-specialised, a kSymStages-deep ring of
// shared-memory stages per block.  Warp 0 (producer) fills a stage with bulk
// asynchronous copies (cp.async.bulk on the TMA engine, no multicast): a tile
// of whole rows is one contiguous span of the block storage and moves in one
// copy of up to 16 KB (a tile of a wide or large self block moves row by row),
// plus one copy each for the tile's column and row values of x and for the
// slots of its partials, all counted on the stage's "full" mbarrier.  It reads
// the tile headers a batch of 32 ahead, so no global load stands between two
// tiles.  Warps 1-4 (consumers) compute from shared memory: 64 threads the row
// sums, 64 the column sums (two threads per row or column when the tile has
// at most 32; the diagonal of a self tile counts once, in its row), release the
// stage on its "empty" mbarrier and write the partials to their slots.
// k_near_reduce then adds each target's consecutive slots in a fixed order: no
// atomics, a deterministic product.  HBM traffic: the block entries once (half
// the block-row form), x from L2.
//
// Every mbarrier wait is bounded (about a second).  A consumer group that gives
// up sets *err and returns; so does the producer, after bounded waits for the
// copies it still has in flight.
constexpr int kSymConsumers = 128;
constexpr int kSymThreads = 32 + kSymConsumers;
constexpr int kSymStages = 2;
constexpr int kSymXc = kNearTileEntries;  // entry offsets within a stage
constexpr int kSymXr = kSymXc + kNearTileCols;
constexpr int kSymSlot = kSymXr + kNearTileRows;
constexpr int kSymStageEntries = kSymSlot + (kNearTileRows + kNearTileCols) * 4 / 16;
constexpr size_t kSymSmemBytes = sizeof(double2) * kSymStageEntries * kSymStages;
static_assert(kNearTileCols == 64 && kNearTileRows == 64, "k_near_sym maps 64 row and 64 column threads");
static_assert(kNearTileRowsSplit <= 32, "a mode-2 tile's rows are copied by one lane each");
static_assert((kSymStageEntries * sizeof(double2)) % 16 == 0, "bulk copies need 16-byte aligned stages");

__device__ __forceinline__ long long packed_row(int i, int kind) {
    return kind == 1 ? static_cast<long long>(i) * (i - 1) / 2 : static_cast<long long>(i) * (i + 1) / 2;
}

// Tile row r: its entries (from column j0 on) and where they start in the stage.
__device__ __forceinline__ int tile_row_len(const DevNearTile& T, int r) {
    if (T.kind == 0) return T.nj;
    return max(0, min(T.nj, T.i0 + r + (T.kind == 2 ? 1 : 0) - T.j0));
}
__device__ __forceinline__ int tile_row_start(const DevNearTile& T, int r) {
    return T.mode == 1 ? static_cast<int>(packed_row(T.i0 + r, T.kind) - packed_row(T.i0, T.kind)) : r * T.nj;
}
// First tile row holding an off-diagonal entry in tile column c.
__device__ __forceinline__ int tile_col_start(const DevNearTile& T, int c) {
    return T.kind == 0 ? 0 : max(0, T.j0 + c - T.i0 + 1);
}
// Entries the tile holds.
__device__ __forceinline__ int tile_entries(const DevNearTile& T) {
    return T.mode == 0 ? T.ni * T.nj : static_cast<int>(packed_row(T.i0 + T.ni, T.kind) - packed_row(T.i0, T.kind));
}

// OR of v over the consumer threads (named barrier 1), which all call it.
__device__ __forceinline__ bool consumers_any(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(static_cast<uint32_t>(v)), "n"(kSymConsumers)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void consumers_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(kSymConsumers) : "memory");
}

__global__ void __launch_bounds__(kSymThreads, 5)
k_near_sym(const DevNearTile* __restrict__ tiles, int ntiles, const double2* __restrict__ Z,
           const double2* __restrict__ x, const int* __restrict__ slots, double2* __restrict__ part,
           int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char sym_smem[];
    double2* stages = reinterpret_cast<double2*>(sym_smem);
    __shared__ __align__(8) unsigned long long full[kSymStages], empty[kSymStages];
    __shared__ DevNearTile hdr[kSymStages];
    __shared__ DevNearTile hbuf[32];  // producer's header batch
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int step = gridDim.x;
    if (tid == 0) {
        for (int s = 0; s < kSymStages; ++s) {
            mbar_init(smem_addr(&full[s]), 1);
            mbar_init(smem_addr(&empty[s]), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == 0) {  // ---- producer warp
        // Lane k holds the k-th header of the next batch in registers (loaded
        // a whole batch ahead) and parks it in hbuf when the batch starts.
        int it = 0;
        DevNearTile Tn{};
        if (blockIdx.x + lane * step < ntiles) Tn = tiles[blockIdx.x + lane * step];
        for (int t = blockIdx.x; t < ntiles; t += step, ++it) {
            if ((it & 31) == 0) {
                __syncwarp();
                hbuf[lane] = Tn;
                __syncwarp();
                const int tb = t + (32 + lane) * step;
                if (tb < ntiles) Tn = tiles[tb];
            }
            const DevNearTile T = hbuf[it & 31];
            const int s = it % kSymStages;
            if (it >= kSymStages && !mbar_wait_bounded(smem_addr(&empty[s]), ((it / kSymStages) - 1) & 1)) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    for (int k = 1; k <= kSymStages && k <= it; ++k)  // copies still in flight
                        mbar_wait_bounded(smem_addr(&full[(it - k) % kSymStages]), ((it - k) / kSymStages) & 1);
                }
                return;
            }
            double2* st = stages + static_cast<size_t>(s) * kSymStageEntries;
            int nv = 0, total;
            long long off = 0;
            if (T.mode == 2) {
                if (lane < T.ni) {
                    const int il = T.i0 + lane;
                    nv = tile_row_len(T, lane);
                    off = T.z + (T.kind == 0 ? static_cast<long long>(il) * T.ld : packed_row(il, T.kind)) + T.j0;
                }
                total = nv;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
            } else {
                total = tile_entries(T);
            }
            const int nslot = (T.ni + T.nj + 3) & ~3;
            const uint32_t bytes = static_cast<uint32_t>((total + T.nj + T.ni) * sizeof(double2) + nslot * sizeof(int));
            const uint32_t b = smem_addr(&full[s]);
            if (lane == 0) {
                hdr[s] = T;
                mbar_arrive_expect_tx(b, bytes);
            }
            __syncwarp();
            if (T.mode == 2) {
                if (nv > 0) bulk_load(smem_addr(st + lane * T.nj), Z + off, static_cast<uint32_t>(nv * sizeof(double2)), b);
            } else if (lane == 0) {
                bulk_load(smem_addr(st), Z + T.z, static_cast<uint32_t>(total * sizeof(double2)), b);
            }
            if (lane == 31) bulk_load(smem_addr(st + kSymXc), x + T.c0 + T.j0, static_cast<uint32_t>(T.nj * sizeof(double2)), b);
            if (lane == 30) bulk_load(smem_addr(st + kSymXr), x + T.r0 + T.i0, static_cast<uint32_t>(T.ni * sizeof(double2)), b);
            if (lane == 29) bulk_load(smem_addr(st + kSymSlot), slots + T.slot, static_cast<uint32_t>(nslot * sizeof(int)), b);
        }
        return;
    }

    // ---- consumers: threads 0-63 rows, 64-127 columns
    const int ct = tid - 32;
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += step, ++it) {
        const int s = it % kSymStages;
        const bool ok = mbar_wait_bounded(smem_addr(&full[s]), (it / kSymStages) & 1);
        if (consumers_any(!ok)) {
            if (ct == 0) atomicExch(err, 1);
            return;
        }
        const DevNearTile T = hdr[s];
        const double2* zt = stages + static_cast<size_t>(s) * kSymStageEntries;
        const double2* xc = zt + kSymXc;
        const double2* xr = zt + kSymXr;
        const int* sl = reinterpret_cast<const int*>(zt + kSymSlot);
        int my_slot = -1;
        double2 sum;
        if (ct < 64) {  // row sums: G adjacent lanes per row, G = 64 / rows rounded down to 1, 2, 4 or 8
            const int G = T.ni <= 8 ? 8 : T.ni <= 16 ? 4 : T.ni <= 32 ? 2 : 1;
            const int r = ct / G, h = ct & (G - 1);
            double2 a0 = z0(), a1 = z0(), a2 = z0(), a3 = z0();
            if (r < T.ni) {
                const int len = tile_row_len(T, r);
                const int seg = (len + G - 1) / G;
                const int k0 = min(len, h * seg), k1 = min(len, k0 + seg);
                const int L = k1 - k0;
                const double2* zr = zt + tile_row_start(T, r) + k0;
                const double2* xk = xc + k0;
                // rows nj apart with nj even share banks: start each row at its
                // own offset (any fixed order of the sum is as good)
                const int q = (T.mode != 1 && !(T.nj & 1) && L > 0) ? r % L : 0;
                int n = 0;
                for (; n + 3 < L; n += 4) {
                    int k = q + n;
                    k -= k >= L ? L : 0;
                    a0 = cfma(zr[k], xk[k], a0);
                    k = k + 1 == L ? 0 : k + 1;
                    a1 = cfma(zr[k], xk[k], a1);
                    k = k + 1 == L ? 0 : k + 1;
                    a2 = cfma(zr[k], xk[k], a2);
                    k = k + 1 == L ? 0 : k + 1;
                    a3 = cfma(zr[k], xk[k], a3);
                }
                for (; n < L; ++n) {
                    int k = q + n;
                    k -= k >= L ? L : 0;
                    a0 = cfma(zr[k], xk[k], a0);
                }
                if (h == 0) my_slot = sl[r];
            }
            sum = cadd(cadd(a0, a1), cadd(a2, a3));
            for (int o = G >> 1; o > 0; o >>= 1) {  // the row's G segments, a fixed order
                const double2 v = make_double2(__shfl_xor_sync(0xffffffffu, sum.x, o),
                                               __shfl_xor_sync(0xffffffffu, sum.y, o));
                sum = cadd(sum, v);
            }
        } else {  // column sums: G adjacent lanes per column, G = 64 / columns rounded down to 1, 2, 4 or 8
            const int cc = ct - 64;
            const int G = T.nj <= 8 ? 8 : T.nj <= 16 ? 4 : T.nj <= 32 ? 2 : 1;
            const int c = cc / G, h = cc & (G - 1);
            double2 a0 = z0(), a1 = z0(), a2 = z0(), a3 = z0();
            if (c < T.nj) {
                const int rs = tile_col_start(T, c);
                const int seg = (max(0, T.ni - rs) + G - 1) / G;
                const int ra = min(T.ni, rs + h * seg), rb = min(T.ni, ra + seg);
                // walk down the column: rows nj apart, or (packed) one longer each
                const int inc = T.mode == 1 ? 1 : 0;
                int stride = T.mode == 1 ? T.i0 + ra + (T.kind == 2 ? 1 : 0) : T.nj;
                const double2* zc = zt + tile_row_start(T, ra) + c;
                int r = ra;
                for (; r + 3 < rb; r += 4) {
                    a0 = cfma(*zc, xr[r], a0);
                    zc += stride;
                    stride += inc;
                    a1 = cfma(*zc, xr[r + 1], a1);
                    zc += stride;
                    stride += inc;
                    a2 = cfma(*zc, xr[r + 2], a2);
                    zc += stride;
                    stride += inc;
                    a3 = cfma(*zc, xr[r + 3], a3);
                    zc += stride;
                    stride += inc;
                }
                for (; r < rb; ++r) {
                    a0 = cfma(*zc, xr[r], a0);
                    zc += stride;
                    stride += inc;
                }
                if (h == 0) my_slot = sl[T.ni + c];
            }
            sum = cadd(cadd(a0, a1), cadd(a2, a3));
            for (int o = G >> 1; o > 0; o >>= 1) {
                const double2 v = make_double2(__shfl_xor_sync(0xffffffffu, sum.x, o),
                                               __shfl_xor_sync(0xffffffffu, sum.y, o));
                sum = cadd(sum, v);
            }
        }
        consumers_sync();  // stage s read by every consumer
        if (ct == 0) mbar_arrive(smem_addr(&empty[s]));
        if (my_slot >= 0) part[my_slot] = sum;
    }
}

// The same tiles, stages and partial slots with one consumer warp per tile:
// warp w of the kNwConsumers takes the block's tiles w, w + kNwConsumers, ...
// in its own two stages of the ring (no barrier between consumer warps).
// Lane l owns tile columns l and l + 32: their x values stay in registers and
// their column sums accumulate in registers over the whole tile.  Rows go in
// batches of eight: each lane forms its part of the eight row sums from the
// same entries it read for the column sums (every entry read from shared
// memory once), and a reduce-scatter over the warp (three halving exchanges,
// then two butterflies) leaves row rb + ((l >> 2) & 7) complete in lanes with
// l & 3 == 0.  A self tile's diagonal counts once, in its row.
constexpr int kNwConsumers = 4;
constexpr int kNwThreads = 32 * (1 + kNwConsumers);
constexpr int kNwStages = 2 * kNwConsumers;
constexpr size_t kNwSmemBytes = sizeof(double2) * kSymStageEntries * kNwStages;

__device__ __forceinline__ double2 shfl_xor2(double2 v, int m) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

__global__ void __launch_bounds__(kNwThreads, 1)
k_near_warp(const DevNearTile* __restrict__ tiles, int ntiles, const double2* __restrict__ Z,
            const double2* __restrict__ x, const int* __restrict__ slots, double2* __restrict__ part,
            int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char nw_smem[];
    double2* stages = reinterpret_cast<double2*>(nw_smem);
    __shared__ __align__(8) unsigned long long full[kNwStages], empty[kNwStages];
    __shared__ DevNearTile hdr[kNwStages];
    __shared__ DevNearTile hbuf[32];  // producer's header batch
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int step = gridDim.x;
    if (tid == 0) {
        for (int s = 0; s < kNwStages; ++s) {
            mbar_init(smem_addr(&full[s]), 1);
            mbar_init(smem_addr(&empty[s]), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == 0) {  // ---- producer warp: as in k_near_sym, over kNwStages stages
        int it = 0;
        DevNearTile Tn{};
        if (blockIdx.x + lane * step < ntiles) Tn = tiles[blockIdx.x + lane * step];
        for (int t = blockIdx.x; t < ntiles; t += step, ++it) {
            if ((it & 31) == 0) {
                __syncwarp();
                hbuf[lane] = Tn;
                __syncwarp();
                const int tb = t + (32 + lane) * step;
                if (tb < ntiles) Tn = tiles[tb];
            }
            const DevNearTile T = hbuf[it & 31];
            const int s = it % kNwStages;
            if (it >= kNwStages && !mbar_wait_bounded(smem_addr(&empty[s]), ((it / kNwStages) - 1) & 1)) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    for (int k = 1; k <= kNwStages && k <= it; ++k)  // copies still in flight
                        mbar_wait_bounded(smem_addr(&full[(it - k) % kNwStages]), ((it - k) / kNwStages) & 1);
                }
                return;
            }
            double2* st = stages + static_cast<size_t>(s) * kSymStageEntries;
            int nv = 0, total;
            long long off = 0;
            if (T.mode == 2) {
                if (lane < T.ni) {
                    const int il = T.i0 + lane;
                    nv = tile_row_len(T, lane);
                    off = T.z + (T.kind == 0 ? static_cast<long long>(il) * T.ld : packed_row(il, T.kind)) + T.j0;
                }
                total = nv;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
            } else {
                total = tile_entries(T);
            }
            const int nslot = (T.ni + T.nj + 3) & ~3;
            const uint32_t bytes = static_cast<uint32_t>((total + T.nj + T.ni) * sizeof(double2) + nslot * sizeof(int));
            const uint32_t b = smem_addr(&full[s]);
            if (lane == 0) {
                hdr[s] = T;
                mbar_arrive_expect_tx(b, bytes);
            }
            __syncwarp();
            if (T.mode == 2) {
                if (nv > 0) bulk_load(smem_addr(st + lane * T.nj), Z + off, static_cast<uint32_t>(nv * sizeof(double2)), b);
            } else if (lane == 0) {
                bulk_load(smem_addr(st), Z + T.z, static_cast<uint32_t>(total * sizeof(double2)), b);
            }
            if (lane == 31) bulk_load(smem_addr(st + kSymXc), x + T.c0 + T.j0, static_cast<uint32_t>(T.nj * sizeof(double2)), b);
            if (lane == 30) bulk_load(smem_addr(st + kSymXr), x + T.r0 + T.i0, static_cast<uint32_t>(T.ni * sizeof(double2)), b);
            if (lane == 29) bulk_load(smem_addr(st + kSymSlot), slots + T.slot, static_cast<uint32_t>(nslot * sizeof(int)), b);
        }
        return;
    }

    // ---- consumer warps
    const int cw = warp - 1;
    const int c0 = lane, c1 = lane + 32;
    for (int it = cw, t = blockIdx.x + cw * step; t < ntiles; it += kNwConsumers, t += kNwConsumers * step) {
        const int s = it % kNwStages;
        const bool ok = mbar_wait_bounded(smem_addr(&full[s]), (it / kNwStages) & 1);
        if (__any_sync(0xffffffffu, !ok)) {
            if (lane == 0) atomicExch(err, 1);
            return;
        }
        const DevNearTile T = hdr[s];
        const double2* zt = stages + static_cast<size_t>(s) * kSymStageEntries;
        const double2* xr = zt + kSymXr;
        const int* sl = reinterpret_cast<const int*>(zt + kSymSlot);
        const double2 xc0 = c0 < T.nj ? zt[kSymXc + c0] : z0();
        const double2 xc1 = c1 < T.nj ? zt[kSymXc + c1] : z0();
        // a row's entry at tile column c also enters column c's sum unless it is
        // on or above a self tile's diagonal
        const int dcol = T.j0 - T.i0;  // row r, column c is below the diagonal iff r > c + dcol
        double2 ca0 = z0(), ca1 = z0(), cb0 = z0(), cb1 = z0();
        for (int rb = 0; rb < T.ni; rb += 8) {
            double2 p[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int r = rb + j;
                double2 za = z0(), zb = z0(), xv = z0();
                if (r < T.ni) {
                    const int len = tile_row_len(T, r);
                    const double2* zr = zt + tile_row_start(T, r);
                    if (c0 < len) za = zr[c0];
                    if (c1 < len) zb = zr[c1];
                    xv = xr[r];
                }
                p[j] = cfma(za, xc0, cmul(zb, xc1));
                const bool ia = T.kind == 0 || r > c0 + dcol, ib = T.kind == 0 || r > c1 + dcol;
                if (j & 1) {
                    if (ia) cb0 = cfma(za, xv, cb0);
                    if (ib) cb1 = cfma(zb, xv, cb1);
                } else {
                    if (ia) ca0 = cfma(za, xv, ca0);
                    if (ib) ca1 = cfma(zb, xv, ca1);
                }
            }
            // reduce-scatter of p[0..7] over the warp
            const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4;
            double2 q[4], u[2], w;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double2 send = h4 ? p[k] : p[k + 4];
                const double2 keep = h4 ? p[k + 4] : p[k];
                q[k] = cadd(keep, shfl_xor2(send, 16));
            }
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const double2 send = h3 ? q[k] : q[k + 2];
                const double2 keep = h3 ? q[k + 2] : q[k];
                u[k] = cadd(keep, shfl_xor2(send, 8));
            }
            {
                const double2 send = h2 ? u[0] : u[1];
                const double2 keep = h2 ? u[1] : u[0];
                w = cadd(keep, shfl_xor2(send, 4));
            }
            w = cadd(w, shfl_xor2(w, 1));
            w = cadd(w, shfl_xor2(w, 2));
            const int r = rb + ((lane >> 2) & 7);
            if ((lane & 3) == 0 && r < T.ni) {
                const int slot = sl[r];
                if (slot >= 0) part[slot] = w;
            }
        }
        if (c0 < T.nj && sl[T.ni + c0] >= 0) part[sl[T.ni + c0]] = cadd(ca0, cb0);
        if (c1 < T.nj && sl[T.ni + c1] >= 0) part[sl[T.ni + c1]] = cadd(ca1, cb1);
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_addr(&empty[s]));
    }
}

// The same tiles and partial slots read straight from global memory into
// registers: no shared-memory stage and no producer warp, so residency is set
// by registers alone.  Warp w of the grid takes tiles w, w + (warps in the
// grid), ...; per tile, lane l owns columns l and l + 32 (x values and column
// sums in registers), rows go in batches of eight (each lane loads its one or
// two entries of each of the eight rows: coalesced 16-byte loads, all sixteen
// issued before use) and the row sums are formed by the reduce-scatter of
// k_near_warp.  A self tile's diagonal counts once, in its row.
constexpr int kNdThreads = 128;

__device__ __forceinline__ long long tile_row_global(const DevNearTile& T, int r) {
    if (T.mode == 0) return T.z + static_cast<long long>(r) * T.nj;
    if (T.mode == 1) return T.z + packed_row(T.i0 + r, T.kind) - packed_row(T.i0, T.kind);
    const int il = T.i0 + r;
    return T.z + (T.kind == 0 ? static_cast<long long>(il) * T.ld : packed_row(il, T.kind)) + T.j0;
}

__global__ void __launch_bounds__(kNdThreads)
k_near_direct(const DevNearTile* __restrict__ tiles, int ntiles, const double2* __restrict__ Z,
              const double2* __restrict__ x, const int* __restrict__ slots, double2* __restrict__ part) {
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (kNdThreads / 32);
    const int c0 = lane, c1 = lane + 32;
    for (int t = blockIdx.x * (kNdThreads / 32) + (threadIdx.x >> 5); t < ntiles; t += nwarps) {
        const DevNearTile T = tiles[t];
        const double2* xr = x + T.r0 + T.i0;
        const int* sl = slots + T.slot;
        const double2 xc0 = c0 < T.nj ? x[T.c0 + T.j0 + c0] : z0();
        const double2 xc1 = c1 < T.nj ? x[T.c0 + T.j0 + c1] : z0();
        const int dcol = T.j0 - T.i0;  // row r, column c is below the diagonal iff r > c + dcol
        double2 ca0 = z0(), ca1 = z0(), cb0 = z0(), cb1 = z0();
        for (int rb = 0; rb < T.ni; rb += 8) {
            double2 za[8], zb[8], xv[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int r = rb + j;
                za[j] = z0();
                zb[j] = z0();
                xv[j] = z0();
                if (r < T.ni) {
                    const int len = tile_row_len(T, r);
                    const double2* zr = Z + tile_row_global(T, r);
                    if (c0 < len) za[j] = __ldcs(zr + c0);
                    if (c1 < len) zb[j] = __ldcs(zr + c1);
                    xv[j] = xr[r];
                }
            }
            double2 p[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int r = rb + j;
                p[j] = cfma(za[j], xc0, cmul(zb[j], xc1));
                const bool ia = T.kind == 0 || r > c0 + dcol, ib = T.kind == 0 || r > c1 + dcol;
                if (j & 1) {
                    if (ia) cb0 = cfma(za[j], xv[j], cb0);
                    if (ib) cb1 = cfma(zb[j], xv[j], cb1);
                } else {
                    if (ia) ca0 = cfma(za[j], xv[j], ca0);
                    if (ib) ca1 = cfma(zb[j], xv[j], ca1);
                }
            }
            // reduce-scatter of p[0..7] over the warp (as in k_near_warp)
            const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4;
            double2 q[4], u[2], w;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double2 send = h4 ? p[k] : p[k + 4];
                const double2 keep = h4 ? p[k + 4] : p[k];
                q[k] = cadd(keep, shfl_xor2(send, 16));
            }
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const double2 send = h3 ? q[k] : q[k + 2];
                const double2 keep = h3 ? q[k + 2] : q[k];
                u[k] = cadd(keep, shfl_xor2(send, 8));
            }
            {
                const double2 send = h2 ? u[0] : u[1];
                const double2 keep = h2 ? u[1] : u[0];
                w = cadd(keep, shfl_xor2(send, 4));
            }
            w = cadd(w, shfl_xor2(w, 1));
            w = cadd(w, shfl_xor2(w, 2));
            const int r = rb + ((lane >> 2) & 7);
            if ((lane & 3) == 0 && r < T.ni) {
                const int slot = sl[r];
                if (slot >= 0) part[slot] = w;
            }
        }
        if (c0 < T.nj) {
            const int slot = sl[T.ni + c0];
            if (slot >= 0) part[slot] = cadd(ca0, cb0);
        }
        if (c1 < T.nj) {
            const int slot = sl[T.ni + c1];
            if (slot >= 0) part[slot] = cadd(ca1, cb1);
        }
    }
}

// y[t] = sum of target t's consecutive partial slots: eight lanes per target,
// a fixed shuffle tree, so the order never changes.
constexpr int kReduceLanes = 8;

__global__ void k_near_reduce(const int* __restrict__ ptr, const double2* __restrict__ part, int n,
                              double2* __restrict__ y) {
    const long long g = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int t = static_cast<int>(g / kReduceLanes);
    const int l = static_cast<int>(g % kReduceLanes);
    double2 acc = z0();
    if (t < n) {
        const int p0 = ptr[t] + l, p1 = ptr[t + 1];
        double2 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = p0 + u * kReduceLanes < p1 ? part[p0 + u * kReduceLanes] : z0();
        acc = cadd(cadd(v[0], v[1]), cadd(v[2], v[3]));
        for (int p = p0 + 4 * kReduceLanes; p < p1; p += kReduceLanes) acc = cadd(acc, part[p]);
    }
#pragma unroll
    for (int o = kReduceLanes / 2; o > 0; o >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
    }
    if (t < n && l == 0) y[t] = acc;
}

// ------------------------------------------------------------ setup kernels
struct DevFarLeafGeom {
    double c[3];
};

// Radiation patterns R_n(dir) = T(dir) . e_n(dir) (Leaf::buildRadPats,
// src/fmm/leaf.cpp:185-207) with e_n = e^{ik khat.(c - r_n)} phat_n for a
// dipole (Dipole::getRadAlongDir, src/sources/dipole.h:47-51) and
// e^{ik khat.c} conj(I_n(k khat)) for an RWG (src/sources/rwg.h:23-25).
__global__ void k_patterns(const DevGeomLevel* __restrict__ lvs, const DevFarLeaf* __restrict__ leaves,
                           const DevFarLeafGeom* __restrict__ geo, DevSources S, double2* __restrict__ pat) {
    const DevFarLeaf lf = leaves[blockIdx.x];
    const DevGeomLevel lv = lvs[lf.level];
    const double* c = geo[blockIdx.x].c;
    const int ndir = lv.ndir;
    for (int e = threadIdx.x; e < lf.nsrc * ndir; e += blockDim.x) {
        const int s = e / ndir, d = e - s * ndir;
        const int src = lf.src0 + s;
        const double kv[3] = {lv.khat[3 * d] * S.k, lv.khat[3 * d + 1] * S.k, lv.khat[3 * d + 2] * S.k};
        zd v[3];
        if (S.kind == kDipole) {
            const double* r = S.pos + 3 * src;
            const double dx[3] = {c[0] - r[0], c[1] - r[1], c[2] - r[2]};
            const zd ph = expi(dot3(kv, dx));
            for (int a = 0; a < 3; ++a) v[a] = ph * S.phat[3 * src + a];
        } else {
            zd I[3];
            rwg_plane_wave_integral(S.rwg[src], S.tris, kv, I);
            const zd ph = expi(dot3(kv, c));
            for (int a = 0; a < 3; ++a) v[a] = ph * conj(I[a]);
        }
        zd out[2];
        thph_apply(lv.thph + 6 * d, v, out);
        double2* o = pat + (lf.pat_off + static_cast<long long>(s) * ndir + d) * 2;
        o[0] = make_double2(out[0].x, out[0].y);
        o[1] = make_double2(out[1].x, out[1].y);
    }
}

// True when some triangle of RWG a shares a vertex with some triangle of b.
__device__ bool rwg_touching(const DevSources& S, const RwgGeom& a, const RwgGeom& b) {
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int u = 0; u < 3; ++u)
                for (int v = 0; v < 3; ++v)
                    if (S.tri_v[3 * a.tri[i] + u] == S.tri_v[3 * b.tri[j] + v]) return true;
    return false;
}

// Z_mn (the operator is A = C k Z) for obs m, src n (Dipole/RWG::getIntegratedRad,
// src/sources/dipole.h:62-70, src/sources/rwg.cpp:92-140).  Coincident
// sources and coincident triangles contribute nothing, unless self_terms is
// set: then a dipole's diagonal is Z_mm = 1, and RWG pairs whose triangles
// touch take the symmetrised mixed-potential value (rwg_mpie).
__device__ zd near_entry(const DevSources& S, int m, int n) {
    if (S.kind == kDipole) {
        const double* a = S.pos + 3 * m;
        const double* b = S.pos + 3 * n;
        if (a[0] == b[0] && a[1] == b[1] && a[2] == b[2]) {
            return mkz(S.self_terms ? 1.0 : 0.0);
        }
        const double X[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
        return dyadic_uv(X, S.k, S.phat + 3 * m, S.phat + 3 * n);
    }
    const RwgGeom& go = S.rwg[m];
    const RwgGeom& gs = S.rwg[n];
    if (S.self_terms && rwg_touching(S, go, gs))
        return 0.5 * (rwg_mpie(go, gs, S.tri_p, S.tri_quad, S.quad_w, S.nq, S.k) +
                      rwg_mpie(gs, go, S.tri_p, S.tri_quad, S.quad_w, S.nq, S.k));
    if (go.center[0] == gs.center[0] && go.center[1] == gs.center[1] && go.center[2] == gs.center[2])
        return mkz(0);
    zd acc = mkz(0);
    for (int ot = 0; ot < 2; ++ot) {
        for (int st = 0; st < 2; ++st) {
            if (go.tri[ot] == gs.tri[st]) continue;
            const double sgn = (ot ^ st) ? -1.0 : 1.0;
            const double* qo = S.tri_quad + static_cast<size_t>(go.tri[ot]) * S.nq * 3;
            const double* qs = S.tri_quad + static_cast<size_t>(gs.tri[st]) * S.nq * 3;
            for (int p = 0; p < S.nq; ++p) {
                const double* ro = qo + 3 * p;
                const double u[3] = {ro[0] - go.xpm[ot][0], ro[1] - go.xpm[ot][1], ro[2] - go.xpm[ot][2]};
                zd inner = mkz(0);
                for (int q = 0; q < S.nq; ++q) {
                    const double* rs = qs + 3 * q;
                    const double v[3] = {rs[0] - gs.xpm[st][0], rs[1] - gs.xpm[st][1], rs[2] - gs.xpm[st][2]};
                    const double X[3] = {ro[0] - rs[0], ro[1] - rs[1], ro[2] - rs[2]};
                    inner += S.quad_w[q] * dyadic_uv(X, S.k, u, v);
                }
                acc += (sgn * S.quad_w[p]) * inner;
            }
        }
    }
    return (go.leng * gs.leng) * acc;
}

// Rows of the dense operator: y_i = C k sum_n Z(m_i, n) x_n with every
// interaction evaluated directly by near_entry (FP64, O(N) work per row), the
// reference against which the MLFMA product's error is stated.  rows: tree
// slots; x in caller order.  One block per row, a fixed reduction tree.
constexpr int kDenseThreads = 256;

__global__ void __launch_bounds__(kDenseThreads)
k_dense_rows(DevSources S, const int* __restrict__ rows, const int* __restrict__ perm, const double2* __restrict__ x,
             int n, double2 ck, double2* __restrict__ y) {
    __shared__ double2 red[kDenseThreads];
    const int m = rows[blockIdx.x];
    zd acc = mkz(0);
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const double2 xv = x[perm[t]];
        acc += near_entry(S, m, t) * zd{xv.x, xv.y};
    }
    red[threadIdx.x] = make_double2(acc.x, acc.y);
    __syncthreads();
    for (int w = kDenseThreads / 2; w > 0; w >>= 1) {
        if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) y[blockIdx.x] = cmul(ck, red[0]);
}

// The same entries written out: out[i * ld + perm[t]] = C k Z[rows[i]][t],
// one thread per column.
__global__ void __launch_bounds__(kDenseThreads)
k_dense_block(DevSources S, const int* __restrict__ rows, const int* __restrict__ perm, int n, double2 ck,
              double2* __restrict__ out, long long ld) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int m = rows[blockIdx.y];
    const zd z = near_entry(S, m, t);
    out[static_cast<long long>(blockIdx.y) * ld + perm[t]] = cmul(ck, make_double2(z.x, z.y));
}

// Far field of currents I (caller order) along unit directions khat:
// F = C k (I - khat khat^T) sum_n I_n f_n(k khat), with f_n = e^{-i r_n . k khat}
// phat_n for a dipole (Dipole::getFarAlongDir, src/sources/dipole.h:53-57)
// and conj(I_n(k khat)) for an RWG (RWG::getFarAlongDir, src/sources/rwg.h:27-29);
// the sum and projection are those of Node::printFarSols
// (src/fmm/node.cpp:155-164).  One block per direction.
constexpr int kFarThreads = 256;

__global__ void __launch_bounds__(kFarThreads)
k_farfield(DevSources S, const int* __restrict__ perm, const double2* __restrict__ cur, int n,
           const double* __restrict__ khat, double2 ck, double2* __restrict__ out) {
    __shared__ double2 red[3][kFarThreads];
    const int d = blockIdx.x;
    const double kh[3] = {khat[3 * d], khat[3 * d + 1], khat[3 * d + 2]};
    const double kr[3] = {kh[0] * S.k, kh[1] * S.k, kh[2] * S.k};
    zd acc[3] = {mkz(0), mkz(0), mkz(0)};
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const double2 cv = cur[perm[t]];
        const zd c = zd{cv.x, cv.y};
        if (S.kind == kDipole) {
            const zd ph = c * expi(-dot3(S.pos + 3 * t, kr));
            for (int a = 0; a < 3; ++a) acc[a] += ph * S.phat[3 * t + a];
        } else {
            zd I[3];
            rwg_plane_wave_integral(S.rwg[t], S.tris, kr, I);
            for (int a = 0; a < 3; ++a) acc[a] += c * conj(I[a]);
        }
    }
    for (int a = 0; a < 3; ++a) red[a][threadIdx.x] = make_double2(acc[a].x, acc[a].y);
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (static_cast<int>(threadIdx.x) < s)
            for (int a = 0; a < 3; ++a) red[a][threadIdx.x] = cadd(red[a][threadIdx.x], red[a][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double2 v[3] = {red[0][0], red[1][0], red[2][0]};
        const double proj = kh[0] * v[0].x + kh[1] * v[1].x + kh[2] * v[2].x;
        const double proji = kh[0] * v[0].y + kh[1] * v[1].y + kh[2] * v[2].y;
        for (int a = 0; a < 3; ++a) {
            const double2 t = make_double2(v[a].x - kh[a] * proj, v[a].y - kh[a] * proji);
            out[3 * d + a] = cmul(ck, t);
        }
    }
}

// Adjoint of the far-field map: g = M^H F for F (ndir x 3) along unit
// directions khat, M the linear map of k_farfield (currents -> far field):
//   g_n = conj(C k) sum_d conj(f_n(k khat_d)) . (I - khat_d khat_d^T) F_d,
// written in caller order.  PF holds the projected F_d (ndir x 3), formed
// first by k_project.  One thread per unknown.  No counterpart in the
// reference (the far-field power gradient uses it).
__global__ void k_project(const double* __restrict__ khat, const double2* __restrict__ F, int ndir,
                          double2* __restrict__ PF) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ndir) return;
    const double* kh = khat + 3 * d;
    const double2* v = F + 3 * d;
    const double pr = kh[0] * v[0].x + kh[1] * v[1].x + kh[2] * v[2].x;
    const double pi = kh[0] * v[0].y + kh[1] * v[1].y + kh[2] * v[2].y;
    for (int a = 0; a < 3; ++a) PF[3 * d + a] = make_double2(v[a].x - kh[a] * pr, v[a].y - kh[a] * pi);
}

__global__ void k_farfield_adj(DevSources S, const int* __restrict__ perm, int n, const double* __restrict__ khat,
                               const double2* __restrict__ PF, int ndir, double2 ck, double2* __restrict__ g) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    zd acc = mkz(0);
    for (int d = 0; d < ndir; ++d) {
        const double kr[3] = {khat[3 * d] * S.k, khat[3 * d + 1] * S.k, khat[3 * d + 2] * S.k};
        zd cf[3];  // conj(f_t(k khat_d))
        if (S.kind == kDipole) {
            const zd ph = expi(dot3(S.pos + 3 * t, kr));
            for (int a = 0; a < 3; ++a) cf[a] = ph * S.phat[3 * t + a];
        } else {
            rwg_plane_wave_integral(S.rwg[t], S.tris, kr, cf);  // f = conj(I)
        }
        for (int a = 0; a < 3; ++a) {
            const double2 p = PF[3 * d + a];
            acc += cf[a] * zd{p.x, p.y};
        }
    }
    const zd r = zd{ck.x, -ck.y} * acc;
    g[perm[t]] = make_double2(r.x, r.y);
}

// Entries of the stored blocks: thread per entry.  A self block is packed
// lower-triangular: row i starts at i(i-1)/2 (strict) or i(i+1)/2 (with its
// diagonal).  Each value is Z_mn for the block's row m and column n, used as
// Z_nm as well.
__global__ void k_near_blocks_assemble(const DevNearBlock* __restrict__ blocks, int nblocks, long long total,
                                       DevSources S, double2* __restrict__ Z) {
    const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= total) return;
    int lo = 0, hi = nblocks - 1;
    while (lo < hi) {  // last block with off <= e
        const int mid = (lo + hi + 1) >> 1;
        if (blocks[mid].off <= e) lo = mid; else hi = mid - 1;
    }
    const DevNearBlock B = blocks[lo];
    const long long loc = e - B.off;
    int i, j;
    if (B.kind == 0) {
        i = static_cast<int>(loc / B.ncol);
        j = static_cast<int>(loc - static_cast<long long>(i) * B.ncol);
    } else {
        // largest i with packed_row(i) <= loc (estimate, then correct by one)
        const double q = sqrt(1.0 + 8.0 * static_cast<double>(loc));
        i = static_cast<int>(B.kind == 1 ? (1.0 + q) * 0.5 : (q - 1.0) * 0.5);
        while (i > 0 && packed_row(i, B.kind) > loc) --i;
        while (packed_row(i + 1, B.kind) <= loc) ++i;
        j = static_cast<int>(loc - packed_row(i, B.kind));
    }
    const zd z = near_entry(S, B.row0 + i, B.col0 + j);
    Z[e] = make_double2(z.x, z.y);
}

// Entries of the block rows: thread per entry.
__global__ void k_near_rows_assemble(const DevNearRow* __restrict__ rows, int nrows, long long total,
                                     const int* __restrict__ cols, DevSources S, double2* __restrict__ Z) {
    const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= total) return;
    int lo = 0, hi = nrows - 1;
    while (lo < hi) {  // last row block with off <= e
        const int mid = (lo + hi + 1) >> 1;
        if (rows[mid].off <= e) lo = mid; else hi = mid - 1;
    }
    const DevNearRow R = rows[lo];
    const long long loc = e - R.off;
    const int i = static_cast<int>(loc / R.ncol);
    const int k = static_cast<int>(loc - static_cast<long long>(i) * R.ncol);
    const zd z = near_entry(S, R.row0 + i, cols[R.col_off + k]);
    Z[e] = make_double2(z.x, z.y);
}

}  // namespace
}  // namespace mlfma

namespace mlfma {
namespace {

// ------------------------------------------------------------ leaf block-Jacobi preconditioner
// M = the diagonal blocks of A = C k Z + diag(loads), one per leaf: its
// inverse from the leaf's stored self block (packed lower triangle, used
// symmetrically, as the near field applies it), by Gauss-Jordan elimination
// with partial pivoting in shared memory.  A leaf larger than kBjMax sources,
// without a self block, or with a (numerically) singular block keeps the
// identity.
constexpr int kBjMax = 64;
constexpr int kBjThreads = 256;

__global__ void __launch_bounds__(kBjThreads)
k_bj_build(const DevBjLeaf* __restrict__ leaves, const double2* __restrict__ Z, double2 ck,
           const double2* __restrict__ loads, double2* __restrict__ inv, int* __restrict__ ok) {
    extern __shared__ double2 aug[];  // nb x 2 nb: [block | identity]
    __shared__ double piv_v[kBjThreads];
    __shared__ int piv_i[kBjThreads];
    __shared__ int singular;
    const DevBjLeaf L = leaves[blockIdx.x];
    const int nb = L.nb, w = 2 * nb;
    if (L.zoff < 0 || nb > kBjMax) {
        if (threadIdx.x == 0) ok[blockIdx.x] = 0;
        return;
    }
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        const int i = e / nb, j = e - i * nb;
        const int hi = max(i, j), lo = min(i, j);
        double2 z = make_double2(0.0, 0.0);
        if (hi != lo || L.kind == 2) z = Z[L.zoff + packed_row(hi, L.kind) + lo];
        double2 a = cmul(ck, z);
        if (i == j && loads) a = cadd(a, loads[L.row0 + i]);
        aug[i * w + j] = a;
        aug[i * w + nb + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    }
    if (threadIdx.x == 0) singular = 0;
    __syncthreads();
    for (int c = 0; c < nb; ++c) {
        // pivot: largest |a_rc| for r >= c
        double best = -1.0;
        int bi = c;
        for (int r = c + threadIdx.x; r < nb; r += blockDim.x) {
            const double2 v = aug[r * w + c];
            const double m = v.x * v.x + v.y * v.y;
            if (m > best) { best = m; bi = r; }
        }
        piv_v[threadIdx.x] = best;
        piv_i[threadIdx.x] = bi;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s && piv_v[threadIdx.x + s] > piv_v[threadIdx.x]) {
                piv_v[threadIdx.x] = piv_v[threadIdx.x + s];
                piv_i[threadIdx.x] = piv_i[threadIdx.x + s];
            }
            __syncthreads();
        }
        const int p = piv_i[0];
        if (!(piv_v[0] > 1e-300)) {
            if (threadIdx.x == 0) singular = 1;
            break;  // uniform: every thread read the same piv_v[0]
        }
        if (p != c)
            for (int j = threadIdx.x; j < w; j += blockDim.x) {
                const double2 t = aug[c * w + j];
                aug[c * w + j] = aug[p * w + j];
                aug[p * w + j] = t;
            }
        __syncthreads();
        const double2 d = aug[c * w + c];
        const double dm = d.x * d.x + d.y * d.y;
        const double2 dinv = make_double2(d.x / dm, -d.y / dm);
        __syncthreads();
        for (int j = threadIdx.x; j < w; j += blockDim.x) aug[c * w + j] = cmul(aug[c * w + j], dinv);
        __syncthreads();
        // eliminate column c from every other row (its factor read before the row changes)
        for (int e = threadIdx.x; e < nb * w; e += blockDim.x) {
            const int r = e / w, j = e - r * w;
            if (r == c || j == c) continue;
            const double2 f = aug[r * w + c];
            aug[r * w + j] = cadd(aug[r * w + j], cmul(make_double2(-f.x, -f.y), aug[c * w + j]));
        }
        __syncthreads();
        for (int r = threadIdx.x; r < nb; r += blockDim.x)
            if (r != c) aug[r * w + c] = make_double2(0.0, 0.0);
        __syncthreads();
    }
    __syncthreads();
    const bool good = singular == 0;
    if (good)
        for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
            const int i = e / nb, j = e - i * nb;
            inv[L.ioff + e] = aug[i * w + nb + j];
        }
    if (threadIdx.x == 0) ok[blockIdx.x] = good ? 1 : 0;
}

// y = M^{-1} x (tree order): per leaf its inverse block, or a copy.
__global__ void __launch_bounds__(kBjThreads)
k_bj_apply(const DevBjLeaf* __restrict__ leaves, const int* __restrict__ ok, const double2* __restrict__ inv,
           const double2* __restrict__ x, double2* __restrict__ y) {
    __shared__ double2 xs[kBjMax];
    const DevBjLeaf L = leaves[blockIdx.x];
    const int nb = L.nb;
    if (!ok[blockIdx.x]) {
        for (int i = threadIdx.x; i < nb; i += blockDim.x) y[L.row0 + i] = x[L.row0 + i];
        return;
    }
    for (int i = threadIdx.x; i < nb; i += blockDim.x) xs[i] = x[L.row0 + i];
    __syncthreads();
    // 4 threads per row, a shuffle sum
    const int row = threadIdx.x >> 2, part = threadIdx.x & 3;
    for (int r = row; r < nb + ((nb & 63) ? 64 - (nb & 63) : 0); r += kBjThreads / 4) {
        double2 acc = make_double2(0.0, 0.0);
        if (r < nb) {
            const double2* m = inv + L.ioff + static_cast<long long>(r) * nb;
            for (int j = part; j < nb; j += 4) acc = cfma(m[j], xs[j], acc);
        }
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 2);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 2);
        if (r < nb && part == 0) y[L.row0 + r] = acc;
    }
}

}  // namespace
}  // namespace mlfma
