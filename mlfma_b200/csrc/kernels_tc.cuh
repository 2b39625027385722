// Interpolation (M2M) and anterpolation (L2L) of the complex-float far field
// on the tensor cores: tcgen05.mma, kind::tf32, split-precision 3xTF32
// products accumulated in FP32 in tensor memory.  Included once, by kernels.cu.
//
// Each stage is a separable pair of contractions over one axis of the
// (theta, phi) grid, applied to every box of a level at once:
//   M2M  (Stem::buildMpoleCoeffs + addInterpCoeffs, src/fmm/stem.cpp:72-184):
//        Z_P = sum_children shift_up(child) .* A_child   (child grid)
//        pass THETA: theta rows of the child grid -> parent theta rows (pole
//                    reflection: the source row read at phi + pi, sign folded)
//        pass PHI:   child phi columns -> parent phi columns (periodic)
//   L2L  (Stem::getShiftedLocalCoeffs + addAnterpCoeffs, src/fmm/stem.cpp:109-244):
//        per (parent, child): shift_down(child) .* B_P      (parent grid)
//        pass PHI_T:   parent phi columns -> child phi columns
//        pass THETA_T: parent theta rows -> child theta rows (reflection), added
//                      to the child's local pattern
// The interpolation weights are the same for every box of a transition, so a
// pass is a GEMM  D[row][i] = sum_k X[row][k] W[i][k]  whose rows are
// (box, position on the other axis, float of the complex pattern entries) and
// whose K is the contracted axis (with the reflected source rows appended).
// Summing the shifted children before the theta pass is exact algebra (the
// interpolation is linear and the same for every child) and interpolates once
// per parent instead of once per child.
//
// One CTA = 4 warps, persistent over 128-row tiles.  Every thread stages one
// row of the tile (loads, shift, child sum, hi/lo split) into shared memory;
// thread 0 issues the MMAs (A: the tile; B: the weights, bulk-copied once per
// CTA; both K-major without swizzle, the layout valid for TF32) and commits them to
// an mbarrier; then each warp reads its 32 TMEM lanes (one row per thread) and
// writes the outputs.  Every mbarrier wait is bounded: a CTA that gives up sets
// *err, releases its tensor memory and returns.
#pragma once

#include <cstdint>

#include "bulk_copy.cuh"
#include "device.cuh"
#include "tc_plan.hpp"

namespace mlfma {

namespace {

// ------------------------------------------------------------ tcgen05 helpers
__device__ __forceinline__ uint32_t tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-wide: allocate ncols TMEM columns, address written to *slot (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D (+)= A B, one thread.
__device__ __forceinline__ void umma_tf32(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
// Arrives on the mbarrier when every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
// 16 consecutive 32-bit columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor (sm_100 form, version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (static_cast<uint64_t>(layout) << 61);
}
// Instruction descriptor: kind::tf32, FP32 accumulator, A and B K-major, M = 128.
__host__ __device__ constexpr uint32_t tc_idesc(int npad) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (0u << 15) | (0u << 16) | (static_cast<uint32_t>(npad >> 3) << 17) |
           (static_cast<uint32_t>(kTcRows >> 4) << 24);
}

// Stages four consecutive contraction values of row m (kq: their 16-byte
// piece within the chunk), split hi + lo, as two 16-byte stores.
__device__ __forceinline__ void tc_stage4(unsigned char* a_hi, unsigned char* a_lo, int m, int kq, int kc_max,
                                          const float* v) {
    uint4 h, l;
    uint32_t* hp = &h.x;
    uint32_t* lp = &l.x;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        hp[u] = tf32_rna(v[u]);
        lp[u] = tf32_rna(v[u] - __uint_as_float(hp[u]));
    }
    const uint32_t o = tc_a_offset(m, kq, kc_max);
    // explicit shared-memory stores: the global loads of the next values need
    // not wait for them (volatile asm keeps them ordered with the fences)
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(smem_addr(a_hi) + o), "r"(h.x), "r"(h.y), "r"(h.z),
                 "r"(h.w));
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(smem_addr(a_lo) + o), "r"(l.x), "r"(l.y), "r"(l.z),
                 "r"(l.w));
}

// One thread: the 3xTF32 MMAs of a staged chunk, D (+)= A_chunk W_chunk^T with
// D = A_hi W_lo + A_lo W_hi + A_hi W_hi (small products first); k0: the
// chunk's first contraction index; first: the chunk starts the accumulation.
__device__ __forceinline__ void tc_issue_chunk(uint32_t tmem, uint32_t s_ahi, uint32_t s_alo, uint32_t s_w,
                                               uint32_t wbytes, int Kpad, int k0, int kc, int kc_max, uint32_t idesc,
                                               bool first) {
    const uint32_t sbo_a = static_cast<uint32_t>(kc_max) * 32u, sbo_w = static_cast<uint32_t>(Kpad) * 32u;
    for (int kk = 0; kk < kc / 8; ++kk) {
        const uint64_t ahi = umma_desc(s_ahi + kk * 256, 128, sbo_a, 0);
        const uint64_t alo = umma_desc(s_alo + kk * 256, 128, sbo_a, 0);
        const uint32_t kb = static_cast<uint32_t>(k0 / 8 + kk) * 256u;  // two 16-byte K pieces
        const uint64_t bhi = umma_desc(s_w + kb, 128, sbo_w, 0);
        const uint64_t blo = umma_desc(s_w + wbytes + kb, 128, sbo_w, 0);
        umma_tf32(tmem, alo, bhi, idesc, (first && kk == 0) ? 0u : 1u);
        umma_tf32(tmem, ahi, blo, idesc, 1u);
        umma_tf32(tmem, ahi, bhi, idesc, 1u);
    }
}

constexpr int kTcThreads = 128;

template <int KIND>
__global__ void __launch_bounds__(kTcThreads)
k_tc_pass(TcArgs a, int* __restrict__ err) {
    extern __shared__ unsigned char tc_smem_raw[];
    __shared__ __align__(8) unsigned long long bar_w, bar_mma;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    // shared memory: weights (hi, lo), the A tile (hi, lo; 1 KB aligned), krow
    const uint32_t raw = smem_addr(tc_smem_raw);
    unsigned char* base = tc_smem_raw + (((raw + 1023u) & ~1023u) - raw);
    const uint32_t wbytes = static_cast<uint32_t>(tc_w_bytes(a.Npad, a.Kpad));
    const uint32_t abytes = static_cast<uint32_t>(tc_a_bytes(a.Kpad));
    unsigned char* a_hi = base + ((2u * wbytes + 1023u) & ~1023u);
    unsigned char* a_lo = a_hi + abytes;
    int* krow_s = reinterpret_cast<int*>(a_lo + abytes);
    const uint32_t s_w = smem_addr(base), s_ahi = smem_addr(a_hi), s_alo = smem_addr(a_lo);

    uint32_t ncols = 32;
    while (ncols < static_cast<uint32_t>(a.Npad)) ncols <<= 1;
    if (warp == 0) tmem_alloc(&tmem_slot, ncols);
    if (tid == 0) {
        mbar_init(smem_addr(&bar_w), 1);
        mbar_init(smem_addr(&bar_mma), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (KIND == kTcTheta || KIND == kTcThetaT)
        for (int i = tid; i < a.K; i += blockDim.x) krow_s[i] = a.krow[i];
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    // the weights, once per CTA (one bulk copy of both halves)
    if (tid == 0) {
        mbar_arrive_expect_tx(smem_addr(&bar_w), 2u * wbytes);
        bulk_load(s_w, a.w, 2u * wbytes, smem_addr(&bar_w));
    }
    bool ok = mbar_wait_bounded(smem_addr(&bar_w), 0);
    ok = __syncthreads_and(ok);
    bool w_done = ok, mma_pending = false;
    const uint32_t idesc = tc_idesc(a.Npad);
    const int kc_max = a.Kpad < kTcKChunk ? a.Kpad : kTcKChunk;
    const long long nrows = static_cast<long long>(a.J) * a.Q * a.nitems;
    const long long ntiles = (nrows + kTcRows - 1) / kTcRows;
    uint32_t phase = 0;
    for (long long tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
        const TcRow r = tc_row(a, tile * kTcRows + tid);
        const TcItem it = tc_item<KIND>(a, r);
        for (int k0 = 0; k0 < a.Kpad && ok; k0 += kTcKChunk) {
            const int kc = min(kTcKChunk, a.Kpad - k0);
            // this row's contraction values of the chunk, eight at a time (all
            // their loads in flight together), split hi + lo
            for (int kq = 0; kq < kc / 4; kq += 2) {
                float v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = tc_load<KIND>(a, r, k0 + 4 * kq + u, krow_s, it);
                tc_stage4(a_hi, a_lo, tid, kq, kc_max, v);
                tc_stage4(a_hi, a_lo, tid, kq + 1, kc_max, v + 4);
            }
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                tc_issue_chunk(tmem, s_ahi, s_alo, s_w, wbytes, a.Kpad, k0, kc, kc_max, idesc, k0 == 0);
                umma_commit(smem_addr(&bar_mma));
            }
            mma_pending = true;
            ok = mbar_wait_bounded(smem_addr(&bar_mma), phase);
            ok = __syncthreads_and(ok);
            if (ok) {
                phase ^= 1u;
                mma_pending = false;
            }
            tc_fence_after();
        }
        if (!ok) break;
        // epilogue: this thread's TMEM lane (its row), 16 columns at a time
        const uint32_t lane_addr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
        for (int i0 = 0; i0 < a.Npad; i0 += 16) {
            float v[16];
            tmem_ld16(lane_addr + i0, v);
            if (r.live) {
                if (KIND == kTcThetaT) {
                    // accumulated outputs: every old value loaded before the stores
                    float old[16];
#pragma unroll
                    for (int u = 0; u < 16; ++u) old[u] = i0 + u < a.N ? tc_peek_out(a, r, i0 + u, it) : 0.f;
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                        if (i0 + u < a.N) tc_put_out(a, r, i0 + u, old[u] + v[u], it);
                } else {
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                        if (i0 + u < a.N) tc_store<KIND>(a, r, i0 + u, v[u], it);
                }
            }
        }
        tc_fence_before();
        __syncthreads();  // TMEM read and the A tile free before the next tile's MMAs
        tc_fence_after();
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 2);
        // work still in flight: wait for it (bounded) before the memory goes
        if (!w_done) mbar_wait_bounded(smem_addr(&bar_w), 0);
        if (mma_pending) mbar_wait_bounded(smem_addr(&bar_mma), phase);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

}  // namespace
}  // namespace mlfma
