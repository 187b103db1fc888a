// Split-BF16 exchange on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// K = sum_q X_q X_q^T with X_q = B_q C (the factored form of the reference's
// K = sum_P B_P D B_P, hafnium/scf/coulomb_exchange.py:184-190). Every operand is
// split into two BF16 parts, x = hi + lo, and each product keeps the three
// leading terms hi*hi + hi*lo + lo*hi, accumulated in FP32 in tensor memory:
//
//   stage 1  X[(q,p)][i] = sum_r B[(q,p)][r] C[r][i]   one GEMM, M = rows (q,p),
//            A = BF16 copies of B stored in full (both triangles, K-major),
//            B-operand = C^T; the epilogue splits X into BF16 hi/lo, p-major.
//   stage 2  K[p][p'] += sum_(q,i) X[p][(q,i)] s_i X[p'][(q,i)], split over k,
//            upper 128-row tiles only; every (tile, split) writes its FP32 sum
//            to its own slice of a partial buffer, which a second kernel adds
//            into K in FP64 in a fixed order (s_i = +-1 for a signed factor,
//            whose stage 1 also writes X diag(s)).
//
// A persistent CTA per SM walks 128 x BN output tiles: warp 4 drives TMA (no
// multicast), warp 5 allocates TMEM and one thread issues tcgen05.mma
// (kind::f16, BF16 inputs, FP32 accumulate, M = 128) into one of two TMEM
// accumulators, warps 0-3 drain the other with tcgen05.ld meanwhile.
// Shared-memory tiles use the 128-byte swizzle that both TMA and the UMMA
// descriptors understand. Every mbarrier wait is bounded: past the limit the
// waiting thread records an error and stops waiting, so a fault in the
// pipeline ends the kernel instead of hanging the GPU.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>

#include "jk.cuh"
#include "tc_exchange.cuh"

namespace hf {

namespace {

constexpr int BM = 128;
constexpr int BK = 64;  // one 128-byte swizzle row of BF16

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: gives up after wait_ns, or as soon as another thread has
// recorded an error, and records its own failure; returns whether the phase
// completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, uint64_t wait_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t start = global_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 0) {
            if (*(volatile int*)err != 0) return false;
            if (global_ns() - start > wait_ns) {
                atomicExch(err, 1);
                return false;
            }
        }
    }
}

// Wait for copies already issued to land before the CTA exits: bounded by
// wait_ns only (an error recorded elsewhere does not cut it short, since the
// copies still write this CTA's shared memory).
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity, int* err, uint64_t wait_ns) {
    if (mbar_try_wait(bar, parity)) return;
    const uint64_t start = global_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return;
        if ((i & 255) == 0 && global_ns() - start > wait_ns) {
            atomicExch(err, 1);
            return;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];\n" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// K-major, 128-byte swizzle UMMA shared-memory descriptor: rows of 128 bytes,
// 8-row groups 1024 bytes apart (SBO), version 1, layout type 2.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D FP32, A/B BF16, both K-major, N = bn, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int bn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
        "}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct TcParams {
    int m_tiles, n_tiles;     // output tiles of 128 x bn
    int bn;                   // N tile (multiple of 16, <= 256)
    int k_tiles;              // k tiles of 64 per work item (split range)
    int k_tiles_total;
    int splits;               // k splits (stage 2)
    int items;                // work items = output tiles x splits (stage 2: upper tiles only)
    int mode;                 // 0: stage-1 epilogue, 1: stage-2 epilogue
    int stages;
    // stage 1: output row m = q_local * npad + p, column i -> X[p][q_local * ldq + i]
    __nv_bfloat16* xh;
    __nv_bfloat16* xl;
    // signed factor (optional): X diag(sign) written beside X for stage 2's B operand
    __nv_bfloat16* xsh;
    __nv_bfloat16* xsl;
    const double* sign;  // [opad]
    int64_t ldx;  // row stride of X (= qchunk * opad)
    int npad, opad;
    int ocols;    // valid columns (the rest of the tile is padding)
    // stage 2: K[p][p'] += acc (upper tiles only)
    double* kout;
    int64_t ldk;
    // stage 2 with per-split partial sums: kpart[split][p][p'] (FP32, row stride ldk) instead
    // of FP64 atomics into kout; summed into kout by k_reduce_partials
    float* kpart;
    int* err;
    uint64_t wait_ns;  // limit of every mbarrier wait
    int stall;         // self-test: the MMA thread first waits on a barrier that nothing completes
};

// Work item -> (m tile, n tile, split). Stage 1: m-major, n inner (neighbouring
// items share the A rows through L2). Stage 2: split-major over the output
// tiles that touch the upper triangle, enumerated row by row.
__device__ __forceinline__ void decode_item(const TcParams& P, int w, int& mt, int& nt, int& split) {
    if (P.mode == 0) {
        mt = w / P.n_tiles;
        nt = w - mt * P.n_tiles;
        split = 0;
        return;
    }
    const int per_split = P.items / P.splits;
    split = w / per_split;
    int r = w - split * per_split;
    for (mt = 0; mt < P.m_tiles; ++mt) {
        const int first = (mt * BM) / P.bn;  // first n tile with (nt + 1) bn > mt BM
        const int count = P.n_tiles - first;
        if (r < count) {
            nt = first + r;
            return;
        }
        r -= count;
    }
    nt = 0;  // not reached for w < items
}

// Persistent: one CTA per SM walks the work items; the TMEM accumulator is
// double buffered so the epilogue of one item overlaps the MMAs of the next.
// Warp 4: TMA producer; warp 5: TMEM allocation and the MMA-issuing thread;
// warps 0-3: epilogue (TMEM lane = output row).
__global__ void __launch_bounds__(192, 1) k_tc_split3(const __grid_constant__ CUtensorMap mAh,
                                                      const __grid_constant__ CUtensorMap mAl,
                                                      const __grid_constant__ CUtensorMap mBh,
                                                      const __grid_constant__ CUtensorMap mBl, TcParams P) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte alignment for the swizzled tiles
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int a_bytes = BM * BK * 2;       // 16 KB
    const int b_bytes = P.bn * BK * 2;     // bn * 128
    const int stage_bytes = 2 * a_bytes + 2 * b_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + P.stages * stage_bytes);
    uint64_t* empty = full + P.stages;
    uint64_t* acc_full = empty + P.stages;   // [2]
    uint64_t* acc_empty = acc_full + 2;      // [2]
    uint64_t* mma_done = acc_empty + 2;
    uint64_t* never = mma_done + 1;          // no thread ever arrives here (the stall self-test)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(never + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < P.stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 128);
        }
        mbar_init(mma_done, 1);
        mbar_init(never, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 4 && lane == 0) {
        prefetch_map(&mAh);
        prefetch_map(&mAl);
        prefetch_map(&mBh);
        prefetch_map(&mBl);
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 4) {
        if (lane == 0) {
            int it = 0, issued = 0;
            bool ok = true;
            for (int w = blockIdx.x; ok && w < P.items; w += gridDim.x) {
                int mt, nt, split;
                decode_item(P, w, mt, nt, split);
                const int kt0 = split * P.k_tiles, kt1 = min(P.k_tiles_total, kt0 + P.k_tiles);
                for (int kt = kt0; kt < kt1; ++kt, ++it) {
                    const int s = it % P.stages;
                    const uint32_t ph = (it / P.stages) & 1;
                    if (!mbar_wait(&empty[s], ph ^ 1, P.err, P.wait_ns)) {
                        ok = false;
                        break;
                    }
                    uint8_t* base = smem + s * stage_bytes;
                    mbar_expect_tx(&full[s], stage_bytes);
                    const int kx = kt * BK;
                    tma_load_2d(base, &mAh, &full[s], kx, mt * BM);
                    tma_load_2d(base + a_bytes, &mAl, &full[s], kx, mt * BM);
                    tma_load_2d(base + 2 * a_bytes, &mBh, &full[s], kx, nt * P.bn);
                    tma_load_2d(base + 2 * a_bytes + b_bytes, &mBl, &full[s], kx, nt * P.bn);
                    issued = it + 1;
                }
            }
            // Before the CTA can exit, every copy this thread issued has landed
            // (already true on the normal path, where the MMA thread consumed them).
            for (int j = max(0, issued - P.stages); j < issued; ++j)
                mbar_drain(&full[j % P.stages], (j / P.stages) & 1, P.err, P.wait_ns);
        }
    } else if (warp == 5) {
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(P.bn);
            int it = 0, local = 0;
            // the stall self-test: a wait that runs out, recorded like any other
            bool ok = !(P.stall && !mbar_wait(never, 0, P.err, P.wait_ns));
            for (int w = blockIdx.x; ok && w < P.items; w += gridDim.x, ++local) {
                int mt, nt, split;
                decode_item(P, w, mt, nt, split);
                const int kt0 = split * P.k_tiles, kt1 = min(P.k_tiles_total, kt0 + P.k_tiles);
                const int buf = local & 1;
                // the epilogue has drained this buffer's previous item
                if (!mbar_wait(&acc_empty[buf], ((local >> 1) & 1) ^ 1, P.err, P.wait_ns)) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t acc_tmem = tmem + (uint32_t)(buf * 256);
                for (int kt = kt0; kt < kt1; ++kt, ++it) {
                    const int s = it % P.stages;
                    const uint32_t ph = (it / P.stages) & 1;
                    if (!mbar_wait(&full[s], ph, P.err, P.wait_ns)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    uint8_t* base = smem + s * stage_bytes;
                    const uint64_t ah = umma_desc(smem_u32(base)), al = umma_desc(smem_u32(base + a_bytes));
                    const uint64_t bh = umma_desc(smem_u32(base + 2 * a_bytes));
                    const uint64_t bl = umma_desc(smem_u32(base + 2 * a_bytes + b_bytes));
#pragma unroll
                    for (int k = 0; k < BK / 16; ++k) {
                        const uint64_t adv = (uint64_t)(k * 32) >> 4;  // 16 BF16 = 32 bytes along the swizzled row
                        const uint32_t acc = (kt > kt0 || k > 0) ? 1u : 0u;
                        umma_bf16(acc_tmem, ah + adv, bh + adv, idesc, acc);
                        umma_bf16(acc_tmem, ah + adv, bl + adv, idesc, 1u);
                        umma_bf16(acc_tmem, al + adv, bh + adv, idesc, 1u);
                    }
                    umma_commit(&empty[s]);
                }
                if (ok) umma_commit(&acc_full[buf]);
            }
            // Arrives once every MMA issued above has completed, also on the error
            // path, so TMEM is never freed under a running MMA.
            umma_commit(mma_done);
        }
    } else {
        // epilogue: warps 0-3 own TMEM lanes 32w .. 32w+31 (output rows)
        int local = 0;
        for (int w = blockIdx.x; w < P.items; w += gridDim.x, ++local) {
            int mt, nt, split;
            decode_item(P, w, mt, nt, split);
            const int buf = local & 1;
            bool ready = mbar_wait(&acc_full[buf], (local >> 1) & 1, P.err, P.wait_ns) && *(volatile int*)P.err == 0;
            // tcgen05.ld is warp-collective: the whole warp reads or none of it does
            ready = __all_sync(0xffffffffu, ready);
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            if (!ready) break;
            const int m0 = mt * BM, n0 = nt * P.bn;
            const int row = m0 + warp * 32 + lane;
            const uint32_t acc_tmem = tmem + (uint32_t)(buf * 256) + ((uint32_t)(warp * 32) << 16);
            for (int c = 0; c < P.bn; c += 16) {
                float v[16];
                tmem_ld16(acc_tmem + (uint32_t)c, v);
                if (P.mode == 0) {
                    const int ql = row / P.npad, p = row % P.npad;
                    const int i0 = n0 + c;
                    if (row < P.m_tiles * BM) {
                        // 16 columns of one row: 32 contiguous bytes per part, stored as two
                        // 16-byte vectors (the row stride, opad and i0 are multiples of 16)
                        const int64_t off = (int64_t)p * P.ldx + (int64_t)ql * P.opad + i0;
                        alignas(16) __nv_bfloat162 hv[8], lv[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * j]), h1 = __float2bfloat16_rn(v[2 * j + 1]);
                            const __nv_bfloat16 l0 = __float2bfloat16_rn(v[2 * j] - __bfloat162float(h0));
                            const __nv_bfloat16 l1 = __float2bfloat16_rn(v[2 * j + 1] - __bfloat162float(h1));
                            hv[j] = __halves2bfloat162(h0, h1);
                            lv[j] = __halves2bfloat162(l0, l1);
                        }
                        uint4* dh = reinterpret_cast<uint4*>(P.xh + off);
                        uint4* dl = reinterpret_cast<uint4*>(P.xl + off);
                        dh[0] = reinterpret_cast<const uint4*>(hv)[0];
                        dh[1] = reinterpret_cast<const uint4*>(hv)[1];
                        dl[0] = reinterpret_cast<const uint4*>(lv)[0];
                        dl[1] = reinterpret_cast<const uint4*>(lv)[1];
                        if (P.xsh) {
                            // negating both parts negates the split value exactly
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                const bool m0 = P.sign[i0 + 2 * j] < 0.0, m1 = P.sign[i0 + 2 * j + 1] < 0.0;
                                const __nv_bfloat16 h0 = __low2bfloat16(hv[j]), h1 = __high2bfloat16(hv[j]);
                                const __nv_bfloat16 l0 = __low2bfloat16(lv[j]), l1 = __high2bfloat16(lv[j]);
                                hv[j] = __halves2bfloat162(m0 ? __hneg(h0) : h0, m1 ? __hneg(h1) : h1);
                                lv[j] = __halves2bfloat162(m0 ? __hneg(l0) : l0, m1 ? __hneg(l1) : l1);
                            }
                            uint4* sh = reinterpret_cast<uint4*>(P.xsh + off);
                            uint4* sl = reinterpret_cast<uint4*>(P.xsl + off);
                            sh[0] = reinterpret_cast<const uint4*>(hv)[0];
                            sh[1] = reinterpret_cast<const uint4*>(hv)[1];
                            sl[0] = reinterpret_cast<const uint4*>(lv)[0];
                            sl[1] = reinterpret_cast<const uint4*>(lv)[1];
                        }
                    }
                } else if (P.kpart) {
                    // 16 columns of this row's partial sum: four 16-byte vectors (ldk is a
                    // multiple of 128 and n0 + c of 16, so they are aligned)
                    float4* d4 = reinterpret_cast<float4*>(P.kpart + ((int64_t)split * P.ldk + row) * P.ldk + n0 + c);
                    d4[0] = make_float4(v[0], v[1], v[2], v[3]);
                    d4[1] = make_float4(v[4], v[5], v[6], v[7]);
                    d4[2] = make_float4(v[8], v[9], v[10], v[11]);
                    d4[3] = make_float4(v[12], v[13], v[14], v[15]);
                } else {
                    double* dst = P.kout + (int64_t)row * P.ldk + n0 + c;
#pragma unroll
                    for (int j = 0; j < 16; ++j) atomicAdd(dst + j, (double)v[j]);
                }
            }
            // this buffer is free for the item after next
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            mbar_arrive(&acc_empty[buf]);
        }
    }
    if (warp == 5 && lane == 0) mbar_drain(mma_done, 0, P.err, P.wait_ns);
    __syncthreads();
    if (warp == 5) {
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
    }
}

// Full BF16 hi/lo copies of B: Bh[q][p][r] from the FP64 upper-tile packing.
// One CTA per (packed tile (I, J), q): the 64x64 FP64 tile is read once with
// 16-byte loads, staged in shared memory, and written as the (I, J) block and,
// off the diagonal, the transposed (J, I) block, 128-byte rows of BF16 pairs.
// Only the nt(nt+1)/2 packed tiles are read; rows and columns beyond nt*64
// (when npad > nt*64) are zeroed by the host beforehand.
__global__ void __launch_bounds__(256) k_split_b_tiles(const double* __restrict__ B, int64_t ldb, int nt,
                                                       int npad, int q0, __nv_bfloat16* __restrict__ bh,
                                                       __nv_bfloat16* __restrict__ bl) {
    __shared__ double s[64][65];
    const int tile = blockIdx.x;
    const int ql = blockIdx.y;
    int I = 0, rem = tile;
    while (rem >= nt - I) {
        rem -= nt - I;
        ++I;
    }
    const int J = I + rem;
    const double2* src = reinterpret_cast<const double2*>(B + (int64_t)(q0 + ql) * ldb + (int64_t)tile * 4096);
    for (int k = threadIdx.x; k < 2048; k += 256) {
        const double2 v = src[k];
        const int a = (2 * k) >> 6, b = (2 * k) & 63;
        s[a][b] = v.x;
        s[a][b + 1] = v.y;
    }
    __syncthreads();
    const int64_t base = (int64_t)ql * npad * npad;
    for (int k = threadIdx.x; k < 2048; k += 256) {
        const int a = k >> 5, b = (k & 31) * 2;
        const double x0 = s[a][b], x1 = s[a][b + 1];
        const __nv_bfloat162 h = __halves2bfloat162(__double2bfloat16(x0), __double2bfloat16(x1));
        const __nv_bfloat162 l = __halves2bfloat162(__double2bfloat16(x0 - (double)__low2float(h)),
                                                    __double2bfloat16(x1 - (double)__high2float(h)));
        const int64_t o = base + (int64_t)(I * 64 + a) * npad + J * 64 + b;
        *reinterpret_cast<__nv_bfloat162*>(bh + o) = h;
        *reinterpret_cast<__nv_bfloat162*>(bl + o) = l;
    }
    if (I == J) return;
    for (int k = threadIdx.x; k < 2048; k += 256) {
        const int a = k >> 5, b = (k & 31) * 2;
        const double x0 = s[b][a], x1 = s[b + 1][a];
        const __nv_bfloat162 h = __halves2bfloat162(__double2bfloat16(x0), __double2bfloat16(x1));
        const __nv_bfloat162 l = __halves2bfloat162(__double2bfloat16(x0 - (double)__low2float(h)),
                                                    __double2bfloat16(x1 - (double)__high2float(h)));
        const int64_t o = base + (int64_t)(J * 64 + a) * npad + I * 64 + b;
        *reinterpret_cast<__nv_bfloat162*>(bh + o) = h;
        *reinterpret_cast<__nv_bfloat162*>(bl + o) = l;
    }
}

// C^T in FP64 ([opad][npad]) -> BF16 hi/lo.
__global__ void k_split_ct(const double* __restrict__ ct, int64_t count, __nv_bfloat16* __restrict__ h,
                           __nv_bfloat16* __restrict__ l) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const double x = ct[e];
    const __nv_bfloat16 hi = __double2bfloat16(x);
    h[e] = hi;
    l[e] = __double2bfloat16(x - (double)__bfloat162float(hi));
}

// Kp[p][p'] += sum_s part[s][p][p'] over the elements of the stage-2 tiles that
// touch the upper triangle ((p' / bn + 1) bn > (p / 128) 128), in a fixed order.
__global__ void k_reduce_partials(const float* __restrict__ part, int splits, int64_t npad, int bn,
                                  double* __restrict__ Kp) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= npad * npad) return;
    const int64_t row = e / npad, col = e % npad;
    if ((col / bn + 1) * bn <= (row / BM) * BM) return;
    double sum = 0.0;
    for (int k = 0; k < splits; ++k) sum += (double)part[(int64_t)k * npad * npad + e];
    Kp[e] += sum;
}

__global__ void k_symmetrize_upper128(const double* __restrict__ Kp, int64_t ldk, int64_t n, double* __restrict__ K) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t mu = e / n, nu = e % n;
    // element-level mirror: K is exactly symmetric (every mu <= nu lies in a computed tile)
    K[e] = mu <= nu ? Kp[mu * ldk + nu] : Kp[nu * ldk + mu];
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 2D BF16 tensor map: rows x cols (cols contiguous), box 64 cols x box_rows, 128B swizzle.
bool make_map(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {cols * 2};
    cuuint32_t box[2] = {BK, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

size_t smem_for(int bn, int stages) { return (size_t)stages * (2 * BM * BK * 2 + 2 * bn * BK * 2) + 1024 + 256; }

int sm_count() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        return 148;
    return sms;
}

// One persistent CTA per SM (at most one per work item).
cudaError_t launch_tc(const CUtensorMap& ah, const CUtensorMap& al, const CUtensorMap& bh, const CUtensorMap& bl,
                      const TcParams& P, cudaStream_t stream) {
    const size_t smem = smem_for(P.bn, P.stages);
    cudaError_t e = cudaFuncSetAttribute(k_tc_split3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (P.items < 1) return cudaSuccess;
    const int grid = std::min(P.items, sm_count());
    k_tc_split3<<<grid, 192, smem, stream>>>(ah, al, bh, bl, P);
    return cudaGetLastError();
}

// As many pipeline stages (<= 4) as fit in 220 KB of shared memory; the
// launch adds 1280 bytes of alignment slack and barriers (227 KB is the limit).
int stages_for(int bn) {
    const size_t per = 2 * BM * BK * 2 + 2 * (size_t)bn * BK * 2;
    return (int)std::max<size_t>(2, std::min<size_t>(4, (220 * 1024) / per));
}

}  // namespace

TcPlan tc_plan(int64_t n, int naux, int64_t ncols) {
    TcPlan t{};
    t.npad = (n + 127) / 128 * 128;
    const int64_t o = std::max<int64_t>(ncols, 1);
    t.n_tiles1 = (int)((o + 255) / 256);
    t.bn1 = (int)(((o + t.n_tiles1 - 1) / t.n_tiles1 + 15) / 16 * 16);
    t.opad = t.bn1 * t.n_tiles1;
    t.naux = naux;
    return t;
}

namespace {
// Stage 2's column tile width, its tiles touching the upper triangle, and the
// largest k split it uses (two CTAs' worth of items per SM).
void stage2_shape(int64_t npad, int& bn2, int& upper, int& splits_max) {
    // the n tiles must cover npad exactly (an odd multiple of 128 takes 128-wide tiles)
    bn2 = npad % 256 == 0 ? 256 : 128;
    const int m_tiles = (int)(npad / BM), n_tiles = (int)(npad / bn2);
    upper = 0;
    for (int mt = 0; mt < m_tiles; ++mt)
        for (int nt = 0; nt < n_tiles; ++nt)
            if ((nt + 1) * bn2 > mt * BM) ++upper;
    splits_max = std::max(1, (2 * 148 + upper - 1) / upper);
}
}  // namespace

size_t tc_partial_bytes(int64_t npad) {
    int bn2, upper, splits_max;
    stage2_shape(npad, bn2, upper, splits_max);
    return ((size_t)splits_max * npad * npad * sizeof(float) + 255) / 256 * 256;
}

size_t tc_b_bytes(int64_t n, int naux) {
    const int64_t npad = (n + 127) / 128 * 128;
    return sizeof(__nv_bfloat16) * 2 * (size_t)npad * npad * naux;
}

cudaError_t tc_split_b(const JkPlan& p, int64_t npad, void* bf16_b, cudaStream_t stream) {
    __nv_bfloat16* bh = static_cast<__nv_bfloat16*>(bf16_b);
    const int64_t per_q = npad * npad;
    __nv_bfloat16* bl = bh + per_q * p.naux;
    if (npad > (int64_t)p.nt * 64) {
        cudaError_t e = cudaMemsetAsync(bf16_b, 0, tc_b_bytes(npad, p.naux), stream);
        if (e != cudaSuccess) return e;
    }
    const int ntiles = p.nt * (p.nt + 1) / 2;
    const int qblock = 65535;
    for (int q0 = 0; q0 < p.naux; q0 += qblock) {
        const int qc = std::min(qblock, p.naux - q0);
        k_split_b_tiles<<<dim3(ntiles, qc), 256, 0, stream>>>(p.B, p.ldb, p.nt, (int)npad, q0, bh + per_q * q0,
                                                             bl + per_q * q0);
    }
    return cudaGetLastError();
}

cudaError_t exchange_build_bf16(const TcPlan& t, const void* bf16_b, const double* Ct_fp64, int64_t ct_ld,
                                double* K, double* Kp, void* work, size_t work_bytes, const TcWait& wait,
                                cudaStream_t stream, int64_t n, const double* sign) {
    (void)ct_ld;
    const int64_t npad = t.npad;
    const __nv_bfloat16* bh = static_cast<const __nv_bfloat16*>(bf16_b);
    const __nv_bfloat16* bl = bh + npad * npad * t.naux;
    // work: Ct hi/lo [opad][npad] | stage-2 partial sums | X hi/lo [npad][qchunk*opad]
    __nv_bfloat16* cth = static_cast<__nv_bfloat16*>(work);
    __nv_bfloat16* ctl = cth + (int64_t)t.opad * npad;
    const size_t ct_bytes = sizeof(__nv_bfloat16) * 2 * (size_t)t.opad * npad;
    const size_t part_bytes = tc_partial_bytes(npad);
    const size_t head = (ct_bytes + 255) / 256 * 256 + part_bytes;
    float* kpart = reinterpret_cast<float*>(static_cast<uint8_t*>(work) + (ct_bytes + 255) / 256 * 256);
    __nv_bfloat16* xbase = reinterpret_cast<__nv_bfloat16*>(static_cast<uint8_t*>(work) + head);
    if (work_bytes <= head) return cudaErrorInvalidValue;
    const size_t per_q = sizeof(__nv_bfloat16) * (sign ? 4 : 2) * (size_t)npad * t.opad;
    int qchunk = (int)std::min<size_t>((work_bytes - head) / per_q, (size_t)t.naux);
    if (qchunk < 1) return cudaErrorInvalidValue;
    const int64_t cnt = (int64_t)t.opad * npad;
    k_split_ct<<<(unsigned)((cnt + 255) / 256), 256, 0, stream>>>(Ct_fp64, cnt, cth, ctl);
    cudaMemsetAsync(Kp, 0, sizeof(double) * npad * npad, stream);
    CUtensorMap mCh, mCl;
    if (!make_map(&mCh, cth, t.opad, npad, t.bn1) || !make_map(&mCl, ctl, t.opad, npad, t.bn1))
        return cudaErrorInvalidValue;
    for (int q0 = 0; q0 < t.naux; q0 += qchunk) {
        const int qc = std::min(qchunk, t.naux - q0);
        const int64_t ldx = (int64_t)qc * t.opad;
        __nv_bfloat16* xh = xbase;
        __nv_bfloat16* xl = xbase + npad * ldx;
        __nv_bfloat16* xsh = sign ? xl + npad * ldx : nullptr;
        __nv_bfloat16* xsl = sign ? xsh + npad * ldx : nullptr;
        // stage 1: rows (q, p) of the full BF16 B for q in [q0, q0 + qc)
        CUtensorMap mAh, mAl;
        const uint64_t rows = (uint64_t)qc * npad;
        if (!make_map(&mAh, bh + (int64_t)q0 * npad * npad, rows, npad, BM) ||
            !make_map(&mAl, bl + (int64_t)q0 * npad * npad, rows, npad, BM))
            return cudaErrorInvalidValue;
        TcParams P{};
        P.m_tiles = (int)(rows / BM);
        P.n_tiles = t.n_tiles1;
        P.bn = t.bn1;
        P.k_tiles_total = (int)(npad / BK);
        P.k_tiles = P.k_tiles_total;
        P.splits = 1;
        P.items = P.m_tiles * P.n_tiles;
        P.mode = 0;
        P.stages = stages_for(P.bn);
        P.xh = xh;
        P.xl = xl;
        P.xsh = xsh;
        P.xsl = xsl;
        P.sign = sign;
        P.ldx = ldx;
        P.npad = (int)npad;
        P.opad = t.opad;
        P.ocols = t.opad;
        P.err = wait.err;
        P.wait_ns = wait.wait_ns;
        P.stall = q0 == 0 ? wait.stall : 0;
        cudaError_t e = launch_tc(mAh, mAl, mCh, mCl, P, stream);
        if (e != cudaSuccess) return e;
        // stage 2: K += X X^T over this chunk, split over k
        int bn2, upper, splits_max;
        stage2_shape(npad, bn2, upper, splits_max);
        CUtensorMap mXh, mXl, mXh2, mXl2;
        // B operand: X diag(sign) when the factor is signed
        if (!make_map(&mXh, xh, npad, ldx, BM) || !make_map(&mXl, xl, npad, ldx, BM) ||
            !make_map(&mXh2, sign ? xsh : xh, npad, ldx, bn2) || !make_map(&mXl2, sign ? xsl : xl, npad, ldx, bn2))
            return cudaErrorInvalidValue;
        TcParams Q{};
        Q.m_tiles = (int)(npad / BM);
        Q.n_tiles = (int)(npad / bn2);
        Q.bn = bn2;
        Q.k_tiles_total = (int)((ldx + BK - 1) / BK);  // the ragged last tile reads zeros past ldx
        const int splits = std::max(1, std::min(Q.k_tiles_total, splits_max));
        Q.k_tiles = (Q.k_tiles_total + splits - 1) / splits;
        Q.splits = (Q.k_tiles_total + Q.k_tiles - 1) / Q.k_tiles;  // every split has k tiles
        Q.items = upper * Q.splits;
        Q.mode = 1;
        Q.stages = stages_for(bn2);
        Q.kout = Kp;
        Q.ldk = npad;
        Q.kpart = kpart;
        Q.err = wait.err;
        Q.wait_ns = wait.wait_ns;
        Q.stall = 0;
        e = launch_tc(mXh, mXl, mXh2, mXl2, Q, stream);
        if (e != cudaSuccess) return e;
        k_reduce_partials<<<(unsigned)((npad * npad + 255) / 256), 256, 0, stream>>>(kpart, Q.splits, npad, bn2, Kp);
    }
    k_symmetrize_upper128<<<(unsigned)((n * n + 255) / 256), 256, 0, stream>>>(Kp, npad, n, K);
    return cudaGetLastError();
}

}  // namespace hf
