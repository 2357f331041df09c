// bg_umma.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05) for
// the learned proposal network.
//
//   C[M, N] = A[M, K] . B[N, K]^T      A, B bf16, both K-major (rows of K
//                                      contiguous), accumulation FP32 in TMEM
//
// One CTA of 128 threads computes a 128 x NT tile.  The K dimension is
// streamed in chunks of 64 through a 3-stage ring of shared-memory tiles
// filled with cp.async (16-byte pieces; rows past M or N are zero-filled).
// Tiles use the canonical K-major layout without swizzle: 8-row x 16-byte
// core matrices, core matrices along K 128 bytes apart (leading byte offset)
// and 8-row groups 1024 bytes apart (stride byte offset).  Thread 0 issues
// four tcgen05.mma (K = 16 each) per chunk and commits them to the chunk's
// mbarrier; a stage is refilled only after that mbarrier completes.  The
// accumulator lives in TMEM (lane = tile row, one column per output column)
// and is read back by every warp for its 32 rows with tcgen05.ld; the
// epilogue is fused (bias, ReLU, ReLU gradient, transposed copies, column
// sums).  Row-major results go through the idle stage buffers: each warp
// stages its 32 x NT block in shared memory and writes whole rows with
// 16-byte stores; the ReLU mask of the gradient epilogue is read the same
// way.  Transposed copies are written from registers (32 consecutive rows
// of one column per warp store).
//
// With TMA (template flag, when the operands' rows are 16-byte aligned) the
// stages are filled by cp.async.bulk.tensor from 2-D tensor maps (K inner,
// rows outer) in boxes of 8 K-elements x all tile rows: each box lands as
// one 16-byte K-slab of every row, so core matrices are 128 bytes apart
// along M (stride byte offset) and one slab (rows x 16 bytes) apart along K
// (leading byte offset).  Thread 0 alone runs the pipeline: it arms a
// stage's full mbarrier with the expected bytes, issues the 16 boxes, and,
// kStages-1 chunks later, waits for the stage, issues its MMAs and commits
// them to the stage's empty mbarrier, which the next fill of the stage waits
// for -- no block-wide barrier inside the K loop.  No multicast.
//
// Every wait on an mbarrier is bounded; a wait that gives up records an
// error code and the CTA leaves after its copies in flight have landed and
// its TMEM is released.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace umma {

constexpr int kM = 128;          // rows per CTA tile (UMMA M)
constexpr int kKc = 64;          // K elements per stage
constexpr int kStages = 3;
constexpr int kThreads = 128;
constexpr uint32_t kLBO = 128;   // bytes between core matrices along K
constexpr uint32_t kSBO = 1024;  // bytes between 8-row groups
constexpr long long kSpinLimit = 1ll << 24;

enum Epi : int {
    EPI_F32 = 0,        // C fp32 (optionally per split), no bias
    EPI_BIAS_F32 = 1,   // C fp32 = acc + bias[n]
    EPI_RELU_BF16 = 2,  // H bf16 = relu(acc + bias[n]), and H^T
    EPI_DRELU_BF16 = 3  // G bf16 = acc * (act[m][n] > 0), and G^T
};

struct GemmArgs {
    const __nv_bfloat16 *A;   // [M][lda]
    const __nv_bfloat16 *B;   // [N][ldb]
    int M, N, K, lda, ldb;
    int k_per_split;          // K range of one grid.z slice (multiple of kKc)
    float *C;                 // fp32 out [split][M][ldc]
    int ldc;
    long long split_stride;   // elements between split slices of C
    const float *bias;        // [N] or null
    __nv_bfloat16 *H;         // bf16 out [M][ldh]
    int ldh;
    __nv_bfloat16 *HT;        // bf16 transposed out [N][ldht] or null
    int ldht;
    const __nv_bfloat16 *act; // [M][ldact] for EPI_DRELU_BF16
    int ldact;
    int n_valid;              // columns >= n_valid are written as 0 (bf16 outs) / skipped (fp32)
    float *colsum;            // EPI_DRELU_BF16: column sums of the bf16 result over each 32-row
    int colsum_ld;            //   quarter of a row tile, at colsum[(4 * row tile + quarter) * colsum_ld + col] (or null)
    int *err;                 // error flag (device)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo = kLBO, uint32_t sbo = kSBO) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // sm100 descriptor version; base offset 0, no swizzle
    return d;
}

// K-major tile in the 128-byte swizzled layout: each row's 64 bf16 of a
// K-chunk are one 128-byte line, 8-row atoms of 1024 bytes (stride byte
// offset), the 16-byte pieces of a line XOR-permuted by the row within the
// atom.  The K-step of one MMA (16 elements) advances the start address by
// 32 bytes inside the line; the tiles are 1024-byte aligned (base offset 0).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;                          // leading byte offset: unused for swizzled K-major
    d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;   // stride byte offset: one 8-row atom
    d |= (uint64_t)1 << 46;                          // sm100 descriptor version
    d |= (uint64_t)2 << 61;                          // layout: 128-byte swizzle
    return d;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

// One 2-D box of a tensor map into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// kind::f16 instruction descriptor: D f32, A bf16, B bf16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t tile_off(int r, int q) {
    return (uint32_t)((r >> 3) * kSBO + q * kLBO + (r & 7) * 16);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

// Bounded wait for the completion of phase `parity`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 columns of the warp's 32 TMEM lanes into registers, without waiting
// (tcgen05.wait::ld before the registers are read)
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Shared memory of one CTA: the stage ring, the mbarriers, the TMEM base.
template <int NT>
struct Smem {
    alignas(1024) unsigned char a[kStages][kM * kKc * 2];
    alignas(1024) unsigned char b[kStages][NT * kKc * 2];
    alignas(8) unsigned long long bar[kStages];   // stage consumed (MMAs committed)
    alignas(8) unsigned long long full[kStages];  // stage filled (TMA path)
    alignas(8) unsigned long long done;           // every MMA finished (TMA path)
    float bias[NT];
    uint32_t tmem_base;
    int failed;
};

template <int NT>
__device__ __forceinline__ void load_stage(Smem<NT> &sm, int st, const GemmArgs &g, int m0, int n0, int k0) {
    const int tid = threadIdx.x;
    const uint32_t a_base = smem_u32(sm.a[st]);
    const uint32_t b_base = smem_u32(sm.b[st]);
    // A: 128 rows x 8 pieces of 16 bytes
#pragma unroll
    for (int p = tid; p < kM * 8; p += kThreads) {
        const int r = p >> 3, q = p & 7;
        const int row = m0 + r;
        const bool ok = row < g.M;
        const __nv_bfloat16 *src = g.A + (long long)(ok ? row : 0) * g.lda + k0 + q * 8;
        cp_async16(a_base + tile_off(r, q), src, ok);
    }
#pragma unroll
    for (int p = tid; p < NT * 8; p += kThreads) {
        const int r = p >> 3, q = p & 7;
        const int row = n0 + r;
        const bool ok = row < g.N;
        const __nv_bfloat16 *src = g.B + (long long)(ok ? row : 0) * g.ldb + k0 + q * 8;
        cp_async16(b_base + tile_off(r, q), src, ok);
    }
}

template <int NT, int EPI, bool TMA>
__global__ void __launch_bounds__(kThreads, 1) k_gemm(const GemmArgs g, const __grid_constant__ CUtensorMap ta,
                                                      const __grid_constant__ CUtensorMap tb) {
    extern __shared__ unsigned char smem_raw[];
    Smem<NT> &sm = *reinterpret_cast<Smem<NT> *>(
        (void *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
    constexpr uint32_t kCols = NT < 32 ? 32 : NT;   // TMEM columns: power of two >= 32
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kM, n0 = blockIdx.y * NT;
    const int kbeg = blockIdx.z * g.k_per_split;
    const int kend = min(g.K, kbeg + g.k_per_split);
    const int nk = (kend - kbeg) / kKc;

    if ((EPI == EPI_RELU_BF16 || EPI == EPI_BIAS_F32) && tid < NT)
        sm.bias[tid] = (n0 + tid < g.N) ? g.bias[n0 + tid] : 0.f;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&sm.bar[s]), 1);
            mbar_init(smem_u32(&sm.full[s]), 1);
        }
        mbar_init(smem_u32(&sm.done), 1);
        sm.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = sm.tmem_base;
    constexpr uint32_t idesc = idesc_bf16(kM, NT);

    if constexpr (TMA) {
        if (tid == 0) {
            constexpr uint32_t kLboA = kM * 16, kLboB = NT * 16;     // one 16-byte K-slab of all rows
            constexpr uint32_t kBytes = (kM + NT) * kKc * 2;
            bool ok = true;
            int issued = 0, consumed = 0;
            for (int c = 0; c < nk + kStages - 1 && ok; ++c) {
                if (c < nk) {
                    const int st = c % kStages;
                    // the MMAs of chunk c - kStages read this stage
                    if (c >= kStages && !mbar_wait(smem_u32(&sm.bar[st]), (uint32_t)(((c / kStages) - 1) & 1))) {
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&sm.full[st]);
                    mbar_expect_tx(fb, kBytes);
                    const uint32_t a_addr = smem_u32(sm.a[st]), b_addr = smem_u32(sm.b[st]);
                    const int kx = kbeg + c * kKc;
#pragma unroll
                    for (int q = 0; q < kKc / 8; ++q) {
                        tma_load_2d(a_addr + q * kLboA, &ta, kx + q * 8, m0, fb);
                        tma_load_2d(b_addr + q * kLboB, &tb, kx + q * 8, n0, fb);
                    }
                    issued = c + 1;
                }
                const int cc = c - (kStages - 1);
                if (cc >= 0) {
                    const int st = cc % kStages;
                    if (!mbar_wait(smem_u32(&sm.full[st]), (uint32_t)((cc / kStages) & 1))) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t a_addr = smem_u32(sm.a[st]), b_addr = smem_u32(sm.b[st]);
#pragma unroll
                    for (int j = 0; j < kKc / 16; ++j)
                        umma_bf16(tmem, smem_desc(a_addr + j * 2 * kLboA, kLboA, 128),
                                  smem_desc(b_addr + j * 2 * kLboB, kLboB, 128), idesc, (cc > 0 || j > 0) ? 1u : 0u);
                    umma_commit(smem_u32(&sm.bar[st]));
                    consumed = cc + 1;
                }
            }
            if (!ok) {
                // let the boxes in flight land before the CTA leaves
                for (int c = consumed; c < issued; ++c) mbar_wait(smem_u32(&sm.full[c % kStages]), (uint32_t)((c / kStages) & 1));
                sm.failed = 1;
            }
            umma_commit(smem_u32(&sm.done));     // arrives once every MMA issued above has finished
        }
        if (!mbar_wait(smem_u32(&sm.done), 0u)) atomicExch(&sm.failed, 1);
        __syncthreads();
    } else {
        // prologue: chunks 0 .. kStages-2
#pragma unroll
        for (int s = 0; s < kStages - 1; ++s) {
            if (s < nk) load_stage(sm, s, g, m0, n0, kbeg + s * kKc);
            cp_async_commit();
        }
        bool ok = true;
        for (int c = 0; c < nk; ++c) {
            const int lc = c + kStages - 1;
            if (lc < nk) {
                const int st = lc % kStages;
                if (lc >= kStages) {
                    // the MMAs of chunk lc - kStages read this stage
                    if (!mbar_wait(smem_u32(&sm.bar[st]), (uint32_t)(((lc - kStages) / kStages) & 1))) ok = false;
                }
                load_stage(sm, st, g, m0, n0, kbeg + lc * kKc);
            }
            cp_async_commit();
            cp_async_wait<kStages - 1>();
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            if (!ok) atomicExch(&sm.failed, 1);
            __syncthreads();
            if (sm.failed) break;
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const int st = c % kStages;
                const uint32_t a_addr = smem_u32(sm.a[st]), b_addr = smem_u32(sm.b[st]);
#pragma unroll
                for (int j = 0; j < kKc / 16; ++j)
                    umma_bf16(tmem, smem_desc(a_addr + j * 2 * kLBO), smem_desc(b_addr + j * 2 * kLBO), idesc,
                              (c > 0 || j > 0) ? 1u : 0u);
                umma_commit(smem_u32(&sm.bar[st]));
            }
        }
        // all MMAs done: the last commit covers every earlier one
        if (!sm.failed && nk > 0) {
            const int st = (nk - 1) % kStages;
            if (!mbar_wait(smem_u32(&sm.bar[st]), (uint32_t)(((nk - 1) / kStages) & 1))) atomicExch(&sm.failed, 1);
        }
        cp_async_wait<0>();
        __syncthreads();
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (sm.failed) {
        if (tid == 0 && g.err) atomicExch(g.err, 1);
    } else {
        // epilogue: warp w owns tile rows 32w .. 32w+31, TMEM lanes alike
        constexpr bool kBF = (EPI == EPI_RELU_BF16 || EPI == EPI_DRELU_BF16);
        constexpr int kEsz = kBF ? 2 : 4;
        constexpr int kRowE = NT + 16 / kEsz;                   // staged row: NT elements + 16 bytes
        constexpr int kPieces = NT * kEsz / 16;                 // 16-byte pieces per row
        static_assert(4 * 32 * kRowE * kEsz + 4 * NT * 4 <= sizeof(((Smem<NT> *)0)->a) +
                                                             sizeof(((Smem<NT> *)0)->b),
                      "epilogue staging exceeds the stage buffers");
        unsigned char *stage = &sm.a[0][0] + (size_t)warp * 32 * kRowE * kEsz;
        float *red = reinterpret_cast<float *>(&sm.a[0][0] + (size_t)4 * 32 * kRowE * kEsz);
        const int wrow0 = m0 + warp * 32;
        const int row = wrow0 + lane;
        const bool row_ok = row < g.M;
        // row-major destination of this epilogue
        unsigned char *dst = nullptr;
        int ldo = 0, col_limit = g.N;
        if (EPI == EPI_F32 || EPI == EPI_BIAS_F32) {
            dst = reinterpret_cast<unsigned char *>(g.C + (long long)blockIdx.z * g.split_stride);
            ldo = g.ldc;
            col_limit = min(g.N, g.n_valid);
        } else {
            dst = reinterpret_cast<unsigned char *>(g.H);
            ldo = g.ldh;
        }
        const bool vec_out = (((size_t)ldo * kEsz) % 16 == 0) && (((uintptr_t)dst & 15) == 0);
        if (EPI == EPI_DRELU_BF16) {
            // the mask source, rows of act, into the staging rows
            const bool vec_in = (((size_t)g.ldact * 2) % 16 == 0) && (((uintptr_t)g.act & 15) == 0);
            for (int p = lane; p < 32 * kPieces; p += 32) {
                const int r = p / kPieces, q = p % kPieces;
                const int grow = wrow0 + r, gcol = n0 + q * 8;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (grow < g.M) {
                    const __nv_bfloat16 *src = g.act + (long long)grow * g.ldact + gcol;
                    if (vec_in && gcol + 8 <= g.N) {
                        v = *reinterpret_cast<const uint4 *>(src);
                    } else {
                        __nv_bfloat16 t[8];
#pragma unroll
                        for (int e = 0; e < 8; ++e) t[e] = gcol + e < g.N ? src[e] : __float2bfloat16_rn(0.f);
                        v = *reinterpret_cast<uint4 *>(t);
                    }
                }
                *reinterpret_cast<uint4 *>(stage + ((size_t)r * kRowE + q * 8) * 2) = v;
            }
            __syncwarp();
        }
#pragma unroll 1
        for (int cb = 0; cb < NT; cb += 16) {
            float v[16];
            if (nk > 0) {
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.f;
            }
            unsigned char *srow = stage + ((size_t)lane * kRowE + cb) * kEsz;
            if (kBF) {
                __nv_bfloat16 hv[16];
                __nv_bfloat16 av[16];
                if (EPI == EPI_DRELU_BF16) {
                    *reinterpret_cast<uint4 *>(av) = *reinterpret_cast<const uint4 *>(srow);
                    *reinterpret_cast<uint4 *>(av + 8) = *reinterpret_cast<const uint4 *>(srow + 16);
                }
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int col = n0 + cb + i;
                    float x = v[i];
                    if (EPI == EPI_RELU_BF16) {
                        x = col < g.N ? x + sm.bias[cb + i] : 0.f;
                        x = x > 0.f ? x : 0.f;
                    } else {
                        x = __bfloat162float(av[i]) > 0.f ? x : 0.f;
                    }
                    if (col >= g.n_valid || col >= g.N || !row_ok) x = 0.f;
                    hv[i] = __float2bfloat16_rn(x);
                    if (g.HT && row_ok && col < g.N) g.HT[(long long)col * g.ldht + row] = hv[i];
                }
                *reinterpret_cast<uint4 *>(srow) = *reinterpret_cast<uint4 *>(hv);
                *reinterpret_cast<uint4 *>(srow + 16) = *reinterpret_cast<uint4 *>(hv + 8);
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int col = n0 + cb + i;
                    if (EPI == EPI_BIAS_F32 && col < g.N) v[i] += sm.bias[cb + i];
                }
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4 *>(srow + i * 4) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            }
        }
        __syncwarp();
        if (EPI == EPI_DRELU_BF16 && g.colsum) {
            // column sums of the bf16 results over the CTA's rows, fixed order
            for (int c = lane; c < NT; c += 32) {
                float sum = 0.f;
                for (int r = 0; r < 32; ++r)
                    sum += __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(stage + ((size_t)r * kRowE + c) * 2));
                red[warp * NT + c] = sum;
            }
        }
        // whole rows out with 16-byte stores
        for (int p = lane; p < 32 * kPieces; p += 32) {
            const int r = p / kPieces, q = p % kPieces;
            const int grow = wrow0 + r;
            if (grow >= g.M) continue;
            constexpr int kPer = 16 / kEsz;
            const int gcol = n0 + q * kPer;
            const unsigned char *src = stage + ((size_t)r * kRowE + q * kPer) * kEsz;
            unsigned char *d = dst + ((size_t)grow * ldo + gcol) * kEsz;
            if (vec_out && gcol + kPer <= col_limit) {
                *reinterpret_cast<uint4 *>(d) = *reinterpret_cast<const uint4 *>(src);
            } else {
                for (int e = 0; e < kPer && gcol + e < col_limit; ++e)
                    for (int by = 0; by < kEsz; ++by) d[e * kEsz + by] = src[e * kEsz + by];
            }
        }
        if (EPI == EPI_DRELU_BF16 && g.colsum) {
            __syncwarp();
            // this warp's 32-row column sums: row (4 blockIdx.x + warp) of colsum
            for (int c = lane; c < NT; c += 32) {
                const int col = n0 + c;
                if (col < g.N) g.colsum[(long long)(4 * blockIdx.x + warp) * g.colsum_ld + col] = red[warp * NT + c];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

template <int NT>
constexpr size_t smem_bytes() {
    return sizeof(Smem<NT>) + 1024;
}

// ---------------------------------------------------------------------------
// Persistent, warp-specialised form of the same product (TMA operands only,
// stages in the 128-byte swizzled K-major layout: one TMA box per operand and
// K-chunk instead of eight 16-byte-wide ones; 6-8 stages in flight).
// A grid of at most one CTA per SM walks the output tiles (consecutive CTAs
// take consecutive row tiles of one column tile, so they share the B tile in
// L2).  Six warps per CTA:
//   warp 0  producer: one thread fills a PStages-deep ring of operand
//           stages with TMA boxes (full[s] armed with the expected bytes,
//           refilled after empty[s], which the MMAs of the stage commit to);
//   warp 1  MMA: one thread issues the four tcgen05.mma of each K-chunk into
//           one of two TMEM accumulators (2 x NT columns) and commits the
//           finished tile to acc_full[buf];
//   warps 2-5  epilogue: tcgen05.ld of their 32-lane quarter, the fused
//           epilogue, stores straight from registers (each thread writes 16
//           consecutive columns of its row: whole 32-byte sectors; the
//           transposed copy is one 64-byte run per column and warp), then
//           acc_empty[buf] frees the accumulator.
// So the epilogue of tile i runs while the MMAs of tile i+1 accumulate into
// the other buffer, and TMEM allocation, barrier set-up and pipeline fill are
// paid once per CTA instead of once per tile.  Every wait is bounded; a wait
// that gives up marks the CTA failed, the roles leave their loops, the
// producer waits for its boxes in flight, the MMA thread for its MMAs, and
// the TMEM is released.
constexpr int kPThreads = 320;          // producer, MMA, eight epilogue warps (two per TMEM lane quarter)
// operand stages in flight: as many as fit in 100 KB, so that the CTA of the
// next product (launched early, programmatic dependent launch) fits beside it
template <int NT> struct PStages { static constexpr int value = (192 * 1024) / ((kM + NT) * kKc * 2); };

// Programmatic dependent launch: the kernel lets the next one in its stream
// start launching, and waits for the previous one to finish (and its writes
// to be visible) before touching global memory.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

template <int NT>
struct PSmem {
    static constexpr int S = PStages<NT>::value;
    alignas(1024) unsigned char a[S][kM * kKc * 2];
    alignas(1024) unsigned char b[S][NT * kKc * 2];
    alignas(8) unsigned long long full[S];
    alignas(8) unsigned long long empty[S];
    alignas(8) unsigned long long acc_full[2];
    alignas(8) unsigned long long acc_empty[2];
    alignas(8) unsigned long long done;
    float red[4][NT];          // per-quarter column sums (EPI_DRELU_BF16)
    uint32_t tmem_base;
    int failed;
};

template <int NT>
constexpr size_t psmem_bytes() {
    return sizeof(PSmem<NT>) + 1024;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

// tile t -> (row tile, column tile, split): row tiles vary fastest
__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int &mt, int &nt, int &z) {
    mt = t % tiles_m;
    const int r = t / tiles_m;
    nt = r % tiles_n;
    z = r / tiles_n;
}

// The ReLU mask source of a DRELU epilogue, 16 columns of the thread's row
// from c0 on (0 past the matrix), read before the accumulator is ready.
__device__ __forceinline__ void p_load_act(const GemmArgs &g, int row, int c0, uint4 (&u)[2]) {
    u[0] = make_uint4(0, 0, 0, 0);
    u[1] = make_uint4(0, 0, 0, 0);
    if (row >= g.M) return;
    const __nv_bfloat16 *src = g.act + (long long)row * g.ldact + c0;
    if (((((uintptr_t)src) & 15) == 0) && c0 + 16 <= g.N) {
        u[0] = *reinterpret_cast<const uint4 *>(src);
        u[1] = *reinterpret_cast<const uint4 *>(src + 8);
    } else {
        __nv_bfloat16 *h = reinterpret_cast<__nv_bfloat16 *>(u);
        for (int i = 0; i < 16 && c0 + i < g.N; ++i) h[i] = src[i];
    }
}

template <int NT, int EPI>
__device__ __forceinline__ void p_epilogue_chunk(const GemmArgs &g, const float (&v)[16], int row, int n0, int cb,
                                                 int ntile_m, int quarter, int lane, PSmem<NT> &sm, int z,
                                                 const uint4 (&actu)[2]) {
    constexpr bool kBF = (EPI == EPI_RELU_BF16 || EPI == EPI_DRELU_BF16);
    const bool row_ok = row < g.M;
    const int c0 = n0 + cb;
    if (kBF) {
        __nv_bfloat16 hv[16];
        float act[16];
        if (EPI == EPI_DRELU_BF16) {
            const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(actu);
#pragma unroll
            for (int i = 0; i < 16; ++i) act[i] = __bfloat162float(h[i]);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int col = c0 + i;
            float x = v[i];
            if (EPI == EPI_RELU_BF16) {
                x = col < g.N ? x + __ldg(g.bias + col) : 0.f;
                x = x > 0.f ? x : 0.f;
            } else {
                x = act[i] > 0.f ? x : 0.f;
            }
            if (col >= g.n_valid || col >= g.N || !row_ok) x = 0.f;
            hv[i] = __float2bfloat16_rn(x);
        }
        if (row_ok) {
            __nv_bfloat16 *d = g.H + (long long)row * g.ldh + c0;
            if (((((uintptr_t)d) & 15) == 0) && c0 + 16 <= g.N) {
                reinterpret_cast<uint4 *>(d)[0] = reinterpret_cast<const uint4 *>(hv)[0];
                reinterpret_cast<uint4 *>(d)[1] = reinterpret_cast<const uint4 *>(hv)[1];
            } else {
                for (int i = 0; i < 16 && c0 + i < g.N; ++i) d[i] = hv[i];
            }
            if (g.HT)
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (c0 + i < g.N) g.HT[(long long)(c0 + i) * g.ldht + row] = hv[i];
        }
        if (EPI == EPI_DRELU_BF16 && g.colsum) {
            // column sums of the bf16 results over the quarter's 32 rows
            // (a fixed butterfly order, so the result is deterministic)
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float s = __bfloat162float(hv[i]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                if (lane == 0) sm.red[quarter][cb + i] = s;
            }
        }
    } else {
        if (row_ok) {
            const int limit = min(g.N, g.n_valid);
            float o[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) o[i] = (EPI == EPI_BIAS_F32 && c0 + i < g.N) ? v[i] + __ldg(g.bias + c0 + i) : v[i];
            float *d = g.C + (long long)z * g.split_stride + (long long)row * g.ldc + c0;
            if (((((uintptr_t)d) & 15) == 0) && c0 + 16 <= limit) {
#pragma unroll
                for (int i = 0; i < 16; i += 4) reinterpret_cast<float4 *>(d)[i / 4] = make_float4(o[i], o[i + 1], o[i + 2], o[i + 3]);
            } else {
                for (int i = 0; i < 16 && c0 + i < limit; ++i) d[i] = o[i];
            }
        }
    }
}

template <int NT, int EPI>
__global__ void __launch_bounds__(kPThreads, 1) k_gemm_p(const GemmArgs g, const __grid_constant__ CUtensorMap ta,
                                                        const __grid_constant__ CUtensorMap tb, int tiles_m,
                                                        int tiles_n, int splits) {
    extern __shared__ unsigned char smem_raw[];
    PSmem<NT> &sm = *reinterpret_cast<PSmem<NT> *>((void *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
    constexpr uint32_t kCols = 2 * NT < 32 ? 32 : 2 * NT;     // two accumulators, power of two
    constexpr uint32_t idesc = idesc_bf16(kM, NT);
    constexpr uint32_t kBytes = (kM + NT) * kKc * 2;
    constexpr int kPStages = PSmem<NT>::S;
    static_assert(NT % 32 == 0, "two epilogue warps per lane quarter split the columns in halves of 16-column chunks");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = tiles_m * tiles_n * splits;
    const int nk = g.k_per_split / kKc;
    pdl_launch_dependents();
    if (tid == 0) {
        // the tensor maps' descriptors into the TMA unit's cache ahead of the first box
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    }

    if (tid == 0) {
        for (int s = 0; s < kPStages; ++s) {
            mbar_init(smem_u32(&sm.full[s]), 1);
            mbar_init(smem_u32(&sm.empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&sm.acc_full[b]), 1);
            mbar_init(smem_u32(&sm.acc_empty[b]), 8);
        }
        mbar_init(smem_u32(&sm.done), 1);
        sm.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = sm.tmem_base;
    // set-up done: from here on the previous kernel's results are read
    pdl_wait();

    if (warp == 0) {
        if (lane == 0) {
            // ---- producer
            long long it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int mt, nt, z;
                tile_coords(t, tiles_m, tiles_n, mt, nt, z);
                const int m0 = mt * kM, n0 = nt * NT, kbeg = z * g.k_per_split;
                for (int c = 0; c < nk; ++c, ++it) {
                    const int st = (int)(it % kPStages);
                    const long long use = it / kPStages;
                    if (use >= 1 && !mbar_wait(smem_u32(&sm.empty[st]), (uint32_t)((use - 1) & 1))) { ok = false; break; }
                    if (*(volatile int *)&sm.failed) { ok = false; break; }
                    const uint32_t fb = smem_u32(&sm.full[st]);
                    mbar_expect_tx(fb, kBytes);
                    const int kx = kbeg + c * kKc;
                    // one box of 64 K-elements (a 128-byte line) x all tile rows per operand
                    tma_load_2d(smem_u32(sm.a[st]), &ta, kx, m0, fb);
                    tma_load_2d(smem_u32(sm.b[st]), &tb, kx, n0, fb);
                }
            }
            if (!ok) atomicExch(&sm.failed, 1);
            // the last boxes issued into each stage have landed before the CTA leaves
            for (long long j = (it > kPStages ? it - kPStages : 0); j < it; ++j)
                mbar_wait(smem_u32(&sm.full[j % kPStages]), (uint32_t)((j / kPStages) & 1));
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issue
            long long it = 0;
            int ti = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++ti) {
                const int buf = ti & 1, use = ti >> 1;
                if (use >= 1 && !mbar_wait(smem_u32(&sm.acc_empty[buf]), (uint32_t)((use - 1) & 1))) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(buf * NT);
                for (int c = 0; c < nk; ++c, ++it) {
                    const int st = (int)(it % kPStages);
                    if (!mbar_wait(smem_u32(&sm.full[st]), (uint32_t)((it / kPStages) & 1))) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t a_addr = smem_u32(sm.a[st]), b_addr = smem_u32(sm.b[st]);
#pragma unroll
                    for (int j = 0; j < kKc / 16; ++j)
                        umma_bf16(acc, smem_desc_sw128(a_addr + j * 32), smem_desc_sw128(b_addr + j * 32), idesc,
                                  (c > 0 || j > 0) ? 1u : 0u);
                    umma_commit(smem_u32(&sm.empty[st]));
                }
                if (!ok) break;
                umma_commit(smem_u32(&sm.acc_full[buf]));
            }
            if (!ok) atomicExch(&sm.failed, 1);
            umma_commit(smem_u32(&sm.done));    // arrives once every MMA issued above has finished
            if (!mbar_wait(smem_u32(&sm.done), 0u)) atomicExch(&sm.failed, 1);
        }
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31, the
        // columns of its half (warps 2-5 the first, 6-9 the second)
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        constexpr int kQ = NT / 32;                              // 16-column chunks per half
        int ti = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++ti) {
            const int buf = ti & 1, use = ti >> 1;
            int mt, nt, z;
            tile_coords(t, tiles_m, tiles_n, mt, nt, z);
            const int m0 = mt * kM, n0 = nt * NT;
            const int row = m0 + quarter * 32 + lane;
            // the mask source is read while the MMAs of the tile run
            uint4 actu[kQ][2];
            if (EPI == EPI_DRELU_BF16)
#pragma unroll
                for (int q = 0; q < kQ; ++q) p_load_act(g, row, n0 + 16 * (half * kQ + q), actu[q]);
            bool ok = mbar_wait(smem_u32(&sm.acc_full[buf]), (uint32_t)(use & 1));
            ok = __all_sync(0xffffffffu, ok);
            if (!ok || *(volatile int *)&sm.failed) { if (lane == 0) atomicExch(&sm.failed, 1); break; }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            // the whole row of the tile out of TMEM with one wait, and the
            // accumulator handed back to the MMA warp before the stores
            uint32_t raw[kQ][16];
#pragma unroll
            for (int q = 0; q < kQ; ++q)
                tmem_ld16_nowait(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * NT + 16 * (half * kQ + q)), raw[q]);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&sm.acc_empty[buf]));
#pragma unroll
            for (int q = 0; q < kQ; ++q) {
                float v[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(raw[q][i]);
                p_epilogue_chunk<NT, EPI>(g, v, row, n0, 16 * (half * kQ + q), mt, quarter, lane, sm, z, actu[q]);
            }
            if (EPI == EPI_DRELU_BF16 && g.colsum) {
                // this quarter's 32-row column sums: row (4 mt + quarter) of colsum
                __syncwarp();
                for (int c = half * (NT / 2) + lane; c < (half + 1) * (NT / 2); c += 32)
                    if (n0 + c < g.N) g.colsum[(long long)(4 * mt + quarter) * g.colsum_ld + n0 + c] = sm.red[quarter][c];
                __syncwarp();
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (sm.failed && tid == 0 && g.err) atomicExch(g.err, 1);
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

}  // namespace umma
