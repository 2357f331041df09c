// bg_mlp.cu -- the learned proposal network for model fitting: a 4-layer MLP
// (64 -> 512 -> 512 -> 512 -> 10, ReLU) whose output is a diagonal Gaussian
// over the fitted parameters (5 means, 5 log standard deviations), trained by
// Gaussian negative log-likelihood with Adam.
//
// Every matrix product, forward and backward, runs in one hand-written
// tcgen05 kernel (bg_umma.cuh) with BF16 operands and FP32 accumulation:
//
//   forward   H_l = relu(H_{l-1} W_l^T + b_l)          A = H_{l-1}, B = W_l
//   backward  G_l = (G_{l+1} W_{l+1}) * [H_l > 0]       A = G_{l+1}, B = W_{l+1}^T
//             dW_l = G_l^T H_{l-1}                      A = G_l^T,  B = H_{l-1}^T
//
// so each layer keeps its activations and gradients in both layouts (the
// epilogues write the transposed copy), and the weights exist as FP32
// master copies plus BF16 copies in both layouts, refreshed by the Adam
// kernel.  The output layer is padded from 10 to 64 rows (zero rows, zero
// gradients) so every K is a multiple of 64.  Weight gradients split the
// batch reduction over grid.z and are summed in a fixed order by the Adam
// kernel (deterministic).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "bg_common.cuh"
#include "bg_umma.cuh"
#include "../../include/brian_b200.h"

namespace {

int fail(int code, const std::string &m) { return bg_internal_fail(code, m.c_str()); }

#define MCK(call)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(BG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

constexpr int kIn = 64, kHid = 512, kOutPad = 64, kNLayer = 4;
constexpr int kSplits = 8;
// Output tile width of the network's GEMMs: 64 columns keeps 256 CTAs in
// flight per 4096-row product (two or three per SM), so one CTA's load
// latency overlaps another's tensor-core work.
constexpr int kNT = 64;

typedef __nv_bfloat16 bf16;

// ------------------------------------------------------------------ kernels
// Batch rows idx[0..B) of the normalised training set -> X (bf16), X^T, Y.
__global__ void k_gather(const float *Xall, const float *Yall, const int64_t *idx, int B, int ydim, bf16 *X, bf16 *XT,
                         float *Y) {
    const int b = blockIdx.x;
    const int64_t r = idx[b];
    for (int j = threadIdx.x; j < kIn; j += blockDim.x) {
        const bf16 v = __float2bfloat16_rn(Xall[r * kIn + j]);
        X[(int64_t)b * kIn + j] = v;
        XT[(int64_t)j * B + b] = v;
    }
    for (int j = threadIdx.x; j < ydim; j += blockDim.x) Y[(int64_t)b * ydim + j] = Yall[r * ydim + j];
}

// Gaussian NLL per sample, mean over the batch:
//   sum_d 0.5 ((y_d - mu_d) e^{-s_d})^2 + s_d,  s = clamp(log sigma, -7, 7)
// gradients (already divided by B) into dOUT (bf16, both layouts; the
// padded columns stay zero from allocation) and per-block column sums of the
// bf16 gradients into colsum[blockIdx.x][64] (the output bias gradient).
__global__ void __launch_bounds__(256) k_nll(const float *OUT, const float *Y, int B, int ydim, bf16 *dO, bf16 *dOT,
                                             float *colsum, float *loss_sum) {
    umma::pdl_launch_dependents();
    umma::pdl_wait();
    constexpr int kMaxY = kOutPad / 2;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ float red[8][kOutPad];
    __shared__ float lred[8];
    float l = 0.f;
    float gcol[kOutPad];
#pragma unroll
    for (int j = 0; j < kOutPad; ++j) gcol[j] = 0.f;
    if (b < B) {
        const float inv_b = 1.0f / (float)B;
        for (int j = 0; j < ydim && j < kMaxY; ++j) {
            const float mu = OUT[(int64_t)b * kOutPad + j];
            const float sr = OUT[(int64_t)b * kOutPad + ydim + j];
            const float s = fminf(fmaxf(sr, -7.f), 7.f);
            const float r = (Y[(int64_t)b * ydim + j] - mu) * expf(-s);
            l += 0.5f * r * r + s;
            const bf16 g = __float2bfloat16_rn(-r * expf(-s) * inv_b);                                  // d/d mu
            const bf16 gs = __float2bfloat16_rn((sr > -7.f && sr < 7.f) ? (1.f - r * r) * inv_b : 0.f);  // d/d log sigma
            dO[(int64_t)b * kOutPad + j] = g;
            dO[(int64_t)b * kOutPad + ydim + j] = gs;
            dOT[(int64_t)j * B + b] = g;
            dOT[(int64_t)(ydim + j) * B + b] = gs;
            gcol[j] = __bfloat162float(g);
            gcol[ydim + j] = __bfloat162float(gs);
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < kOutPad; ++j) {
        if (j >= 2 * ydim) break;
        float v = gcol[j];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][j] = v;
    }
    float lv = l;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lv += __shfl_xor_sync(0xffffffffu, lv, off);
    if (lane == 0) lred[warp] = lv;
    __syncthreads();
    if ((int)threadIdx.x < 2 * ydim) {
        float v = 0.f;
        for (int w = 0; w < 8; ++w) v += red[w][threadIdx.x];
        colsum[(int64_t)blockIdx.x * kOutPad + threadIdx.x] = v;
    }
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int w = 0; w < 8; ++w) v += lred[w];
        atomicAdd(loss_sum, v / (float)B);
    }
}

__global__ void k_to_bf16(const float *W, int rows, int cols, bf16 *Wb, bf16 *WbT) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)rows * cols) return;
    const int r = (int)(i / cols), c = (int)(i % cols);
    const bf16 h = __float2bfloat16_rn(W[i]);
    Wb[i] = h;
    if (WbT) WbT[(int64_t)c * rows + r] = h;
}

// Adam over every parameter tensor of the network in one launch: segment k
// of the flat index space is tensor k (W0, b0, W1, b1, ...), whose gradient
// is the sum of `splits` partial slices.  The step count t comes from device
// memory (the step runs as a captured graph), c1 = 1 - b1^t, c2 = 1 - b2^t.
struct AdamSeg {
    float *P, *m, *v; const float *grad; int splits; int64_t split_stride; int rows, cols, rows_train;
    bf16 *Pb, *PbT;
};
struct AdamAll {
    AdamSeg seg[2 * kNLayer];
    int64_t off[2 * kNLayer + 1];
    const int64_t *step;
    float lr, b1, b2, eps;
    float scale;                   // gradient multiplier (1: exact; 1/ranks after a summing all-reduce)
};
__global__ void k_adam_all(const __grid_constant__ AdamAll a) {
    umma::pdl_launch_dependents();
    umma::pdl_wait();
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 >= a.off[2 * kNLayer]) return;
    int k = 0;
#pragma unroll
    for (int q = 1; q < 2 * kNLayer; ++q) k += i0 >= a.off[q] ? 1 : 0;
    const AdamSeg &sg = a.seg[k];
    const int64_t i = i0 - a.off[k];
    const int r = (int)(i / sg.cols);
    if (r < sg.rows_train) {
        const float t = (float)*a.step;
        const float c1 = 1.f - powf(a.b1, t), c2 = 1.f - powf(a.b2, t);
        float g = 0.f;
        for (int s = 0; s < sg.splits; ++s) g += sg.grad[s * sg.split_stride + i];
        g *= a.scale;
        const float mi = a.b1 * sg.m[i] + (1.f - a.b1) * g;
        const float vi = a.b2 * sg.v[i] + (1.f - a.b2) * g * g;
        sg.m[i] = mi;
        sg.v[i] = vi;
        sg.P[i] -= a.lr * (mi / c1) / (sqrtf(vi / c2) + a.eps);
    }
    if (sg.Pb) sg.Pb[i] = __float2bfloat16_rn(sg.P[i]);   // the transposed copy: k_transpose_all
}

// The transposed bf16 copies of the updated weights (PbT[c][r] = Pb[r][c]),
// 32 x 32 tiles through shared memory so that both the reads and the writes
// are coalesced; block b is a tile of the first segments with a PbT.
__global__ void __launch_bounds__(256) k_transpose_all(const __grid_constant__ AdamAll a) {
    umma::pdl_launch_dependents();
    umma::pdl_wait();
    __shared__ bf16 tile[32][33];
    int b = blockIdx.x, k = 0;
    for (; k < 2 * kNLayer; ++k) {
        const AdamSeg &sg = a.seg[k];
        if (!sg.PbT) continue;
        const int nt = ((sg.rows + 31) / 32) * ((sg.cols + 31) / 32);
        if (b < nt) break;
        b -= nt;
    }
    if (k == 2 * kNLayer) return;
    const AdamSeg &sg = a.seg[k];
    const int tcols = (sg.cols + 31) / 32;
    const int r0 = (b / tcols) * 32, c0 = (b % tcols) * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int r = r0 + ty + j, c = c0 + tx;
        if (r < sg.rows && c < sg.cols) tile[ty + j][tx] = sg.Pb[(int64_t)r * sg.cols + c];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int c = c0 + ty + j, r = r0 + tx;
        if (r < sg.rows && c < sg.cols) sg.PbT[(int64_t)c * sg.rows + r] = tile[tx][ty + j];
    }
}

// The bias gradients, each the sum of its layer's column-sum partials (one
// per 32 or 256 batch rows), in one fixed order: block b sums 32 columns of
// one layer, warp w the partials w, w + 8, ... of them (coalesced rows), and
// warp 0 adds the eight warp sums in warp order.
struct BiasRed {
    const float *p[kNLayer]; int nblk[kNLayer], ld[kNLayer], rows[kNLayer];
    int blk0[kNLayer + 1];          // first block of each layer
    float *out;                     // [kNLayer][kHid]
};
__global__ void __launch_bounds__(256) k_bias_reduce(const __grid_constant__ BiasRed r) {
    umma::pdl_launch_dependents();
    umma::pdl_wait();
    __shared__ float red[8][32];
    int l = 0;
    while (l + 1 < kNLayer && (int)blockIdx.x >= r.blk0[l + 1]) ++l;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = ((int)blockIdx.x - r.blk0[l]) * 32 + lane;
    float g = 0.f;
    if (i < r.rows[l]) {
#pragma unroll 8
        for (int s = warp; s < r.nblk[l]; s += 8) g += r.p[l][(int64_t)s * r.ld[l] + i];
    }
    red[warp][lane] = g;
    __syncthreads();
    if (warp == 0 && i < r.rows[l]) {
        float t = red[0][lane];
#pragma unroll
        for (int w = 1; w < 8; ++w) t += red[w][lane];
        r.out[l * kHid + i] = t;
    }
}

// The gradient of every tensor as one flat vector in the optimiser's segment
// order (W0, b0, W1, b1, ...): each entry the sum of its partial slices in
// the order Adam sums them, so an update from the flat vector (scale 1)
// equals the fused one.  Data-parallel training all-reduces this vector.
__global__ void k_grad_flat(const __grid_constant__ AdamAll a, float *flat) {
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 >= a.off[2 * kNLayer]) return;
    int k = 0;
#pragma unroll
    for (int q = 1; q < 2 * kNLayer; ++q) k += i0 >= a.off[q] ? 1 : 0;
    const AdamSeg &sg = a.seg[k];
    const int64_t i = i0 - a.off[k];
    float g = 0.f;
    for (int s = 0; s < sg.splits; ++s) g += sg.grad[s * sg.split_stride + i];
    flat[i0] = g;
}

// One training step's bookkeeping: the batch index within the epoch and the
// optimiser step, advanced after the step's kernels.
__global__ void k_step_advance(int64_t *batch_index, int64_t *opt_step) {
    umma::pdl_launch_dependents();
    umma::pdl_wait();
    *batch_index += 1;
    *opt_step += 1;
}

// The epoch's batch order: rows sorted by a Philox draw keyed (seed, epoch, row).
__global__ void k_perm_keys(uint64_t seed, int64_t epoch, int64_t n, unsigned long long *keys, int64_t *vals) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t c[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), (uint32_t)epoch, (uint32_t)((uint64_t)epoch >> 32)};
        bg_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        keys[i] = ((unsigned long long)c[0] << 32) | c[1];
        vals[i] = i;
    }
}

// Batch rows idx[base .. base+B) with base = B * batch_index (a device
// counter, so the gather can sit in a captured graph).
__global__ void k_gather_at(const float *Xall, const float *Yall, const int64_t *perm, const int64_t *batch_index,
                            int B, int ydim, bf16 *X, bf16 *XT, float *Y) {
    const int b = blockIdx.x;
    const int64_t r = perm[*batch_index * B + b];
    for (int j = threadIdx.x; j < kIn; j += blockDim.x) {
        const bf16 v = __float2bfloat16_rn(Xall[r * kIn + j]);
        X[(int64_t)b * kIn + j] = v;
        XT[(int64_t)j * B + b] = v;
    }
    for (int j = threadIdx.x; j < ydim; j += blockDim.x) Y[(int64_t)b * ydim + j] = Yall[r * ydim + j];
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link against the driver library); null when unavailable.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
        cudaGetLastError();
    }
    return fn;
}

// 2-D map of a row-major bf16 matrix [rows][ld] over its first `cols`
// columns, zero fill past the edges: boxes of 8 columns x box_rows rows
// (no swizzle), or with sw128 of 64 columns (one 128-byte line) x box_rows
// rows landing in the 128-byte swizzled layout.
bool tile_map(CUtensorMap *m, const bf16 *base, int rows, int cols, int ld, int box_rows, bool sw128 = false) {
    EncodeTiledFn f = encode_tiled();
    if (!f || ((uintptr_t)base & 15) || ((size_t)ld * 2) % 16 || cols % (sw128 ? 64 : 8)) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {sw128 ? 64u : 8u, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, sw128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NT, int EPI, bool TMA>
int launch_gemm_as(const umma::GemmArgs &g, int splits, cudaStream_t st, const CUtensorMap &ta,
                   const CUtensorMap &tb) {
    static bool attr_set = false;
    constexpr size_t smem = umma::smem_bytes<NT>();
    if (!attr_set) {
        MCK(cudaFuncSetAttribute(umma::k_gemm<NT, EPI, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
    }
    dim3 grid((unsigned)((g.M + umma::kM - 1) / umma::kM), (unsigned)((g.N + NT - 1) / NT), (unsigned)splits);
    umma::k_gemm<NT, EPI, TMA><<<grid, umma::kThreads, smem, st>>>(g, ta, tb);
    MCK(cudaGetLastError());
    return BG_OK;
}

// Launch with programmatic stream serialization: the kernel may start while
// the previous one in the stream finishes; it waits (griddepcontrol.wait)
// before reading anything that one wrote.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args &&...args) {
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

int sm_count_mlp() {
    static int n = 0;
    if (!n) { int dev = 0; cudaGetDevice(&dev); cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev); if (n <= 0) n = 148; }
    return n;
}

// The persistent warp-specialised kernel over all tiles of the product.
template <int NT, int EPI>
int launch_gemm_persistent(const umma::GemmArgs &g, int splits, cudaStream_t st, const CUtensorMap &ta,
                           const CUtensorMap &tb) {
    static bool attr_set = false;
    constexpr size_t smem = umma::psmem_bytes<NT>();
    if (!attr_set) {
        MCK(cudaFuncSetAttribute(umma::k_gemm_p<NT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
    }
    const int tiles_m = (g.M + umma::kM - 1) / umma::kM, tiles_n = (g.N + NT - 1) / NT;
    const int ntiles = tiles_m * tiles_n * splits;
    const int grid = std::max(1, std::min(ntiles, sm_count_mlp()));
    MCK(launch_pdl(umma::k_gemm_p<NT, EPI>, dim3(grid), dim3(umma::kPThreads), smem, st, g, ta, tb, tiles_m, tiles_n,
                   splits));
    return BG_OK;
}

// TMA-fed persistent kernel when both operands allow a tensor map (16-byte
// aligned rows, K a multiple of 8) and every split has K-chunks, else the
// one-tile-per-CTA kernel with cp.async stages.
template <int NT, int EPI>
int launch_gemm(const umma::GemmArgs &g, int splits, cudaStream_t st) {
    CUtensorMap ta, tb;
    memset(&ta, 0, sizeof ta);
    memset(&tb, 0, sizeof tb);
    if (g.k_per_split >= umma::kKc && g.k_per_split % umma::kKc == 0 && (long long)g.k_per_split * splits == g.K &&
        tile_map(&ta, g.A, g.M, g.K, g.lda, umma::kM, true) && tile_map(&tb, g.B, g.N, g.K, g.ldb, NT, true))
        return launch_gemm_persistent<NT, EPI>(g, splits, st, ta, tb);
    memset(&ta, 0, sizeof ta);
    memset(&tb, 0, sizeof tb);
    return launch_gemm_as<NT, EPI, false>(g, splits, st, ta, tb);
}

umma::GemmArgs gemm_args(const bf16 *A, int lda, const bf16 *B, int ldb, int M, int N, int K, int *err) {
    umma::GemmArgs g;
    memset(&g, 0, sizeof g);
    g.A = A;
    g.B = B;
    g.M = M;
    g.N = N;
    g.K = K;
    g.lda = lda;
    g.ldb = ldb;
    g.k_per_split = K;
    g.n_valid = N;
    g.err = err;
    return g;
}

template <typename T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

template <typename T>
int dalloc(T **p, size_t n) {
    dfree(*p);
    if (n == 0) return BG_OK;
    if (cudaMalloc((void **)p, n * sizeof(T)) != cudaSuccess) return fail(BG_ENOMEM, "mlp: cudaMalloc failed");
    cudaMemset(*p, 0, n * sizeof(T));
    return BG_OK;
}

}  // namespace

struct bg_mlp {
    int device = 0;
    int ydim = 5;
    cudaStream_t stream = nullptr;
    int *err = nullptr;
    // parameters: layer l has W[l] [rows][cols] (fp32 master), b[l]
    int rows[kNLayer] = {kHid, kHid, kHid, kOutPad};
    int cols[kNLayer] = {kIn, kHid, kHid, kHid};
    float *W[kNLayer] = {}, *b[kNLayer] = {}, *mW[kNLayer] = {}, *vW[kNLayer] = {}, *mb[kNLayer] = {},
          *vb[kNLayer] = {};
    bf16 *Wb[kNLayer] = {}, *WbT[kNLayer] = {};
    float *gW = nullptr;                  // weight-gradient scratch: per layer, kSplits partial slices
    float *gWl[kNLayer] = {};             //   layer l's region of gW
    int64_t *dBatchIdx = nullptr;         // device counters of a training step: batch within the epoch,
    int64_t *dOptStep = nullptr;          //   optimiser step
    // epoch order: Philox keys sorted with their row indices
    unsigned long long *pkeys = nullptr, *pkeys_out = nullptr; int64_t *pvals = nullptr, *perm = nullptr;
    void *sort_tmp = nullptr; size_t sort_tmp_bytes = 0;
    // one training step captured as a graph (rebuilt when the batch size changes)
    cudaGraphExec_t step_graph = nullptr; int graph_batch = 0; float graph_lr = 0.f;
    float *cs[kNLayer] = {};              // bias-gradient partials per layer [row blocks][512]
    float *gbias = nullptr;               // their sums, [kNLayer][512]
    int64_t step = 0;
    // batch buffers
    int B = 0;
    bf16 *X = nullptr, *XT = nullptr, *H[3] = {}, *HT[3] = {}, *G[3] = {}, *GT[3] = {}, *dO = nullptr, *dOT = nullptr;
    float *OUT = nullptr, *Y = nullptr, *loss = nullptr;
    int64_t *idx = nullptr;
    // training set
    int64_t nset = 0;
    float *Xall = nullptr, *Yall = nullptr;
    float last_forward_ms = 0;
    float *gflat = nullptr; int64_t nflat = 0;   // flat gradient (data-parallel steps)
};

namespace {

int ensure_batch(bg_mlp *h, int B) {
    if (B == h->B) return BG_OK;
    // the batch buffers move: a captured training step holds their addresses
    if (h->step_graph) {
        cudaStreamSynchronize(h->stream);
        cudaGraphExecDestroy(h->step_graph);
        h->step_graph = nullptr;
        h->graph_batch = 0;
    }
    int rc = 0;
    if ((rc = dalloc(&h->X, (size_t)B * kIn))) return rc;
    if ((rc = dalloc(&h->XT, (size_t)B * kIn))) return rc;
    for (int l = 0; l < 3; ++l) {
        if ((rc = dalloc(&h->H[l], (size_t)B * kHid))) return rc;
        if ((rc = dalloc(&h->HT[l], (size_t)B * kHid))) return rc;
        if ((rc = dalloc(&h->G[l], (size_t)B * kHid))) return rc;
        if ((rc = dalloc(&h->GT[l], (size_t)B * kHid))) return rc;
    }
    if ((rc = dalloc(&h->dO, (size_t)B * kOutPad))) return rc;
    if ((rc = dalloc(&h->dOT, (size_t)B * kOutPad))) return rc;
    if ((rc = dalloc(&h->OUT, (size_t)B * kOutPad))) return rc;
    if ((rc = dalloc(&h->Y, (size_t)B * h->ydim))) return rc;
    if ((rc = dalloc(&h->idx, (size_t)B))) return rc;
    for (int l = 0; l < kNLayer; ++l)
        if ((rc = dalloc(&h->cs[l], (size_t)((B + 31) / 32) * kHid))) return rc;
    if (!h->gbias && (rc = dalloc(&h->gbias, (size_t)kNLayer * kHid))) return rc;
    h->B = B;
    return BG_OK;
}

// forward of the batch in h->X -> h->OUT
int forward(bg_mlp *h, int B) {
    const bf16 *in = h->X;
    int K = kIn;
    for (int l = 0; l < 3; ++l) {
        umma::GemmArgs g = gemm_args(in, K, h->Wb[l], K, B, kHid, K, h->err);
        g.bias = h->b[l];
        g.H = h->H[l];
        g.ldh = kHid;
        g.HT = h->HT[l];
        g.ldht = B;
        int rc = launch_gemm<kNT, umma::EPI_RELU_BF16>(g, 1, h->stream);
        if (rc) return rc;
        in = h->H[l];
        K = kHid;
    }
    umma::GemmArgs g = gemm_args(in, kHid, h->Wb[3], kHid, B, kOutPad, kHid, h->err);
    g.bias = h->b[3];
    g.C = h->OUT;
    g.ldc = kOutPad;
    return launch_gemm<64, umma::EPI_BIAS_F32>(g, 1, h->stream);
}

// Bias-gradient partials of layer l: per-block column sums written by the
// loss kernel (output layer, blocks of 256 rows, 64 columns) or by the
// ReLU-gradient epilogue that produced G[l] (blocks of 32 rows).
void bias_partials(const bg_mlp *h, int l, int B, const float **p, int *nblk, int *ld) {
    *p = h->cs[l];
    if (l == kNLayer - 1) {
        *nblk = (B + 255) / 256;
        *ld = kOutPad;
    } else {
        *nblk = 4 * ((B + umma::kM - 1) / umma::kM);
        *ld = kHid;
    }
}

// the bias gradients' sums (k_bias_reduce) for Adam and the flat gradient
int reduce_bias(bg_mlp *h, int B, bool pdl) {
    BiasRed r;
    memset(&r, 0, sizeof r);
    for (int l = 0; l < kNLayer; ++l) {
        bias_partials(h, l, B, &r.p[l], &r.nblk[l], &r.ld[l]);
        r.rows[l] = h->rows[l];
        r.blk0[l + 1] = r.blk0[l] + (r.rows[l] + 31) / 32;
    }
    r.out = h->gbias;
    const dim3 grid((unsigned)r.blk0[kNLayer]), block(256);
    if (pdl) MCK(launch_pdl(k_bias_reduce, grid, block, 0, h->stream, r));
    else k_bias_reduce<<<grid, block, 0, h->stream>>>(r);
    MCK(cudaGetLastError());
    return BG_OK;
}

// backward from the loss gradient in h->dO / h->dOT: weight gradients of
// layer l into its region of h->gW (kSplits partial slices over the batch),
// bias gradients as the column-sum partials, and the input gradient of every
// hidden layer (read against the weights before any update)
int backward(bg_mlp *h, int B) {
    int rc = 0;
    const int splits = kSplits;
    const int kper = B / splits;
    const bf16 *gin = h->dO;
    const bf16 *ginT = h->dOT;
    int gK = kOutPad;
    for (int l = 3; l >= 0; --l) {
        // dW_l = gin^T . input_l   (input_l = H[l-1] or X)
        const bf16 *inT = l > 0 ? h->HT[l - 1] : h->XT;
        const int nin = l > 0 ? kHid : kIn;
        {
            umma::GemmArgs g = gemm_args(ginT, B, inT, B, h->rows[l], nin, B, h->err);
            g.k_per_split = kper;
            g.C = h->gWl[l];
            g.ldc = nin;
            g.split_stride = (int64_t)h->rows[l] * h->cols[l];
            if (nin == kIn) rc = launch_gemm<64, umma::EPI_F32>(g, splits, h->stream);
            else rc = launch_gemm<kNT, umma::EPI_F32>(g, splits, h->stream);
            if (rc) return rc;
        }
        // gradient into the previous hidden layer; its epilogue also sums the
        // columns for layer l-1's bias
        if (l > 0) {
            umma::GemmArgs g = gemm_args(gin, gK, h->WbT[l], h->rows[l], B, kHid, gK, h->err);
            g.act = h->H[l - 1];
            g.ldact = kHid;
            g.H = h->G[l - 1];
            g.ldh = kHid;
            g.HT = h->GT[l - 1];
            g.ldht = B;
            g.colsum = h->cs[l - 1];
            g.colsum_ld = kHid;
            if ((rc = launch_gemm<kNT, umma::EPI_DRELU_BF16>(g, 1, h->stream))) return rc;
            gin = h->G[l - 1];
            ginT = h->GT[l - 1];
            gK = kHid;
        }
    }
    return BG_OK;
}

// Adam's tensor descriptors: gradients from the partial slices of a batch
// of B rows, or (flat != null) from a flat gradient vector
AdamAll adam_desc(bg_mlp *h, int B, float lr, const float *flat, float scale) {
    AdamAll a;
    memset(&a, 0, sizeof a);
    int64_t off = 0;
    for (int l = 0; l < kNLayer; ++l) {
        const int rows_train = l == 3 ? 2 * h->ydim : h->rows[l];
        AdamSeg &w = a.seg[2 * l];
        w.P = h->W[l]; w.m = h->mW[l]; w.v = h->vW[l]; w.grad = h->gWl[l]; w.splits = kSplits;
        w.split_stride = (int64_t)h->rows[l] * h->cols[l]; w.rows = h->rows[l]; w.cols = h->cols[l];
        w.rows_train = rows_train; w.Pb = h->Wb[l]; w.PbT = h->WbT[l];
        a.off[2 * l] = off;
        off += (int64_t)h->rows[l] * h->cols[l];
        AdamSeg &bb = a.seg[2 * l + 1];
        bb.P = h->b[l]; bb.m = h->mb[l]; bb.v = h->vb[l];
        bb.grad = h->gbias + (int64_t)l * kHid; bb.splits = 1; bb.split_stride = 0;   // k_bias_reduce's sums
        bb.rows = h->rows[l]; bb.cols = 1; bb.rows_train = rows_train;
        a.off[2 * l + 1] = off;
        off += h->rows[l];
    }
    a.off[2 * kNLayer] = off;
    a.step = h->dOptStep;
    a.lr = lr; a.b1 = 0.9f; a.b2 = 0.999f; a.eps = 1e-8f; a.scale = scale;
    if (flat)
        for (int k = 0; k < 2 * kNLayer; ++k) { a.seg[k].grad = flat + a.off[k]; a.seg[k].splits = 1; a.seg[k].split_stride = 0; }
    return a;
}

// Adam on every tensor in one launch (the step count is read on the device)
int adam_all(bg_mlp *h, int B, float lr, const float *flat = nullptr, float scale = 1.f) {
    const AdamAll a = adam_desc(h, B, lr, flat, scale);
    const int64_t off = a.off[2 * kNLayer];
    MCK(launch_pdl(k_adam_all, dim3((unsigned)((off + 255) / 256)), dim3(256), 0, h->stream, a));
    int tiles = 0;
    for (int k = 0; k < 2 * kNLayer; ++k)
        if (a.seg[k].PbT) tiles += ((a.seg[k].rows + 31) / 32) * ((a.seg[k].cols + 31) / 32);
    if (tiles) MCK(launch_pdl(k_transpose_all, dim3((unsigned)tiles), dim3(32, 8), 0, h->stream, a));
    return BG_OK;
}

// one training step on batch `*dBatchIdx` of h->perm: gather, forward, loss,
// backward, Adam, counters
int train_step(bg_mlp *h, int B, float lr) {
    k_gather_at<<<B, 64, 0, h->stream>>>(h->Xall, h->Yall, h->perm, h->dBatchIdx, B, h->ydim, h->X, h->XT, h->Y);
    int rc = forward(h, B);
    if (rc) return rc;
    MCK(launch_pdl(k_nll, dim3((B + 255) / 256), dim3(256), 0, h->stream, (const float *)h->OUT, (const float *)h->Y, B,
                   h->ydim, h->dO, h->dOT, h->cs[kNLayer - 1], h->loss));
    if ((rc = backward(h, B))) return rc;
    if ((rc = reduce_bias(h, B, true))) return rc;
    // Adam's step count t is the step being taken (1 for the first)
    MCK(launch_pdl(k_step_advance, dim3(1), dim3(1), 0, h->stream, h->dBatchIdx, h->dOptStep));
    if ((rc = adam_all(h, B, lr))) return rc;
    MCK(cudaGetLastError());
    return BG_OK;
}

// the epoch order buffers and the sort's scratch, kept for later calls
int ensure_perm(bg_mlp *h) {
    if (h->perm) return BG_OK;
    int rc;
    if ((rc = dalloc(&h->pkeys, (size_t)h->nset)) || (rc = dalloc(&h->pkeys_out, (size_t)h->nset)) ||
        (rc = dalloc(&h->pvals, (size_t)h->nset)) || (rc = dalloc(&h->perm, (size_t)h->nset)))
        return rc;
    size_t bytes = 0;
    MCK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, h->pkeys, h->pkeys_out, h->pvals, h->perm, (int)h->nset));
    MCK(cudaMalloc(&h->sort_tmp, bytes));
    h->sort_tmp_bytes = bytes;
    return BG_OK;
}

// the epoch's order: rows sorted by Philox keys (seed, epoch, row)
int epoch_perm(bg_mlp *h, uint64_t seed, int64_t ep) {
    k_perm_keys<<<(unsigned)std::min<int64_t>((h->nset + 255) / 256, 4096), 256, 0, h->stream>>>(
        seed, ep, h->nset, h->pkeys, h->pvals);
    MCK(cudaGetLastError());
    MCK(cub::DeviceRadixSort::SortPairs(h->sort_tmp, h->sort_tmp_bytes, h->pkeys, h->pkeys_out, h->pvals, h->perm,
                                        (int)h->nset, 0, 64, h->stream));
    return BG_OK;
}

int check_err(bg_mlp *h) {
    int e = 0;
    MCK(cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(BG_ETIMEOUT, "mlp: a tensor-core wait gave up");
    return BG_OK;
}

}  // namespace

extern "C" {

BG_API int bg_mlp_create(bg_mlp **out, int device, int ydim) {
    if (!out || ydim <= 0 || 2 * ydim > kOutPad) return fail(BG_EINVAL, "mlp: bad arguments");
    *out = nullptr;
    MCK(cudaSetDevice(device));
    bg_mlp *h = new bg_mlp();
    h->device = device;
    h->ydim = ydim;
    int rc = 0;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) rc = fail(BG_ECUDA, "mlp: stream");
    if (!rc) rc = dalloc(&h->err, 1);
    for (int l = 0; l < kNLayer && !rc; ++l) {
        const size_t n = (size_t)h->rows[l] * h->cols[l];
        if (!rc) rc = dalloc(&h->W[l], n);
        if (!rc) rc = dalloc(&h->mW[l], n);
        if (!rc) rc = dalloc(&h->vW[l], n);
        if (!rc) rc = dalloc(&h->b[l], (size_t)h->rows[l]);
        if (!rc) rc = dalloc(&h->mb[l], (size_t)h->rows[l]);
        if (!rc) rc = dalloc(&h->vb[l], (size_t)h->rows[l]);
        if (!rc) rc = dalloc(&h->Wb[l], n);
        if (!rc) rc = dalloc(&h->WbT[l], n);
    }
    {
        size_t tot = 0;
        for (int l = 0; l < kNLayer; ++l) tot += (size_t)kSplits * h->rows[l] * h->cols[l];
        tot = std::max(tot, (size_t)kSplits * kHid * kHid);
        if (!rc) rc = dalloc(&h->gW, tot);
        size_t o = 0;
        for (int l = 0; l < kNLayer && !rc; ++l) { h->gWl[l] = h->gW + o; o += (size_t)kSplits * h->rows[l] * h->cols[l]; }
    }
    if (!rc) rc = dalloc(&h->dBatchIdx, 1);
    if (!rc) rc = dalloc(&h->dOptStep, 1);
    if (!rc) rc = dalloc(&h->loss, 1);
    if (rc) {
        bg_mlp_destroy(h);
        return rc;
    }
    *out = h;
    return BG_OK;
}

BG_API int bg_mlp_destroy(bg_mlp *h) {
    if (!h) return BG_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int l = 0; l < kNLayer; ++l) {
        dfree(h->W[l]); dfree(h->b[l]); dfree(h->mW[l]); dfree(h->vW[l]); dfree(h->mb[l]); dfree(h->vb[l]);
        dfree(h->Wb[l]); dfree(h->WbT[l]);
    }
    for (int l = 0; l < 3; ++l) { dfree(h->H[l]); dfree(h->HT[l]); dfree(h->G[l]); dfree(h->GT[l]); }
    dfree(h->X); dfree(h->XT); dfree(h->dO); dfree(h->dOT); dfree(h->OUT); dfree(h->Y); dfree(h->idx);
    for (int l = 0; l < kNLayer; ++l) dfree(h->cs[l]);
    dfree(h->gW); dfree(h->gflat); dfree(h->loss); dfree(h->err); dfree(h->Xall); dfree(h->Yall);
    dfree(h->dBatchIdx); dfree(h->dOptStep); dfree(h->pkeys); dfree(h->pkeys_out); dfree(h->pvals); dfree(h->perm);
    if (h->sort_tmp) cudaFree(h->sort_tmp);
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return BG_OK;
}

BG_API int bg_mlp_set_params(bg_mlp *h, int layer, const float *W, const float *b) {
    if (!h || layer < 0 || layer >= kNLayer || !W || !b) return fail(BG_EINVAL, "mlp: bad parameter set");
    MCK(cudaSetDevice(h->device));
    const size_t n = (size_t)h->rows[layer] * h->cols[layer];
    MCK(cudaMemcpy(h->W[layer], W, n * sizeof(float), cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(h->b[layer], b, (size_t)h->rows[layer] * sizeof(float), cudaMemcpyHostToDevice));
    MCK(cudaMemset(h->mW[layer], 0, n * sizeof(float)));
    MCK(cudaMemset(h->vW[layer], 0, n * sizeof(float)));
    MCK(cudaMemset(h->mb[layer], 0, (size_t)h->rows[layer] * sizeof(float)));
    MCK(cudaMemset(h->vb[layer], 0, (size_t)h->rows[layer] * sizeof(float)));
    k_to_bf16<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->W[layer], h->rows[layer], h->cols[layer],
                                                                    h->Wb[layer], h->WbT[layer]);
    MCK(cudaGetLastError());
    MCK(cudaMemsetAsync(h->dOptStep, 0, sizeof(int64_t), h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    h->step = 0;
    return BG_OK;
}

BG_API int bg_mlp_get_params(bg_mlp *h, int layer, float *W, float *b) {
    if (!h || layer < 0 || layer >= kNLayer) return fail(BG_EINVAL, "mlp: bad layer");
    MCK(cudaSetDevice(h->device));
    MCK(cudaStreamSynchronize(h->stream));
    if (W) MCK(cudaMemcpy(W, h->W[layer], (size_t)h->rows[layer] * h->cols[layer] * sizeof(float),
                          cudaMemcpyDeviceToHost));
    if (b) MCK(cudaMemcpy(b, h->b[layer], (size_t)h->rows[layer] * sizeof(float), cudaMemcpyDeviceToHost));
    return BG_OK;
}

BG_API int bg_mlp_forward(bg_mlp *h, const float *X, int64_t n, float *out) {
    if (!h || !X || n <= 0 || !out) return fail(BG_EINVAL, "mlp: bad forward call");
    MCK(cudaSetDevice(h->device));
    const int B = (int)((n + 127) / 128 * 128);
    int rc = ensure_batch(h, B);
    if (rc) return rc;
    std::vector<bf16> xb((size_t)B * kIn, __float2bfloat16_rn(0.f)), xt((size_t)B * kIn, __float2bfloat16_rn(0.f));
    for (int64_t r = 0; r < n; ++r)
        for (int j = 0; j < kIn; ++j) {
            const bf16 v = __float2bfloat16_rn(X[r * kIn + j]);
            xb[(size_t)r * kIn + j] = v;
            xt[(size_t)j * B + r] = v;
        }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, h->stream);
    MCK(cudaMemcpyAsync(h->X, xb.data(), xb.size() * sizeof(bf16), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(h->XT, xt.data(), xt.size() * sizeof(bf16), cudaMemcpyHostToDevice, h->stream));
    if ((rc = forward(h, B))) return rc;
    std::vector<float> o((size_t)B * kOutPad);
    MCK(cudaMemcpyAsync(o.data(), h->OUT, o.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    cudaEventRecord(e1, h->stream);
    MCK(cudaStreamSynchronize(h->stream));
    cudaEventElapsedTime(&h->last_forward_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if ((rc = check_err(h))) return rc;
    for (int64_t r = 0; r < n; ++r)
        for (int j = 0; j < 2 * h->ydim; ++j) out[r * 2 * h->ydim + j] = o[(size_t)r * kOutPad + j];
    return BG_OK;
}

BG_API int bg_mlp_last_forward_ms(bg_mlp *h, float *ms) {
    if (!h || !ms) return fail(BG_EINVAL, "mlp: bad arguments");
    *ms = h->last_forward_ms;
    return BG_OK;
}

BG_API int bg_mlp_set_data(bg_mlp *h, const float *X, const float *Y, int64_t n) {
    if (!h || !X || !Y || n <= 0) return fail(BG_EINVAL, "mlp: bad training set");
    MCK(cudaSetDevice(h->device));
    MCK(cudaStreamSynchronize(h->stream));
    // the training set moves: the epoch-order buffers and the captured step
    // (which holds its addresses) are rebuilt by the next bg_mlp_train
    dfree(h->pkeys); dfree(h->pkeys_out); dfree(h->pvals); dfree(h->perm);
    if (h->sort_tmp) { cudaFree(h->sort_tmp); h->sort_tmp = nullptr; h->sort_tmp_bytes = 0; }
    if (h->step_graph) { cudaGraphExecDestroy(h->step_graph); h->step_graph = nullptr; h->graph_batch = 0; }
    int rc = dalloc(&h->Xall, (size_t)n * kIn);
    if (!rc) rc = dalloc(&h->Yall, (size_t)n * h->ydim);
    if (rc) return rc;
    MCK(cudaMemcpy(h->Xall, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(h->Yall, Y, (size_t)n * h->ydim * sizeof(float), cudaMemcpyHostToDevice));
    h->nset = n;
    return BG_OK;
}

BG_API int bg_mlp_train(bg_mlp *h, int epochs, int batch, float lr, uint64_t seed, float *epoch_loss,
                        float *gpu_ms) {
    if (!h || epochs < 0 || batch < 128 || batch % 128 != 0 || (batch / kSplits) % umma::kKc != 0)
        return fail(BG_EINVAL, "mlp: batch must be a multiple of 512 (128 rows x 8 batch splits of 64)");
    if (h->nset < batch) return fail(BG_ESTATE, "mlp: training set smaller than one batch");
    MCK(cudaSetDevice(h->device));
    int rc = ensure_batch(h, batch);
    if (rc) return rc;
    const int64_t steps = h->nset / batch;
    if ((rc = ensure_perm(h))) return rc;
    cudaEvent_t e0, e1;
    MCK(cudaEventCreate(&e0));
    MCK(cudaEventCreate(&e1));
    MCK(cudaEventRecord(e0, h->stream));
    for (int ep = 0; ep < epochs && !rc; ++ep) {
        if ((rc = epoch_perm(h, seed, ep))) break;
        MCK(cudaMemsetAsync(h->loss, 0, sizeof(float), h->stream));
        MCK(cudaMemsetAsync(h->dBatchIdx, 0, sizeof(int64_t), h->stream));
        for (int64_t s = 0; s < steps && !rc; ++s) {
            if (h->step_graph && h->graph_batch == batch && h->graph_lr == lr) {
                MCK(cudaGraphLaunch(h->step_graph, h->stream));
            } else if (s == 0) {
                // the first step runs directly (kernel attributes, tensor maps)
                rc = train_step(h, batch, lr);
            } else {
                // capture one step and replay it for the rest of training
                if (h->step_graph) { cudaGraphExecDestroy(h->step_graph); h->step_graph = nullptr; }
                cudaGraph_t graph = nullptr;
                MCK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
                rc = train_step(h, batch, lr);
                cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
                if (!rc && ce != cudaSuccess) rc = fail(BG_ECUDA, std::string("mlp: step capture: ") + cudaGetErrorString(ce));
                if (!rc && cudaGraphInstantiate(&h->step_graph, graph, 0) != cudaSuccess)
                    rc = fail(BG_ECUDA, "mlp: step graph instantiation failed");
                if (graph) cudaGraphDestroy(graph);
                if (rc) break;
                h->graph_batch = batch;
                h->graph_lr = lr;
                MCK(cudaGraphLaunch(h->step_graph, h->stream));
            }
        }
        h->step += steps;
        float ls = 0;
        cudaMemcpyAsync(&ls, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream);
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (!rc && e != cudaSuccess) rc = fail(BG_ECUDA, std::string("mlp: training failed: ") + cudaGetErrorString(e));
        if (!rc) rc = check_err(h);
        if (epoch_loss) epoch_loss[ep] = ls / (float)steps;
    }
    cudaEventRecord(e1, h->stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (gpu_ms) *gpu_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

BG_API int bg_mlp_epoch_order(bg_mlp *h, uint64_t seed, int64_t epoch) {
    if (!h || epoch < 0) return fail(BG_EINVAL, "mlp: bad epoch");
    if (h->nset <= 0) return fail(BG_ESTATE, "mlp: no training set");
    MCK(cudaSetDevice(h->device));
    int rc = ensure_perm(h);
    if (!rc) rc = epoch_perm(h, seed, epoch);
    if (!rc) MCK(cudaStreamSynchronize(h->stream));
    return rc;
}

BG_API int bg_mlp_step_gradients(bg_mlp *h, int batch, int64_t row0, float *loss, void **grad, int64_t *ngrad) {
    if (!h || batch < 128 || batch % 128 != 0 || (batch / kSplits) % umma::kKc != 0)
        return fail(BG_EINVAL, "mlp: batch must be a multiple of 512 (128 rows x 8 batch splits of 64)");
    if (!h->perm) return fail(BG_ESTATE, "mlp: no epoch order (bg_mlp_epoch_order)");
    if (row0 < 0 || row0 % batch != 0 || row0 + batch > h->nset) return fail(BG_EINVAL, "mlp: rows outside the epoch");
    MCK(cudaSetDevice(h->device));
    int rc = ensure_batch(h, batch);
    if (rc) return rc;
    const int64_t nflat = adam_desc(h, batch, 0.f, nullptr, 1.f).off[2 * kNLayer];
    if (h->nflat != nflat) {
        if ((rc = dalloc(&h->gflat, (size_t)nflat))) return rc;
        h->nflat = nflat;
    }
    const int64_t bidx = row0 / batch;
    MCK(cudaMemcpyAsync(h->dBatchIdx, &bidx, sizeof(int64_t), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemsetAsync(h->loss, 0, sizeof(float), h->stream));
    k_gather_at<<<batch, 64, 0, h->stream>>>(h->Xall, h->Yall, h->perm, h->dBatchIdx, batch, h->ydim, h->X, h->XT, h->Y);
    if ((rc = forward(h, batch))) return rc;
    k_nll<<<(batch + 255) / 256, 256, 0, h->stream>>>(h->OUT, h->Y, batch, h->ydim, h->dO, h->dOT,
                                                       h->cs[kNLayer - 1], h->loss);
    if ((rc = backward(h, batch))) return rc;
    if ((rc = reduce_bias(h, batch, false))) return rc;
    const AdamAll a = adam_desc(h, batch, 0.f, nullptr, 1.f);
    k_grad_flat<<<(unsigned)((nflat + 255) / 256), 256, 0, h->stream>>>(a, h->gflat);
    MCK(cudaGetLastError());
    float ls = 0;
    MCK(cudaMemcpyAsync(&ls, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    if ((rc = check_err(h))) return rc;
    if (loss) *loss = ls;
    if (grad) *grad = h->gflat;
    if (ngrad) *ngrad = nflat;
    return BG_OK;
}

BG_API int bg_mlp_apply_gradients(bg_mlp *h, const void *grad, float lr, float scale) {
    if (!h || !grad) return fail(BG_EINVAL, "mlp: no gradient");
    if (!h->gflat || h->B <= 0) return fail(BG_ESTATE, "mlp: no step gradients yet");
    MCK(cudaSetDevice(h->device));
    // Adam's step count t is the step being taken (1 for the first)
    MCK(launch_pdl(k_step_advance, dim3(1), dim3(1), 0, h->stream, h->dBatchIdx, h->dOptStep));
    int rc = adam_all(h, h->B, lr, (const float *)grad, scale);
    if (rc) return rc;
    MCK(cudaStreamSynchronize(h->stream));
    h->step += 1;
    return BG_OK;
}

// One forward + backward on the first `n` rows of the training set (no
// update), for gradient checks: loss, dW_l (summed) and db_l of every layer.
BG_API int bg_mlp_gradients(bg_mlp *h, int batch, float *loss, float *const *dW, float *const *db) {
    if (!h || batch < 128 || batch % 512 != 0 || h->nset < batch) return fail(BG_EINVAL, "mlp: bad gradient call");
    MCK(cudaSetDevice(h->device));
    int rc = ensure_batch(h, batch);
    if (rc) return rc;
    std::vector<int64_t> idx(batch);
    for (int i = 0; i < batch; ++i) idx[i] = i;
    MCK(cudaMemcpyAsync(h->idx, idx.data(), batch * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemsetAsync(h->loss, 0, sizeof(float), h->stream));
    k_gather<<<batch, 64, 0, h->stream>>>(h->Xall, h->Yall, h->idx, batch, h->ydim, h->X, h->XT, h->Y);
    if ((rc = forward(h, batch))) return rc;
    k_nll<<<(batch + 255) / 256, 256, 0, h->stream>>>(h->OUT, h->Y, batch, h->ydim, h->dO, h->dOT,
                                                       h->cs[kNLayer - 1], h->loss);
    // run the backward pass layer by layer, reading each layer's gradient
    // before the next layer reuses the scratch
    const int splits = kSplits;
    const int kper = batch / splits;
    const bf16 *gin = h->dO, *ginT = h->dOT;
    int gK = kOutPad;
    for (int l = 3; l >= 0; --l) {
        const bf16 *inT = l > 0 ? h->HT[l - 1] : h->XT;
        const int nin = l > 0 ? kHid : kIn;
        umma::GemmArgs g = gemm_args(ginT, batch, inT, batch, h->rows[l], nin, batch, h->err);
        g.k_per_split = kper;
        g.C = h->gW;
        g.ldc = nin;
        g.split_stride = (int64_t)kHid * kHid;
        rc = nin == kIn ? launch_gemm<64, umma::EPI_F32>(g, splits, h->stream)
                        : launch_gemm<kNT, umma::EPI_F32>(g, splits, h->stream);
        if (rc) return rc;
        std::vector<float> part((size_t)splits * kHid * kHid);
        MCK(cudaMemcpyAsync(part.data(), h->gW, part.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        MCK(cudaStreamSynchronize(h->stream));
        const size_t n = (size_t)h->rows[l] * nin;
        if (dW && dW[l])
            for (size_t i = 0; i < n; ++i) {
                float s = 0;
                for (int z = 0; z < splits; ++z) s += part[(size_t)z * kHid * kHid + i];
                dW[l][i] = s;
            }
        if (db && db[l]) {
            // the bias gradient: fixed-order sum of the column-sum partials
            const float *bp;
            int nblk, ld;
            bias_partials(h, l, batch, &bp, &nblk, &ld);
            std::vector<float> cp((size_t)nblk * ld);
            MCK(cudaMemcpy(cp.data(), bp, cp.size() * sizeof(float), cudaMemcpyDeviceToHost));
            for (int r = 0; r < h->rows[l]; ++r) {
                float s = 0;
                for (int z = 0; z < nblk; ++z) s += r < ld ? cp[(size_t)z * ld + r] : 0.f;
                db[l][r] = s;
            }
        }
        if (l > 0) {
            umma::GemmArgs g2 = gemm_args(gin, gK, h->WbT[l], h->rows[l], batch, kHid, gK, h->err);
            g2.act = h->H[l - 1];
            g2.ldact = kHid;
            g2.H = h->G[l - 1];
            g2.ldh = kHid;
            g2.HT = h->GT[l - 1];
            g2.ldht = batch;
            g2.colsum = h->cs[l - 1];
            g2.colsum_ld = kHid;
            if ((rc = launch_gemm<kNT, umma::EPI_DRELU_BF16>(g2, 1, h->stream))) return rc;
            gin = h->G[l - 1];
            ginT = h->GT[l - 1];
            gK = kHid;
        }
    }
    if (loss) MCK(cudaMemcpy(loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost));
    MCK(cudaStreamSynchronize(h->stream));
    return check_err(h);
}

// Plain GEMM on device buffers: C[M][N] = A[M][K] . B[N][K]^T (bf16 in,
// fp32 out), K a multiple of 64; the tensor-core kernel of the network.
BG_API int bg_gemm_bf16(int64_t M, int64_t N, int64_t K, const void *A, const void *B, float *C, void *stream) {
    if (M <= 0 || N <= 0 || K <= 0 || K % 64 != 0 || !A || !B || !C) return fail(BG_EINVAL, "gemm: bad shape");
    // the error flag of the tensor-core waits: one per device, kept for the process
    static int *flags[64] = {nullptr};
    int dev = 0;
    MCK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(BG_EINVAL, "gemm: device index");
    if (!flags[dev]) MCK(cudaMalloc((void **)&flags[dev], sizeof(int)));
    int *err = flags[dev];
    cudaStream_t st = (cudaStream_t)stream;
    MCK(cudaMemsetAsync(err, 0, sizeof(int), st));
    umma::GemmArgs g = gemm_args((const bf16 *)A, (int)K, (const bf16 *)B, (int)K, (int)M, (int)N, (int)K, err);
    g.C = C;
    g.ldc = (int)N;
    int rc = launch_gemm<128, umma::EPI_F32>(g, 1, st);
    cudaError_t e = cudaStreamSynchronize(st);
    int ev = 0;
    cudaMemcpy(&ev, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(BG_ECUDA, std::string("gemm: ") + cudaGetErrorString(e));
    if (ev) return fail(BG_ETIMEOUT, "gemm: a tensor-core wait gave up");
    return BG_OK;
}

}  // extern "C"
