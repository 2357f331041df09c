// bg_batch.cu -- instances of the batch kernel (one per precision, number of
// state variables and block shape) and their launcher.
#include "bg_batch.cuh"

namespace {

template <typename T, int NV, int SH>
const void *batch_fn() {
    constexpr bg::BatchShape sh = bg::kBatchShapes[SH];
    return (const void *)bg::k_batch<T, NV, sh.threads, sh.npt>;
}

template <typename T, int NV>
const void *batch_fn_shape(int shape) {
    switch (shape) {
    case 0: return batch_fn<T, NV, 0>();
    case 1: return batch_fn<T, NV, 1>();
    case 2: return batch_fn<T, NV, 2>();
    case 3: return batch_fn<T, NV, 3>();
    case 4: return batch_fn<T, NV, 4>();
    case 5: return batch_fn<T, NV, 5>();
    default: return nullptr;
    }
}
static_assert(bg::kBatchNumShapes == 6, "one case per shape");

template <typename T>
const void *batch_fn_nv(int nvar, int shape) {
    switch (nvar) {
    case 1: return batch_fn_shape<T, 1>(shape);
    case 2: return batch_fn_shape<T, 2>(shape);
    case 3: return batch_fn_shape<T, 3>(shape);
    case 4: return batch_fn_shape<T, 4>(shape);
    default: return nullptr;
    }
}

const void *batch_kernel(int precision, int nvar, int shape) {
    return precision == 64 ? batch_fn_nv<double>(nvar, shape) : batch_fn_nv<float>(nvar, shape);
}

}  // namespace

int bg_batch_prepare_shape(int precision, int nvar, int shape, size_t smem) {
    const void *k = batch_kernel(precision, nvar, shape);
    if (!k) return 0;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) { cudaGetLastError(); return 0; }
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t room = optin > (int)fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
    if (smem > room) return 0;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (int)room;
}

cudaError_t bg_batch_launch(int precision, int nvar, int shape, const void *nets, const int32_t *order, int blocks,
                            int lanes, int dry, size_t smem, cudaStream_t s) {
    const void *k = batch_kernel(precision, nvar, shape);
    if (!k || blocks <= 0) return cudaErrorInvalidValue;
    const int threads = bg::kBatchShapes[shape].threads;
    void *args[] = {(void *)&nets, (void *)&order, (void *)&lanes, (void *)&dry};
    return cudaLaunchKernel(k, dim3((unsigned)blocks), dim3((unsigned)threads), args, smem, s);
}
