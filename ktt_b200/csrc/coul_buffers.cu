// coul_buffers.cu -- device buffers behind the C ABI (declared in include/coulktt.h).
//
// The C++ ktt::Tuner surface keeps its kernel arguments in device memory through these calls, so
// that it links against this library's C ABI only.  (KTT's CUDA engine wraps the same driver calls
// in its CudaBuffer class: Source/ComputeEngine/Cuda/Buffers/CudaBuffer.cpp.)
#include <cuda_runtime.h>

#include "coul_internal.h"

using namespace coul;

extern "C" {

COUL_API int coul_buffer_alloc(coul_ctx* ctx, size_t bytes, void** d_ptr)
{
    if (ctx == nullptr || d_ptr == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "NULL argument");
    *d_ptr = nullptr;
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    cudaError_t e = cudaMalloc(d_ptr, bytes > 0 ? bytes : 16);
    if (e != cudaSuccess)
        return set_error(COUL_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return COUL_OK;
}

COUL_API int coul_buffer_free(coul_ctx* ctx, void* d_ptr)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (d_ptr == nullptr)
        return COUL_OK;
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    cudaStreamSynchronize(ctx->stream);
    cudaError_t e = cudaFree(d_ptr);
    return e == cudaSuccess ? COUL_OK : cuda_error(e, "cudaFree");
}

static int copy(coul_ctx* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, bool wait)
{
    if (ctx == nullptr || (bytes > 0 && (dst == nullptr || src == nullptr)))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "NULL argument");
    if (bytes == 0)
        return COUL_OK;
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, ctx->stream);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaMemcpyAsync");
    if (wait && (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return cuda_error(e, "cudaStreamSynchronize");
    return COUL_OK;
}

COUL_API int coul_buffer_upload(coul_ctx* ctx, void* d_dst, const void* h_src, size_t bytes)
{
    return copy(ctx, d_dst, h_src, bytes, cudaMemcpyHostToDevice, true);
}

COUL_API int coul_buffer_download(coul_ctx* ctx, void* h_dst, const void* d_src, size_t bytes)
{
    return copy(ctx, h_dst, d_src, bytes, cudaMemcpyDeviceToHost, true);
}

COUL_API int coul_buffer_copy(coul_ctx* ctx, void* d_dst, const void* d_src, size_t bytes)
{
    return copy(ctx, d_dst, d_src, bytes, cudaMemcpyDeviceToDevice, false);
}

COUL_API int coul_buffer_memset(coul_ctx* ctx, void* d_dst, int value, size_t bytes)
{
    if (ctx == nullptr || (bytes > 0 && d_dst == nullptr))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "NULL argument");
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    cudaError_t e = cudaMemsetAsync(d_dst, value, bytes, ctx->stream);
    return e == cudaSuccess ? COUL_OK : cuda_error(e, "cudaMemsetAsync");
}

}  // extern "C"
