// coul_internal.h -- state and helpers shared by the translation units behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "coul_forward.cuh"
#include "coulktt.h"

struct coul_batch;

struct coul_ctx {
    int device = 0;
    void* user_context = nullptr;  // the caller's CUcontext (coul_ctx_create_on), else the primary context
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;  // the stream every call of this context is enqueued on
    cudaEvent_t ev_start = nullptr; // bracket the most recent timed call
    cudaEvent_t ev_stop = nullptr;
    bool have_timing = false;
    int* d_status = nullptr;  // device status word written by kernels whose bounded waits expire
    float* d_atoms_cache = nullptr;  // buffers of the host-pointer convenience calls
    size_t atoms_cap = 0;
    float* d_out_cache = nullptr;
    size_t out_cap = 0;
    int sm_count = 0;
    int cc_major = 0;
    int cc_minor = 0;
    std::vector<std::function<void()>> cleanups;  // frees buffers owned by other units (run at destroy)
    void* adjoint_workspace = nullptr;            // FP64 partials of coul_adjoint_3d (coul_adjoint.cu)
    void* split_workspace_state = nullptr;        // partial blocks and counters of the queue and balanced forms
    std::vector<coul_batch*> batches;             // live batches (their device resources go with the context)
    struct Occupancy {
        const void* kernel;
        int threads;
        size_t smem;
        int blocks_per_sm;
    };
    std::vector<Occupancy> occupancy_cache;       // persistent forms' resident blocks (coul_capi.cu)
};

namespace coul {

int set_error(int status, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);
int ctx_activate(coul_ctx* ctx);
int ctx_begin_timing(coul_ctx* ctx);
int ctx_end_timing(coul_ctx* ctx);
bool aligned16(const void* p);
int validate_tune(const coul_tune* t, int mode, int soa, const VariantEntry** out);
int validate_grid(const coul_grid* g);
int launch_forward(coul_ctx* ctx, const VariantEntry* v, const FwdParams& prm, int mode, const coul_tune* t);
int queue_split_setup(coul_ctx* ctx, const VariantEntry* v, FwdLaunch& L, const coul_tune* t);
int balanced_split_setup(coul_ctx* ctx, const VariantEntry* v, FwdLaunch& L, const coul_tune* t);
// Releases the device resources of the context's live batches and detaches them (coul_batched.cu);
// their handles stay valid for coul_batch_destroy.  Called by coul_ctx_destroy, context current.
void orphan_batches(coul_ctx* ctx);

}  // namespace coul
