// coul_profiler.cu -- hardware counters around the context's launches (coul_profiler_* in
// include/coulktt.h).
//
// KTT collects counters through CUPTI's profiler API with one kernel run per pass
// (Source/ComputeEngine/Cuda/Cupti/CuptiMetricInterface.cpp:21-120, CuptiInstance.cpp, CuptiPass.cpp);
// this file does the same with CUPTI's range profiler: a host object turns the metric names into a
// configuration image for the device's chip, the range profiler is enabled on the CUDA context with
// one user range and user replay, the caller reruns its launches once per pass between
// begin_pass / end_pass, and the decoded counter data are evaluated to one value per metric.
// libcupti is opened at run time so that the library loads without it.  Nothing here touches the
// device's clocks or other settings.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <dlfcn.h>

#include <cuda.h>
#include <cupti_profiler_host.h>
#include <cupti_profiler_target.h>
#include <cupti_range_profiler.h>
#include <cupti_target.h>

#include "coul_internal.h"

namespace {

struct CuptiApi {
    bool loaded = false;
    std::string error;
    decltype(&cuptiGetResultString) GetResultString = nullptr;
    decltype(&cuptiProfilerInitialize) ProfilerInitialize = nullptr;
    decltype(&cuptiDeviceGetChipName) DeviceGetChipName = nullptr;
    decltype(&cuptiProfilerGetCounterAvailability) GetCounterAvailability = nullptr;
    decltype(&cuptiProfilerHostInitialize) HostInitialize = nullptr;
    decltype(&cuptiProfilerHostDeinitialize) HostDeinitialize = nullptr;
    decltype(&cuptiProfilerHostConfigAddMetrics) HostConfigAddMetrics = nullptr;
    decltype(&cuptiProfilerHostGetConfigImageSize) HostGetConfigImageSize = nullptr;
    decltype(&cuptiProfilerHostGetConfigImage) HostGetConfigImage = nullptr;
    decltype(&cuptiProfilerHostGetNumOfPasses) HostGetNumOfPasses = nullptr;
    decltype(&cuptiProfilerHostEvaluateToGpuValues) HostEvaluateToGpuValues = nullptr;
    decltype(&cuptiRangeProfilerEnable) RangeEnable = nullptr;
    decltype(&cuptiRangeProfilerDisable) RangeDisable = nullptr;
    decltype(&cuptiRangeProfilerGetCounterDataSize) RangeGetCounterDataSize = nullptr;
    decltype(&cuptiRangeProfilerCounterDataImageInitialize) RangeCounterDataImageInitialize = nullptr;
    decltype(&cuptiRangeProfilerSetConfig) RangeSetConfig = nullptr;
    decltype(&cuptiRangeProfilerStart) RangeStart = nullptr;
    decltype(&cuptiRangeProfilerStop) RangeStop = nullptr;
    decltype(&cuptiRangeProfilerPushRange) RangePushRange = nullptr;
    decltype(&cuptiRangeProfilerPopRange) RangePopRange = nullptr;
    decltype(&cuptiRangeProfilerDecodeData) RangeDecodeData = nullptr;
    decltype(&cuptiRangeProfilerGetCounterDataInfo) RangeGetCounterDataInfo = nullptr;
    CUresult (*CtxGetCurrent)(CUcontext*) = nullptr;
};

template <typename F>
bool bind(void* lib, const char* name, F& fn)
{
    fn = reinterpret_cast<F>(dlsym(lib, name));
    return fn != nullptr;
}

const CuptiApi& cupti()
{
    static CuptiApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void* lib = dlopen("libcupti.so.12", RTLD_NOW | RTLD_LOCAL);
        if (lib == nullptr)
            lib = dlopen("libcupti.so", RTLD_NOW | RTLD_LOCAL);
        if (lib == nullptr) {
            api.error = std::string("libcupti could not be opened: ") + dlerror();
            return;
        }
        bool ok = bind(lib, "cuptiGetResultString", api.GetResultString) &&
                  bind(lib, "cuptiProfilerInitialize", api.ProfilerInitialize) &&
                  bind(lib, "cuptiDeviceGetChipName", api.DeviceGetChipName) &&
                  bind(lib, "cuptiProfilerGetCounterAvailability", api.GetCounterAvailability) &&
                  bind(lib, "cuptiProfilerHostInitialize", api.HostInitialize) &&
                  bind(lib, "cuptiProfilerHostDeinitialize", api.HostDeinitialize) &&
                  bind(lib, "cuptiProfilerHostConfigAddMetrics", api.HostConfigAddMetrics) &&
                  bind(lib, "cuptiProfilerHostGetConfigImageSize", api.HostGetConfigImageSize) &&
                  bind(lib, "cuptiProfilerHostGetConfigImage", api.HostGetConfigImage) &&
                  bind(lib, "cuptiProfilerHostGetNumOfPasses", api.HostGetNumOfPasses) &&
                  bind(lib, "cuptiProfilerHostEvaluateToGpuValues", api.HostEvaluateToGpuValues) &&
                  bind(lib, "cuptiRangeProfilerEnable", api.RangeEnable) &&
                  bind(lib, "cuptiRangeProfilerDisable", api.RangeDisable) &&
                  bind(lib, "cuptiRangeProfilerGetCounterDataSize", api.RangeGetCounterDataSize) &&
                  bind(lib, "cuptiRangeProfilerCounterDataImageInitialize", api.RangeCounterDataImageInitialize) &&
                  bind(lib, "cuptiRangeProfilerSetConfig", api.RangeSetConfig) &&
                  bind(lib, "cuptiRangeProfilerStart", api.RangeStart) &&
                  bind(lib, "cuptiRangeProfilerStop", api.RangeStop) &&
                  bind(lib, "cuptiRangeProfilerPushRange", api.RangePushRange) &&
                  bind(lib, "cuptiRangeProfilerPopRange", api.RangePopRange) &&
                  bind(lib, "cuptiRangeProfilerDecodeData", api.RangeDecodeData) &&
                  bind(lib, "cuptiRangeProfilerGetCounterDataInfo", api.RangeGetCounterDataInfo);
        if (!ok) {
            api.error = "libcupti lacks the range profiler API (CUDA 12.6 or newer is needed)";
            return;
        }
        // the driver (loaded by the runtime on a GPU machine) gives the context query; host-only use
        // (coul_profiler_supported) works without it
        void* driver = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
        if (driver == nullptr || !bind(driver, "cuCtxGetCurrent", api.CtxGetCurrent))
            api.CtxGetCurrent = nullptr;
        api.loaded = true;
    });
    return api;
}

int cupti_error(CUptiResult r, const char* what)
{
    const char* s = nullptr;
    if (cupti().GetResultString != nullptr)
        cupti().GetResultString(r, &s);
    return coul::set_error(COUL_ERR_CUDA, std::string("CUPTI ") + what + ": " +
                                              (s != nullptr ? std::string(s) : "error " + std::to_string(static_cast<int>(r))));
}

#define CUPTI_TRY(call, what)                          \
    do {                                               \
        const CUptiResult r_ = (call);                 \
        if (r_ != CUPTI_SUCCESS)                       \
            return cupti_error(r_, what);              \
    } while (0)

std::mutex g_active_mutex;
bool g_active = false;  // one range profiler per process

// Creates a host object for `chip`; availability may be null (host-only use).
int host_object(const char* chip, const uint8_t* availability, CUpti_Profiler_Host_Object** out)
{
    CUpti_Profiler_Host_Initialize_Params p{CUpti_Profiler_Host_Initialize_Params_STRUCT_SIZE};
    p.profilerType = CUPTI_PROFILER_TYPE_RANGE_PROFILER;
    p.pChipName = chip;
    p.pCounterAvailabilityImage = availability;
    CUPTI_TRY(cupti().HostInitialize(&p), "host initialisation");
    *out = p.pHostObject;
    return COUL_OK;
}

void host_release(CUpti_Profiler_Host_Object* host)
{
    if (host == nullptr)
        return;
    CUpti_Profiler_Host_Deinitialize_Params p{CUpti_Profiler_Host_Deinitialize_Params_STRUCT_SIZE};
    p.pHostObject = host;
    cupti().HostDeinitialize(&p);
}

// valid[i] = 1 when the chip accepts metric i on its own (a fresh host object per name, so one
// rejected name does not spoil the others).
int check_metrics(const char* chip, const uint8_t* availability, const char* const* metrics, int n, int* valid)
{
    for (int i = 0; i < n; ++i) {
        CUpti_Profiler_Host_Object* host = nullptr;
        int rc = host_object(chip, availability, &host);
        if (rc)
            return rc;
        CUpti_Profiler_Host_ConfigAddMetrics_Params p{CUpti_Profiler_Host_ConfigAddMetrics_Params_STRUCT_SIZE};
        p.pHostObject = host;
        const char* name = metrics[i];
        p.ppMetricNames = &name;
        p.numMetrics = 1;
        valid[i] = cupti().HostConfigAddMetrics(&p) == CUPTI_SUCCESS ? 1 : 0;
        host_release(host);
    }
    return COUL_OK;
}

}  // namespace

struct coul_profiler {
    coul_ctx* ctx = nullptr;
    CUpti_Profiler_Host_Object* host = nullptr;
    CUpti_RangeProfiler_Object* range = nullptr;
    std::vector<std::string> names;        // requested metrics
    std::vector<int> valid;                // accepted by the chip
    std::vector<const char*> collected;    // the accepted ones, in order
    std::vector<uint8_t> config;
    std::vector<uint8_t> counter_data;
    int passes = 0;
    bool in_pass = false;
    bool done = false;
};

namespace {

void release(coul_profiler* p)
{
    if (p->range != nullptr) {
        if (p->in_pass) {
            CUpti_RangeProfiler_PopRange_Params pop{CUpti_RangeProfiler_PopRange_Params_STRUCT_SIZE};
            pop.pRangeProfilerObject = p->range;
            cupti().RangePopRange(&pop);
            CUpti_RangeProfiler_Stop_Params stop{CUpti_RangeProfiler_Stop_Params_STRUCT_SIZE};
            stop.pRangeProfilerObject = p->range;
            cupti().RangeStop(&stop);
        }
        CUpti_RangeProfiler_Disable_Params d{CUpti_RangeProfiler_Disable_Params_STRUCT_SIZE};
        d.pRangeProfilerObject = p->range;
        cupti().RangeDisable(&d);
        p->range = nullptr;
    }
    host_release(p->host);
    p->host = nullptr;
}

int create(coul_profiler* p, const char* const* metrics, int n)
{
    const CuptiApi& api = cupti();
    coul_ctx* ctx = p->ctx;
    static std::once_flag init_once;
    static CUptiResult init_result = CUPTI_SUCCESS;
    std::call_once(init_once, [&] {
        CUpti_Profiler_Initialize_Params ip{CUpti_Profiler_Initialize_Params_STRUCT_SIZE};
        init_result = api.ProfilerInitialize(&ip);
    });
    CUPTI_TRY(init_result, "profiler initialisation");

    // the runtime's primary context of the device, current after activation
    cudaError_t e = cudaFree(nullptr);
    if (e != cudaSuccess)
        return coul::cuda_error(e, "context initialisation");
    CUcontext cu = nullptr;
    if (api.CtxGetCurrent == nullptr)
        return coul::set_error(COUL_ERR_UNSUPPORTED, "libcuda.so.1 does not export cuCtxGetCurrent");
    if (api.CtxGetCurrent(&cu) != CUDA_SUCCESS || cu == nullptr)
        return coul::set_error(COUL_ERR_CUDA, "no current CUDA context for the profiler");

    CUpti_Device_GetChipName_Params chip{CUpti_Device_GetChipName_Params_STRUCT_SIZE};
    chip.deviceIndex = static_cast<size_t>(ctx->device);
    CUPTI_TRY(api.DeviceGetChipName(&chip), "chip name");

    CUpti_Profiler_GetCounterAvailability_Params av{CUpti_Profiler_GetCounterAvailability_Params_STRUCT_SIZE};
    av.ctx = cu;
    CUPTI_TRY(api.GetCounterAvailability(&av), "counter availability size");
    std::vector<uint8_t> availability(av.counterAvailabilityImageSize);
    av.pCounterAvailabilityImage = availability.data();
    CUPTI_TRY(api.GetCounterAvailability(&av), "counter availability");

    p->names.assign(metrics, metrics + n);
    p->valid.assign(static_cast<size_t>(n), 0);
    int rc = check_metrics(chip.pChipName, availability.data(), metrics, n, p->valid.data());
    if (rc)
        return rc;
    for (int i = 0; i < n; ++i)
        if (p->valid[static_cast<size_t>(i)])
            p->collected.push_back(p->names[static_cast<size_t>(i)].c_str());
    if (p->collected.empty())
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, std::string("no requested metric is offered by ") + chip.pChipName);

    if ((rc = host_object(chip.pChipName, availability.data(), &p->host)))
        return rc;
    CUpti_Profiler_Host_ConfigAddMetrics_Params add{CUpti_Profiler_Host_ConfigAddMetrics_Params_STRUCT_SIZE};
    add.pHostObject = p->host;
    add.ppMetricNames = p->collected.data();
    add.numMetrics = p->collected.size();
    CUPTI_TRY(api.HostConfigAddMetrics(&add), "metric configuration");
    CUpti_Profiler_Host_GetConfigImageSize_Params cs{CUpti_Profiler_Host_GetConfigImageSize_Params_STRUCT_SIZE};
    cs.pHostObject = p->host;
    CUPTI_TRY(api.HostGetConfigImageSize(&cs), "configuration image size");
    p->config.resize(cs.configImageSize);
    CUpti_Profiler_Host_GetConfigImage_Params ci{CUpti_Profiler_Host_GetConfigImage_Params_STRUCT_SIZE};
    ci.pHostObject = p->host;
    ci.configImageSize = p->config.size();
    ci.pConfigImage = p->config.data();
    CUPTI_TRY(api.HostGetConfigImage(&ci), "configuration image");
    CUpti_Profiler_Host_GetNumOfPasses_Params np{CUpti_Profiler_Host_GetNumOfPasses_Params_STRUCT_SIZE};
    np.configImageSize = p->config.size();
    np.pConfigImage = p->config.data();
    CUPTI_TRY(api.HostGetNumOfPasses(&np), "pass count");
    p->passes = static_cast<int>(np.numOfPasses);

    CUpti_RangeProfiler_Enable_Params en{CUpti_RangeProfiler_Enable_Params_STRUCT_SIZE};
    en.ctx = cu;
    CUPTI_TRY(api.RangeEnable(&en), "range profiler enable");
    p->range = en.pRangeProfilerObject;

    CUpti_RangeProfiler_GetCounterDataSize_Params ds{CUpti_RangeProfiler_GetCounterDataSize_Params_STRUCT_SIZE};
    ds.pRangeProfilerObject = p->range;
    ds.pMetricNames = p->collected.data();
    ds.numMetrics = p->collected.size();
    ds.maxNumOfRanges = 1;
    ds.maxNumRangeTreeNodes = 1;
    CUPTI_TRY(api.RangeGetCounterDataSize(&ds), "counter data size");
    p->counter_data.resize(ds.counterDataSize);
    CUpti_RangeProfiler_CounterDataImage_Initialize_Params di{
        CUpti_RangeProfiler_CounterDataImage_Initialize_Params_STRUCT_SIZE};
    di.pRangeProfilerObject = p->range;
    di.counterDataSize = p->counter_data.size();
    di.pCounterData = p->counter_data.data();
    CUPTI_TRY(api.RangeCounterDataImageInitialize(&di), "counter data image");

    // one user range per pass, the caller replaying the launches (auto ranges record nothing here)
    CUpti_RangeProfiler_SetConfig_Params sc{CUpti_RangeProfiler_SetConfig_Params_STRUCT_SIZE};
    sc.pRangeProfilerObject = p->range;
    sc.configSize = p->config.size();
    sc.pConfig = p->config.data();
    sc.counterDataImageSize = p->counter_data.size();
    sc.pCounterDataImage = p->counter_data.data();
    sc.range = CUPTI_UserRange;
    sc.replayMode = CUPTI_UserReplay;
    sc.maxRangesPerPass = 1;
    sc.numNestingLevels = 1;
    sc.minNestingLevel = 1;
    sc.passIndex = 0;
    sc.targetNestingLevel = 1;
    CUPTI_TRY(api.RangeSetConfig(&sc), "range profiler configuration");
    return COUL_OK;
}

}  // namespace

COUL_API int coul_profiler_supported(const char* chip, const char* const* metrics, int n_metrics, int* valid)
{
    if (chip == nullptr || n_metrics < 0 || (n_metrics > 0 && (metrics == nullptr || valid == nullptr)))
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "chip, metrics or valid is NULL");
    for (int i = 0; i < n_metrics; ++i)
        if (metrics[i] == nullptr)
            return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "metric name is NULL");
    if (!cupti().loaded)
        return coul::set_error(COUL_ERR_UNSUPPORTED, cupti().error);
    return check_metrics(chip, nullptr, metrics, n_metrics, valid);
}

COUL_API int coul_profiler_create(coul_ctx* ctx, const char* const* metrics, int n_metrics, int* valid,
                                  coul_profiler** out, int* passes)
{
    if (ctx == nullptr || out == nullptr || metrics == nullptr || n_metrics <= 0)
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "ctx, metrics or out is NULL, or no metric named");
    for (int i = 0; i < n_metrics; ++i)
        if (metrics[i] == nullptr)
            return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "metric name is NULL");
    *out = nullptr;
    if (!cupti().loaded)
        return coul::set_error(COUL_ERR_UNSUPPORTED, cupti().error);
    int rc = coul::ctx_activate(ctx);
    if (rc)
        return rc;
    {
        std::lock_guard<std::mutex> lock(g_active_mutex);
        if (g_active)
            return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "another profiler is active in this process");
        g_active = true;
    }
    auto* p = new coul_profiler();
    p->ctx = ctx;
    rc = create(p, metrics, n_metrics);
    if (rc) {
        release(p);
        delete p;
        std::lock_guard<std::mutex> lock(g_active_mutex);
        g_active = false;
        return rc;
    }
    if (valid != nullptr)
        std::memcpy(valid, p->valid.data(), sizeof(int) * static_cast<size_t>(n_metrics));
    if (passes != nullptr)
        *passes = p->passes;
    *out = p;
    return COUL_OK;
}

COUL_API int coul_profiler_begin_pass(coul_profiler* p)
{
    if (p == nullptr || p->range == nullptr)
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "profiler is NULL");
    if (p->in_pass || p->done)
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, p->done ? "every pass is already collected" : "pass already begun");
    int rc = coul::ctx_activate(p->ctx);
    if (rc)
        return rc;
    CUpti_RangeProfiler_Start_Params st{CUpti_RangeProfiler_Start_Params_STRUCT_SIZE};
    st.pRangeProfilerObject = p->range;
    CUPTI_TRY(cupti().RangeStart(&st), "range profiler start");
    CUpti_RangeProfiler_PushRange_Params push{CUpti_RangeProfiler_PushRange_Params_STRUCT_SIZE};
    push.pRangeProfilerObject = p->range;
    push.pRangeName = "ktt";
    const CUptiResult r = cupti().RangePushRange(&push);
    if (r != CUPTI_SUCCESS) {
        CUpti_RangeProfiler_Stop_Params stop{CUpti_RangeProfiler_Stop_Params_STRUCT_SIZE};
        stop.pRangeProfilerObject = p->range;
        cupti().RangeStop(&stop);
        return cupti_error(r, "range push");
    }
    p->in_pass = true;
    return COUL_OK;
}

COUL_API int coul_profiler_end_pass(coul_profiler* p, int* all_passes_done)
{
    if (p == nullptr || p->range == nullptr || !p->in_pass)
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "no pass has begun");
    p->in_pass = false;
    CUpti_RangeProfiler_PopRange_Params pop{CUpti_RangeProfiler_PopRange_Params_STRUCT_SIZE};
    pop.pRangeProfilerObject = p->range;
    const CUptiResult popped = cupti().RangePopRange(&pop);
    CUpti_RangeProfiler_Stop_Params stop{CUpti_RangeProfiler_Stop_Params_STRUCT_SIZE};
    stop.pRangeProfilerObject = p->range;
    CUPTI_TRY(cupti().RangeStop(&stop), "range profiler stop");
    CUPTI_TRY(popped, "range pop");
    p->done = stop.isAllPassSubmitted != 0;
    if (all_passes_done != nullptr)
        *all_passes_done = p->done ? 1 : 0;
    return COUL_OK;
}

COUL_API int coul_profiler_read(coul_profiler* p, double* values)
{
    if (p == nullptr || values == nullptr)
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "profiler or values is NULL");
    if (!p->done)
        return coul::set_error(COUL_ERR_INVALID_ARGUMENT, "passes remain to be run");
    const cudaError_t e = cudaStreamSynchronize(p->ctx->stream);
    if (e != cudaSuccess)
        return coul::cuda_error(e, "profiled launches");
    CUpti_RangeProfiler_DecodeData_Params dd{CUpti_RangeProfiler_DecodeData_Params_STRUCT_SIZE};
    dd.pRangeProfilerObject = p->range;
    CUPTI_TRY(cupti().RangeDecodeData(&dd), "counter decode");
    CUpti_RangeProfiler_GetCounterDataInfo_Params info{CUpti_RangeProfiler_GetCounterDataInfo_Params_STRUCT_SIZE};
    info.pCounterDataImage = p->counter_data.data();
    info.counterDataImageSize = p->counter_data.size();
    CUPTI_TRY(cupti().RangeGetCounterDataInfo(&info), "counter data info");
    if (info.numTotalRanges < 1)
        return coul::set_error(COUL_ERR_CUDA, "the profiled range holds no counter data");
    std::vector<double> collected(p->collected.size(), NAN);
    CUpti_Profiler_Host_EvaluateToGpuValues_Params ev{CUpti_Profiler_Host_EvaluateToGpuValues_Params_STRUCT_SIZE};
    ev.pHostObject = p->host;
    ev.pCounterDataImage = p->counter_data.data();
    ev.counterDataImageSize = p->counter_data.size();
    ev.rangeIndex = 0;
    ev.ppMetricNames = p->collected.data();
    ev.numMetrics = p->collected.size();
    ev.pMetricValues = collected.data();
    CUPTI_TRY(cupti().HostEvaluateToGpuValues(&ev), "metric evaluation");
    size_t k = 0;
    for (size_t i = 0; i < p->names.size(); ++i)
        values[i] = p->valid[i] ? collected[k++] : NAN;
    return COUL_OK;
}

COUL_API int coul_profiler_destroy(coul_profiler* p)
{
    if (p == nullptr)
        return COUL_OK;
    if (p->ctx != nullptr)
        (void)coul::ctx_activate(p->ctx);
    release(p);
    delete p;
    std::lock_guard<std::mutex> lock(g_active_mutex);
    g_active = false;
    return COUL_OK;
}
