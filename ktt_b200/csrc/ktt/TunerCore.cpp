// TunerCore.cpp -- the machinery behind ktt::Tuner (see TunerCore.h for the KTT parts it restates).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "Logger.h"
#include "TunerCore.h"

namespace ktt
{

namespace
{

using Clock = std::chrono::steady_clock;

Nanoseconds ElapsedNs(const Clock::time_point start)
{
    return static_cast<Nanoseconds>(std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - start).count());
}

ResultStatus StatusFromCoul(const int rc)
{
    switch (rc)
    {
    case COUL_ERR_UNSUPPORTED: return ResultStatus::CompilationFailed;
    case COUL_ERR_DEVICE_LIMITS: return ResultStatus::DeviceLimitsExceeded;
    default: return ResultStatus::ComputationFailed;
    }
}

void CheckCoul(const int rc, const std::string& what)
{
    if (rc != COUL_OK)
    {
        throw RunFailure(StatusFromCoul(rc), what + ": " + coul_last_error());
    }
}

// Atom-loop unroll for KTT's INNER_UNROLL_FACTOR: 0 (no pragma) and 1 are none; values above 8
// use the 8-way variant (the register-blocked z loop is always fully unrolled here, so KTT's
// z-loop unroll has no separate counterpart).
int UnrollFor(const uint64_t factor)
{
    if (factor <= 1) return 1;
    if (factor < 4) return 2;
    if (factor < 8) return 4;
    return 8;
}

} // namespace

// ---- compute layer for custom launchers ------------------------------------------------------

class ComputeLayer : public ComputeInterface
{
public:
    ComputeLayer(TunerCore& core, const KernelData& kernel, const KernelConfiguration& configuration, const KernelRunMode mode) :
        m_Core(core), m_Kernel(kernel), m_Configuration(configuration), m_Mode(mode)
    {
        for (const auto id : kernel.definitions)
        {
            m_Global[id] = core.ModifiedSize(kernel, id, ModifierType::Global, configuration);
            m_Local[id] = core.ModifiedSize(kernel, id, ModifierType::Local, configuration);
        }
    }

    void RunKernel(const KernelDefinitionId id) override { RunKernel(id, GetCurrentGlobalSize(id), GetCurrentLocalSize(id)); }
    void RunKernelWithProfiling(const KernelDefinitionId id) override { RunKernel(id); }

    void RunKernelWithProfiling(const KernelDefinitionId id, const DimensionVector& globalSize,
        const DimensionVector& localSize) override
    {
        RunKernel(id, globalSize, localSize);
    }

    uint64_t GetRemainingProfilingRuns([[maybe_unused]] const KernelDefinitionId id) const override { return 0; }
    uint64_t GetRemainingProfilingRuns() const override { return 0; }

    void RunKernel(const KernelDefinitionId id, const DimensionVector& globalSize, const DimensionVector& localSize) override
    {
        const auto start = Clock::now();
        const Nanoseconds duration = m_Core.LaunchDefinition(m_Kernel, id, m_Configuration, globalSize, localSize);
        const Nanoseconds wall = ElapsedNs(start);
        auto it = m_Results.find(id);

        if (it == m_Results.end())
        {
            ComputationResult result(m_Core.Definition(id).name);
            result.SetSizeData(m_Core.GridSize(globalSize, localSize), localSize);
            result.SetDurationData(duration, wall > duration ? wall - duration : 0);
            m_Results.emplace(id, result);
            m_Order.push_back(id);
        }
        else
        {
            const Nanoseconds d = it->second.GetDuration() + duration;
            const Nanoseconds o = it->second.GetOverhead() + (wall > duration ? wall - duration : 0);
            it->second.SetDurationData(d, o);
        }
    }

    // the launch runs on the queue's stream; it completes before the call returns
    ComputeActionId RunKernelAsync(const KernelDefinitionId id, const QueueId queue) override
    {
        m_Core.OnQueue(queue, [&] { RunKernel(id); });
        return m_NextAction++;
    }

    ComputeActionId RunKernelAsync(const KernelDefinitionId id, const QueueId queue,
        const DimensionVector& globalSize, const DimensionVector& localSize) override
    {
        m_Core.OnQueue(queue, [&] { RunKernel(id, globalSize, localSize); });
        return m_NextAction++;
    }

    void WaitForComputeAction([[maybe_unused]] const ComputeActionId id) override { m_Core.Synchronize(); }
    QueueId GetDefaultQueue() const override { return m_Core.QueueIds().front(); }
    std::vector<QueueId> GetAllQueues() const override { return m_Core.QueueIds(); }
    void SynchronizeQueue(const QueueId queue) override { m_Core.SynchronizeQueue(queue); }
    void SynchronizeQueues() override
    {
        for (const auto queue : m_Core.QueueIds())
        {
            m_Core.SynchronizeQueue(queue);
        }
    }
    void SynchronizeDevice() override { m_Core.Synchronize(); }

    const DimensionVector& GetCurrentGlobalSize(const KernelDefinitionId id) const override { return SizeOf(m_Global, id); }
    const DimensionVector& GetCurrentLocalSize(const KernelDefinitionId id) const override { return SizeOf(m_Local, id); }
    const KernelConfiguration& GetCurrentConfiguration() const override { return m_Configuration; }
    KernelRunMode GetRunMode() const override { return m_Mode; }

    void ChangeArguments(const KernelDefinitionId id, const std::vector<ArgumentId>& arguments) override
    {
        m_Core.SetArguments(id, arguments);
    }

    void SwapArguments(const KernelDefinitionId id, const ArgumentId& first, const ArgumentId& second) override
    {
        auto& arguments = m_Core.Definition(id).arguments;
        auto a = std::find(arguments.begin(), arguments.end(), first);
        auto b = std::find(arguments.begin(), arguments.end(), second);

        if (a == arguments.end() || b == arguments.end())
        {
            throw std::runtime_error("SwapArguments: argument not used by the definition");
        }

        std::iter_swap(a, b);
    }

    void UpdateScalarArgument(const ArgumentId& id, const void* data) override
    {
        ArgumentData& argument = m_Core.Argument(id);

        if (argument.memoryType != ArgumentMemoryType::Scalar)
        {
            throw std::runtime_error("Argument " + id + " is not a scalar");
        }

        m_Core.OverrideScalar(id, data);
    }

    void UploadBuffer(const ArgumentId& id) override { m_Core.UploadArgument(m_Core.Argument(id), true); }

    void DownloadBuffer(const ArgumentId& id, void* destination, const size_t dataSize) override
    {
        m_Core.DownloadArgument(m_Core.Argument(id), destination, dataSize);
    }

    void UpdateBuffer(const ArgumentId& id, const void* data, const size_t dataSize) override
    {
        ArgumentData& argument = m_Core.Argument(id);
        m_Core.UpdateArgumentDevice(argument, data, dataSize);
    }

    void CopyBuffer(const ArgumentId& destination, const ArgumentId& source, const size_t dataSize) override
    {
        ArgumentData& dst = m_Core.Argument(destination);
        ArgumentData& src = m_Core.Argument(source);
        m_Core.UploadArgument(dst, false);
        m_Core.UploadArgument(src, false);
        const size_t bytes = dataSize == 0 ? std::min(TunerCore::DeviceBytes(dst), TunerCore::DeviceBytes(src)) : dataSize;
        void* d = dst.ownership == ArgumentOwnership::User ? dst.userDevice : dst.device;
        const void* s = src.ownership == ArgumentOwnership::User ? src.userDevice : src.device;
        CheckCoul(coul_buffer_copy(m_Core.Context(), d, s, bytes), "CopyBuffer");
    }

    void ClearBuffer(const ArgumentId& id) override
    {
        ArgumentData& argument = m_Core.Argument(id);
        m_Core.UploadArgument(argument, false);
        void* d = argument.ownership == ArgumentOwnership::User ? argument.userDevice : argument.device;
        CheckCoul(coul_buffer_memset(m_Core.Context(), d, 0, TunerCore::DeviceBytes(argument)), "ClearBuffer");
    }

    bool HasBuffer(const ArgumentId& id) override
    {
        const ArgumentData& argument = m_Core.Argument(id);
        return argument.ownership == ArgumentOwnership::User || argument.device != nullptr;
    }

    TransferActionId UploadBufferAsync(const ArgumentId& id, const QueueId queue) override
    {
        m_Core.OnQueue(queue, [&] { UploadBuffer(id); });
        return m_NextTransfer++;
    }

    TransferActionId DownloadBufferAsync(const ArgumentId& id, const QueueId queue, void* destination,
        const size_t dataSize) override
    {
        m_Core.OnQueue(queue, [&] { DownloadBuffer(id, destination, dataSize); });
        return m_NextTransfer++;
    }

    TransferActionId UpdateBufferAsync(const ArgumentId& id, const QueueId queue, const void* data, const size_t dataSize) override
    {
        m_Core.OnQueue(queue, [&] { UpdateBuffer(id, data, dataSize); });
        return m_NextTransfer++;
    }

    TransferActionId CopyBufferAsync(const ArgumentId& destination, const ArgumentId& source, const QueueId queue,
        const size_t dataSize) override
    {
        m_Core.OnQueue(queue, [&] { CopyBuffer(destination, source, dataSize); });
        return m_NextTransfer++;
    }

    void WaitForTransferAction([[maybe_unused]] const TransferActionId id) override { m_Core.Synchronize(); }

    void ResizeBuffer(const ArgumentId& id, const size_t newDataSize, const bool preserveData) override
    {
        m_Core.ResizeArgument(m_Core.Argument(id), newDataSize, preserveData);
    }

    void UpdateLocalArgument(const ArgumentId& id, const size_t dataSize) override
    {
        const ArgumentData& argument = m_Core.Argument(id);

        if (argument.memoryType != ArgumentMemoryType::Local || dataSize == 0)
        {
            throw std::runtime_error("Argument " + id + " is not a local memory argument, or the size is zero");
        }

        // A per-run override in KTT (ComputeLayer.cpp:175-186) that sets the launch's dynamic shared
        // memory; the built-in kernels size their own shared memory, so the stored argument is left
        // as it is and nothing carries over to later runs.
    }

    void GetUnifiedMemoryBufferHandle(const ArgumentId& id, [[maybe_unused]] UnifiedBufferMemory& memoryHandle) override
    {
        throw std::runtime_error("Argument " + id + " is not in unified memory (this build keeps arguments in device memory)");
    }

    bool GetProfiling([[maybe_unused]] const KernelId id) override { return m_Core.GetProfiling(); }

    std::vector<ComputationResult> Results() const
    {
        std::vector<ComputationResult> out;

        for (const auto id : m_Order)
        {
            out.push_back(m_Results.at(id));
        }

        return out;
    }

private:
    TunerCore& m_Core;
    const KernelData& m_Kernel;
    KernelConfiguration m_Configuration;
    KernelRunMode m_Mode;
    std::map<KernelDefinitionId, DimensionVector> m_Global;
    std::map<KernelDefinitionId, DimensionVector> m_Local;
    std::map<KernelDefinitionId, ComputationResult> m_Results;
    std::vector<KernelDefinitionId> m_Order;
    ComputeActionId m_NextAction = 0;
    TransferActionId m_NextTransfer = 0;

    static const DimensionVector& SizeOf(const std::map<KernelDefinitionId, DimensionVector>& sizes, const KernelDefinitionId id)
    {
        auto it = sizes.find(id);

        if (it == sizes.end())
        {
            throw std::runtime_error("Definition " + std::to_string(id) + " is not part of the kernel");
        }

        return it->second;
    }
};

// ---- TunerCore --------------------------------------------------------------------------------

TunerCore::TunerCore(const DeviceIndex device, const ComputeApi api) :
    m_Device(device), m_Api(api), m_Context(nullptr), m_GlobalSizeType(GlobalSizeType::OpenCL), m_Profiling(false),
    m_ReadOnlyCache(true), m_ValidationMethod(ValidationMethod::SideBySideComparison), m_ValidationThreshold(1e-4),
    m_ValidationMode(ValidationMode::OfflineTuning | ValidationMode::OnlineTuning), m_NextDefinition(0), m_NextKernel(0),
    m_NextArgument(0)
{
    if (api == ComputeApi::Vulkan)
    {
        throw std::runtime_error("This build has no Vulkan engine; it runs the built-in CUDA kernels for sm_100a");
    }

    if (api == ComputeApi::OpenCL)
    {
        // KTT's OpenCL host programs for this path (Examples/CoulombSum2d/CoulombSum2d.cpp,
        // Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp) run unchanged: their definitions
        // are matched by kernel name and argument list to the same built-in kernels, with KTT's
        // OpenCL global-size convention; the .cl sources are never compiled.
        log::Info("ComputeApi::OpenCL requested: definitions run on the built-in CUDA kernels (sm_100a)");
    }
}

TunerCore::~TunerCore()
{
    if (m_Context != nullptr)
    {
        for (auto& [id, argument] : m_Arguments)
        {
            if (argument.device != nullptr)
            {
                coul_buffer_free(m_Context, argument.device);
            }
        }

        if (m_ScratchDevice != nullptr)
        {
            coul_buffer_free(m_Context, m_ScratchDevice);
        }

        for (auto& [key, batch] : m_Batches)
        {
            coul_batch_destroy(batch);
        }

        coul_ctx_destroy(m_Context);
    }
}

coul_ctx* TunerCore::Context()
{
    if (m_Context == nullptr)
    {
        const int rc = m_UserContext != nullptr
            ? coul_ctx_create_on(m_UserContext, m_Queues.front().second, &m_Context)
            : coul_ctx_create(static_cast<int>(m_Device), &m_Context);

        if (rc != COUL_OK)
        {
            m_Context = nullptr;
            throw RunFailure(ResultStatus::ComputationFailed, std::string("device initialisation failed: ") + coul_last_error());
        }

        int device = 0;
        CheckCoul(coul_ctx_device(m_Context, &device), "device index");
        m_Device = static_cast<DeviceIndex>(device);
    }

    return m_Context;
}

// ---- queues: the caller's streams (KTT: CudaEngine.cpp:67-106 adopts the initializer's context and
// streams; AddComputeQueue / RemoveComputeQueue, Tuner.h:851-863) --

void TunerCore::AdoptContext(const ComputeApiInitializer& initializer, std::vector<QueueId>& assigned)
{
    if (initializer.GetContext() == nullptr || initializer.GetQueues().empty())
    {
        throw std::runtime_error("Compute API initializer needs a context and at least one queue");
    }

    if (m_Api != ComputeApi::CUDA)
    {
        throw std::runtime_error("Compute API initializer: only a CUDA context and CUDA streams can be adopted");
    }

    m_UserContext = initializer.GetContext();
    assigned.clear();

    for (const auto queue : initializer.GetQueues())
    {
        assigned.push_back(AddQueue(queue));
    }
}

QueueId TunerCore::AddQueue(ComputeQueue queue)
{
    if (m_UserContext == nullptr)
    {
        throw std::runtime_error("New queues can only be added to a tuner created with a compute API initializer");
    }

    if (queue == nullptr)
    {
        throw std::runtime_error("Queue must be a stream of the initializer's context");
    }

    for (const auto& [id, stream] : m_Queues)
    {
        if (stream == queue)
        {
            throw std::runtime_error("Queue was already added with id " + std::to_string(id));
        }
    }

    const QueueId id = m_NextQueue++;
    m_Queues.emplace_back(id, queue);
    return id;
}

void TunerCore::RemoveQueue(const QueueId id)
{
    if (m_UserContext == nullptr)
    {
        throw std::runtime_error("Queues can only be removed from a tuner created with a compute API initializer");
    }

    const auto it = std::find_if(m_Queues.begin(), m_Queues.end(), [id](const auto& q) { return q.first == id; });

    if (it == m_Queues.end())
    {
        throw std::runtime_error("Invalid queue id: " + std::to_string(id));
    }

    if (m_Queues.size() == 1)
    {
        throw std::runtime_error("The last queue of a tuner cannot be removed");
    }

    const bool current = m_Context != nullptr && coul_ctx_get_stream(m_Context) == it->second;

    if (m_Context != nullptr)
    {
        CheckCoul(coul_synchronize(m_Context), "synchronize before a queue is removed");
    }

    m_Queues.erase(it);

    if (current)
    {
        CheckCoul(coul_ctx_set_stream(m_Context, m_Queues.front().second), "queue switch");
    }
}

std::vector<QueueId> TunerCore::QueueIds() const
{
    if (m_UserContext == nullptr)
    {
        return {0};
    }

    std::vector<QueueId> ids;

    for (const auto& q : m_Queues)
    {
        ids.push_back(q.first);
    }

    return ids;
}

void TunerCore::OnQueue(const QueueId id, const std::function<void()>& work)
{
    if (m_UserContext == nullptr)
    {
        if (id != 0)
        {
            throw std::runtime_error("Invalid queue id: " + std::to_string(id) + " (this tuner has queue 0)");
        }

        work();
        return;
    }

    const auto it = std::find_if(m_Queues.cbegin(), m_Queues.cend(), [id](const auto& q) { return q.first == id; });

    if (it == m_Queues.cend())
    {
        throw std::runtime_error("Invalid queue id: " + std::to_string(id));
    }

    coul_ctx* ctx = Context();
    void* previous = coul_ctx_get_stream(ctx);
    CheckCoul(coul_ctx_set_stream(ctx, it->second), "queue switch");

    try
    {
        work();
    }
    catch (...)
    {
        coul_ctx_set_stream(ctx, previous);
        throw;
    }

    CheckCoul(coul_ctx_set_stream(ctx, previous), "queue switch");
}

void TunerCore::SynchronizeQueue(const QueueId id)
{
    OnQueue(id, [this] { Synchronize(); });
}

void TunerCore::Synchronize()
{
    if (m_Context != nullptr)
    {
        CheckCoul(coul_synchronize(m_Context), "synchronize");
    }
}

// KTT's CUDA device description (CudaDevice.cpp:26-58) from the C ABI's property query.
DeviceInfo TunerCore::QueryDevice(const DeviceIndex index)
{
    coul_device_props props{};
    CheckCoul(coul_device_query(static_cast<int>(index), &props), "device query");
    DeviceInfo info(index, props.name);
    info.SetVendor("NVIDIA Corporation");
    info.SetExtensions("N/A");
    info.SetDeviceType(DeviceType::GPU);
    info.SetGlobalMemorySize(props.global_memory);
    info.SetLocalMemorySize(props.shared_memory_block);
    info.SetMaxConstantBufferSize(props.constant_memory);
    info.SetMaxWorkGroupSize(static_cast<uint64_t>(props.max_threads_block));
    info.SetMaxComputeUnits(static_cast<uint32_t>(props.sm_count));
    info.SetCudaComputeCapabilityMajor(static_cast<uint32_t>(props.cc_major));
    info.SetCudaComputeCapabilityMinor(static_cast<uint32_t>(props.cc_minor));
    return info;
}

DeviceInfo TunerCore::GetDeviceInfo()
{
    Context();  // the tuner's device must be usable
    return QueryDevice(m_Device);
}

std::vector<DeviceInfo> TunerCore::GetDeviceInfo(const PlatformIndex platform)
{
    if (platform != 0)
    {
        throw std::runtime_error("CUDA has one platform, index 0; requested " + std::to_string(platform));
    }

    int count = 0;
    CheckCoul(coul_device_count(&count), "device count");
    std::vector<DeviceInfo> result;

    for (int i = 0; i < count; ++i)
    {
        result.push_back(QueryDevice(static_cast<DeviceIndex>(i)));
    }

    return result;
}

std::vector<PlatformInfo> TunerCore::GetPlatformInfo()
{
    int count = 0;
    CheckCoul(coul_device_count(&count), "device count");
    coul_device_props props{};
    PlatformInfo info(0, "NVIDIA CUDA");
    info.SetVendor("NVIDIA Corporation");
    info.SetVersion(count > 0 && coul_device_query(0, &props) == COUL_OK ? std::to_string(props.driver_version) : "N/A");
    info.SetExtensions("N/A");
    return {info};
}

std::string TunerCore::DeviceName()
{
    try
    {
        return GetDeviceInfo().GetName();
    }
    catch (const std::exception&)
    {
        return "unavailable";
    }
}

// -- kernels --

KernelDefinitionId TunerCore::AddDefinition(const std::string& name, const std::string& source, const DimensionVector& global,
    const DimensionVector& local, const std::vector<std::string>& typeNames)
{
    if (GetDefinitionId(name, typeNames) != InvalidKernelDefinitionId)
    {
        throw std::runtime_error("Kernel definition with name " + name + " and the same template types already exists");
    }

    DefinitionData data;
    data.id = m_NextDefinition++;
    data.name = name;
    data.source = source;
    data.globalSize = global;
    data.localSize = local;
    data.typeNames = typeNames;
    m_Definitions[data.id] = data;
    return data.id;
}

KernelDefinitionId TunerCore::GetDefinitionId(const std::string& name, const std::vector<std::string>& typeNames) const
{
    for (const auto& [id, data] : m_Definitions)
    {
        if (data.name == name && data.typeNames == typeNames)
        {
            return id;
        }
    }

    return InvalidKernelDefinitionId;
}

void TunerCore::RemoveDefinition(const KernelDefinitionId id)
{
    for (const auto& [kid, kernel] : m_Kernels)
    {
        if (std::find(kernel.definitions.cbegin(), kernel.definitions.cend(), id) != kernel.definitions.cend())
        {
            throw std::runtime_error("Definition " + std::to_string(id) + " is used by kernel " + kernel.name);
        }
    }

    if (m_Definitions.erase(id) == 0)
    {
        throw std::runtime_error("Invalid kernel definition id " + std::to_string(id));
    }
}

DefinitionData& TunerCore::Definition(const KernelDefinitionId id)
{
    auto it = m_Definitions.find(id);

    if (it == m_Definitions.end())
    {
        throw std::runtime_error("Invalid kernel definition id " + std::to_string(id));
    }

    return it->second;
}

const DefinitionData& TunerCore::Definition(const KernelDefinitionId id) const
{
    return const_cast<TunerCore*>(this)->Definition(id);
}

void TunerCore::SetArguments(const KernelDefinitionId id, const std::vector<ArgumentId>& arguments)
{
    for (const auto& a : arguments)
    {
        (void)Argument(a);
    }

    Definition(id).arguments = arguments;
}

KernelId TunerCore::CreateKernel(const std::string& name, const std::vector<KernelDefinitionId>& definitions,
    KernelLauncher launcher)
{
    if (definitions.empty())
    {
        throw std::runtime_error("A kernel needs at least one definition");
    }

    for (const auto id : definitions)
    {
        (void)Definition(id);
    }

    for (const auto& [id, kernel] : m_Kernels)
    {
        if (kernel.name == name)
        {
            throw std::runtime_error("Kernel with name " + name + " already exists");
        }
    }

    KernelData& kernel = m_Kernels[m_NextKernel];
    kernel.id = m_NextKernel++;
    kernel.name = name;
    kernel.definitions = definitions;
    kernel.launcher = std::move(launcher);
    return kernel.id;
}

void TunerCore::RemoveKernel(const KernelId id)
{
    if (m_Kernels.erase(id) == 0)
    {
        throw std::runtime_error("Invalid kernel id " + std::to_string(id));
    }
}

KernelData& TunerCore::Kernel(const KernelId id)
{
    auto it = m_Kernels.find(id);

    if (it == m_Kernels.end())
    {
        throw std::runtime_error("Invalid kernel id " + std::to_string(id));
    }

    return it->second;
}

const KernelData& TunerCore::Kernel(const KernelId id) const { return const_cast<TunerCore*>(this)->Kernel(id); }
void TunerCore::SetLauncher(const KernelId id, KernelLauncher launcher) { Kernel(id).launcher = std::move(launcher); }

void TunerCore::AddParameter(const KernelId id, const std::string& name, const std::vector<ParameterValue>& values,
    const std::string& group)
{
    KernelData& kernel = Kernel(id);

    for (const auto& p : kernel.parameters)
    {
        if (p.name == name)
        {
            throw std::runtime_error("Kernel parameter with name " + name + " already exists");
        }
    }

    if (values.empty())
    {
        throw std::runtime_error("Kernel parameter " + name + " needs at least one value");
    }

    const auto type = ParameterPair::GetTypeFromValue(values.front());

    for (const auto& v : values)
    {
        if (ParameterPair::GetTypeFromValue(v) != type)
        {
            throw std::runtime_error("All values of kernel parameter " + name + " must have the same type");
        }
    }

    kernel.parameters.push_back({name, values, group});
    kernel.space.reset();
}

void TunerCore::AddModifier(const KernelId id, ModifierData modifier)
{
    KernelData& kernel = Kernel(id);

    for (const auto& name : modifier.parameters)
    {
        const bool known = std::any_of(kernel.parameters.cbegin(), kernel.parameters.cend(),
            [&](const KernelParameterInfo& p) { return p.name == name; });

        if (!known)
        {
            throw std::runtime_error("Thread modifier refers to unknown parameter " + name);
        }
    }

    kernel.modifiers.push_back(std::move(modifier));
}

void TunerCore::AddConstraint(const KernelId id, const std::vector<std::string>& parameters, GenericConstraintFunction function,
    const bool basic)
{
    KernelData& kernel = Kernel(id);
    std::string group;
    bool first = true;

    for (const auto& name : parameters)
    {
        auto it = std::find_if(kernel.parameters.cbegin(), kernel.parameters.cend(),
            [&](const KernelParameterInfo& p) { return p.name == name; });

        if (it == kernel.parameters.cend())
        {
            throw std::runtime_error("Constraint refers to unknown parameter " + name);
        }

        if (basic && ParameterPair::GetTypeFromValue(it->values.front()) != ParameterValueType::UnsignedInt)
        {
            throw std::runtime_error("Kernel parameter with name " + name
                + " does not have unsigned integer values and cannot be used by non-generic kernel constraints");
        }

        if (!first && it->group != group)
        {
            throw std::runtime_error("Constraint can only be added between parameters that belong to the same group");
        }

        group = it->group;
        first = false;
    }

    kernel.constraints.push_back({parameters, std::move(function)});
    kernel.space.reset();
}

// -- arguments --

ArgumentId TunerCore::AddArgument(ArgumentData argument, const ArgumentId& customId)
{
    if (argument.memoryType == ArgumentMemoryType::Vector && argument.bytes == 0)
    {
        throw std::runtime_error("Vector argument must have a non-zero size");
    }

    ArgumentId id = customId;

    if (id.empty())
    {
        do
        {
            id = std::to_string(m_NextArgument++);
        } while (m_Arguments.count(id) != 0);
    }
    else if (m_Arguments.count(id) != 0)
    {
        throw std::runtime_error("Argument with id " + id + " already exists");
    }

    argument.id = id;
    m_Arguments[id] = std::move(argument);
    return id;
}

void TunerCore::RemoveArgument(const ArgumentId& id)
{
    for (const auto& [did, definition] : m_Definitions)
    {
        if (std::find(definition.arguments.cbegin(), definition.arguments.cend(), id) != definition.arguments.cend())
        {
            throw std::runtime_error("Argument " + id + " is used by definition " + definition.name);
        }
    }

    auto it = m_Arguments.find(id);

    if (it == m_Arguments.end())
    {
        throw std::runtime_error("Invalid argument id " + id);
    }

    if (it->second.device != nullptr && m_Context != nullptr)
    {
        coul_buffer_free(m_Context, it->second.device);
    }

    m_Arguments.erase(it);
    m_Validation.erase(id);
}

ArgumentData& TunerCore::Argument(const ArgumentId& id)
{
    auto it = m_Arguments.find(id);

    if (it == m_Arguments.end())
    {
        throw std::runtime_error("Invalid argument id " + id);
    }

    return it->second;
}

void TunerCore::UploadArgument(ArgumentData& argument, const bool force)
{
    if (argument.memoryType != ArgumentMemoryType::Vector || argument.ownership == ArgumentOwnership::User)
    {
        return;
    }

    coul_ctx* ctx = Context();

    // A fresh upload starts from the host data at its own size, so a buffer resized by an earlier
    // run's launcher is re-created (KTT re-creates writable buffers per run).
    if (argument.device != nullptr && (force || !argument.deviceCurrent) && argument.deviceBytes != argument.bytes)
    {
        coul_buffer_free(ctx, argument.device);
        argument.device = nullptr;
    }

    if (argument.device == nullptr)
    {
        CheckCoul(coul_buffer_alloc(ctx, argument.bytes, &argument.device), "buffer allocation for argument " + argument.id);
        argument.deviceBytes = argument.bytes;
        argument.deviceCurrent = false;
    }

    if (force || !argument.deviceCurrent)
    {
        CheckCoul(coul_buffer_upload(ctx, argument.device, argument.HostData(), argument.bytes), "upload of argument " + argument.id);
        argument.deviceCurrent = true;
    }
}

size_t TunerCore::DeviceBytes(const ArgumentData& argument)
{
    return argument.ownership != ArgumentOwnership::User && argument.device != nullptr ? argument.deviceBytes : argument.bytes;
}

// ComputeInterface::UpdateBuffer (KTT: CudaEngine.cpp:430-470, UpdateArgument): the device buffer takes
// the data; the host copy is not touched, so a writable argument starts the next run from the
// caller's data again.
void TunerCore::UpdateArgumentDevice(ArgumentData& argument, const void* data, size_t bytes)
{
    if (argument.memoryType != ArgumentMemoryType::Vector)
    {
        throw std::runtime_error("Argument " + argument.id + " is not a vector");
    }

    UploadArgument(argument, false);
    bytes = bytes == 0 ? DeviceBytes(argument) : std::min(bytes, DeviceBytes(argument));
    void* target = argument.ownership == ArgumentOwnership::User ? argument.userDevice : argument.device;
    CheckCoul(coul_buffer_upload(Context(), target, data, bytes), "UpdateBuffer of argument " + argument.id);
}

// ComputeInterface::ResizeBuffer (KTT: Source/Api/ComputeInterface.h:312-318, CudaEngine.cpp:558-569):
// only the tuner-owned device buffer takes the new size (preserved bytes are copied on the device,
// the rest reads as zero).  The host data keep their size; a writable argument is re-created from
// them at the start of the next run, a cached read-only one keeps the resized buffer.
void TunerCore::ResizeArgument(ArgumentData& argument, const size_t bytes, const bool preserve)
{
    if (argument.memoryType != ArgumentMemoryType::Vector || argument.ownership == ArgumentOwnership::User || bytes == 0)
    {
        throw std::runtime_error("Only vector arguments whose buffer the tuner manages can be resized, to a non-zero size ("
            + argument.id + ")");
    }

    UploadArgument(argument, false);
    coul_ctx* ctx = Context();
    void* resized = nullptr;
    CheckCoul(coul_buffer_alloc(ctx, bytes, &resized), "buffer allocation for argument " + argument.id);

    // bytes not preserved read as zero
    CheckCoul(coul_buffer_memset(ctx, resized, 0, bytes), "resize of " + argument.id);

    if (preserve)
    {
        CheckCoul(coul_buffer_copy(ctx, resized, argument.device, std::min(bytes, argument.deviceBytes)), "resize of " + argument.id);
    }

    CheckCoul(coul_synchronize(ctx), "resize of " + argument.id);
    coul_buffer_free(ctx, argument.device);
    argument.device = resized;
    argument.deviceBytes = bytes;
    argument.deviceCurrent = true;
}

void TunerCore::DownloadArgument(ArgumentData& argument, void* destination, size_t bytes)
{
    if (argument.memoryType != ArgumentMemoryType::Vector)
    {
        throw std::runtime_error("Argument " + argument.id + " is not a vector");
    }

    UploadArgument(argument, false);
    bytes = bytes == 0 ? DeviceBytes(argument) : std::min(bytes, DeviceBytes(argument));
    const void* source = argument.ownership == ArgumentOwnership::User ? argument.userDevice : argument.device;
    CheckCoul(coul_buffer_download(Context(), destination, source, bytes), "download of argument " + argument.id);
}

void TunerCore::OverrideScalar(const ArgumentId& id, const void* data)
{
    const ArgumentData& argument = Argument(id);
    const auto* bytes = static_cast<const uint8_t*>(data);
    m_ScalarOverrides[id] = std::vector<uint8_t>(bytes, bytes + argument.bytes);
}

void TunerCore::ClearOverrides()
{
    m_ScalarOverrides.clear();
}

const void* TunerCore::ScalarData(const ArgumentData& argument) const
{
    auto it = m_ScalarOverrides.find(argument.id);
    return it != m_ScalarOverrides.end() ? it->second.data() : argument.owned.data();
}

std::vector<ArgumentId> TunerCore::KernelArguments(const KernelData& kernel) const
{
    std::vector<ArgumentId> ids;

    for (const auto d : kernel.definitions)
    {
        for (const auto& a : Definition(d).arguments)
        {
            if (std::find(ids.cbegin(), ids.cend(), a) == ids.cend())
            {
                ids.push_back(a);
            }
        }
    }

    return ids;
}

void TunerCore::ResetWritableArguments(const KernelData& kernel)
{
    // Writable arguments start every run from the host data (KTT re-uploads them per run,
    // Source/KernelRunner/KernelRunner.cpp:63-90); read-only ones stay cached on the device.
    for (const auto& id : KernelArguments(kernel))
    {
        ArgumentData& argument = Argument(id);

        if (argument.accessType != ArgumentAccessType::ReadOnly || !m_ReadOnlyCache)
        {
            argument.deviceCurrent = false;
        }
    }
}

// -- sizes and launches --

DimensionVector TunerCore::ModifiedSize(const KernelData& kernel, const KernelDefinitionId id, const ModifierType type,
    const KernelConfiguration& configuration) const
{
    // Modifiers per dimension in the order they were added (Source/Kernel/Kernel.cpp:275-308).
    const DefinitionData& definition = Definition(id);
    DimensionVector size = type == ModifierType::Global ? definition.globalSize : definition.localSize;

    for (const auto dimension : {ModifierDimension::X, ModifierDimension::Y, ModifierDimension::Z})
    {
        size_t value = size.GetSize(dimension);

        for (const auto& modifier : kernel.modifiers)
        {
            if (modifier.type != type || modifier.dimension != dimension
                || std::find(modifier.definitions.cbegin(), modifier.definitions.cend(), id) == modifier.definitions.cend())
            {
                continue;
            }

            std::vector<uint64_t> values;

            for (const auto& name : modifier.parameters)
            {
                bool found = false;

                for (const auto& pair : configuration.GetPairs())
                {
                    if (pair.GetName() == name)
                    {
                        values.push_back(pair.GetValueUint());
                        found = true;
                        break;
                    }
                }

                if (!found)
                {
                    throw std::runtime_error("Configuration lacks parameter " + name + " used by a thread modifier");
                }
            }

            value = static_cast<size_t>(modifier.function(value, values));
        }

        size.SetSize(dimension, value);
    }

    return size;
}

Nanoseconds TunerCore::LaunchDefinition(const KernelData& kernel, const KernelDefinitionId id,
    const KernelConfiguration& configuration, const DimensionVector& global, const DimensionVector& local)
{
    (void)kernel;
    const DefinitionData& definition = Definition(id);
    // Local (shared-memory size) and symbol (__constant__ variable) arguments are not kernel function
    // parameters in KTT's CUDA engine (Tuner.h:488-510: local ones go last in SetArguments); the
    // built-in kernels take neither, so they are dropped before the argument list is matched.
    std::vector<ArgumentId> args;

    for (const auto& a : definition.arguments)
    {
        const ArgumentMemoryType type = Argument(a).memoryType;

        if (type != ArgumentMemoryType::Local && type != ArgumentMemoryType::Symbol)
        {
            args.push_back(a);
        }
    }

    coul_ctx* ctx = Context();

    auto parameter = [&](const char* name, const int64_t fallback) -> int64_t
    {
        for (const auto& pair : configuration.GetPairs())
        {
            if (pair.GetName() == name)
            {
                return static_cast<int64_t>(pair.GetValueUint());
            }
        }

        return fallback;
    };

    auto vector = [&](const size_t i) -> float*
    {
        ArgumentData& argument = Argument(args.at(i));

        if (argument.memoryType != ArgumentMemoryType::Vector)
        {
            throw RunFailure(ResultStatus::ComputationFailed, "argument " + std::to_string(i) + " of " + definition.name
                + " must be a vector");
        }

        UploadArgument(argument, false);
        return static_cast<float*>(argument.ownership == ArgumentOwnership::User ? argument.userDevice : argument.device);
    };

    auto scalar = [&](const size_t i) -> double
    {
        const ArgumentData& argument = Argument(args.at(i));

        if (argument.memoryType != ArgumentMemoryType::Scalar)
        {
            throw RunFailure(ResultStatus::ComputationFailed, "argument " + std::to_string(i) + " of " + definition.name
                + " must be a scalar");
        }

        const void* p = ScalarData(argument);

        switch (argument.dataType)
        {
        case ArgumentDataType::Int: return *static_cast<const int32_t*>(p);
        case ArgumentDataType::UnsignedInt: return *static_cast<const uint32_t*>(p);
        case ArgumentDataType::Long: return static_cast<double>(*static_cast<const int64_t*>(p));
        case ArgumentDataType::UnsignedLong: return static_cast<double>(*static_cast<const uint64_t*>(p));
        case ArgumentDataType::Float: return *static_cast<const float*>(p);
        case ArgumentDataType::Double: return *static_cast<const double*>(p);
        default: throw RunFailure(ResultStatus::ComputationFailed, "unsupported scalar type of argument " + argument.id);
        }
    };

    // device scratch of at least `bytes` (kept across launches, grown on demand)
    auto scratch = [&](const size_t bytes) -> float*
    {
        if (m_ScratchBytes < bytes)
        {
            if (m_ScratchDevice != nullptr)
            {
                coul_buffer_free(ctx, m_ScratchDevice);
                m_ScratchDevice = nullptr;
                m_ScratchBytes = 0;
            }

            CheckCoul(coul_buffer_alloc(ctx, bytes, &m_ScratchDevice), "scratch allocation");
            m_ScratchBytes = bytes;
        }

        return static_cast<float*>(m_ScratchDevice);
    };

    auto packedAtoms = [&](const size_t first, const int64_t n) -> const float*
    {
        // KTT's USE_SOA layouts carry the same atoms in four arrays; gather them into float4 on the device.
        if (parameter("USE_SOA", 0) == 0)
        {
            return vector(first);
        }

        float* packed = scratch(static_cast<size_t>(std::max<int64_t>(n, 1)) * 16);
        CheckCoul(coul_pack_atoms(ctx, vector(first + 1), vector(first + 2), vector(first + 3), vector(first + 4), n,
                      packed),
            "pack of four-array atoms");
        return packed;
    };

    coul_tune tune;
    coul_tune_default(&tune);
    tune.block_x = static_cast<int>(parameter("WORK_GROUP_SIZE_X", static_cast<int64_t>(local.GetSizeX())));
    tune.block_y = static_cast<int>(parameter("WORK_GROUP_SIZE_Y", static_cast<int64_t>(local.GetSizeY())));
    tune.unroll = UnrollFor(static_cast<uint64_t>(parameter("INNER_UNROLL_FACTOR", 1)));
    tune.atom_source = static_cast<int>(parameter("USE_CONSTANT_MEMORY", 0));
    tune.precision = static_cast<int>(parameter("PRECISION", 0));
    tune.rsqrt_soft = static_cast<int>(parameter("RSQRT_SOFT", 0));
    tune.atom_split = static_cast<int>(parameter("ATOM_SPLIT", 0));
    tune.split_form = static_cast<int>(parameter("SPLIT_FORM", 0));

    // a 3D launch: the definition's global size, or (for definitions sized by modifier scripts) the
    // launch's, spans more than one z plane
    const bool threeD = definition.globalSize.GetSizeZ() > 1 || global.GetSizeZ() > 1;
    int rc = COUL_OK;

    // The buffers a launch reads and writes must hold what the scalars describe; checked on the
    // host so that a mismatched host program ends with a failed result instead of a device fault.
    auto require = [&](const size_t i, const double bytes, const char* what)
    {
        if (bytes < 0.0 || static_cast<double>(DeviceBytes(Argument(args.at(i)))) < bytes)
        {
            throw RunFailure(ResultStatus::ComputationFailed, definition.name + ": argument " + std::to_string(i) + " ("
                + what + ") is smaller than the sizes given by the scalar arguments");
        }
    };
    auto requireAtoms = [&](const int64_t n)
    {
        if (parameter("USE_SOA", 0) == 0)
        {
            require(0, 16.0 * static_cast<double>(n), "atoms");
        }
        else
        {
            for (size_t i = 1; i <= 4; ++i)
            {
                require(i, 4.0 * static_cast<double>(n), "atom array");
            }
        }
    };

    // The nine-argument directCoulombSum is either KTT's 3D kernel, whose eighth argument is the
    // (cubic) grid size (Examples/CoulombSum3d/CoulombSum3d.cu), or one slice of a 3D map, whose
    // eighth argument is the slice index and which its launcher runs with a global z size of 1
    // (Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp:146-184, .cl:36-41).
    const bool sliceOf3d = definition.name == "directCoulombSum" && args.size() == 9
        && (!threeD || (global.GetSizeZ() == 1 && static_cast<int64_t>(scalar(7)) != static_cast<int64_t>(definition.globalSize.GetSizeX())));

    if (definition.name == "directCoulombSum" && args.size() == 9 && !sliceOf3d)
    {
        // Examples/CoulombSum3d/CoulombSum3d.cu: (atomInfo, X, Y, Z, W, numberOfAtoms, gridSpacing, gridSize, energyGrid)
        const int64_t n = static_cast<int64_t>(scalar(5));
        const int g = static_cast<int>(scalar(7));
        coul_grid grid{g, g, g, static_cast<float>(scalar(6)), {0.0f, 0.0f, 0.0f}};
        requireAtoms(n);
        require(8, 4.0 * g * g * static_cast<double>(g), "energy grid");
        tune.z_iterations = static_cast<int>(parameter("Z_ITERATIONS", 1));
        tune.x_points = static_cast<int>(parameter("X_POINTS", parameter("VECTOR_SIZE", 1)));

        if (parameter("USE_SOA", 0) == 1)
        {
            rc = coul_forward_3d_soa(ctx, vector(1), vector(2), vector(3), vector(4), n, &grid, &tune, 1, vector(8));
        }
        else
        {
            rc = coul_forward_3d(ctx, vector(0), n, &grid, &tune, 1, vector(8));
        }
    }
    else if (definition.name == "directCoulombSum" && (args.size() == 8 || args.size() == 9))
    {
        // 2D slice (Examples/CoulombSum2d/CoulombSum2d.cl): (atomInfo, X, Y, Z, W, numberOfAtoms, gridSpacing, energyGrid),
        // or one slice of a 3D map (Examples/CoulombSum3dIterative/CoulombSum3dIterative.cl) with zIndex before energyGrid.
        const int64_t n = static_cast<int64_t>(scalar(5));
        const int nx = static_cast<int>(definition.globalSize.GetSizeX());
        const int ny = static_cast<int>(definition.globalSize.GetSizeY());
        const int64_t zIndex = args.size() == 9 ? static_cast<int64_t>(scalar(7)) : 0;
        requireAtoms(n);
        require(args.size() - 1, 4.0 * (static_cast<double>(zIndex) + 1.0) * nx * static_cast<double>(ny), "energy grid");
        float* out = vector(args.size() - 1) + zIndex * static_cast<int64_t>(nx) * ny;
        tune.z_iterations = static_cast<int>(parameter("Y_ITERATIONS", 2));
        tune.x_points = static_cast<int>(parameter("X_POINTS", parameter("OUTER_UNROLL_FACTOR", 1)));
        tune.atom_source = COUL_ATOMS_SHARED_TMA;
        rc = coul_forward_2d(ctx, packedAtoms(0, n), n, static_cast<float>(scalar(6)), nx, ny, &tune, 1, out);
    }
    else if (definition.name == "directCoulombSumReference" && args.size() == 5)
    {
        // Examples/CoulombSum3d/CoulombSum3dReference.cu: (atomInfo, numberOfAtoms, gridSpacing, gridSize, energyGrid)
        const int g = static_cast<int>(scalar(3));
        coul_grid grid{g, g, g, static_cast<float>(scalar(2)), {0.0f, 0.0f, 0.0f}};
        require(0, 16.0 * scalar(1), "atoms");
        require(4, 4.0 * g * g * static_cast<double>(g), "energy grid");
        rc = coul_forward_3d_reference(ctx, vector(0), static_cast<int64_t>(scalar(1)), &grid, 1, vector(4));
    }
    else if (definition.name == "directCoulombSumReference" && args.size() == 4 && threeD)
    {
        // Examples/CoulombSum3dIterative/CoulombSum3dIterativeReference.cl: 3D map, sizes from the global size
        coul_grid grid{static_cast<int>(definition.globalSize.GetSizeX()), static_cast<int>(definition.globalSize.GetSizeY()),
            static_cast<int>(definition.globalSize.GetSizeZ()), static_cast<float>(scalar(2)), {0.0f, 0.0f, 0.0f}};
        require(0, 16.0 * scalar(1), "atoms");
        require(3, 4.0 * grid.nx * static_cast<double>(grid.ny) * grid.nz, "energy grid");
        rc = coul_forward_3d_reference(ctx, vector(0), static_cast<int64_t>(scalar(1)), &grid, 1, vector(3));
    }
    else if (definition.name == "directCoulombSumReference" && args.size() == 4)
    {
        // Examples/CoulombSum2d/CoulombSum2dReference.cl: 2D slice, assigns (=) instead of accumulating
        coul_tune reference;
        coul_tune_default(&reference);
        reference.z_iterations = 2;
        reference.x_points = 1;
        require(0, 16.0 * scalar(1), "atoms");
        require(3, 4.0 * static_cast<double>(definition.globalSize.GetSizeX()) * definition.globalSize.GetSizeY(), "energy grid");
        rc = coul_forward_2d(ctx, vector(0), static_cast<int64_t>(scalar(1)), static_cast<float>(scalar(2)),
            static_cast<int>(definition.globalSize.GetSizeX()), static_cast<int>(definition.globalSize.GetSizeY()), &reference, 0,
            vector(3));
    }
    else if (definition.name == "coulombBatch" && args.size() == 6)
    {
        // This library's batched map as a tunable kernel (no KTT counterpart; KTT launches one kernel per
        // problem): (atoms: float4 of all molecules concatenated, atomOffsets: int64[m + 1] in atoms,
        // grids: float[7 m] = nx, ny, nz, spacing, origin x/y/z, maps: float of all maps concatenated (output),
        // mapOffsets: int64[m + 1] in floats, moleculeCount: int).  The tile configuration comes from the same
        // parameters as directCoulombSum; one persistent launch, replayed from a CUDA graph, computes all maps.
        const int m = static_cast<int>(scalar(5));
        const ArgumentData& atomOffsets = Argument(args.at(1));
        const ArgumentData& grids = Argument(args.at(2));
        const ArgumentData& mapOffsets = Argument(args.at(4));

        if (m < 1 || atomOffsets.bytes < static_cast<size_t>(m + 1) * 8 || mapOffsets.bytes < static_cast<size_t>(m + 1) * 8
            || grids.bytes < static_cast<size_t>(m) * 7 * 4 || atomOffsets.dataType != ArgumentDataType::Long
            || mapOffsets.dataType != ArgumentDataType::Long || grids.dataType != ArgumentDataType::Float)
        {
            throw RunFailure(ResultStatus::ComputationFailed, "coulombBatch: offsets must be int64[m + 1], grids float[7 m]");
        }

        const auto* ao = static_cast<const int64_t*>(atomOffsets.HostData());
        const auto* mo = static_cast<const int64_t*>(mapOffsets.HostData());
        const auto* gr = static_cast<const float*>(grids.HostData());
        float* atoms = vector(0);
        float* maps = vector(3);
        tune.z_iterations = static_cast<int>(parameter("Z_ITERATIONS", 8));
        tune.x_points = static_cast<int>(parameter("X_POINTS", parameter("VECTOR_SIZE", 1)));
        tune.atom_source = COUL_ATOMS_SHARED_TMA;
        std::ostringstream key;
        key << static_cast<const void*>(atoms) << '/' << static_cast<const void*>(maps) << '/' << m << '/' << tune.block_x << ','
            << tune.block_y << ',' << tune.z_iterations << ',' << tune.x_points << ',' << tune.unroll << ',' << tune.precision
            << ',' << tune.rsqrt_soft;
        auto it = m_Batches.find(key.str());

        if (it == m_Batches.end())
        {
            std::vector<coul_molecule> molecules(static_cast<size_t>(m));

            for (int i = 0; i < m; ++i)
            {
                coul_molecule& mol = molecules[static_cast<size_t>(i)];
                mol.d_atoms = atoms + ao[i] * 4;
                mol.n_atoms = ao[i + 1] - ao[i];
                mol.grid = coul_grid{static_cast<int>(gr[7 * i]), static_cast<int>(gr[7 * i + 1]), static_cast<int>(gr[7 * i + 2]),
                    gr[7 * i + 3], {gr[7 * i + 4], gr[7 * i + 5], gr[7 * i + 6]}};
                mol.d_out = maps + mo[i];
            }

            coul_batch* batch = nullptr;
            CheckCoul(coul_batch_create(ctx, molecules.data(), m, &tune, &batch), "coulombBatch set-up");
            it = m_Batches.emplace(key.str(), batch).first;
        }

        rc = coul_batch_run(ctx, it->second, COUL_BATCH_GRAPH, 0);
    }
    else if (definition.name == "nbody_kernel" && args.size() == 15)
    {
        // Examples/Nbody/Nbody.cu:260-275: (timeDelta, oldBodyInfo, oldPosX, oldPosY, oldPosZ, mass, newBodyInfo,
        // oldVel, oldVelX, oldVelY, oldVelZ, newVel, damping, softeningSqr, n).  WORK_GROUP_SIZE_X -> block size,
        // OUTER_UNROLL_FACTOR -> bodies per thread, INNER_UNROLL_FACTOR1 -> j-loop unroll, WORK_GROUP_SIZE_Y -> CTAs
        // per cluster splitting the j range; USE_SOA reads the separate arrays (gathered into float4 here);
        // LOCAL_MEM, VECTOR_TYPE and INNER_UNROLL_FACTOR2 have no counterpart (bodies j always come through
        // the TMA-staged shared-memory ring, pairs of bodies i always share packed FP32x2 instructions).
        const int64_t n = static_cast<int64_t>(scalar(14));
        coul_nbody_tune nb;
        coul_nbody_tune_default(&nb);
        nb.block_x = static_cast<int>(parameter("WORK_GROUP_SIZE_X", static_cast<int64_t>(local.GetSizeX())));
        nb.bodies_per_thread = static_cast<int>(parameter("OUTER_UNROLL_FACTOR", 1));
        const int64_t u = parameter("INNER_UNROLL_FACTOR1", 0);
        nb.unroll = u <= 1 ? 1 : (u < 4 ? 2 : 4);
        const int64_t wy = parameter("WORK_GROUP_SIZE_Y", 1);
        nb.j_split = wy >= 2 ? static_cast<int>(wy) : 0;
        const float* pos = vector(1);
        const float* vel = vector(7);

        if (parameter("USE_SOA", 0) == 1)
        {
            float* packed = scratch(static_cast<size_t>(std::max<int64_t>(n, 1)) * 32);
            float* packedVel = packed + std::max<int64_t>(n, 1) * 4;
            CheckCoul(coul_pack_atoms(ctx, vector(2), vector(3), vector(4), vector(5), n, packed), "pack of positions");
            CheckCoul(coul_pack_atoms(ctx, vector(8), vector(9), vector(10), nullptr, n, packedVel), "pack of velocities");
            pos = packed;
            vel = packedVel;
        }

        rc = coul_nbody_step(ctx, pos, vel, n, static_cast<float>(scalar(0)), static_cast<float>(scalar(12)),
            static_cast<float>(scalar(13)), &nb, vector(6), vector(11));
    }
    else if (definition.name == "nbody_kernel_reference" && args.size() == 7)
    {
        // Examples/Nbody/NbodyReference.cu:36-44: (dt, pos_old, pos_new, oldVel, newVel, damping, softeningSqr); the
        // body count is the launch's global size
        const int64_t n = static_cast<int64_t>(global.GetSizeX() * (GetGlobalSizeType() == GlobalSizeType::CUDA
            ? local.GetSizeX() : 1));
        coul_nbody_tune nb;
        coul_nbody_tune_default(&nb);
        rc = coul_nbody_step(ctx, vector(1), vector(3), n, static_cast<float>(scalar(0)), static_cast<float>(scalar(5)),
            static_cast<float>(scalar(6)), &nb, vector(2), vector(4));
    }
    else
    {
        throw RunFailure(ResultStatus::CompilationFailed, "no sm_100a implementation of kernel " + definition.name + " with "
            + std::to_string(args.size()) + " arguments");
    }

    CheckCoul(rc, "launch of " + definition.name);
    CheckCoul(coul_synchronize(ctx), "execution of " + definition.name);
    double ms = 0.0;
    CheckCoul(coul_elapsed_ms(ctx, &ms), "timing of " + definition.name);
    return static_cast<Nanoseconds>(std::llround(ms * 1e6));
}

// -- validation --

void TunerCore::SetValidationMethod(const ValidationMethod method, const double threshold)
{
    if (threshold < 0.0)
    {
        throw std::runtime_error("Validation threshold must be non-negative");
    }

    m_ValidationMethod = method;
    m_ValidationThreshold = threshold;
}

ValidationData& TunerCore::Validation(const ArgumentId& id)
{
    (void)Argument(id);
    return m_Validation[id];
}

void TunerCore::ComputeReference(const ArgumentId& id, ValidationData& data)
{
    ArgumentData& argument = Argument(id);
    const size_t elements = data.range ? data.range : argument.bytes / argument.elementSize;
    data.reference.assign(elements * argument.elementSize, 0);

    if (data.computation)
    {
        data.computation(data.reference.data());
    }
    else if (data.referenceKernel != InvalidKernelId)
    {
        KernelResult result = Run(data.referenceKernel, data.referenceConfiguration, {}, KernelRunMode::ResultValidation);

        if (!result.IsValid())
        {
            throw std::runtime_error("Reference kernel failed for argument " + id);
        }

        DownloadArgument(argument, data.reference.data(), data.reference.size());
    }
    else if (!data.referenceArgument.empty())
    {
        const ArgumentData& other = Argument(data.referenceArgument);
        std::memcpy(data.reference.data(), other.HostData(), std::min(other.bytes, data.reference.size()));
    }

    data.computed = true;
}

bool TunerCore::Compare(const ArgumentData& argument, const ValidationData& data, const void* result, const size_t elements) const
{
    // ResultValidator (Source/KernelRunner/ResultValidator.inl:53-108): floating-point arguments by the
    // configured method and threshold, integer ones exactly, or by the user's comparator.
    if (data.comparator)
    {
        const auto* r = static_cast<const uint8_t*>(result);
        const auto* e = data.reference.data();

        for (size_t i = 0; i < elements; ++i)
        {
            if (!data.comparator(r + i * argument.elementSize, e + i * argument.elementSize))
            {
                log::Warning("Results differ for argument with id " + argument.id + " at index " + std::to_string(i));
                return false;
            }
        }

        return true;
    }

    auto check = [&](auto typed) -> bool
    {
        using T = decltype(typed);
        const T* r = static_cast<const T*>(result);
        const T* e = reinterpret_cast<const T*>(data.reference.data());

        if constexpr (std::is_floating_point_v<T>)
        {
            if (m_ValidationMethod == ValidationMethod::AbsoluteDifference)
            {
                double sum = 0.0;

                for (size_t i = 0; i < elements; ++i)
                {
                    sum += std::fabs(static_cast<double>(r[i]) - static_cast<double>(e[i]));
                }

                if (sum > m_ValidationThreshold)
                {
                    log::Warning("Results differ for argument with id " + argument.id + ", absolute difference is "
                        + std::to_string(sum));
                    return false;
                }

                return true;
            }

            for (size_t i = 0; i < elements; ++i)
            {
                const double difference = std::fabs(static_cast<double>(r[i]) - static_cast<double>(e[i]));
                const bool fail = m_ValidationMethod == ValidationMethod::SideBySideComparison
                    ? !(difference <= m_ValidationThreshold)
                    : (difference > 1e-4 && difference / static_cast<double>(e[i]) > m_ValidationThreshold);

                if (fail)
                {
                    log::Warning("Results differ for argument with id " + argument.id + " at index " + std::to_string(i)
                        + ", reference value: " + std::to_string(e[i]) + ", result value: " + std::to_string(r[i])
                        + ", difference: " + std::to_string(difference));
                    return false;
                }
            }

            return true;
        }
        else
        {
            for (size_t i = 0; i < elements; ++i)
            {
                if (r[i] != e[i])
                {
                    log::Warning("Results differ for argument with id " + argument.id + " at index " + std::to_string(i));
                    return false;
                }
            }

            return true;
        }
    };

    switch (argument.dataType)
    {
    case ArgumentDataType::Float: return check(float{});
    case ArgumentDataType::Double: return check(double{});
    case ArgumentDataType::Int: return check(int32_t{});
    case ArgumentDataType::UnsignedInt: return check(uint32_t{});
    case ArgumentDataType::Long: return check(int64_t{});
    case ArgumentDataType::UnsignedLong: return check(uint64_t{});
    case ArgumentDataType::Short: return check(int16_t{});
    case ArgumentDataType::UnsignedShort: return check(uint16_t{});
    case ArgumentDataType::Char: return check(int8_t{});
    case ArgumentDataType::UnsignedChar: return check(uint8_t{});
    default: return std::memcmp(result, data.reference.data(), elements * argument.elementSize) == 0;
    }
}

bool TunerCore::ValidateOutputs(const KernelData& kernel, const KernelConfiguration& configuration, KernelResult& result)
{
    (void)configuration;
    const auto ids = KernelArguments(kernel);

    for (auto& [id, data] : m_Validation)
    {
        if (std::find(ids.cbegin(), ids.cend(), id) == ids.cend())
        {
            continue;
        }

        ArgumentData& argument = Argument(id);
        const size_t elements = data.range ? data.range : argument.bytes / argument.elementSize;
        std::vector<uint8_t> values(elements * argument.elementSize);
        DownloadArgument(argument, values.data(), values.size());

        if (!data.computed)
        {
            ComputeReference(id, data);
            // the reference run reset the writable arguments; nothing else depends on them now
        }

        if (!Compare(argument, data, values.data(), elements))
        {
            result.SetStatus(ResultStatus::ValidationFailed);
            return false;
        }
    }

    return true;
}

// -- running --

DimensionVector TunerCore::GridSize(const DimensionVector& global, const DimensionVector& local) const
{
    // results record the launch grid in blocks whatever the global size type (KTT divides an
    // OpenCL-style global size by the local size before the launch: CudaKernel.cpp:107-137)
    if (m_GlobalSizeType != GlobalSizeType::OpenCL)
    {
        return global;
    }

    auto blocks = [](const size_t g, const size_t l) { return l == 0 ? g : (g + l - 1) / l; };
    return DimensionVector(blocks(global.GetSizeX(), local.GetSizeX()), blocks(global.GetSizeY(), local.GetSizeY()),
        blocks(global.GetSizeZ(), local.GetSizeZ()));
}

const std::vector<std::string>& TunerCore::DefaultProfilingCounters()
{
    // KTT's default metric list (Source/ComputeEngine/Cuda/Cupti/CuptiMetricInterface.cpp:621-660),
    // the counters its profile-based searcher reads, plus the XU-pipe instruction count that the
    // searcher's B200 analysis adds for the MUFU-bound kernels of this path
    static const std::vector<std::string> counters{
        "dram__throughput.avg.pct_of_peak_sustained_elapsed",
        "dram__sectors_read.sum",
        "dram__sectors_write.sum",
        "lts__t_sectors.avg.pct_of_peak_sustained_elapsed",
        "lts__t_sectors_op_read.sum",
        "lts__t_sectors_op_write.sum",
        "l1tex__t_requests_pipe_lsu_mem_global_op_ld.avg.pct_of_peak_sustained_active",
        "l1tex__t_requests_pipe_lsu_mem_global_op_ld.sum",
        "l1tex__data_pipe_lsu_wavefronts_mem_shared.avg.pct_of_peak_sustained_elapsed",
        "l1tex__data_pipe_lsu_wavefronts_mem_shared_op_ld.sum",
        "l1tex__data_pipe_lsu_wavefronts_mem_shared_op_st.sum",
        "l1tex__t_sectors_pipe_lsu_mem_local_op_ld.sum",
        "l1tex__t_sectors_pipe_lsu_mem_local_op_st.sum",
        "sm__warps_active.avg.pct_of_peak_sustained_active",
        "smsp__cycles_active.avg.pct_of_peak_sustained_elapsed",
        "smsp__sass_thread_inst_executed_op_fp16_pred_on.sum",
        "smsp__sass_thread_inst_executed_op_fp32_pred_on.sum",
        "smsp__sass_thread_inst_executed_op_fp64_pred_on.sum",
        "smsp__sass_thread_inst_executed_op_integer_pred_on.sum",
        "smsp__sass_thread_inst_executed_op_control_pred_on.sum",
        "smsp__sass_thread_inst_executed_op_memory_pred_on.sum",
        "smsp__sass_thread_inst_executed_op_misc_pred_on.sum",
        "smsp__sass_thread_inst_executed_op_conversion_pred_on.sum",
        "smsp__inst_executed.sum",
        "smsp__inst_executed_pipe_fp16.sum",
        "smsp__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active",
        "smsp__inst_executed_pipe_fp64.avg.pct_of_peak_sustained_active",
        "smsp__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active",
        "smsp__inst_executed_pipe_lsu.avg.pct_of_peak_sustained_active",
        "smsp__inst_executed_pipe_tex.avg.pct_of_peak_sustained_active",
        "smsp__issue_active.avg.pct_of_peak_sustained_active",
        "smsp__thread_inst_executed_per_inst_executed.ratio",
        "smsp__thread_inst_executed_per_inst_executed.pct",
        "smsp__inst_executed_pipe_xu.sum",
    };

    return counters;
}

void TunerCore::SetProfilingCounters(const std::vector<std::string>& counters)
{
    if (counters.empty())
    {
        throw std::runtime_error("Number of profiling metrics must be greater than zero");
    }

    m_ProfilingCounters = counters;
}

void TunerCore::SetProfiledDefinitions(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds)
{
    KernelData& kernel = Kernel(id);

    if (definitionIds.empty())
    {
        throw std::runtime_error("Number of profiled definitions must be greater than zero");
    }

    for (const auto definition : definitionIds)
    {
        if (std::find(kernel.definitions.cbegin(), kernel.definitions.cend(), definition) == kernel.definitions.cend())
        {
            throw std::runtime_error("Definition " + std::to_string(definition) + " is not part of kernel " + kernel.name);
        }
    }

    kernel.profiledDefinitions = definitionIds;
}

std::unique_ptr<KernelProfilingData> TunerCore::ProfileExecution(const KernelData& kernel,
    const std::function<std::vector<ComputationResult>()>& execute)
{
    // One user range around a whole execution, replayed once per pass (coul_profiler_* in coulktt.h);
    // the counters cover every launch of the execution.
    const std::vector<std::string>& names = m_ProfilingCounters.empty() ? DefaultProfilingCounters() : m_ProfilingCounters;
    std::vector<const char*> pointers;

    for (const auto& name : names)
    {
        pointers.push_back(name.c_str());
    }

    std::vector<int> valid(names.size(), 0);
    coul_profiler* profiler = nullptr;
    int passes = 0;
    CheckCoul(coul_profiler_create(Context(), pointers.data(), static_cast<int>(pointers.size()), valid.data(), &profiler,
        &passes), "profiler set-up");
    std::unique_ptr<coul_profiler, int (*)(coul_profiler*)> guard(profiler, coul_profiler_destroy);

    for (size_t i = 0; i < names.size(); ++i)
    {
        if (!valid[i] && m_UnsupportedCounters.insert(names[i]).second)
        {
            log::Warning("Metric with name " + names[i] + " is not supported on the current device");
        }
    }

    int done = 0;

    for (int pass = 0; !done; ++pass)
    {
        if (pass > passes + 1)
        {
            throw RunFailure(ResultStatus::ComputationFailed, "profiler asked for more passes than it announced");
        }

        ResetWritableArguments(kernel);
        CheckCoul(coul_profiler_begin_pass(profiler), "profiling pass");

        try
        {
            (void)execute();
        }
        catch (...)
        {
            int ignored = 0;
            (void)coul_profiler_end_pass(profiler, &ignored);
            throw;
        }

        CheckCoul(coul_profiler_end_pass(profiler, &done), "profiling pass");
    }

    std::vector<double> values(names.size(), 0.0);
    CheckCoul(coul_profiler_read(profiler, values.data()), "profiling counters");
    std::vector<KernelProfilingCounter> counters;

    for (size_t i = 0; i < names.size(); ++i)
    {
        if (valid[i])
        {
            counters.emplace_back(names[i], ProfilingCounterType::Double, values[i]);
        }
    }

    log::Debug("Collected " + std::to_string(counters.size()) + " profiling counters in " + std::to_string(passes) + " passes");
    return std::make_unique<KernelProfilingData>(counters);
}

KernelResult TunerCore::Run(const KernelId id, const KernelConfiguration& configuration,
    const std::vector<BufferOutputDescriptor>& output, const KernelRunMode mode)
{
    const KernelData& kernel = Kernel(id);
    KernelResult result(kernel.name, configuration);
    const auto start = Clock::now();
    std::vector<ComputationResult> computations;

    // one execution of the kernel: its launcher, or each definition in turn
    auto execute = [&]() -> std::vector<ComputationResult>
    {
        if (kernel.launcher)
        {
            // overrides a launcher sets hold for this execution only
            struct DropOverrides
            {
                TunerCore& core;
                ~DropOverrides() { core.ClearOverrides(); }
            } drop{*this};
            ClearOverrides();
            ComputeLayer layer(*this, kernel, configuration, mode);
            kernel.launcher(layer);
            return layer.Results();
        }

        std::vector<ComputationResult> list;

        for (const auto definition : kernel.definitions)
        {
            const DimensionVector global = ModifiedSize(kernel, definition, ModifierType::Global, configuration);
            const DimensionVector local = ModifiedSize(kernel, definition, ModifierType::Local, configuration);
            const auto launchStart = Clock::now();
            const Nanoseconds duration = LaunchDefinition(kernel, definition, configuration, global, local);
            const Nanoseconds wall = ElapsedNs(launchStart);
            ComputationResult computation(Definition(definition).name);
            computation.SetSizeData(GridSize(global, local), local);
            computation.SetDurationData(duration, wall > duration ? wall - duration : 0);
            list.push_back(computation);
        }

        return list;
    };

    std::unique_ptr<KernelProfilingData> profilingData;
    Nanoseconds profilingOverhead = 0;

    try
    {
        if (m_Profiling)
        {
            // the profiling passes run first, each from freshly reset arguments, so that the timed
            // execution below and its validation see exactly one run (KTT repeats the whole tuning
            // iteration per pass: Source/TuningRunner/TuningRunner.cpp:40-53)
            const auto profilingStart = Clock::now();

            try
            {
                profilingData = ProfileExecution(kernel, execute);
            }
            catch (const std::exception& failure)
            {
                // no counters (no libcupti, profiling not permitted, ...): the run itself goes on
                if (!m_ProfilingFailureReported)
                {
                    log::Warning(std::string("Profiling counters are not collected: ") + failure.what());
                    m_ProfilingFailureReported = true;
                }
            }

            profilingOverhead = ElapsedNs(profilingStart);
        }

        ResetWritableArguments(kernel);
        computations = execute();

        if (profilingData && !computations.empty())
        {
            // the counters go to the first computation of a profiled definition (by default the
            // kernel's first definition), else to the first computation
            const KernelDefinitionId profiled = kernel.profiledDefinitions.empty() ? kernel.definitions.front()
                : kernel.profiledDefinitions.front();
            const std::string& function = Definition(profiled).name;
            auto target = std::find_if(computations.begin(), computations.end(),
                [&function](const ComputationResult& c) { return c.GetKernelFunction() == function; });
            (target == computations.end() ? computations.front() : *target).SetProfilingData(std::move(profilingData));
        }
    }
    catch (const RunFailure& failure)
    {
        log::Warning("Kernel run failed for kernel " + kernel.name + ", configuration " + configuration.GetString() + ": "
            + failure.what());
        result.SetStatus(failure.status);
        result.SetFailedKernelOverhead(ElapsedNs(start));
        return result;
    }
    catch (const std::exception& failure)
    {
        log::Warning("Kernel run failed for kernel " + kernel.name + ": " + failure.what());
        result.SetStatus(ResultStatus::ComputationFailed);
        result.SetFailedKernelOverhead(ElapsedNs(start));
        return result;
    }

    result.SetResults(computations);
    result.SetProfilingRunsOverhead(profilingOverhead);
    const bool validate = (mode == KernelRunMode::Running && HasFlag(m_ValidationMode, ValidationMode::Running))
        || (mode == KernelRunMode::OfflineTuning && HasFlag(m_ValidationMode, ValidationMode::OfflineTuning))
        || (mode == KernelRunMode::OnlineTuning && HasFlag(m_ValidationMode, ValidationMode::OnlineTuning));

    if (validate)
    {
        const auto validationStart = Clock::now();

        try
        {
            ValidateOutputs(kernel, configuration, result);
        }
        catch (const std::exception& failure)
        {
            log::Warning(std::string("Validation failed: ") + failure.what());
            result.SetStatus(ResultStatus::ValidationFailed);
        }

        result.SetValidationOverhead(ElapsedNs(validationStart));
    }

    const auto transferStart = Clock::now();

    for (const auto& descriptor : output)
    {
        DownloadArgument(Argument(descriptor.GetArgumentId()), descriptor.GetOutputDestination(), descriptor.GetOutputSize());
    }

    result.SetDataMovementOverhead(ElapsedNs(transferStart));
    return result;
}

ConfigurationSpace& TunerCore::Space(const KernelId id)
{
    KernelData& kernel = Kernel(id);

    if (!kernel.space)
    {
        log::Info("Generating configurations for kernel " + kernel.name);
        kernel.space = std::make_unique<ConfigurationSpace>(kernel.parameters, kernel.constraints);
        log::Info("Total count of " + std::to_string(kernel.space->GetConfigurationsCount())
            + " configurations was generated");
    }

    return *kernel.space;
}

void TunerCore::ClearSpace(const KernelId id)
{
    KernelData& kernel = Kernel(id);

    if (kernel.searcher && kernel.searcher->IsInitialized())
    {
        kernel.searcher->Reset();
    }

    kernel.space.reset();
    kernel.searcherActive = false;
}

void TunerCore::SetSearcher(const KernelId id, std::unique_ptr<Searcher> searcher)
{
    ClearSpace(id);
    Kernel(id).searcher = std::move(searcher);
}

// Operator cap on the configurations one Tune call runs, on top of the program's own stop
// condition: KTT_B200_CONFIGURATION_LIMIT=N (a positive integer; unset, empty or 0 = no cap).  It
// lets a KTT host program whose search space and stop condition are fixed in its source run with
// a bounded budget.  No counterpart in KTT.
uint64_t TunerCore::ConfigurationLimitFromEnvironment()
{
    const char* value = std::getenv("KTT_B200_CONFIGURATION_LIMIT");

    if (value == nullptr || *value == '\0')
    {
        return 0;
    }

    char* end = nullptr;
    const unsigned long long n = std::strtoull(value, &end, 10);

    if (end == value || *end != '\0')
    {
        log::Warning(std::string("KTT_B200_CONFIGURATION_LIMIT is not a number, ignored: ") + value);
        return 0;
    }

    return static_cast<uint64_t>(n);
}

std::vector<KernelResult> TunerCore::Tune(const KernelId id, std::unique_ptr<StopCondition> stop)
{
    // The offline tuning loop of Source/TuningRunner/TuningRunner.cpp:17-82.
    KernelData& kernel = Kernel(id);
    ClearSpace(id);
    ConfigurationSpace& space = Space(id);

    if (!kernel.searcher)
    {
        kernel.searcher = std::make_unique<DeterministicSearcher>();
    }

    kernel.searcher->Initialize(space);

    if (stop)
    {
        stop->Initialize(space.GetConfigurationsCount());
    }

    std::vector<KernelResult> results;
    Nanoseconds searcherOverhead = 0;
    const uint64_t limit = ConfigurationLimitFromEnvironment();

    while (!space.IsExhausted())
    {
        if (limit != 0 && results.size() >= limit)
        {
            log::Info("Tuning stopped after " + std::to_string(limit) + " configurations (KTT_B200_CONFIGURATION_LIMIT)");
            break;
        }

        const KernelConfiguration configuration = kernel.searcher->GetCurrentConfiguration();
        KernelResult result = Run(id, configuration, {}, KernelRunMode::OfflineTuning);
        result.SetSearcherOverhead(searcherOverhead);
        space.MarkExplored(space.GetIndex(configuration));

        if (result.IsValid())
        {
            space.UpdateBest(configuration, result.GetTotalDuration());
        }

        log::Info("Tuned configuration " + std::to_string(results.size()) + ": " + configuration.GetString() + " -> "
            + (result.IsValid() ? std::to_string(result.GetTotalDuration() / 1000) + " us" : std::string("failed")));
        results.push_back(result);

        if (stop)
        {
            stop->Update(result);

            if (stop->IsFulfilled())
            {
                log::Info(stop->GetStatusString());
                break;
            }
        }

        if (space.IsExhausted())
        {
            break;
        }

        const auto searcherStart = Clock::now();
        const bool more = kernel.searcher->CalculateNextConfiguration(result);
        searcherOverhead = ElapsedNs(searcherStart);

        if (!more)
        {
            break;
        }
    }

    kernel.searcher->Reset();
    return results;
}

KernelResult TunerCore::TuneIteration(const KernelId id, const std::vector<BufferOutputDescriptor>& output,
    const bool recompute)
{
    // One step of online tuning (Tuner::TuneIteration, Source/Tuner.h:677): the searcher's current
    // configuration is run with output, then the searcher moves on; once the space is exhausted
    // the best configuration keeps being run.
    KernelData& kernel = Kernel(id);
    ConfigurationSpace& space = Space(id);

    if (recompute)
    {
        for (auto& [aid, data] : m_Validation)
        {
            data.computed = false;
        }
    }

    if (!kernel.searcher)
    {
        kernel.searcher = std::make_unique<DeterministicSearcher>();
    }

    if (!kernel.searcher->IsInitialized() && !space.IsExhausted())
    {
        kernel.searcher->Initialize(space);
        kernel.searcherActive = true;
    }

    if (!kernel.searcherActive || space.IsExhausted())
    {
        return Run(id, space.GetBestConfiguration(), output, KernelRunMode::Running);
    }

    const KernelConfiguration configuration = kernel.searcher->GetCurrentConfiguration();
    KernelResult result = Run(id, configuration, output, KernelRunMode::OnlineTuning);
    space.MarkExplored(space.GetIndex(configuration));

    if (result.IsValid())
    {
        space.UpdateBest(configuration, result.GetTotalDuration());
    }

    if (space.IsExhausted() || !kernel.searcher->CalculateNextConfiguration(result))
    {
        kernel.searcherActive = false;
    }

    return result;
}

std::vector<KernelResult> TunerCore::SimulateTuning(const KernelId id, const std::vector<KernelResult>& recorded,
    const uint64_t iterations, StopCondition* stop)
{
    // Replays recorded results through the searcher without running anything
    // (Source/TuningRunner/TuningRunner.cpp:131-201); a stop condition sees the recorded results.
    KernelData& kernel = Kernel(id);
    ClearSpace(id);
    ConfigurationSpace& space = Space(id);

    if (!kernel.searcher)
    {
        kernel.searcher = std::make_unique<DeterministicSearcher>();
    }

    kernel.searcher->Initialize(space);
    std::vector<KernelResult> results;

    if (stop != nullptr)
    {
        stop->Initialize(space.GetConfigurationsCount());
    }

    while (!space.IsExhausted() && (iterations == 0 || results.size() < iterations)
        && (stop == nullptr || !stop->IsFulfilled()))
    {
        const KernelConfiguration configuration = kernel.searcher->GetCurrentConfiguration();
        auto it = std::find_if(recorded.cbegin(), recorded.cend(),
            [&](const KernelResult& r) { return r.GetConfiguration() == configuration; });
        KernelResult result = it != recorded.cend() ? *it : KernelResult(kernel.name, configuration);

        if (it == recorded.cend())
        {
            log::Warning("No recorded result for configuration " + configuration.GetString());
            result.SetStatus(ResultStatus::ComputationFailed);
        }

        space.MarkExplored(space.GetIndex(configuration));

        if (result.IsValid())
        {
            space.UpdateBest(configuration, result.GetTotalDuration());
        }

        results.push_back(result);

        if (stop != nullptr)
        {
            stop->Update(result);

            if (stop->IsFulfilled())
            {
                log::Info(stop->GetStatusString());
                break;
            }
        }

        if (space.IsExhausted() || !kernel.searcher->CalculateNextConfiguration(result))
        {
            break;
        }
    }

    kernel.searcher->Reset();
    return results;
}

KernelConfiguration TunerCore::CreateConfiguration(const KernelId id, const ParameterInput& input) const
{
    const KernelData& kernel = Kernel(id);
    std::vector<ParameterPair> pairs;

    for (const auto& [name, value] : input)
    {
        auto it = std::find_if(kernel.parameters.cbegin(), kernel.parameters.cend(),
            [&](const KernelParameterInfo& p) { return p.name == name; });

        if (it == kernel.parameters.cend())
        {
            throw std::runtime_error("Kernel " + kernel.name + " has no parameter " + name);
        }

        const ParameterPair pair(name, value);
        // the parameter's own value of that number (a signed literal names an unsigned value alike:
        // Python integers arrive as int64)
        auto numeric = [](const ParameterValue& v, double& out)
        {
            if (std::holds_alternative<int64_t>(v)) { out = static_cast<double>(std::get<int64_t>(v)); return true; }
            if (std::holds_alternative<uint64_t>(v)) { out = static_cast<double>(std::get<uint64_t>(v)); return true; }
            if (std::holds_alternative<double>(v)) { out = std::get<double>(v); return true; }
            return false;
        };
        const auto match = std::find_if(it->values.cbegin(), it->values.cend(), [&](const ParameterValue& v)
        {
            double a = 0.0;
            double b = 0.0;
            return pair.HasSameValue(ParameterPair(name, v)) || (numeric(v, a) && numeric(value, b) && a == b);
        });

        if (match == it->values.cend())
        {
            throw std::runtime_error("Value " + pair.GetValueString() + " is not a value of parameter " + name);
        }

        pairs.emplace_back(name, *match);
    }

    for (const auto& p : kernel.parameters)
    {
        const bool given = std::any_of(pairs.cbegin(), pairs.cend(), [&](const ParameterPair& q) { return q.GetName() == p.name; });

        if (!given)
        {
            pairs.emplace_back(p.name, p.values.front());
        }
    }

    return KernelConfiguration(pairs);
}

std::string TunerCore::GetDefinitionSource(const KernelDefinitionId id, const KernelConfiguration& configuration) const
{
    return configuration.GeneratePrefix() + Definition(id).source;
}

std::string TunerCore::GetKernelSource(const KernelId id, const KernelConfiguration& configuration) const
{
    const KernelData& kernel = Kernel(id);
    std::string source;

    for (const auto d : kernel.definitions)
    {
        source += GetDefinitionSource(d, configuration);
    }

    return source;
}

} // namespace ktt
