// Tuner.cpp -- the public ktt::Tuner facade.
//
// Every method forwards to TunerCore inside a try block; failures are logged at Error level and
// turned into the invalid return values of KTT 2.1.0 (Source/Tuner.cpp:40-150): InvalidKernelId,
// InvalidKernelDefinitionId, InvalidArgumentId, an empty configuration, or a KernelResult whose
// status says what went wrong.
#include <fstream>
#include <iterator>
#include <sstream>

#include "Logger.h"
#include "TunerCore.h"

namespace ktt
{

namespace
{

template <typename F, typename R>
R Guarded(F&& f, R fallback)
{
    try
    {
        return f();
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
        return fallback;
    }
}

template <typename F>
void GuardedVoid(F&& f)
{
    try
    {
        f();
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
    }
}

} // namespace

// ---- DeviceInfo ---------------------------------------------------------------------------------

DeviceInfo::DeviceInfo(const DeviceIndex index, const std::string& name, const uint64_t globalMemorySize, const uint32_t smCount,
    const uint32_t ccMajor, const uint32_t ccMinor) :
    m_Index(index), m_Name(name), m_GlobalMemorySize(globalMemorySize), m_SmCount(smCount), m_CcMajor(ccMajor),
    m_CcMinor(ccMinor)
{}

DeviceIndex DeviceInfo::GetIndex() const { return m_Index; }
const std::string& DeviceInfo::GetName() const { return m_Name; }
uint64_t DeviceInfo::GetGlobalMemorySize() const { return m_GlobalMemorySize; }
uint32_t DeviceInfo::GetMaxComputeUnits() const { return m_SmCount; }
uint32_t DeviceInfo::GetCudaComputeCapabilityMajor() const { return m_CcMajor; }
uint32_t DeviceInfo::GetCudaComputeCapabilityMinor() const { return m_CcMinor; }

std::string DeviceInfo::GetString() const
{
    return "Device " + std::to_string(m_Index) + ": " + m_Name + ", compute units " + std::to_string(m_SmCount)
        + ", compute capability " + std::to_string(m_CcMajor) + "." + std::to_string(m_CcMinor);
}

// ---- Tuner ------------------------------------------------------------------------------------

Tuner::Tuner(const PlatformIndex platform, const DeviceIndex device, const ComputeApi api) : Tuner(platform, device, api, 1) {}

Tuner::Tuner([[maybe_unused]] const PlatformIndex platform, const DeviceIndex device, const ComputeApi api,
    [[maybe_unused]] const uint32_t computeQueueCount) :
    m_Core(std::make_unique<TunerCore>(device, api))
{}

Tuner::~Tuner() = default;

KernelDefinitionId Tuner::AddKernelDefinition(const std::string& name, const std::string& source, const DimensionVector& globalSize,
    const DimensionVector& localSize, const std::vector<std::string>& typeNames)
{
    return Guarded([&] { return m_Core->AddDefinition(name, source, globalSize, localSize, typeNames); },
        InvalidKernelDefinitionId);
}

KernelDefinitionId Tuner::AddKernelDefinitionFromFile(const std::string& name, const std::string& filePath,
    const DimensionVector& globalSize, const DimensionVector& localSize, const std::vector<std::string>& typeNames)
{
    return Guarded([&]
    {
        std::ifstream file(filePath);
        std::string source;

        if (file)
        {
            source.assign(std::istreambuf_iterator<char>(file), std::istreambuf_iterator<char>());
        }
        else
        {
            // The kernel runs from its built-in sm_100a implementation; the source text is only kept
            // for GetKernelSource, so a missing file is reported but not fatal.
            log::Warning("Kernel source file " + filePath + " was not found; the definition keeps an empty source");
        }

        return m_Core->AddDefinition(name, source, globalSize, localSize, typeNames);
    }, InvalidKernelDefinitionId);
}

KernelDefinitionId Tuner::GetKernelDefinitionId(const std::string& name, const std::vector<std::string>& typeNames) const
{
    return m_Core->GetDefinitionId(name, typeNames);
}

void Tuner::RemoveKernelDefinition(const KernelDefinitionId id) { GuardedVoid([&] { m_Core->RemoveDefinition(id); }); }

void Tuner::SetArguments(const KernelDefinitionId id, const std::vector<ArgumentId>& argumentIds)
{
    GuardedVoid([&] { m_Core->SetArguments(id, argumentIds); });
}

KernelId Tuner::CreateSimpleKernel(const std::string& name, const KernelDefinitionId definitionId)
{
    return Guarded([&] { return m_Core->CreateKernel(name, {definitionId}, nullptr); }, InvalidKernelId);
}

KernelId Tuner::CreateCompositeKernel(const std::string& name, const std::vector<KernelDefinitionId>& definitionIds,
    KernelLauncher launcher)
{
    return Guarded([&] { return m_Core->CreateKernel(name, definitionIds, launcher); }, InvalidKernelId);
}

void Tuner::RemoveKernel(const KernelId id) { GuardedVoid([&] { m_Core->RemoveKernel(id); }); }
void Tuner::SetLauncher(const KernelId id, KernelLauncher launcher) { GuardedVoid([&] { m_Core->SetLauncher(id, launcher); }); }

void Tuner::AddParameterInternal(const KernelId id, const std::string& name, const std::vector<ParameterValue>& values,
    const std::string& group)
{
    GuardedVoid([&] { m_Core->AddParameter(id, name, values, group); });
}

void Tuner::AddThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds, const ModifierType type,
    const ModifierDimension dimension, const std::vector<std::string>& parameters, ModifierFunction function)
{
    GuardedVoid([&]
    {
        ModifierData data;
        data.type = type;
        data.dimension = dimension;
        data.definitions = definitionIds;
        data.parameters = parameters;
        data.function = function;
        m_Core->AddModifier(id, data);
    });
}

void Tuner::AddThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds, const ModifierType type,
    const ModifierDimension dimension, const std::string& parameter, const ModifierAction action)
{
    AddThreadModifier(id, definitionIds, type, dimension, std::vector<std::string>{parameter},
        [action, dimension](const uint64_t size, const std::vector<uint64_t>& values)
        {
            DimensionVector v;
            v.SetSize(dimension, static_cast<size_t>(size));
            v.ModifyByValue(static_cast<size_t>(values.at(0)), action, dimension);
            return static_cast<uint64_t>(v.GetSize(dimension));
        });
}

void Tuner::AddConstraint(const KernelId id, const std::vector<std::string>& parameters, ConstraintFunction function)
{
    GuardedVoid([&]
    {
        m_Core->AddConstraint(id, parameters, [function](const std::vector<const ParameterValue*>& values)
        {
            std::vector<uint64_t> plain;

            for (const auto* v : values)
            {
                plain.push_back(std::get<uint64_t>(*v));
            }

            return function(plain);
        }, true);
    });
}

void Tuner::AddGenericConstraint(const KernelId id, const std::vector<std::string>& parameters, GenericConstraintFunction function)
{
    GuardedVoid([&] { m_Core->AddConstraint(id, parameters, function, false); });
}

ArgumentId Tuner::AddArgumentWithOwnedData(const size_t elementSize, const ArgumentDataType dataType,
    const ArgumentMemoryType memoryType, const ArgumentAccessType accessType, const void* data, const size_t dataSize,
    const ArgumentId& customId)
{
    return Guarded([&]
    {
        ArgumentData argument;
        argument.dataType = dataType;
        argument.memoryType = memoryType;
        argument.accessType = accessType;
        argument.ownership = ArgumentOwnership::Owned;
        argument.elementSize = elementSize;
        argument.bytes = dataSize;
        argument.owned.assign(static_cast<const uint8_t*>(data), static_cast<const uint8_t*>(data) + dataSize);
        return m_Core->AddArgument(std::move(argument), customId);
    }, InvalidArgumentId);
}

ArgumentId Tuner::AddArgumentWithReferencedData(const size_t elementSize, const ArgumentDataType dataType,
    const ArgumentAccessType accessType, void* data, const size_t dataSize, const ArgumentId& customId)
{
    return Guarded([&]
    {
        ArgumentData argument;
        argument.dataType = dataType;
        argument.memoryType = ArgumentMemoryType::Vector;
        argument.accessType = accessType;
        argument.ownership = ArgumentOwnership::Referenced;
        argument.elementSize = elementSize;
        argument.bytes = dataSize;
        argument.referenced = data;
        return m_Core->AddArgument(std::move(argument), customId);
    }, InvalidArgumentId);
}

ArgumentId Tuner::AddUserArgument(ComputeBuffer buffer, const size_t elementSize, const ArgumentDataType dataType,
    const ArgumentAccessType accessType, const size_t bufferSize, const ArgumentId& customId)
{
    return Guarded([&]
    {
        ArgumentData argument;
        argument.dataType = dataType;
        argument.memoryType = ArgumentMemoryType::Vector;
        argument.accessType = accessType;
        argument.ownership = ArgumentOwnership::User;
        argument.elementSize = elementSize;
        argument.bytes = bufferSize;
        argument.userDevice = buffer;
        argument.deviceCurrent = true;
        return m_Core->AddArgument(std::move(argument), customId);
    }, InvalidArgumentId);
}

void Tuner::RemoveArgument(const ArgumentId& id) { GuardedVoid([&] { m_Core->RemoveArgument(id); }); }
void Tuner::SetReadOnlyArgumentCache(const bool flag) { m_Core->SetReadOnlyCache(flag); }

KernelResult Tuner::Run(const KernelId id, const KernelConfiguration& configuration, const std::vector<BufferOutputDescriptor>& output)
{
    return Guarded([&] { return m_Core->Run(id, configuration, output, KernelRunMode::Running); },
        [&] { KernelResult r("", configuration); r.SetStatus(ResultStatus::ComputationFailed); return r; }());
}

void Tuner::SetProfiling(const bool flag)
{
    // Hardware counters are collected with Nsight Compute on this path; KTT's in-process CUPTI
    // replay is not provided, so profiling requests only record the flag.
    if (flag)
    {
        log::Warning("In-process profiling counters are not collected; use Nsight Compute on the launched kernels");
    }

    m_Core->SetProfiling(flag);
}

bool Tuner::GetProfiling() { return m_Core->GetProfiling(); }

void Tuner::SetValidationMethod(const ValidationMethod method, const double toleranceThreshold)
{
    GuardedVoid([&] { m_Core->SetValidationMethod(method, toleranceThreshold); });
}

void Tuner::SetValidationMode(const ValidationMode mode) { m_Core->SetValidationMode(mode); }

void Tuner::SetValidationRange(const ArgumentId& id, const size_t range)
{
    GuardedVoid([&] { m_Core->Validation(id).range = range; });
}

void Tuner::SetValueComparator(const ArgumentId& id, ValueComparator comparator)
{
    GuardedVoid([&] { m_Core->Validation(id).comparator = comparator; });
}

void Tuner::SetReferenceComputation(const ArgumentId& id, ReferenceComputation computation)
{
    GuardedVoid([&]
    {
        ValidationData& data = m_Core->Validation(id);
        data.computation = computation;
        data.referenceKernel = InvalidKernelId;
        data.referenceArgument.clear();
        data.computed = false;
    });
}

void Tuner::SetReferenceKernel(const ArgumentId& id, const KernelId referenceId, const KernelConfiguration& configuration)
{
    GuardedVoid([&]
    {
        (void)m_Core->Kernel(referenceId);
        ValidationData& data = m_Core->Validation(id);
        data.computation = nullptr;
        data.referenceKernel = referenceId;
        data.referenceConfiguration = configuration;
        data.referenceArgument.clear();
        data.computed = false;
    });
}

void Tuner::SetReferenceArgument(const ArgumentId& id, const ArgumentId& referenceId)
{
    GuardedVoid([&]
    {
        (void)m_Core->Argument(referenceId);
        ValidationData& data = m_Core->Validation(id);
        data.computation = nullptr;
        data.referenceKernel = InvalidKernelId;
        data.referenceArgument = referenceId;
        data.computed = false;
    });
}

std::vector<KernelResult> Tuner::Tune(const KernelId id, std::unique_ptr<StopCondition> stopCondition)
{
    return Guarded([&] { return m_Core->Tune(id, std::move(stopCondition)); }, std::vector<KernelResult>{});
}

KernelResult Tuner::TuneIteration(const KernelId id, const std::vector<BufferOutputDescriptor>& output, const bool recomputeReference)
{
    return Guarded([&] { return m_Core->TuneIteration(id, output, recomputeReference); },
        [&] { KernelResult r; r.SetStatus(ResultStatus::ComputationFailed); return r; }());
}

std::vector<KernelResult> Tuner::SimulateTuning(const KernelId id, const std::vector<KernelResult>& results, const uint64_t iterations)
{
    return Guarded([&] { return m_Core->SimulateTuning(id, results, iterations); }, std::vector<KernelResult>{});
}

void Tuner::SetSearcher(const KernelId id, std::unique_ptr<Searcher> searcher)
{
    GuardedVoid([&] { m_Core->SetSearcher(id, std::move(searcher)); });
}

void Tuner::InitializeConfigurationData(const KernelId id) { GuardedVoid([&] { (void)m_Core->Space(id); }); }
void Tuner::ClearConfigurationData(const KernelId id) { GuardedVoid([&] { m_Core->ClearSpace(id); }); }

uint64_t Tuner::GetConfigurationsCount(const KernelId id) const
{
    return Guarded([&] { return m_Core->Space(id).GetConfigurationsCount(); }, uint64_t{0});
}

KernelConfiguration Tuner::GetBestConfiguration(const KernelId id) const
{
    return Guarded([&] { return m_Core->Space(id).GetBestConfiguration(); }, KernelConfiguration());
}

KernelConfiguration Tuner::CreateConfiguration(const KernelId id, const ParameterInput& parameters) const
{
    return Guarded([&] { return m_Core->CreateConfiguration(id, parameters); }, KernelConfiguration());
}

std::string Tuner::GetKernelSource(const KernelId id, const KernelConfiguration& configuration) const
{
    return Guarded([&] { return m_Core->GetKernelSource(id, configuration); }, std::string());
}

std::string Tuner::GetKernelDefinitionSource(const KernelDefinitionId id, const KernelConfiguration& configuration) const
{
    return Guarded([&] { return m_Core->GetDefinitionSource(id, configuration); }, std::string());
}

void Tuner::SynchronizeQueue([[maybe_unused]] const QueueId id) { GuardedVoid([&] { m_Core->Synchronize(); }); }
void Tuner::SynchronizeQueues() { GuardedVoid([&] { m_Core->Synchronize(); }); }
void Tuner::SynchronizeDevice() { GuardedVoid([&] { m_Core->Synchronize(); }); }
void Tuner::SetCompilerOptions(const std::string& options, [[maybe_unused]] const bool overrideDefault)
{
    m_Core->SetCompilerOptions(options);
}

void Tuner::SetGlobalSizeType(const GlobalSizeType type) { m_Core->SetGlobalSizeType(type); }
void Tuner::SetAutomaticGlobalSizeCorrection([[maybe_unused]] const bool flag) {}
void Tuner::SetKernelCacheCapacity([[maybe_unused]] const uint64_t capacity) {}

DeviceInfo Tuner::GetCurrentDeviceInfo() const
{
    return Guarded([&] { return m_Core->GetDeviceInfo(); }, DeviceInfo(0, "unavailable", 0, 0, 0, 0));
}

void Tuner::SetLoggingLevel(const LoggingLevel level) { log::state().level = level; }
LoggingLevel Tuner::GetLoggingLevel() { return log::state().level; }

void Tuner::SetLoggingTarget(std::ostream& outputTarget)
{
    log::state().file.reset();
    log::state().stream = &outputTarget;
}

void Tuner::SetLoggingTarget(const std::string& filePath)
{
    auto file = std::make_unique<std::ofstream>(filePath);

    if (!*file)
    {
        log::Error("Unable to open log file " + filePath);
        return;
    }

    log::state().stream = file.get();
    log::state().file = std::move(file);
}

} // namespace ktt
