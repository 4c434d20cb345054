// TunerCore.h -- internal state behind ktt::Tuner (not installed; include/ktt/Tuner.h is the API).
//
// Plays the roles of KTT 2.1.0's TunerCore (Source/TunerCore.cpp), KernelManager / Kernel
// (Source/Kernel), KernelArgumentManager (Source/KernelArgument), KernelRunner and ComputeLayer
// (Source/KernelRunner), ResultValidator (Source/KernelRunner/ResultValidator.cpp) and
// TuningRunner (Source/TuningRunner/TuningRunner.cpp), with the CUDA engine replaced by the C ABI of
// libcoulktt.so.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include <coulktt.h>
#include <ktt/Tuner.h>

namespace ktt
{

// Failure carried from deep inside a run to the result status.
struct RunFailure : std::runtime_error
{
    RunFailure(const ResultStatus s, const std::string& what) : std::runtime_error(what), status(s) {}
    ResultStatus status;
};

struct DefinitionData
{
    KernelDefinitionId id = 0;
    std::string name;
    std::string source;
    DimensionVector globalSize;
    DimensionVector localSize;
    std::vector<std::string> typeNames;
    std::vector<ArgumentId> arguments;
};

struct ModifierData
{
    ModifierType type = ModifierType::Global;
    ModifierDimension dimension = ModifierDimension::X;
    std::vector<KernelDefinitionId> definitions;
    std::vector<std::string> parameters;
    ModifierFunction function;
};

struct KernelData
{
    KernelId id = 0;
    std::string name;
    std::vector<KernelDefinitionId> definitions;
    std::vector<KernelParameterInfo> parameters;
    std::vector<KernelConstraintInfo> constraints;
    std::vector<ModifierData> modifiers;
    KernelLauncher launcher;
    std::vector<KernelDefinitionId> profiledDefinitions;  // empty: the first definition
    std::unique_ptr<Searcher> searcher;
    std::unique_ptr<ConfigurationSpace> space;
    bool searcherActive = false;
};

enum class ArgumentOwnership { Owned, Referenced, User };

struct ArgumentData
{
    ArgumentId id;
    ArgumentDataType dataType = ArgumentDataType::Float;
    ArgumentMemoryType memoryType = ArgumentMemoryType::Vector;
    ArgumentAccessType accessType = ArgumentAccessType::ReadOnly;
    ArgumentOwnership ownership = ArgumentOwnership::Owned;
    size_t elementSize = 4;
    std::vector<uint8_t> owned;      // owned host copy (vectors and scalars)
    void* referenced = nullptr;      // caller's host memory (referenced vectors)
    void* userDevice = nullptr;      // caller's device buffer (user vectors)
    size_t bytes = 0;                // data bytes; for local arguments the shared-memory size
    std::string symbolName;          // symbol arguments: the __constant__ variable's name
    void* device = nullptr;          // framework device buffer
    size_t deviceBytes = 0;
    bool deviceCurrent = false;      // device copy matches the host data

    void* HostData() { return ownership == ArgumentOwnership::Referenced ? referenced : owned.data(); }
    const void* HostData() const { return ownership == ArgumentOwnership::Referenced ? referenced : owned.data(); }
};

struct ValidationData
{
    ReferenceComputation computation;
    KernelId referenceKernel = InvalidKernelId;
    KernelConfiguration referenceConfiguration;
    ArgumentId referenceArgument;
    ValueComparator comparator;
    size_t range = 0;  // elements; 0 = whole argument
    std::vector<uint8_t> reference;
    bool computed = false;
};

class ComputeLayer;

class TunerCore
{
public:
    TunerCore(const DeviceIndex device, const ComputeApi api);
    ~TunerCore();

    // kernels and definitions
    KernelDefinitionId AddDefinition(const std::string& name, const std::string& source, const DimensionVector& global,
        const DimensionVector& local, const std::vector<std::string>& typeNames);
    KernelDefinitionId GetDefinitionId(const std::string& name, const std::vector<std::string>& typeNames) const;
    void RemoveDefinition(const KernelDefinitionId id);
    void SetArguments(const KernelDefinitionId id, const std::vector<ArgumentId>& arguments);
    KernelId CreateKernel(const std::string& name, const std::vector<KernelDefinitionId>& definitions, KernelLauncher launcher);
    void RemoveKernel(const KernelId id);
    void SetLauncher(const KernelId id, KernelLauncher launcher);
    void AddParameter(const KernelId id, const std::string& name, const std::vector<ParameterValue>& values,
        const std::string& group);
    void AddModifier(const KernelId id, ModifierData modifier);
    void AddConstraint(const KernelId id, const std::vector<std::string>& parameters, GenericConstraintFunction function,
        const bool basic);

    // arguments
    ArgumentId AddArgument(ArgumentData argument, const ArgumentId& customId);
    void RemoveArgument(const ArgumentId& id);
    void SetReadOnlyCache(const bool flag) { m_ReadOnlyCache = flag; }

    // validation
    void SetValidationMethod(const ValidationMethod method, const double threshold);
    void SetValidationMode(const ValidationMode mode) { m_ValidationMode = mode; }
    ValidationData& Validation(const ArgumentId& id);

    // running
    KernelResult Run(const KernelId id, const KernelConfiguration& configuration, const std::vector<BufferOutputDescriptor>& output,
        const KernelRunMode mode);
    std::vector<KernelResult> Tune(const KernelId id, std::unique_ptr<StopCondition> stop);
    KernelResult TuneIteration(const KernelId id, const std::vector<BufferOutputDescriptor>& output, const bool recompute);
    std::vector<KernelResult> SimulateTuning(const KernelId id, const std::vector<KernelResult>& results, const uint64_t iterations,
        StopCondition* stop);
    void SetSearcher(const KernelId id, std::unique_ptr<Searcher> searcher);
    ConfigurationSpace& Space(const KernelId id);
    void ClearSpace(const KernelId id);
    KernelConfiguration CreateConfiguration(const KernelId id, const ParameterInput& input) const;
    std::string GetKernelSource(const KernelId id, const KernelConfiguration& configuration) const;
    std::string GetDefinitionSource(const KernelDefinitionId id, const KernelConfiguration& configuration) const;

    // device
    coul_ctx* Context();
    void Synchronize();
    DeviceInfo GetDeviceInfo();
    // queues: ids of the caller's streams, or {0} for the tuner's own
    void AdoptContext(const ComputeApiInitializer& initializer, std::vector<QueueId>& assigned);
    QueueId AddQueue(ComputeQueue queue);
    void RemoveQueue(const QueueId id);
    std::vector<QueueId> QueueIds() const;
    void SynchronizeQueue(const QueueId id);
    // runs `work` with the context's calls enqueued on queue `id`
    void OnQueue(const QueueId id, const std::function<void()>& work);
    std::vector<DeviceInfo> GetDeviceInfo(const PlatformIndex platform);
    std::vector<PlatformInfo> GetPlatformInfo();
    static DeviceInfo QueryDevice(const DeviceIndex index);
    std::string DeviceName();
    void SetGlobalSizeType(const GlobalSizeType type) { m_GlobalSizeType = type; }
    GlobalSizeType GetGlobalSizeType() const { return m_GlobalSizeType; }
    void SetProfiling(const bool flag) { m_Profiling = flag; }
    bool GetProfiling() const { return m_Profiling; }
    void SetProfilingCounters(const std::vector<std::string>& counters);
    void SetProfiledDefinitions(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds);
    static const std::vector<std::string>& DefaultProfilingCounters();
    void SetCompilerOptions(const std::string& options) { m_CompilerOptions = options; }
    ComputeApi GetApi() const { return m_Api; }

    // used by the compute layer
    DefinitionData& Definition(const KernelDefinitionId id);
    const DefinitionData& Definition(const KernelDefinitionId id) const;
    KernelData& Kernel(const KernelId id);
    const KernelData& Kernel(const KernelId id) const;
    ArgumentData& Argument(const ArgumentId& id);
    DimensionVector ModifiedSize(const KernelData& kernel, const KernelDefinitionId id, const ModifierType type,
        const KernelConfiguration& configuration) const;
    DimensionVector GridSize(const DimensionVector& global, const DimensionVector& local) const;
    // Runs one definition through its built-in sm_100a implementation; returns the event-timed duration.
    Nanoseconds LaunchDefinition(const KernelData& kernel, const KernelDefinitionId id, const KernelConfiguration& configuration,
        const DimensionVector& global, const DimensionVector& local);
    void UploadArgument(ArgumentData& argument, const bool force);
    void ResizeArgument(ArgumentData& argument, const size_t bytes, const bool preserve);
    void DownloadArgument(ArgumentData& argument, void* destination, size_t bytes);
    // Writes the argument's device buffer only; its host data stays as the caller gave it.
    void UpdateArgumentDevice(ArgumentData& argument, const void* data, size_t bytes);
    // Size of the buffer a launch sees (a resized device buffer keeps its new size until the run ends).
    static size_t DeviceBytes(const ArgumentData& argument);
    // Per-run overrides set from a launcher (KTT: ComputeLayer.cpp:160-190, AddArgumentOverride):
    // they apply to the launches of the current run and are dropped when it ends.
    void OverrideScalar(const ArgumentId& id, const void* data);
    void ClearOverrides();
    const void* ScalarData(const ArgumentData& argument) const;

private:
    DeviceIndex m_Device;
    ComputeContext m_UserContext = nullptr;                  // caller's CUcontext (ComputeApiInitializer)
    std::vector<std::pair<QueueId, ComputeQueue>> m_Queues;  // caller's streams with their ids
    QueueId m_NextQueue = 0;
    ComputeApi m_Api;
    coul_ctx* m_Context;
    GlobalSizeType m_GlobalSizeType;
    bool m_Profiling;
    bool m_ReadOnlyCache;
    std::string m_CompilerOptions;
    ValidationMethod m_ValidationMethod;
    double m_ValidationThreshold;
    ValidationMode m_ValidationMode;
    uint64_t m_NextDefinition;
    uint64_t m_NextKernel;
    uint64_t m_NextArgument;
    std::map<KernelDefinitionId, DefinitionData> m_Definitions;
    std::map<KernelId, KernelData> m_Kernels;
    std::map<ArgumentId, ArgumentData> m_Arguments;
    std::map<ArgumentId, ValidationData> m_Validation;
    void* m_ScratchDevice = nullptr;  // float4 atoms gathered from KTT's four-array layout
    size_t m_ScratchBytes = 0;
    // persistent batches of the coulombBatch definition, one per (arguments, tile configuration)
    std::map<std::string, coul_batch*> m_Batches;
    std::vector<std::string> m_ProfilingCounters;  // empty: the default list
    std::set<std::string> m_UnsupportedCounters;   // reported once each
    bool m_ProfilingFailureReported = false;
    std::map<ArgumentId, std::vector<uint8_t>> m_ScalarOverrides;  // the current run's only

    void ResetWritableArguments(const KernelData& kernel);
    static uint64_t ConfigurationLimitFromEnvironment();
    std::unique_ptr<KernelProfilingData> ProfileExecution(const KernelData& kernel,
        const std::function<std::vector<ComputationResult>()>& execute);
    bool ValidateOutputs(const KernelData& kernel, const KernelConfiguration& configuration, KernelResult& result);
    void ComputeReference(const ArgumentId& id, ValidationData& data);
    bool Compare(const ArgumentData& argument, const ValidationData& data, const void* result, const size_t elements) const;
    std::vector<ArgumentId> KernelArguments(const KernelData& kernel) const;
};

} // namespace ktt
