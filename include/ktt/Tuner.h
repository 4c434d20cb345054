// Tuner.h -- the ktt::Tuner surface of the B200-native Coulomb path.
//
// Drop-in for KTT 2.1.0's Source/Tuner.h:63-1010 for host programs of the direct Coulomb summation
// examples (Examples/CoulombSum3d/CoulombSum3d.cpp, Examples/CoulombSum2d/CoulombSum2d.cpp,
// Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp): same class, method names, argument
// meaning and error convention (every public method catches failures, logs them at Error level and
// returns InvalidKernelId / InvalidKernelDefinitionId / InvalidArgumentId; run failures become a
// KernelResult status, Source/Tuner.cpp:40-150).
//
// What differs underneath: KTT prepends the configuration as "#define NAME VALUE" lines to the
// kernel source and JIT-compiles it with NVRTC.  Here a kernel definition is matched by its
// function name and argument list to a built-in, ahead-of-time compiled sm_100a implementation in
// libcoulktt.so (directCoulombSum / directCoulombSumReference in their 3D, 2D-slice and
// slice-of-3D forms), and the configuration's parameter values select the compiled variant:
//     WORK_GROUP_SIZE_X/Y -> block shape, Z_ITERATIONS -> points per thread along z,
//     VECTOR_SIZE (3D) / OUTER_UNROLL_FACTOR (2D) -> points per thread along x,
//     INNER_UNROLL_FACTOR -> atom-loop unroll, USE_CONSTANT_MEMORY -> atom source,
//     USE_SOA -> which argument layout the 3D kernel reads,
// plus the B200 parameters PRECISION (0 FP32, 1 compensated, 2 FP64 merge, 3 FP64 pairs, 4 FP64 merge with
// the sums in shared memory),
// RSQRT_SOFT (share of reciprocal square roots on the FMA pipe, of 8), ATOM_SPLIT (2 or more: the
// atoms are split into that many chunks per point tile) and SPLIT_FORM (0: a thread-block cluster
// of ATOM_SPLIT CTAs shares each tile, 2..16; 1: a persistent grid takes (tile, chunk) items from a
// device queue, 2..256; 2: one CTA per SM of WORK_GROUP_SIZE_X x WORK_GROUP_SIZE_Y x ATOM_SPLIT
// threads (at most 1,024) takes an equal range of the (tile, atom) space, ATOM_SPLIT = 2..32 atom
// groups sharing each tile's points).  A configuration that maps to no compiled variant
// ends with ResultStatus::CompilationFailed, one beyond the device's launch limits with
// DeviceLimitsExceeded -- the statuses KTT reports for a kernel that fails to compile or launch.
// A definition with no built-in implementation is rejected when it is run.  GetKernelSource still
// returns KTT's "#define" prefix followed by the stored source.
#pragma once

#include <memory>
#include <ostream>
#include <string>
#include <type_traits>
#include <vector>

#include <ktt/ComputeApiInitializer.h>
#include <ktt/ComputeInterface.h>
#include <ktt/Configuration.h>
#include <ktt/ConfigurationSpace.h>
#include <ktt/Results.h>
#include <ktt/Searcher.h>
#include <ktt/StopCondition.h>

namespace ktt
{

class TunerCore;

// Description of a compute device (Source/Api/Info/DeviceInfo.h); for CUDA devices filled as KTT's
// CUDA engine fills it (CudaDevice.cpp:26-58).
class KTT_API DeviceInfo
{
public:
    explicit DeviceInfo(const DeviceIndex index, const std::string& name);
    DeviceInfo(const DeviceIndex index, const std::string& name, const uint64_t globalMemorySize, const uint32_t smCount,
        const uint32_t ccMajor, const uint32_t ccMinor);
    DeviceIndex GetIndex() const;
    const std::string& GetName() const;
    const std::string& GetVendor() const;
    const std::string& GetExtensions() const;
    DeviceType GetDeviceType() const;
    std::string GetDeviceTypeString() const;
    uint64_t GetGlobalMemorySize() const;
    uint64_t GetLocalMemorySize() const;
    uint64_t GetMaxConstantBufferSize() const;
    uint64_t GetMaxWorkGroupSize() const;
    uint32_t GetMaxComputeUnits() const;
    uint32_t GetCudaComputeCapabilityMajor() const;
    uint32_t GetCudaComputeCapabilityMinor() const;
    std::string GetString() const;

    void SetVendor(const std::string& vendor);
    void SetExtensions(const std::string& extensions);
    void SetDeviceType(const DeviceType deviceType);
    void SetGlobalMemorySize(const uint64_t size);
    void SetLocalMemorySize(const uint64_t size);
    void SetMaxConstantBufferSize(const uint64_t size);
    void SetMaxWorkGroupSize(const uint64_t size);
    void SetMaxComputeUnits(const uint32_t units);
    void SetCudaComputeCapabilityMajor(const uint32_t major);
    void SetCudaComputeCapabilityMinor(const uint32_t minor);

private:
    DeviceIndex m_Index;
    std::string m_Name;
    std::string m_Vendor;
    std::string m_Extensions;
    DeviceType m_DeviceType = DeviceType::GPU;
    uint64_t m_GlobalMemorySize = 0;
    uint64_t m_LocalMemorySize = 0;
    uint64_t m_MaxConstantBufferSize = 0;
    uint64_t m_MaxWorkGroupSize = 0;
    uint32_t m_SmCount = 0;
    uint32_t m_CcMajor = 0;
    uint32_t m_CcMinor = 0;
};

// Description of a compute platform (Source/Api/Info/PlatformInfo.h); CUDA has one, "NVIDIA CUDA",
// whose version is the driver's (CudaEngine.cpp:696-707).
class KTT_API PlatformInfo
{
public:
    explicit PlatformInfo(const PlatformIndex index, const std::string& name);
    PlatformIndex GetIndex() const;
    const std::string& GetName() const;
    const std::string& GetVendor() const;
    const std::string& GetVersion() const;
    const std::string& GetExtensions() const;
    std::string GetString() const;

    void SetVendor(const std::string& vendor);
    void SetVersion(const std::string& version);
    void SetExtensions(const std::string& extensions);

private:
    PlatformIndex m_Index;
    std::string m_Name;
    std::string m_Vendor;
    std::string m_Version;
    std::string m_Extensions;
};

class KTT_API Tuner
{
public:
    explicit Tuner(const PlatformIndex platform, const DeviceIndex device, const ComputeApi api);
    explicit Tuner(const PlatformIndex platform, const DeviceIndex device, const ComputeApi api,
        const uint32_t computeQueueCount);
    // On the caller's CUDA context and streams (Tutorials/05ComputeApiInitializer); the queues get ids
    // 0, 1, ... in the initializer's order, also returned in assignedQueueIds.
    explicit Tuner(const ComputeApi api, const ComputeApiInitializer& initializer);
    explicit Tuner(const ComputeApi api, const ComputeApiInitializer& initializer, std::vector<QueueId>& assignedQueueIds);
    ~Tuner();

    // ---- kernels --------------------------------------------------------------------------
    KernelDefinitionId AddKernelDefinition(const std::string& name, const std::string& source,
        const DimensionVector& globalSize, const DimensionVector& localSize, const std::vector<std::string>& typeNames = {});
    KernelDefinitionId AddKernelDefinitionFromFile(const std::string& name, const std::string& filePath,
        const DimensionVector& globalSize, const DimensionVector& localSize, const std::vector<std::string>& typeNames = {});
    // Without sizes: global and local size (1, 1, 1), to be set by thread modifiers (KTT's JSON
    // tuning scripts define their kernels this way).
    KernelDefinitionId AddKernelDefinition(const std::string& name, const std::string& source,
        const std::vector<std::string>& typeNames = {});
    KernelDefinitionId AddKernelDefinitionFromFile(const std::string& name, const std::string& filePath,
        const std::vector<std::string>& typeNames = {});
    KernelDefinitionId GetKernelDefinitionId(const std::string& name, const std::vector<std::string>& typeNames = {}) const;
    void RemoveKernelDefinition(const KernelDefinitionId id);
    void SetArguments(const KernelDefinitionId id, const std::vector<ArgumentId>& argumentIds);
    KernelId CreateSimpleKernel(const std::string& name, const KernelDefinitionId definitionId);
    KernelId CreateCompositeKernel(const std::string& name, const std::vector<KernelDefinitionId>& definitionIds,
        KernelLauncher launcher = nullptr);
    void RemoveKernel(const KernelId id);
    void SetLauncher(const KernelId id, KernelLauncher launcher);

    // ---- tuning parameters -----------------------------------------------------------------
    template <typename T>
    void AddParameter(const KernelId id, const std::string& name, const std::vector<T>& values, const std::string& group = "")
    {
        std::vector<ParameterValue> parameterValues;

        for (const auto& value : values)
        {
            if constexpr (std::is_same_v<T, std::string> || std::is_same_v<T, bool> || std::is_same_v<T, double>)
            {
                parameterValues.push_back(value);
            }
            else if constexpr (std::is_same_v<T, float>)
            {
                parameterValues.push_back(static_cast<double>(value));
            }
            else if constexpr (std::is_signed_v<T>)
            {
                parameterValues.push_back(static_cast<int64_t>(value));
            }
            else
            {
                parameterValues.push_back(static_cast<uint64_t>(value));
            }
        }

        AddParameterInternal(id, name, parameterValues, group);
    }

    void AddThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds, const ModifierType type,
        const ModifierDimension dimension, const std::vector<std::string>& parameters, ModifierFunction function);
    void AddThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds, const ModifierType type,
        const ModifierDimension dimension, const std::string& parameter, const ModifierAction action);
    void AddConstraint(const KernelId id, const std::vector<std::string>& parameters, ConstraintFunction function);
    void AddGenericConstraint(const KernelId id, const std::vector<std::string>& parameters, GenericConstraintFunction function);

    // Script forms.  KTT evaluates these strings with embedded Python; here the Python expression
    // subset of KTT's scripts (arithmetic, comparisons, and/or/not, conditional expressions, lists,
    // comprehensions, min/max/range/...) is parsed and evaluated natively.  A values script yields
    // a list; a modifier script sees every tuning parameter by name and the incoming size as
    // "defaultSize"; a constraint script sees the named parameters.
    void AddScriptParameter(const KernelId id, const std::string& name, const ParameterValueType valueType,
        const std::string& valueScript, const std::string& group = "");
    void AddScriptThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds, const ModifierType type,
        const ModifierDimension dimension, const std::string& script);
    void AddScriptConstraint(const KernelId id, const std::vector<std::string>& parameters, const std::string& script);

    // ---- arguments -------------------------------------------------------------------------
    template <typename T>
    ArgumentId AddArgumentVector(const std::vector<T>& data, const ArgumentAccessType accessType, const ArgumentId& customId = "")
    {
        return AddArgumentWithOwnedData(sizeof(T), DeriveDataType<T>(), ArgumentMemoryType::Vector, accessType, data.data(),
            data.size() * sizeof(T), customId);
    }

    // Referenced host data (the tuner reads and writes the caller's vector).
    template <typename T>
    ArgumentId AddArgumentVector(std::vector<T>& data, const ArgumentAccessType accessType, const ArgumentMemoryLocation memoryLocation,
        const ArgumentManagementType managementType, const bool referenceUserData, const ArgumentId& customId = "")
    {
        (void)memoryLocation;
        (void)managementType;

        if (!referenceUserData)
        {
            return AddArgumentVector(static_cast<const std::vector<T>&>(data), accessType, customId);
        }

        return AddArgumentWithReferencedData(sizeof(T), DeriveDataType<T>(), accessType, data.data(), data.size() * sizeof(T),
            customId);
    }

    // User device buffer (a CUDA device pointer the caller owns; the tuner never frees it).
    template <typename T>
    ArgumentId AddArgumentVector(ComputeBuffer buffer, const size_t bufferSize, const ArgumentAccessType accessType,
        const ArgumentId& customId = "")
    {
        return AddUserArgument(buffer, sizeof(T), DeriveDataType<T>(), accessType, bufferSize, customId);
    }

    template <typename T>
    ArgumentId AddArgumentScalar(const T& data, const ArgumentId& customId = "")
    {
        return AddArgumentWithOwnedData(sizeof(T), DeriveDataType<T>(), ArgumentMemoryType::Scalar, ArgumentAccessType::ReadOnly,
            &data, sizeof(T), customId);
    }

    // Scalar of raw bytes (data type Custom).
    ArgumentId AddArgumentScalar(const void* data, const size_t dataSize, const ArgumentId& customId = "");

    // Local (CUDA: dynamic shared) memory of localMemorySize bytes; placed last in SetArguments.  The
    // built-in kernels stage their operands in shared memory of their own, so such an argument is
    // accepted and does not change a launch.
    template <typename T>
    ArgumentId AddArgumentLocal(const size_t localMemorySize, const ArgumentId& customId = "")
    {
        return AddSpecialArgument(sizeof(T), DeriveDataType<T>(), ArgumentMemoryType::Local, nullptr, localMemorySize,
            "", customId);
    }

    // Value for a __constant__ variable named symbolName (CUDA); not a kernel function parameter.
    template <typename T>
    ArgumentId AddArgumentSymbol(const T& data, const ArgumentId& customId = "", const std::string& symbolName = "")
    {
        return AddSpecialArgument(sizeof(T), DeriveDataType<T>(), ArgumentMemoryType::Symbol, &data, sizeof(T), symbolName,
            customId);
    }

    // Vector argument read from a raw binary file, or generated by a script evaluated once per
    // element index (bound to "i") and converted to dataType.
    ArgumentId AddArgumentVectorFromFile(const std::string& filePath, const ArgumentDataType dataType, const size_t elementSize,
        const ArgumentAccessType accessType, const ArgumentMemoryLocation memoryLocation = ArgumentMemoryLocation::Device,
        const ArgumentManagementType managementType = ArgumentManagementType::Framework, const ArgumentId& customId = "");
    ArgumentId AddArgumentVectorFromGenerator(const std::string& generatorFunction, const ArgumentDataType dataType,
        const size_t bufferSize, const size_t elementSize, const ArgumentAccessType accessType,
        const ArgumentMemoryLocation memoryLocation = ArgumentMemoryLocation::Device,
        const ArgumentManagementType managementType = ArgumentManagementType::Framework, const ArgumentId& customId = "");
    // Writes the argument's current data (from the device once it has been used there) to a raw file.
    void SaveArgumentVector(const ArgumentId& id, const std::string& filePath);

    void RemoveArgument(const ArgumentId& id);
    void SetReadOnlyArgumentCache(const bool flag);

    // ---- running and validation ------------------------------------------------------------
    KernelResult Run(const KernelId id, const KernelConfiguration& configuration, const std::vector<BufferOutputDescriptor>& output);
    // Profiled runs collect hardware counters with CUPTI's range profiler: before the timed run the
    // kernel's whole execution (its launcher, or each definition) is replayed once per counter pass,
    // each time from reset arguments, and the counters are attached to the first ComputationResult.
    // Where counters cannot be collected (no libcupti, profiling not permitted) runs go on without
    // them after one warning.
    void SetProfiling(const bool flag);
    bool GetProfiling();
    // Counters to collect (names of CUPTI's metrics; ones the device does not offer are dropped with
    // a warning); by default KTT's list plus the XU-pipe instruction count.
    void SetProfilingCounters(const std::vector<std::string>& counters);
    // Definitions of a composite kernel whose computation results carry the counters (by default the
    // first definition).  One counter set is collected per execution, over all of its launches, and
    // attached to the first computation of the first of these definitions.
    void SetProfiledDefinitions(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds);
    void SetValidationMethod(const ValidationMethod method, const double toleranceThreshold);
    void SetValidationMode(const ValidationMode mode);
    void SetValidationRange(const ArgumentId& id, const size_t range);
    void SetValueComparator(const ArgumentId& id, ValueComparator comparator);
    void SetReferenceComputation(const ArgumentId& id, ReferenceComputation computation);
    void SetReferenceKernel(const ArgumentId& id, const KernelId referenceId, const KernelConfiguration& configuration);
    void SetReferenceArgument(const ArgumentId& id, const ArgumentId& referenceId);

    // ---- tuning ----------------------------------------------------------------------------
    std::vector<KernelResult> Tune(const KernelId id, std::unique_ptr<StopCondition> stopCondition = nullptr);
    KernelResult TuneIteration(const KernelId id, const std::vector<BufferOutputDescriptor>& output,
        const bool recomputeReference = false);
    std::vector<KernelResult> SimulateTuning(const KernelId id, const std::vector<KernelResult>& results,
        std::unique_ptr<StopCondition> stopCondition = nullptr);
    // The same, stopping after `iterations` replayed configurations (0 = until the space is exhausted).
    std::vector<KernelResult> SimulateTuning(const KernelId id, const std::vector<KernelResult>& results,
        const uint64_t iterations);
    void SetSearcher(const KernelId id, std::unique_ptr<Searcher> searcher);
    // KTT's profile-based searcher (ProfileBasedSearcher.h) with the counter model at modelPath (the
    // JSON forest of ktt_b200/profile_model.py; for a KTT model path "X.sav", "X.sav.json").
    // useBuiltinModule has no effect: the searcher is native code.
    void SetProfileBasedSearcher(const KernelId id, const std::string& modelPath, const bool useBuiltinModule = true,
        const uint32_t batchSize = 5, const uint32_t neighborSize = 100, const uint32_t randomSize = 10);
    void InitializeConfigurationData(const KernelId id);
    void ClearConfigurationData(const KernelId id);
    uint64_t GetConfigurationsCount(const KernelId id) const;
    KernelConfiguration GetBestConfiguration(const KernelId id) const;
    KernelConfiguration CreateConfiguration(const KernelId id, const ParameterInput& parameters) const;
    std::string GetKernelSource(const KernelId id, const KernelConfiguration& configuration) const;
    std::string GetKernelDefinitionSource(const KernelDefinitionId id, const KernelConfiguration& configuration) const;

    // ---- output ----------------------------------------------------------------------------
    static void SetTimeUnit(const TimeUnit unit);
    void SaveResults(const std::vector<KernelResult>& results, const std::string& filePath, const OutputFormat format,
        const UserData& data = {}) const;
    std::vector<KernelResult> LoadResults(const std::string& filePath, const OutputFormat format) const;
    std::vector<KernelResult> LoadResults(const std::string& filePath, const OutputFormat format, UserData& data) const;

    // ---- queues, device, compiler and logging ----------------------------------------------
    // Queues of a tuner created from a ComputeApiInitializer: another of the caller's streams, or one
    // removed again (the last one stays); without an initializer the tuner has queue 0 only.
    QueueId AddComputeQueue(ComputeQueue queue);
    void RemoveComputeQueue(const QueueId id);
    // Compute and transfer actions complete before the call that started them returns, so these only
    // wait for the device.
    void WaitForComputeAction(const ComputeActionId id);
    void WaitForTransferAction(const TransferActionId id);
    void SynchronizeQueue(const QueueId id);
    void SynchronizeQueues();
    void SynchronizeDevice();
    void SetCompilerOptions(const std::string& options, const bool overrideDefault = false);
    void SetGlobalSizeType(const GlobalSizeType type);
    void SetAutomaticGlobalSizeCorrection(const bool flag);
    void SetKernelCacheCapacity(const uint64_t capacity);
    // All platforms (CUDA: one) and the devices of one platform, as Tutorials/01ComputeApiInfo prints them.
    std::vector<PlatformInfo> GetPlatformInfo() const;
    std::vector<DeviceInfo> GetDeviceInfo(const PlatformIndex platform) const;
    DeviceInfo GetCurrentDeviceInfo() const;

    static void SetLoggingLevel(const LoggingLevel level);
    static LoggingLevel GetLoggingLevel();
    static void SetLoggingTarget(std::ostream& outputTarget);
    static void SetLoggingTarget(const std::string& filePath);

private:
    std::unique_ptr<TunerCore> m_Core;

    ArgumentId AddArgumentWithOwnedData(const size_t elementSize, const ArgumentDataType dataType,
        const ArgumentMemoryType memoryType, const ArgumentAccessType accessType, const void* data, const size_t dataSize,
        const ArgumentId& customId);
    ArgumentId AddArgumentWithReferencedData(const size_t elementSize, const ArgumentDataType dataType,
        const ArgumentAccessType accessType, void* data, const size_t dataSize, const ArgumentId& customId);
    ArgumentId AddSpecialArgument(const size_t elementSize, const ArgumentDataType dataType, const ArgumentMemoryType memoryType,
        const void* data, const size_t dataSize, const std::string& symbolName, const ArgumentId& customId);
    ArgumentId AddUserArgument(ComputeBuffer buffer, const size_t elementSize, const ArgumentDataType dataType,
        const ArgumentAccessType accessType, const size_t bufferSize, const ArgumentId& customId);
    void AddParameterInternal(const KernelId id, const std::string& name, const std::vector<ParameterValue>& values,
        const std::string& group);

    template <typename T>
    static ArgumentDataType DeriveDataType()
    {
        if constexpr (std::is_same_v<T, float>) return ArgumentDataType::Float;
        else if constexpr (std::is_same_v<T, double>) return ArgumentDataType::Double;
        else if constexpr (std::is_same_v<T, int32_t>) return ArgumentDataType::Int;
        else if constexpr (std::is_same_v<T, uint32_t>) return ArgumentDataType::UnsignedInt;
        else if constexpr (std::is_same_v<T, int64_t>) return ArgumentDataType::Long;
        else if constexpr (std::is_same_v<T, uint64_t>) return ArgumentDataType::UnsignedLong;
        else if constexpr (std::is_same_v<T, int16_t>) return ArgumentDataType::Short;
        else if constexpr (std::is_same_v<T, uint16_t>) return ArgumentDataType::UnsignedShort;
        else if constexpr (std::is_same_v<T, int8_t> || std::is_same_v<T, char>) return ArgumentDataType::Char;
        else if constexpr (std::is_same_v<T, uint8_t>) return ArgumentDataType::UnsignedChar;
        else return ArgumentDataType::Custom;
    }
};

} // namespace ktt
