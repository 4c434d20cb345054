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
// plus the B200 parameters PRECISION (0 FP32, 1 compensated, 2 FP64 merge), RSQRT_SOFT (share of
// reciprocal square roots on the FMA pipe, of 8) and ATOM_SPLIT (2..8: a thread-block cluster of
// that many CTAs shares each point tile, each streaming a share of the atoms).  A configuration that maps to no compiled variant
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

#include <ktt/ComputeInterface.h>
#include <ktt/Configuration.h>
#include <ktt/ConfigurationSpace.h>
#include <ktt/Results.h>
#include <ktt/Searcher.h>
#include <ktt/StopCondition.h>

namespace ktt
{

class TunerCore;

class KTT_API DeviceInfo
{
public:
    DeviceInfo(const DeviceIndex index, const std::string& name, const uint64_t globalMemorySize, const uint32_t smCount,
        const uint32_t ccMajor, const uint32_t ccMinor);
    DeviceIndex GetIndex() const;
    const std::string& GetName() const;
    uint64_t GetGlobalMemorySize() const;
    uint32_t GetMaxComputeUnits() const;
    uint32_t GetCudaComputeCapabilityMajor() const;
    uint32_t GetCudaComputeCapabilityMinor() const;
    std::string GetString() const;

private:
    DeviceIndex m_Index;
    std::string m_Name;
    uint64_t m_GlobalMemorySize;
    uint32_t m_SmCount;
    uint32_t m_CcMajor;
    uint32_t m_CcMinor;
};

class KTT_API Tuner
{
public:
    explicit Tuner(const PlatformIndex platform, const DeviceIndex device, const ComputeApi api);
    explicit Tuner(const PlatformIndex platform, const DeviceIndex device, const ComputeApi api,
        const uint32_t computeQueueCount);
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
    void SynchronizeQueue(const QueueId id);
    void SynchronizeQueues();
    void SynchronizeDevice();
    void SetCompilerOptions(const std::string& options, const bool overrideDefault = false);
    void SetGlobalSizeType(const GlobalSizeType type);
    void SetAutomaticGlobalSizeCorrection(const bool flag);
    void SetKernelCacheCapacity(const uint64_t capacity);
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
