// Results.h -- results and output descriptors of the ktt:: surface.
//
// Interfaces of KTT 2.1.0 Source/Api/Output/ComputationResult.h, KernelCompilationData.h,
// KernelResult.h (durations and overheads, TotalDuration = kernel durations + extra duration:
// Source/Api/Output/KernelResult.cpp:108-242), KernelProfilingCounter.h, KernelProfilingData.h,
// ProfilingCounterType.h and BufferOutputDescriptor.h.
#pragma once

#include <memory>
#include <string>
#include <variant>
#include <vector>

#include <ktt/Configuration.h>

namespace ktt
{

// Properties of the compiled kernel variant a computation ran.
class KTT_API KernelCompilationData
{
public:
    KernelCompilationData();

    uint64_t m_MaxWorkGroupSize;
    uint64_t m_LocalMemorySize;
    uint64_t m_PrivateMemorySize;
    uint64_t m_ConstantMemorySize;
    uint64_t m_RegistersCount;
};

enum class ProfilingCounterType
{
    Int,
    UnsignedInt,
    Double,
    Percent,
    Throughput,
    UtilizationLevel
};

// One hardware counter of a profiled run (CUPTI metrics arrive as Double).
class KTT_API KernelProfilingCounter
{
public:
    KernelProfilingCounter();
    explicit KernelProfilingCounter(const std::string& name, const ProfilingCounterType type, const int64_t value);
    explicit KernelProfilingCounter(const std::string& name, const ProfilingCounterType type, const uint64_t value);
    explicit KernelProfilingCounter(const std::string& name, const ProfilingCounterType type, const double value);

    const std::string& GetName() const;
    ProfilingCounterType GetType() const;
    int64_t GetValueInt() const;
    uint64_t GetValueUint() const;
    double GetValueDouble() const;

    bool operator==(const KernelProfilingCounter& other) const;
    bool operator!=(const KernelProfilingCounter& other) const;
    bool operator<(const KernelProfilingCounter& other) const;

private:
    std::string m_Name;
    ProfilingCounterType m_Type;
    std::variant<int64_t, uint64_t, double> m_Value;
};

// The counters of one profiled computation; while passes remain it holds their count instead
// (valid once it has no remaining runs).
class KTT_API KernelProfilingData
{
public:
    KernelProfilingData();
    explicit KernelProfilingData(const uint64_t remainingRuns);
    explicit KernelProfilingData(const std::vector<KernelProfilingCounter>& counters);

    bool IsValid() const;
    bool HasCounter(const std::string& name) const;
    const KernelProfilingCounter& GetCounter(const std::string& name) const;
    const std::vector<KernelProfilingCounter>& GetCounters() const;
    void SetCounters(const std::vector<KernelProfilingCounter>& counters);
    void AddCounter(const KernelProfilingCounter& counter);
    bool HasRemainingProfilingRuns() const;
    uint64_t GetRemainingProfilingRuns() const;
    void DecreaseRemainingProfilingRuns();

private:
    std::vector<KernelProfilingCounter> m_Counters;
    uint64_t m_RemainingRuns;
};

class KTT_API ComputationResult
{
public:
    ComputationResult();
    explicit ComputationResult(const std::string& kernelFunction);
    ComputationResult(const ComputationResult& other);
    ComputationResult& operator=(const ComputationResult& other);

    void SetDurationData(const Nanoseconds duration, const Nanoseconds overhead,
        const Nanoseconds compilationOverhead = 0);
    void SetSizeData(const DimensionVector& globalSize, const DimensionVector& localSize);
    void SetCompilationData(std::unique_ptr<KernelCompilationData> data);
    void SetProfilingData(std::unique_ptr<KernelProfilingData> data);

    const std::string& GetKernelFunction() const;
    const DimensionVector& GetGlobalSize() const;
    const DimensionVector& GetLocalSize() const;
    Nanoseconds GetDuration() const;
    Nanoseconds GetOverhead() const;
    Nanoseconds GetCompilationOverhead() const;
    bool HasCompilationData() const;
    const KernelCompilationData& GetCompilationData() const;
    bool HasProfilingData() const;
    const KernelProfilingData& GetProfilingData() const;
    bool HasRemainingProfilingRuns() const;
    bool HasPowerData() const;

private:
    std::string m_KernelFunction;
    DimensionVector m_GlobalSize;
    DimensionVector m_LocalSize;
    Nanoseconds m_Duration;
    Nanoseconds m_Overhead;
    Nanoseconds m_CompilationOverhead;
    std::unique_ptr<KernelCompilationData> m_CompilationData;
    std::unique_ptr<KernelProfilingData> m_ProfilingData;
};

class KTT_API KernelResult
{
public:
    KernelResult();
    explicit KernelResult(const std::string& kernelName, const KernelConfiguration& configuration);
    explicit KernelResult(const std::string& kernelName, const KernelConfiguration& configuration,
        const std::vector<ComputationResult>& results);

    void SetStatus(const ResultStatus status);
    void SetExtraDuration(const Nanoseconds duration);
    void SetDataMovementOverhead(const Nanoseconds overhead);
    void SetValidationOverhead(const Nanoseconds overhead);
    void SetSearcherOverhead(const Nanoseconds overhead);
    void SetFailedKernelOverhead(const Nanoseconds overhead);
    void SetProfilingRunsOverhead(const Nanoseconds overhead);
    void SetResults(const std::vector<ComputationResult>& results);

    const std::string& GetKernelName() const;
    const std::vector<ComputationResult>& GetResults() const;
    const KernelConfiguration& GetConfiguration() const;
    ResultStatus GetStatus() const;
    Nanoseconds GetKernelDuration() const;
    Nanoseconds GetKernelOverhead() const;
    Nanoseconds GetKernelCompilationOverhead() const;
    Nanoseconds GetExtraDuration() const;
    Nanoseconds GetDataMovementOverhead() const;
    Nanoseconds GetValidationOverhead() const;
    Nanoseconds GetSearcherOverhead() const;
    Nanoseconds GetFailedKernelOverhead() const;
    Nanoseconds GetProfilingRunsOverhead() const;
    Nanoseconds GetCompilationOverhead() const;
    Nanoseconds GetTotalDuration() const;
    Nanoseconds GetTotalOverhead() const;
    bool IsValid() const;
    bool HasRemainingProfilingRuns() const;

private:
    KernelConfiguration m_Configuration;
    std::vector<ComputationResult> m_Results;
    std::string m_KernelName;
    Nanoseconds m_ExtraDuration;
    Nanoseconds m_DataMovementOverhead;
    Nanoseconds m_ValidationOverhead;
    Nanoseconds m_SearcherOverhead;
    Nanoseconds m_FailedKernelOverhead;
    Nanoseconds m_ProfilingRunsOverhead;
    ResultStatus m_Status;
};

class KTT_API BufferOutputDescriptor
{
public:
    explicit BufferOutputDescriptor(const ArgumentId& id, void* outputDestination);
    explicit BufferOutputDescriptor(const ArgumentId& id, void* outputDestination, const size_t outputSize);

    const ArgumentId& GetArgumentId() const;
    void* GetOutputDestination() const;
    size_t GetOutputSize() const;

private:
    ArgumentId m_ArgumentId;
    void* m_OutputDestination;
    size_t m_OutputSize;
};

} // namespace ktt
