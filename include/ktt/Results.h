// Results.h -- results and output descriptors of the ktt:: surface.
//
// Interfaces of KTT 2.1.0 Source/Api/Output/ComputationResult.h, KernelCompilationData.h,
// KernelResult.h (durations and overheads, TotalDuration = kernel durations + extra duration:
// Source/Api/Output/KernelResult.cpp:108-242) and BufferOutputDescriptor.h.
#pragma once

#include <memory>
#include <string>
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

    const std::string& GetKernelFunction() const;
    const DimensionVector& GetGlobalSize() const;
    const DimensionVector& GetLocalSize() const;
    Nanoseconds GetDuration() const;
    Nanoseconds GetOverhead() const;
    Nanoseconds GetCompilationOverhead() const;
    bool HasCompilationData() const;
    const KernelCompilationData& GetCompilationData() const;
    bool HasProfilingData() const;
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
