// Results.cpp -- ComputationResult, KernelResult, BufferOutputDescriptor (see include/ktt/Results.h).
//
// Duration bookkeeping as in KTT 2.1.0 Source/Api/Output/KernelResult.cpp:108-242: the kernel
// duration of a result is the sum of its computations' durations, the total duration adds the
// extra duration, the total overhead sums every overhead, and a result is valid when its status is Ok.
#include <algorithm>
#include <stdexcept>

#include <ktt/Results.h>

namespace ktt
{

// ---- profiling counters (Source/Api/Output/KernelProfilingCounter.cpp, KernelProfilingData.cpp) ----

KernelProfilingCounter::KernelProfilingCounter() : m_Type(ProfilingCounterType::Double), m_Value(0.0) {}

KernelProfilingCounter::KernelProfilingCounter(const std::string& name, const ProfilingCounterType type, const int64_t value) :
    m_Name(name), m_Type(type), m_Value(value)
{}

KernelProfilingCounter::KernelProfilingCounter(const std::string& name, const ProfilingCounterType type, const uint64_t value) :
    m_Name(name), m_Type(type), m_Value(value)
{}

KernelProfilingCounter::KernelProfilingCounter(const std::string& name, const ProfilingCounterType type, const double value) :
    m_Name(name), m_Type(type), m_Value(value)
{}

const std::string& KernelProfilingCounter::GetName() const { return m_Name; }
ProfilingCounterType KernelProfilingCounter::GetType() const { return m_Type; }

int64_t KernelProfilingCounter::GetValueInt() const
{
    if (!std::holds_alternative<int64_t>(m_Value))
    {
        throw std::runtime_error("Profiling counter " + m_Name + " does not hold a signed integer value");
    }

    return std::get<int64_t>(m_Value);
}

uint64_t KernelProfilingCounter::GetValueUint() const
{
    if (!std::holds_alternative<uint64_t>(m_Value))
    {
        throw std::runtime_error("Profiling counter " + m_Name + " does not hold an unsigned integer value");
    }

    return std::get<uint64_t>(m_Value);
}

double KernelProfilingCounter::GetValueDouble() const
{
    if (!std::holds_alternative<double>(m_Value))
    {
        throw std::runtime_error("Profiling counter " + m_Name + " does not hold a floating-point value");
    }

    return std::get<double>(m_Value);
}

bool KernelProfilingCounter::operator==(const KernelProfilingCounter& other) const { return m_Name == other.m_Name; }
bool KernelProfilingCounter::operator!=(const KernelProfilingCounter& other) const { return !(*this == other); }
bool KernelProfilingCounter::operator<(const KernelProfilingCounter& other) const { return m_Name < other.m_Name; }

KernelProfilingData::KernelProfilingData() : m_RemainingRuns(0) {}
KernelProfilingData::KernelProfilingData(const uint64_t remainingRuns) : m_RemainingRuns(remainingRuns) {}
KernelProfilingData::KernelProfilingData(const std::vector<KernelProfilingCounter>& counters) :
    m_Counters(counters), m_RemainingRuns(0)
{}

bool KernelProfilingData::IsValid() const { return m_RemainingRuns == 0; }

bool KernelProfilingData::HasCounter(const std::string& name) const
{
    return std::any_of(m_Counters.cbegin(), m_Counters.cend(), [&name](const auto& c) { return c.GetName() == name; });
}

const KernelProfilingCounter& KernelProfilingData::GetCounter(const std::string& name) const
{
    const auto it = std::find_if(m_Counters.cbegin(), m_Counters.cend(), [&name](const auto& c) { return c.GetName() == name; });

    if (it == m_Counters.cend())
    {
        throw std::runtime_error("Profiling counter with name " + name + " was not found");
    }

    return *it;
}

const std::vector<KernelProfilingCounter>& KernelProfilingData::GetCounters() const { return m_Counters; }

void KernelProfilingData::SetCounters(const std::vector<KernelProfilingCounter>& counters)
{
    m_Counters = counters;
    m_RemainingRuns = 0;
}

void KernelProfilingData::AddCounter(const KernelProfilingCounter& counter) { m_Counters.push_back(counter); }
bool KernelProfilingData::HasRemainingProfilingRuns() const { return m_RemainingRuns > 0; }
uint64_t KernelProfilingData::GetRemainingProfilingRuns() const { return m_RemainingRuns; }

void KernelProfilingData::DecreaseRemainingProfilingRuns()
{
    if (m_RemainingRuns > 0)
    {
        --m_RemainingRuns;
    }
}

KernelCompilationData::KernelCompilationData() :
    m_MaxWorkGroupSize(0), m_LocalMemorySize(0), m_PrivateMemorySize(0), m_ConstantMemorySize(0), m_RegistersCount(0)
{}

ComputationResult::ComputationResult() : ComputationResult("") {}

ComputationResult::ComputationResult(const std::string& kernelFunction) :
    m_KernelFunction(kernelFunction), m_Duration(InvalidDuration), m_Overhead(0), m_CompilationOverhead(0)
{}

ComputationResult::ComputationResult(const ComputationResult& other) :
    m_KernelFunction(other.m_KernelFunction), m_GlobalSize(other.m_GlobalSize), m_LocalSize(other.m_LocalSize),
    m_Duration(other.m_Duration), m_Overhead(other.m_Overhead), m_CompilationOverhead(other.m_CompilationOverhead)
{
    if (other.m_CompilationData)
    {
        m_CompilationData = std::make_unique<KernelCompilationData>(*other.m_CompilationData);
    }

    if (other.m_ProfilingData)
    {
        m_ProfilingData = std::make_unique<KernelProfilingData>(*other.m_ProfilingData);
    }
}

ComputationResult& ComputationResult::operator=(const ComputationResult& other)
{
    if (this != &other)
    {
        m_KernelFunction = other.m_KernelFunction;
        m_GlobalSize = other.m_GlobalSize;
        m_LocalSize = other.m_LocalSize;
        m_Duration = other.m_Duration;
        m_Overhead = other.m_Overhead;
        m_CompilationOverhead = other.m_CompilationOverhead;
        m_CompilationData = other.m_CompilationData ? std::make_unique<KernelCompilationData>(*other.m_CompilationData)
                                                    : nullptr;
        m_ProfilingData = other.m_ProfilingData ? std::make_unique<KernelProfilingData>(*other.m_ProfilingData) : nullptr;
    }

    return *this;
}

void ComputationResult::SetDurationData(const Nanoseconds duration, const Nanoseconds overhead,
    const Nanoseconds compilationOverhead)
{
    m_Duration = duration;
    m_Overhead = overhead;
    m_CompilationOverhead = compilationOverhead;
}

void ComputationResult::SetSizeData(const DimensionVector& globalSize, const DimensionVector& localSize)
{
    m_GlobalSize = globalSize;
    m_LocalSize = localSize;
}

void ComputationResult::SetCompilationData(std::unique_ptr<KernelCompilationData> data) { m_CompilationData = std::move(data); }
void ComputationResult::SetProfilingData(std::unique_ptr<KernelProfilingData> data) { m_ProfilingData = std::move(data); }
const std::string& ComputationResult::GetKernelFunction() const { return m_KernelFunction; }
const DimensionVector& ComputationResult::GetGlobalSize() const { return m_GlobalSize; }
const DimensionVector& ComputationResult::GetLocalSize() const { return m_LocalSize; }
Nanoseconds ComputationResult::GetDuration() const { return m_Duration; }
Nanoseconds ComputationResult::GetOverhead() const { return m_Overhead; }
Nanoseconds ComputationResult::GetCompilationOverhead() const { return m_CompilationOverhead; }
bool ComputationResult::HasCompilationData() const { return m_CompilationData != nullptr; }

const KernelCompilationData& ComputationResult::GetCompilationData() const
{
    static const KernelCompilationData empty;
    return m_CompilationData ? *m_CompilationData : empty;
}

bool ComputationResult::HasProfilingData() const { return m_ProfilingData != nullptr; }

const KernelProfilingData& ComputationResult::GetProfilingData() const
{
    if (!m_ProfilingData)
    {
        throw std::runtime_error("Computation result of " + m_KernelFunction + " has no profiling data");
    }

    return *m_ProfilingData;
}

bool ComputationResult::HasRemainingProfilingRuns() const
{
    return m_ProfilingData != nullptr && m_ProfilingData->HasRemainingProfilingRuns();
}
bool ComputationResult::HasPowerData() const { return false; }

// ---- KernelResult ---------------------------------------------------------------------------

KernelResult::KernelResult() : KernelResult("", KernelConfiguration()) {}

KernelResult::KernelResult(const std::string& kernelName, const KernelConfiguration& configuration) :
    KernelResult(kernelName, configuration, {})
{}

KernelResult::KernelResult(const std::string& kernelName, const KernelConfiguration& configuration,
    const std::vector<ComputationResult>& results) :
    m_Configuration(configuration), m_Results(results), m_KernelName(kernelName), m_ExtraDuration(0),
    m_DataMovementOverhead(0), m_ValidationOverhead(0), m_SearcherOverhead(0), m_FailedKernelOverhead(0),
    m_ProfilingRunsOverhead(0), m_Status(ResultStatus::Ok)
{}

void KernelResult::SetStatus(const ResultStatus status) { m_Status = status; }
void KernelResult::SetExtraDuration(const Nanoseconds duration) { m_ExtraDuration = duration; }
void KernelResult::SetDataMovementOverhead(const Nanoseconds overhead) { m_DataMovementOverhead = overhead; }
void KernelResult::SetValidationOverhead(const Nanoseconds overhead) { m_ValidationOverhead = overhead; }
void KernelResult::SetSearcherOverhead(const Nanoseconds overhead) { m_SearcherOverhead = overhead; }
void KernelResult::SetFailedKernelOverhead(const Nanoseconds overhead) { m_FailedKernelOverhead = overhead; }
void KernelResult::SetProfilingRunsOverhead(const Nanoseconds overhead) { m_ProfilingRunsOverhead = overhead; }
void KernelResult::SetResults(const std::vector<ComputationResult>& results) { m_Results = results; }

const std::string& KernelResult::GetKernelName() const { return m_KernelName; }
const std::vector<ComputationResult>& KernelResult::GetResults() const { return m_Results; }
const KernelConfiguration& KernelResult::GetConfiguration() const { return m_Configuration; }
ResultStatus KernelResult::GetStatus() const { return m_Status; }

Nanoseconds KernelResult::GetKernelDuration() const
{
    Nanoseconds total = 0;

    for (const auto& result : m_Results)
    {
        if (result.GetDuration() == InvalidDuration)
        {
            return InvalidDuration;
        }

        total += result.GetDuration();
    }

    return total;
}

Nanoseconds KernelResult::GetKernelOverhead() const
{
    Nanoseconds total = 0;

    for (const auto& result : m_Results)
    {
        total += result.GetOverhead();
    }

    return total;
}

Nanoseconds KernelResult::GetKernelCompilationOverhead() const
{
    Nanoseconds total = 0;

    for (const auto& result : m_Results)
    {
        total += result.GetCompilationOverhead();
    }

    return total;
}

Nanoseconds KernelResult::GetExtraDuration() const { return m_ExtraDuration; }
Nanoseconds KernelResult::GetDataMovementOverhead() const { return m_DataMovementOverhead; }
Nanoseconds KernelResult::GetValidationOverhead() const { return m_ValidationOverhead; }
Nanoseconds KernelResult::GetSearcherOverhead() const { return m_SearcherOverhead; }
Nanoseconds KernelResult::GetFailedKernelOverhead() const { return m_FailedKernelOverhead; }
Nanoseconds KernelResult::GetProfilingRunsOverhead() const { return m_ProfilingRunsOverhead; }
Nanoseconds KernelResult::GetCompilationOverhead() const { return GetKernelCompilationOverhead(); }

Nanoseconds KernelResult::GetTotalDuration() const
{
    const Nanoseconds kernel = GetKernelDuration();
    return kernel == InvalidDuration ? InvalidDuration : kernel + m_ExtraDuration;
}

Nanoseconds KernelResult::GetTotalOverhead() const
{
    return GetKernelOverhead() + m_DataMovementOverhead + m_ValidationOverhead + m_SearcherOverhead + m_FailedKernelOverhead
        + m_ProfilingRunsOverhead;
}

bool KernelResult::IsValid() const { return m_Status == ResultStatus::Ok; }
bool KernelResult::HasRemainingProfilingRuns() const
{
    return std::any_of(m_Results.cbegin(), m_Results.cend(), [](const auto& r) { return r.HasRemainingProfilingRuns(); });
}

// ---- BufferOutputDescriptor -----------------------------------------------------------------

BufferOutputDescriptor::BufferOutputDescriptor(const ArgumentId& id, void* outputDestination) :
    BufferOutputDescriptor(id, outputDestination, 0)
{}

BufferOutputDescriptor::BufferOutputDescriptor(const ArgumentId& id, void* outputDestination, const size_t outputSize) :
    m_ArgumentId(id), m_OutputDestination(outputDestination), m_OutputSize(outputSize)
{}

const ArgumentId& BufferOutputDescriptor::GetArgumentId() const { return m_ArgumentId; }
void* BufferOutputDescriptor::GetOutputDestination() const { return m_OutputDestination; }
size_t BufferOutputDescriptor::GetOutputSize() const { return m_OutputSize; }

} // namespace ktt
