// StopCondition.cpp -- stop conditions (see include/ktt/StopCondition.h); semantics of KTT 2.1.0
// Source/Api/StopCondition/{ConfigurationCount,ConfigurationDuration,ConfigurationFraction,
// TuningDuration,UnionCondition}.cpp.
#include <algorithm>
#include <limits>

#include <ktt/StopCondition.h>

namespace ktt
{

ConfigurationCount::ConfigurationCount(const uint64_t count) : m_CurrentCount(0), m_TargetCount(count) {}
bool ConfigurationCount::IsFulfilled() const { return m_CurrentCount >= m_TargetCount; }

void ConfigurationCount::Initialize(const uint64_t configurationsCount)
{
    m_CurrentCount = 0;
    m_TargetCount = std::min(m_TargetCount, configurationsCount);
}

void ConfigurationCount::Update([[maybe_unused]] const KernelResult& result) { ++m_CurrentCount; }

std::string ConfigurationCount::GetStatusString() const
{
    return "Current count of explored configurations: " + std::to_string(m_CurrentCount) + " / "
        + std::to_string(m_TargetCount);
}

ConfigurationDuration::ConfigurationDuration(const double duration) :
    m_BestDuration(std::numeric_limits<double>::max()), m_TargetDuration(std::max(0.0, duration))
{}

bool ConfigurationDuration::IsFulfilled() const { return m_BestDuration <= m_TargetDuration; }
void ConfigurationDuration::Initialize([[maybe_unused]] const uint64_t configurationsCount)
{
    m_BestDuration = std::numeric_limits<double>::max();
}

void ConfigurationDuration::Update(const KernelResult& result)
{
    if (result.IsValid())
    {
        // durations are kept in nanoseconds; the target is in milliseconds
        m_BestDuration = std::min(m_BestDuration, static_cast<double>(result.GetTotalDuration()) / 1e6);
    }
}

std::string ConfigurationDuration::GetStatusString() const
{
    return "Current best known configuration duration: " + std::to_string(m_BestDuration) + "ms, target duration: "
        + std::to_string(m_TargetDuration) + "ms";
}

ConfigurationFraction::ConfigurationFraction(const double fraction) :
    m_CurrentCount(0), m_TotalCount(0), m_TargetFraction(std::clamp(fraction, 0.0, 1.0))
{}

bool ConfigurationFraction::IsFulfilled() const
{
    return m_TotalCount == 0 || static_cast<double>(m_CurrentCount) / static_cast<double>(m_TotalCount) >= m_TargetFraction;
}

void ConfigurationFraction::Initialize(const uint64_t configurationsCount)
{
    m_CurrentCount = 0;
    m_TotalCount = configurationsCount;
}

void ConfigurationFraction::Update([[maybe_unused]] const KernelResult& result) { ++m_CurrentCount; }

std::string ConfigurationFraction::GetStatusString() const
{
    const double fraction = m_TotalCount ? static_cast<double>(m_CurrentCount) / static_cast<double>(m_TotalCount) : 1.0;
    return "Current fraction of explored configurations: " + std::to_string(fraction) + " / "
        + std::to_string(m_TargetFraction);
}

TuningDuration::TuningDuration(const double duration) : m_PassedTime(0.0), m_TargetTime(std::max(0.0, duration)) {}
bool TuningDuration::IsFulfilled() const { return m_PassedTime > m_TargetTime; }

void TuningDuration::Initialize([[maybe_unused]] const uint64_t configurationsCount)
{
    m_InitialTime = std::chrono::steady_clock::now();
    m_PassedTime = 0.0;
}

void TuningDuration::Update([[maybe_unused]] const KernelResult& result)
{
    const auto now = std::chrono::steady_clock::now();
    m_PassedTime = std::chrono::duration<double>(now - m_InitialTime).count();
}

std::string TuningDuration::GetStatusString() const
{
    return "Current tuning time: " + std::to_string(m_PassedTime) + "s / " + std::to_string(m_TargetTime) + "s";
}

UnionCondition::UnionCondition(std::vector<std::shared_ptr<StopCondition>> conditions) : m_Conditions(std::move(conditions)) {}

bool UnionCondition::IsFulfilled() const
{
    return std::any_of(m_Conditions.cbegin(), m_Conditions.cend(), [](const auto& c) { return c->IsFulfilled(); });
}

void UnionCondition::Initialize(const uint64_t configurationsCount)
{
    for (auto& condition : m_Conditions)
    {
        condition->Initialize(configurationsCount);
    }
}

void UnionCondition::Update(const KernelResult& result)
{
    for (auto& condition : m_Conditions)
    {
        condition->Update(result);
    }
}

std::string UnionCondition::GetStatusString() const
{
    std::string result;

    for (const auto& condition : m_Conditions)
    {
        result += condition->GetStatusString() + "\n";
    }

    return result;
}

} // namespace ktt
