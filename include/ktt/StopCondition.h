// StopCondition.h -- tuning stop conditions of the ktt:: surface.
//
// Interfaces and semantics of KTT 2.1.0 Source/Api/StopCondition/*.h: a condition is initialised
// with the size of the configuration space, updated with each KernelResult, and asked whether the
// tuning should stop.  ConfigurationCount counts tested configurations, ConfigurationDuration stops
// once a valid configuration at or below the given duration (ms) is found, ConfigurationFraction
// after a fraction of the space, TuningDuration after the given wall-clock seconds, UnionCondition
// when any member condition is fulfilled.
#pragma once

#include <chrono>
#include <memory>
#include <string>
#include <vector>

#include <ktt/Results.h>

namespace ktt
{

class KTT_API StopCondition
{
public:
    virtual ~StopCondition() = default;
    virtual bool IsFulfilled() const = 0;
    virtual void Initialize(const uint64_t configurationsCount) = 0;
    virtual void Update(const KernelResult& result) = 0;
    virtual std::string GetStatusString() const = 0;
};

class KTT_API ConfigurationCount : public StopCondition
{
public:
    explicit ConfigurationCount(const uint64_t count);
    bool IsFulfilled() const override;
    void Initialize(const uint64_t configurationsCount) override;
    void Update(const KernelResult& result) override;
    std::string GetStatusString() const override;

private:
    uint64_t m_CurrentCount;
    uint64_t m_TargetCount;
};

class KTT_API ConfigurationDuration : public StopCondition
{
public:
    explicit ConfigurationDuration(const double duration);
    bool IsFulfilled() const override;
    void Initialize(const uint64_t configurationsCount) override;
    void Update(const KernelResult& result) override;
    std::string GetStatusString() const override;

private:
    double m_BestDuration;
    double m_TargetDuration;
};

class KTT_API ConfigurationFraction : public StopCondition
{
public:
    explicit ConfigurationFraction(const double fraction);
    bool IsFulfilled() const override;
    void Initialize(const uint64_t configurationsCount) override;
    void Update(const KernelResult& result) override;
    std::string GetStatusString() const override;

private:
    uint64_t m_CurrentCount;
    uint64_t m_TotalCount;
    double m_TargetFraction;
};

class KTT_API TuningDuration : public StopCondition
{
public:
    explicit TuningDuration(const double duration);
    bool IsFulfilled() const override;
    void Initialize(const uint64_t configurationsCount) override;
    void Update(const KernelResult& result) override;
    std::string GetStatusString() const override;

private:
    std::chrono::steady_clock::time_point m_InitialTime;
    double m_PassedTime;
    double m_TargetTime;
};

class KTT_API UnionCondition : public StopCondition
{
public:
    explicit UnionCondition(std::vector<std::shared_ptr<StopCondition>> conditions);
    bool IsFulfilled() const override;
    void Initialize(const uint64_t configurationsCount) override;
    void Update(const KernelResult& result) override;
    std::string GetStatusString() const override;

private:
    std::vector<std::shared_ptr<StopCondition>> m_Conditions;
};

} // namespace ktt
