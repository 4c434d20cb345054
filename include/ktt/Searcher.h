// Searcher.h -- configuration searchers of the ktt:: surface.
//
// Searcher base class with the query interface of KTT 2.1.0 Source/Api/Searcher/Searcher.h:22-136
// (configurations addressed by index in the configuration space, random choice among unexplored
// ones, neighbours within a number of differing parameters), and the three searchers of
// Source/Api/Searcher: DeterministicSearcher (indices in order, DeterministicSearcher.cpp:10-26),
// RandomSearcher (uniform among unexplored, RandomSearcher.cpp:10-24) and McmcSearcher (Markov chain
// Monte Carlo with 10 random boot steps, neighbours within 2 differing parameters and escape
// probability 0.02, McmcSearcher.cpp:58-188, McmcSearcher.h:56-58).
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <random>
#include <set>
#include <vector>

#include <ktt/Results.h>

namespace ktt
{

class ConfigurationSpace;

class KTT_API Searcher
{
public:
    Searcher();
    virtual ~Searcher() = default;

    virtual void OnInitialize();
    virtual void OnReset();
    virtual bool CalculateNextConfiguration(const KernelResult& previousResult) = 0;
    virtual KernelConfiguration GetCurrentConfiguration() const = 0;

    KernelConfiguration GetConfiguration(const uint64_t index) const;
    uint64_t GetIndex(const KernelConfiguration& configuration) const;
    KernelConfiguration GetRandomConfiguration() const;
    std::vector<KernelConfiguration> GetNeighbourConfigurations(const KernelConfiguration& configuration,
        const uint64_t maxDifferences, const size_t maxNeighbours = 3) const;
    uint64_t GetConfigurationsCount() const;
    uint64_t GetUnexploredConfigurationsCount() const;
    const std::set<uint64_t>& GetExploredIndices() const;
    bool IsInitialized() const;

    // Called by the tuner.
    void Initialize(const ConfigurationSpace& space);
    void Reset();

private:
    const ConfigurationSpace* m_Space;
};

class KTT_API DeterministicSearcher : public Searcher
{
public:
    DeterministicSearcher();
    void OnReset() override;
    bool CalculateNextConfiguration(const KernelResult& previousResult) override;
    KernelConfiguration GetCurrentConfiguration() const override;

private:
    uint64_t m_Index;
};

class KTT_API RandomSearcher : public Searcher
{
public:
    RandomSearcher();
    void OnInitialize() override;
    bool CalculateNextConfiguration(const KernelResult& previousResult) override;
    KernelConfiguration GetCurrentConfiguration() const override;

private:
    KernelConfiguration m_CurrentConfiguration;
};

class KTT_API McmcSearcher : public Searcher
{
public:
    McmcSearcher(const KernelConfiguration& start = {});
    // Seeded variant: the same seed reproduces the same walk (KTT seeds from the clock).
    McmcSearcher(const KernelConfiguration& start, const uint64_t seed);

    void OnInitialize() override;
    void OnReset() override;
    bool CalculateNextConfiguration(const KernelResult& previousResult) override;
    KernelConfiguration GetCurrentConfiguration() const override;

private:
    uint64_t m_Index;
    size_t m_VisitedStatesCount;
    size_t m_OriginState;
    size_t m_CurrentState;
    size_t m_Boot;
    double m_BestTime;
    KernelConfiguration m_Start;
    std::map<size_t, double> m_ExecutionTimes;
    std::default_random_engine m_Generator;
    std::uniform_int_distribution<size_t> m_IntDistribution;
    std::uniform_real_distribution<double> m_ProbabilityDistribution;

    inline static size_t m_MaximumDifferences = 2;
    inline static size_t m_BootIterations = 10;
    inline static double m_EscapeProbability = 0.02;
};

} // namespace ktt
