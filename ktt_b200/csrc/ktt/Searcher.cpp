// Searcher.cpp -- Searcher base, DeterministicSearcher, RandomSearcher, McmcSearcher.
//
// The MCMC walk restates KTT 2.1.0 Source/Api/Searcher/McmcSearcher.cpp:58-188: after 10 boot steps
// that visit random unexplored configurations and keep the fastest as the origin, each step
// records the last configuration's time (+inf when it failed), moves the origin to the last state
// when it was at least as fast (or, with probability 0.02, regardless), and proposes a random
// unexplored neighbour of the origin within 2 differing parameters; with no such neighbour it
// restarts from a random unexplored configuration.
#include <chrono>
#include <limits>
#include <stdexcept>

#include <ktt/ConfigurationSpace.h>
#include <ktt/Searcher.h>

namespace ktt
{

Searcher::Searcher() : m_Space(nullptr) {}
void Searcher::OnInitialize() {}
void Searcher::OnReset() {}

KernelConfiguration Searcher::GetConfiguration(const uint64_t index) const { return m_Space->GetConfiguration(index); }
uint64_t Searcher::GetIndex(const KernelConfiguration& configuration) const { return m_Space->GetIndex(configuration); }
KernelConfiguration Searcher::GetRandomConfiguration() const { return m_Space->GetRandomConfiguration(); }

std::vector<KernelConfiguration> Searcher::GetNeighbourConfigurations(const KernelConfiguration& configuration,
    const uint64_t maxDifferences, const size_t maxNeighbours) const
{
    return m_Space->GetNeighbours(configuration, maxDifferences, maxNeighbours);
}

uint64_t Searcher::GetConfigurationsCount() const { return m_Space->GetConfigurationsCount(); }

uint64_t Searcher::GetUnexploredConfigurationsCount() const
{
    return m_Space->GetConfigurationsCount() - m_Space->GetExplored().size();
}

const std::set<uint64_t>& Searcher::GetExploredIndices() const { return m_Space->GetExplored(); }
bool Searcher::IsInitialized() const { return m_Space != nullptr; }

void Searcher::Initialize(const ConfigurationSpace& space)
{
    m_Space = &space;
    OnInitialize();
}

void Searcher::Reset()
{
    OnReset();
    m_Space = nullptr;
}

// ---- DeterministicSearcher ------------------------------------------------------------------

DeterministicSearcher::DeterministicSearcher() : m_Index(0) {}
void DeterministicSearcher::OnReset() { m_Index = 0; }

bool DeterministicSearcher::CalculateNextConfiguration([[maybe_unused]] const KernelResult& previousResult)
{
    ++m_Index;
    return m_Index < GetConfigurationsCount();
}

KernelConfiguration DeterministicSearcher::GetCurrentConfiguration() const { return GetConfiguration(m_Index); }

// ---- RandomSearcher -------------------------------------------------------------------------

RandomSearcher::RandomSearcher() = default;
void RandomSearcher::OnInitialize() { m_CurrentConfiguration = GetRandomConfiguration(); }

bool RandomSearcher::CalculateNextConfiguration([[maybe_unused]] const KernelResult& previousResult)
{
    if (GetUnexploredConfigurationsCount() == 0)
    {
        return false;
    }

    m_CurrentConfiguration = GetRandomConfiguration();
    return true;
}

KernelConfiguration RandomSearcher::GetCurrentConfiguration() const { return m_CurrentConfiguration; }

// ---- McmcSearcher ---------------------------------------------------------------------------

McmcSearcher::McmcSearcher(const KernelConfiguration& start) :
    McmcSearcher(start, static_cast<uint64_t>(std::chrono::system_clock::now().time_since_epoch().count()))
{}

McmcSearcher::McmcSearcher(const KernelConfiguration& start, const uint64_t seed) :
    m_Index(0), m_VisitedStatesCount(0), m_OriginState(0), m_CurrentState(0), m_Boot(0),
    m_BestTime(std::numeric_limits<double>::max()), m_Start(start),
    m_Generator(static_cast<std::default_random_engine::result_type>(seed)), m_ProbabilityDistribution(0.0, 1.0)
{}

void McmcSearcher::OnInitialize()
{
    m_IntDistribution = std::uniform_int_distribution<size_t>(0, GetConfigurationsCount() - 1);
    size_t initialState = 0;

    if (m_Start.IsValid())
    {
        initialState = GetIndex(m_Start);
    }
    else
    {
        initialState = m_IntDistribution(m_Generator);
        m_Boot = m_BootIterations;
    }

    m_OriginState = initialState;
    m_CurrentState = initialState;
    m_Index = initialState;
}

void McmcSearcher::OnReset()
{
    m_Index = 0;
    m_VisitedStatesCount = 0;
    m_OriginState = 0;
    m_CurrentState = 0;
    m_BestTime = std::numeric_limits<double>::max();
    m_ExecutionTimes.clear();
}

bool McmcSearcher::CalculateNextConfiguration(const KernelResult& previousResult)
{
    ++m_VisitedStatesCount;
    const double infinity = std::numeric_limits<double>::max();
    m_ExecutionTimes[m_Index] = previousResult.IsValid() ? static_cast<double>(previousResult.GetTotalDuration()) : infinity;

    auto timeOf = [this, infinity](size_t state) -> double&
    {
        auto it = m_ExecutionTimes.find(state);
        return it == m_ExecutionTimes.end() ? (m_ExecutionTimes[state] = infinity) : it->second;
    };

    if (m_Boot > 0)
    {
        if (timeOf(m_CurrentState) <= timeOf(m_OriginState))
        {
            m_OriginState = m_CurrentState;
            m_BestTime = timeOf(m_CurrentState);
        }

        --m_Boot;

        if (GetExploredIndices().size() >= GetConfigurationsCount())
        {
            return false;
        }

        while (GetExploredIndices().count(m_Index) != 0)
        {
            m_Index = m_IntDistribution(m_Generator);
        }

        m_CurrentState = m_Index;
        return true;
    }

    if (timeOf(m_CurrentState) <= timeOf(m_OriginState) || m_ProbabilityDistribution(m_Generator) < m_EscapeProbability)
    {
        m_OriginState = m_CurrentState;

        if (timeOf(m_CurrentState) < m_BestTime)
        {
            m_BestTime = timeOf(m_CurrentState);
        }
    }

    if (GetExploredIndices().size() >= GetConfigurationsCount())
    {
        return false;
    }

    const auto neighbourConfigurations = GetNeighbourConfigurations(GetConfiguration(m_OriginState), m_MaximumDifferences,
        std::numeric_limits<size_t>::max());
    std::vector<size_t> neighbours;

    for (const auto& neighbour : neighbourConfigurations)
    {
        neighbours.push_back(static_cast<size_t>(GetIndex(neighbour)));
    }

    if (neighbours.empty())
    {
        while (GetExploredIndices().count(m_OriginState) != 0)
        {
            m_OriginState = m_IntDistribution(m_Generator);
        }

        m_Index = m_OriginState;
        m_CurrentState = m_OriginState;
        return true;
    }

    m_CurrentState = neighbours.at(m_IntDistribution(m_Generator) % neighbours.size());
    m_Index = m_CurrentState;
    return true;
}

KernelConfiguration McmcSearcher::GetCurrentConfiguration() const { return GetConfiguration(m_Index); }

} // namespace ktt
