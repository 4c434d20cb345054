// ConfigurationSpace.h -- the set of valid configurations of one kernel, addressed by index.
//
// Restates what KTT 2.1.0 builds in Source/TuningRunner/ConfigurationData.cpp:31-278 from the
// parameter groups (Kernel::GenerateParameterGroups, Source/Kernel/Kernel.cpp:238-256), subgroups
// (KernelParameterGroup::GenerateSubgroups, Source/Kernel/KernelParameterGroup.cpp) and
// configuration trees (Source/TuningRunner/ConfigurationTree.cpp, ConfigurationForest.cpp):
//   * parameters are grouped by their group name; groups are tuned one after another: the space is
//     the concatenation of the groups' spaces (count = sum), and a configuration of one group is
//     completed with the best configuration found so far for the other groups;
//   * inside a group, parameters linked by constraints form a subgroup (connected components of
//     the "shares a constraint" relation); every other parameter is a subgroup of its own;
//   * a subgroup's valid value combinations are enumerated depth-first: parameters of constraints
//     with fewer parameters first (in constraint order), then the rest, the first parameter being
//     the outermost loop, each constraint evaluated as soon as all its parameters are assigned;
//   * a group's configuration index is mixed-radix over its subgroups, the first subgroup varying
//     fastest.
// KTT orders subgroups by heap-pointer order (std::set of pointers), which is not reproducible;
// here constrained subgroups come in the order of their first constraint, then unconstrained
// parameters in the order they were added.  The set of configurations and the enumeration order
// inside each subgroup are KTT's.
#pragma once

#include <cstdint>
#include <map>
#include <random>
#include <set>
#include <string>
#include <vector>

#include <ktt/Configuration.h>

namespace ktt
{

struct KTT_API KernelParameterInfo
{
    std::string name;
    std::vector<ParameterValue> values;
    std::string group;
};

struct KTT_API KernelConstraintInfo
{
    std::vector<std::string> parameters;
    GenericConstraintFunction function;
};

class KTT_API ConfigurationSpace
{
public:
    ConfigurationSpace(const std::vector<KernelParameterInfo>& parameters,
        const std::vector<KernelConstraintInfo>& constraints, const uint64_t seed = 0);

    uint64_t GetConfigurationsCount() const;
    KernelConfiguration GetConfiguration(const uint64_t index) const;
    uint64_t GetIndex(const KernelConfiguration& configuration) const;
    bool IsValid(const KernelConfiguration& configuration) const;
    KernelConfiguration GetRandomConfiguration() const;
    std::vector<KernelConfiguration> GetNeighbours(const KernelConfiguration& configuration, const uint64_t maxDifferences,
        const size_t maxNeighbours) const;

    void MarkExplored(const uint64_t index);
    const std::set<uint64_t>& GetExplored() const;
    bool IsExhausted() const;
    void UpdateBest(const KernelConfiguration& configuration, const Nanoseconds duration);
    KernelConfiguration GetBestConfiguration() const;
    Nanoseconds GetBestDuration() const;

    // Layout, for inspection: per group, its subgroups as lists of parameter names in enumeration order.
    std::vector<std::vector<std::vector<std::string>>> GetLayout() const;

private:
    struct Subgroup
    {
        std::vector<size_t> parameters;                 // indices into m_Parameters, enumeration order
        std::vector<std::vector<size_t>> combinations;  // value indices per valid combination, DFS order
    };

    struct Group
    {
        std::string name;
        std::vector<Subgroup> subgroups;
        uint64_t count = 1;
    };

    std::vector<KernelParameterInfo> m_Parameters;
    std::vector<KernelConstraintInfo> m_Constraints;
    std::vector<Group> m_Groups;
    std::set<uint64_t> m_Explored;
    KernelConfiguration m_Best;
    Nanoseconds m_BestDuration;
    mutable std::mt19937_64 m_Generator;

    size_t ParameterIndex(const std::string& name) const;
    KernelConfiguration GroupConfiguration(const size_t group, uint64_t local) const;
    bool LocalIndex(const size_t group, const KernelConfiguration& configuration, uint64_t& local) const;
    bool ConstraintsHold(const KernelConfiguration& configuration) const;
};

} // namespace ktt
