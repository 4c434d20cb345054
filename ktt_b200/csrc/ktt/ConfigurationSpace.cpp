// ConfigurationSpace.cpp -- see include/ktt/ConfigurationSpace.h for the construction rules and the
// KTT 2.1.0 sources they restate.
#include <algorithm>
#include <functional>
#include <limits>
#include <map>
#include <stdexcept>

#include <ktt/ConfigurationSpace.h>

namespace ktt
{

ConfigurationSpace::ConfigurationSpace(const std::vector<KernelParameterInfo>& parameters,
    const std::vector<KernelConstraintInfo>& constraints, const uint64_t seed) :
    m_Parameters(parameters), m_Constraints(constraints), m_BestDuration(InvalidDuration), m_Generator(seed)
{
    for (const auto& constraint : m_Constraints)
    {
        for (const auto& name : constraint.parameters)
        {
            (void)ParameterIndex(name);
        }
    }

    // groups by name, in name order (KTT iterates a std::map keyed by group name)
    std::map<std::string, std::vector<size_t>> groups;

    for (size_t i = 0; i < m_Parameters.size(); ++i)
    {
        if (m_Parameters[i].values.empty())
        {
            throw std::runtime_error("Parameter " + m_Parameters[i].name + " has no values");
        }

        groups[m_Parameters[i].group].push_back(i);
    }

    for (const auto& [groupName, members] : groups)
    {
        Group group;
        group.name = groupName;

        // constraints that touch this group, in the order they were added
        std::vector<size_t> groupConstraints;

        for (size_t c = 0; c < m_Constraints.size(); ++c)
        {
            for (const auto& name : m_Constraints[c].parameters)
            {
                if (std::find(members.cbegin(), members.cend(), ParameterIndex(name)) != members.cend())
                {
                    groupConstraints.push_back(c);
                    break;
                }
            }
        }

        // subgroups: connected components over shared constraints, seeded in constraint order
        std::vector<bool> used(m_Constraints.size(), false);
        std::vector<bool> covered(m_Parameters.size(), false);
        std::vector<std::pair<std::vector<size_t>, std::vector<size_t>>> components;  // (parameters, constraints)

        for (const size_t seedConstraint : groupConstraints)
        {
            if (used[seedConstraint])
            {
                continue;
            }

            std::vector<size_t> compConstraints{seedConstraint};
            std::vector<size_t> compParameters;
            used[seedConstraint] = true;
            bool added = true;

            while (added)
            {
                added = false;

                for (const size_t c : compConstraints)
                {
                    for (const auto& name : m_Constraints[c].parameters)
                    {
                        const size_t p = ParameterIndex(name);

                        if (std::find(compParameters.cbegin(), compParameters.cend(), p) == compParameters.cend())
                        {
                            compParameters.push_back(p);
                        }
                    }
                }

                for (const size_t c : groupConstraints)
                {
                    if (used[c])
                    {
                        continue;
                    }

                    const bool touches = std::any_of(m_Constraints[c].parameters.cbegin(), m_Constraints[c].parameters.cend(),
                        [&](const std::string& name)
                        {
                            return std::find(compParameters.cbegin(), compParameters.cend(), ParameterIndex(name))
                                != compParameters.cend();
                        });

                    if (touches)
                    {
                        used[c] = true;
                        compConstraints.push_back(c);
                        added = true;
                    }
                }
            }

            for (const size_t p : compParameters)
            {
                covered[p] = true;
            }

            components.emplace_back(compParameters, compConstraints);
        }

        for (const size_t p : members)
        {
            if (!covered[p])
            {
                components.push_back({{p}, {}});
            }
        }

        for (auto& [compParameters, compConstraints] : components)
        {
            Subgroup subgroup;

            // enumeration order: parameters of constraints with fewer parameters first (stable), then the rest
            std::vector<size_t> sortedConstraints = compConstraints;
            std::stable_sort(sortedConstraints.begin(), sortedConstraints.end(), [this](size_t a, size_t b)
            {
                return m_Constraints[a].parameters.size() < m_Constraints[b].parameters.size();
            });

            for (const size_t c : sortedConstraints)
            {
                for (const auto& name : m_Constraints[c].parameters)
                {
                    const size_t p = ParameterIndex(name);

                    if (std::find(subgroup.parameters.cbegin(), subgroup.parameters.cend(), p) == subgroup.parameters.cend())
                    {
                        subgroup.parameters.push_back(p);
                    }
                }
            }

            for (const size_t p : members)
            {
                if (std::find(compParameters.cbegin(), compParameters.cend(), p) != compParameters.cend()
                    && std::find(subgroup.parameters.cbegin(), subgroup.parameters.cend(), p) == subgroup.parameters.cend())
                {
                    subgroup.parameters.push_back(p);
                }
            }

            // each constraint is evaluated at the level where its last parameter gets assigned
            std::map<size_t, std::vector<size_t>> evaluationLevel;

            for (const size_t c : compConstraints)
            {
                size_t level = 0;

                for (const auto& name : m_Constraints[c].parameters)
                {
                    const size_t p = ParameterIndex(name);
                    const size_t position = static_cast<size_t>(
                        std::find(subgroup.parameters.cbegin(), subgroup.parameters.cend(), p) - subgroup.parameters.cbegin());
                    level = std::max(level, position);
                }

                evaluationLevel[level].push_back(c);
            }

            std::vector<size_t> indices;
            std::function<void(size_t)> enumerate = [&](size_t level)
            {
                if (level == subgroup.parameters.size())
                {
                    subgroup.combinations.push_back(indices);
                    return;
                }

                const auto& parameter = m_Parameters[subgroup.parameters[level]];

                for (size_t v = 0; v < parameter.values.size(); ++v)
                {
                    indices.push_back(v);
                    bool ok = true;
                    auto it = evaluationLevel.find(level);

                    if (it != evaluationLevel.end())
                    {
                        for (const size_t c : it->second)
                        {
                            std::vector<const ParameterValue*> values;

                            for (const auto& name : m_Constraints[c].parameters)
                            {
                                const size_t p = ParameterIndex(name);
                                const size_t position = static_cast<size_t>(std::find(subgroup.parameters.cbegin(),
                                    subgroup.parameters.cend(), p) - subgroup.parameters.cbegin());
                                values.push_back(&m_Parameters[p].values[indices[position]]);
                            }

                            ok = ok && m_Constraints[c].function(values);
                        }
                    }

                    if (ok)
                    {
                        enumerate(level + 1);
                    }

                    indices.pop_back();
                }
            };

            enumerate(0);
            group.count *= subgroup.combinations.size();
            group.subgroups.push_back(std::move(subgroup));
        }

        m_Groups.push_back(std::move(group));
    }

    // the initial "best" configuration: the first configuration of every group
    for (size_t g = 0; g < m_Groups.size(); ++g)
    {
        if (m_Groups[g].count > 0)
        {
            m_Best.Merge(GroupConfiguration(g, 0));
        }
    }
}

size_t ConfigurationSpace::ParameterIndex(const std::string& name) const
{
    for (size_t i = 0; i < m_Parameters.size(); ++i)
    {
        if (m_Parameters[i].name == name)
        {
            return i;
        }
    }

    throw std::runtime_error("Unknown parameter " + name);
}

uint64_t ConfigurationSpace::GetConfigurationsCount() const
{
    if (m_Parameters.empty())
    {
        return 1;
    }

    uint64_t total = 0;

    for (const auto& group : m_Groups)
    {
        total += group.count;
    }

    return total;
}

KernelConfiguration ConfigurationSpace::GroupConfiguration(const size_t group, uint64_t local) const
{
    std::vector<ParameterPair> pairs;

    for (const auto& subgroup : m_Groups[group].subgroups)
    {
        const uint64_t n = subgroup.combinations.size();
        const auto& combination = subgroup.combinations[local % n];
        local /= n;

        for (size_t k = 0; k < subgroup.parameters.size(); ++k)
        {
            const auto& parameter = m_Parameters[subgroup.parameters[k]];
            pairs.emplace_back(parameter.name, parameter.values[combination[k]]);
        }
    }

    return KernelConfiguration(pairs);
}

KernelConfiguration ConfigurationSpace::GetConfiguration(const uint64_t index) const
{
    if (index >= GetConfigurationsCount())
    {
        throw std::runtime_error("Invalid configuration index " + std::to_string(index));
    }

    if (m_Parameters.empty())
    {
        return KernelConfiguration();
    }

    uint64_t local = index;

    for (size_t g = 0; g < m_Groups.size(); ++g)
    {
        if (local < m_Groups[g].count)
        {
            KernelConfiguration result = GroupConfiguration(g, local);
            result.Merge(m_Best);
            return result;
        }

        local -= m_Groups[g].count;
    }

    throw std::runtime_error("Invalid configuration index");
}

bool ConfigurationSpace::LocalIndex(const size_t group, const KernelConfiguration& configuration, uint64_t& local) const
{
    local = 0;
    uint64_t multiplier = 1;

    for (const auto& subgroup : m_Groups[group].subgroups)
    {
        std::vector<size_t> indices;

        for (const size_t p : subgroup.parameters)
        {
            const auto& parameter = m_Parameters[p];
            bool found = false;

            for (const auto& pair : configuration.GetPairs())
            {
                if (pair.GetName() != parameter.name)
                {
                    continue;
                }

                for (size_t v = 0; v < parameter.values.size(); ++v)
                {
                    if (pair.HasSameValue(ParameterPair(parameter.name, parameter.values[v])))
                    {
                        indices.push_back(v);
                        found = true;
                        break;
                    }
                }

                break;
            }

            if (!found)
            {
                return false;
            }
        }

        const auto it = std::find(subgroup.combinations.cbegin(), subgroup.combinations.cend(), indices);

        if (it == subgroup.combinations.cend())
        {
            return false;
        }

        local += multiplier * static_cast<uint64_t>(it - subgroup.combinations.cbegin());
        multiplier *= subgroup.combinations.size();
    }

    return true;
}

uint64_t ConfigurationSpace::GetIndex(const KernelConfiguration& configuration) const
{
    if (m_Parameters.empty())
    {
        return 0;
    }

    // the group whose parameters lead the configuration (KTT: the first pair belongs to the local tree)
    if (configuration.GetPairs().empty())
    {
        throw std::runtime_error("Empty configuration");
    }

    const std::string& lead = configuration.GetPairs().front().GetName();
    uint64_t offset = 0;

    for (size_t g = 0; g < m_Groups.size(); ++g)
    {
        const bool owns = std::any_of(m_Groups[g].subgroups.cbegin(), m_Groups[g].subgroups.cend(), [&](const Subgroup& s)
        {
            return std::any_of(s.parameters.cbegin(), s.parameters.cend(),
                [&](size_t p) { return m_Parameters[p].name == lead; });
        });

        if (owns)
        {
            uint64_t local = 0;

            if (!LocalIndex(g, configuration, local))
            {
                throw std::runtime_error("Configuration is not in the space: " + configuration.GetString());
            }

            return offset + local;
        }

        offset += m_Groups[g].count;
    }

    throw std::runtime_error("Configuration is not in the space: " + configuration.GetString());
}

bool ConfigurationSpace::ConstraintsHold(const KernelConfiguration& configuration) const
{
    for (const auto& constraint : m_Constraints)
    {
        std::vector<const ParameterValue*> values;

        for (const auto& name : constraint.parameters)
        {
            const ParameterValue* value = nullptr;

            for (const auto& pair : configuration.GetPairs())
            {
                if (pair.GetName() == name)
                {
                    value = &pair.GetValue();
                    break;
                }
            }

            if (value == nullptr)
            {
                return false;
            }

            values.push_back(value);
        }

        if (!constraint.function(values))
        {
            return false;
        }
    }

    return true;
}

bool ConfigurationSpace::IsValid(const KernelConfiguration& configuration) const
{
    for (const auto& parameter : m_Parameters)
    {
        bool found = false;

        for (const auto& pair : configuration.GetPairs())
        {
            if (pair.GetName() != parameter.name)
            {
                continue;
            }

            found = std::any_of(parameter.values.cbegin(), parameter.values.cend(),
                [&](const ParameterValue& v) { return pair.HasSameValue(ParameterPair(parameter.name, v)); });
            break;
        }

        if (!found)
        {
            return false;
        }
    }

    return ConstraintsHold(configuration);
}

KernelConfiguration ConfigurationSpace::GetRandomConfiguration() const
{
    const uint64_t total = GetConfigurationsCount();

    if (m_Explored.size() >= total)
    {
        throw std::runtime_error("All configurations have been explored");
    }

    std::uniform_int_distribution<uint64_t> distribution(0, total - 1);

    // rejection sampling while the space is sparsely explored, then a uniform pick among the rest
    if (m_Explored.size() * 2 < total)
    {
        while (true)
        {
            const uint64_t index = distribution(m_Generator);

            if (m_Explored.count(index) == 0)
            {
                return GetConfiguration(index);
            }
        }
    }

    std::vector<uint64_t> remaining;

    for (uint64_t i = 0; i < total; ++i)
    {
        if (m_Explored.count(i) == 0)
        {
            remaining.push_back(i);
        }
    }

    std::uniform_int_distribution<size_t> pick(0, remaining.size() - 1);
    return GetConfiguration(remaining[pick(m_Generator)]);
}

std::vector<KernelConfiguration> ConfigurationSpace::GetNeighbours(const KernelConfiguration& configuration,
    const uint64_t maxDifferences, const size_t maxNeighbours) const
{
    // Breadth first over the number of changed parameters (KTT Kernel::EnumerateNeighbours,
    // Source/Kernel/Kernel.cpp:371-428): all configurations differing in 1 parameter, then in 2, ...,
    // keeping the valid, unexplored ones.  Parameters in name order, values in their declared order.
    std::vector<size_t> order(m_Parameters.size());

    for (size_t i = 0; i < order.size(); ++i)
    {
        order[i] = i;
    }

    std::sort(order.begin(), order.end(), [this](size_t a, size_t b) { return m_Parameters[a].name < m_Parameters[b].name; });

    std::vector<KernelConfiguration> result;
    std::vector<size_t> chosen;

    std::function<bool(size_t, size_t, const KernelConfiguration&)> recurse =
        [&](size_t start, size_t remaining, const KernelConfiguration& current) -> bool
    {
        if (remaining == 0)
        {
            if (IsValid(current) && m_Explored.count(GetIndex(current)) == 0)
            {
                if (result.size() >= maxNeighbours)
                {
                    return false;
                }

                KernelConfiguration merged = current;
                merged.Merge(m_Best);
                result.push_back(merged);
            }

            return true;
        }

        for (size_t o = start; o < order.size(); ++o)
        {
            const auto& parameter = m_Parameters[order[o]];
            std::vector<ParameterPair> values;

            for (const auto& v : parameter.values)
            {
                values.emplace_back(parameter.name, v);
            }

            bool present = false;

            for (const auto& pair : current.GetPairs())
            {
                present = present || pair.GetName() == parameter.name;
            }

            if (!present)
            {
                continue;
            }

            for (const auto& neighbour : current.GenerateNeighbours(parameter.name, values))
            {
                if (!recurse(o + 1, remaining - 1, neighbour))
                {
                    return false;
                }
            }
        }

        return true;
    };

    for (uint64_t d = 1; d <= maxDifferences; ++d)
    {
        if (!recurse(0, static_cast<size_t>(d), configuration))
        {
            break;
        }
    }

    return result;
}

void ConfigurationSpace::MarkExplored(const uint64_t index) { m_Explored.insert(index); }
const std::set<uint64_t>& ConfigurationSpace::GetExplored() const { return m_Explored; }
bool ConfigurationSpace::IsExhausted() const { return m_Explored.size() >= GetConfigurationsCount(); }

void ConfigurationSpace::UpdateBest(const KernelConfiguration& configuration, const Nanoseconds duration)
{
    if (duration < m_BestDuration)
    {
        m_BestDuration = duration;
        m_Best = configuration;
    }
}

KernelConfiguration ConfigurationSpace::GetBestConfiguration() const { return m_Best; }
Nanoseconds ConfigurationSpace::GetBestDuration() const { return m_BestDuration; }

std::vector<std::vector<std::vector<std::string>>> ConfigurationSpace::GetLayout() const
{
    std::vector<std::vector<std::vector<std::string>>> layout;

    for (const auto& group : m_Groups)
    {
        std::vector<std::vector<std::string>> subgroups;

        for (const auto& subgroup : group.subgroups)
        {
            std::vector<std::string> names;

            for (const size_t p : subgroup.parameters)
            {
                names.push_back(m_Parameters[p].name);
            }

            subgroups.push_back(names);
        }

        layout.push_back(subgroups);
    }

    return layout;
}

} // namespace ktt
