// CPU tests of the ktt:: surface (no GPU needed): configuration space, searchers, stop conditions,
// result files and the error convention.  Driven by tests/test_tuner_cpu.py; each test is selected
// by name on the command line and exits 0 on success.
//
//   tuner_cpu_tests <test> [fixture-dir]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include <Ktt.h>

namespace
{

int failures = 0;

#define CHECK(cond)                                                                                      \
    do                                                                                                   \
    {                                                                                                    \
        if (!(cond))                                                                                     \
        {                                                                                                \
            std::cerr << __FILE__ << ":" << __LINE__ << ": check failed: " #cond << std::endl;           \
            ++failures;                                                                                  \
        }                                                                                                \
    } while (0)

std::string fixtureDir = "tests/golden";
std::string workDir = "/tmp";

// The tuning space of the CUDA 3D Coulomb example (parameters, thread modifiers and constraints
// as in Examples/CoulombSum3d/CoulombSum3d.cpp:137-216 for the CUDA back-end).
struct Coulomb3dSpace
{
    ktt::Tuner tuner{0, 0, ktt::ComputeApi::CUDA};
    ktt::KernelDefinitionId definition;
    ktt::KernelId kernel;

    Coulomb3dSpace()
    {
        tuner.SetGlobalSizeType(ktt::GlobalSizeType::CUDA);
        definition = tuner.AddKernelDefinition("directCoulombSum", "/* source */", ktt::DimensionVector(256, 256, 256),
            ktt::DimensionVector());
        kernel = tuner.CreateSimpleKernel("CoulombSum", definition);
        tuner.AddParameter(kernel, "WORK_GROUP_SIZE_X", std::vector<uint64_t>{16, 32});
        tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::X, "WORK_GROUP_SIZE_X",
            ktt::ModifierAction::Multiply);
        tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::X, "WORK_GROUP_SIZE_X",
            ktt::ModifierAction::DivideCeil);
        tuner.AddParameter(kernel, "WORK_GROUP_SIZE_Y", std::vector<uint64_t>{1, 2, 4, 8});
        tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
            ktt::ModifierAction::Multiply);
        tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
            ktt::ModifierAction::DivideCeil);
        tuner.AddParameter(kernel, "WORK_GROUP_SIZE_Z", std::vector<uint64_t>{1});
        tuner.AddParameter(kernel, "Z_ITERATIONS", std::vector<uint64_t>{1, 2, 4, 8, 16, 32});
        tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::Z, "Z_ITERATIONS",
            ktt::ModifierAction::DivideCeil);
        tuner.AddParameter(kernel, "INNER_UNROLL_FACTOR", std::vector<uint64_t>{0, 1, 2, 4, 8, 16, 32});
        tuner.AddParameter(kernel, "USE_CONSTANT_MEMORY", std::vector<uint64_t>{0});
        tuner.AddParameter(kernel, "USE_SOA", std::vector<uint64_t>{0, 1});
        tuner.AddParameter(kernel, "VECTOR_SIZE", std::vector<uint64_t>{1});
        tuner.AddConstraint(kernel, {"INNER_UNROLL_FACTOR", "Z_ITERATIONS"},
            [](const std::vector<uint64_t>& v) { return v.at(0) < v.at(1); });
        tuner.AddConstraint(kernel, {"WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"},
            [](const std::vector<uint64_t>& v) { return v.at(0) * v.at(1) >= 64; });
    }
};

std::string Key(const ktt::KernelConfiguration& configuration)
{
    std::vector<std::string> items;

    for (const auto& pair : configuration.GetPairs())
    {
        items.push_back(pair.GetString());
    }

    std::sort(items.begin(), items.end());
    std::string key;

    for (const auto& item : items)
    {
        key += item + ";";
    }

    return key;
}

// The recorded 2080 Ti results in KTT's own JSON layout (written by tests/test_tuner_cpu.py).
std::vector<ktt::KernelResult> Recorded(ktt::Tuner& tuner)
{
    return tuner.LoadResults(workDir + "/coulomb_2080_ktt_format.json", ktt::OutputFormat::JSON);
}

// ---- tests ------------------------------------------------------------------------------------

void TestPrefix()
{
    // Tests/KernelManagerTests.cpp:57-81
    std::vector<ktt::ParameterPair> pairs;
    pairs.emplace_back("param_two", static_cast<uint64_t>(5));
    pairs.emplace_back("param_one", static_cast<uint64_t>(2));
    ktt::KernelConfiguration configuration(pairs);
    CHECK(configuration.GeneratePrefix() == "#define param_two 5\n#define param_one 2\n");
    CHECK(configuration.GetString() == "param_two 5, param_one 2");

    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    const auto definition = tuner.AddKernelDefinition("simpleKernel", "__global__ void simpleKernel() {}",
        ktt::DimensionVector(1024), ktt::DimensionVector(8, 8));
    const auto kernel = tuner.CreateSimpleKernel("kernel", definition);
    tuner.AddParameter(kernel, "param_one", std::vector<uint64_t>{1, 2, 3});
    tuner.AddParameter(kernel, "param_two", std::vector<uint64_t>{5, 10});
    CHECK(tuner.GetKernelSource(kernel, configuration) == "#define param_two 5\n#define param_one 2\n__global__ void simpleKernel() {}");
}

void TestCoulombSpaceMatchesRecordedSpace()
{
    Coulomb3dSpace s;
    CHECK(s.tuner.GetConfigurationsCount(s.kernel) == 210);
    std::set<std::string> ours;
    ktt::Tuner& tuner = s.tuner;
    const auto results = Recorded(tuner);
    CHECK(results.size() == 210);
    std::set<std::string> recorded;

    for (const auto& r : results)
    {
        recorded.insert(Key(r.GetConfiguration()));
    }

    // every configuration of the space, enumerated through a deterministic simulated run
    const auto walked = tuner.SimulateTuning(s.kernel, results);
    CHECK(walked.size() == 210);

    for (const auto& r : walked)
    {
        ours.insert(Key(r.GetConfiguration()));
    }

    CHECK(ours.size() == 210);
    CHECK(ours == recorded);
}

void TestSubgroupEnumerationOrder()
{
    // Inside a constrained subgroup the first parameter of the constraint is the outer loop:
    // (INNER_UNROLL_FACTOR, Z_ITERATIONS) enumerate as (0,1), (0,2), ..., (0,32), (1,2), ...
    std::vector<ktt::KernelParameterInfo> parameters{
        {"Z_ITERATIONS", {uint64_t{1}, uint64_t{2}, uint64_t{4}}, ""},
        {"INNER_UNROLL_FACTOR", {uint64_t{0}, uint64_t{1}, uint64_t{2}}, ""}};
    std::vector<ktt::KernelConstraintInfo> constraints{{{"INNER_UNROLL_FACTOR", "Z_ITERATIONS"},
        [](const std::vector<const ktt::ParameterValue*>& v) { return std::get<uint64_t>(*v[0]) < std::get<uint64_t>(*v[1]); }}};
    ktt::ConfigurationSpace space(parameters, constraints);
    CHECK(space.GetConfigurationsCount() == 6);
    const std::vector<std::pair<uint64_t, uint64_t>> expected{{0, 1}, {0, 2}, {0, 4}, {1, 2}, {1, 4}, {2, 4}};

    for (uint64_t i = 0; i < 6; ++i)
    {
        const auto c = space.GetConfiguration(i);
        CHECK(c.GetPairs()[0].GetName() == "INNER_UNROLL_FACTOR");
        CHECK(c.GetPairs()[0].GetValueUint() == expected[i].first);
        CHECK(c.GetPairs()[1].GetValueUint() == expected[i].second);
        CHECK(space.GetIndex(c) == i);
    }

    // the first subgroup varies fastest; unconstrained parameters follow in the order they were added
    std::vector<ktt::KernelParameterInfo> p2{{"A", {uint64_t{1}, uint64_t{2}}, ""}, {"B", {uint64_t{7}, uint64_t{8}, uint64_t{9}}, ""}};
    ktt::ConfigurationSpace s2(p2, {});
    CHECK(s2.GetConfigurationsCount() == 6);
    CHECK(s2.GetConfiguration(1).GetPairs()[0].GetValueUint() == 2);
    CHECK(s2.GetConfiguration(1).GetPairs()[1].GetValueUint() == 7);
    CHECK(s2.GetConfiguration(2).GetPairs()[1].GetValueUint() == 8);
}

void TestGroups()
{
    // parameters in different groups are tuned one group after the other: count is the sum
    std::vector<ktt::KernelParameterInfo> parameters{{"A", {uint64_t{1}, uint64_t{2}, uint64_t{3}}, "g1"},
        {"B", {uint64_t{1}, uint64_t{2}}, "g2"}, {"C", {uint64_t{5}, uint64_t{6}}, "g2"}};
    ktt::ConfigurationSpace space(parameters, {});
    CHECK(space.GetConfigurationsCount() == 3 + 4);
    const auto c = space.GetConfiguration(4);  // second configuration of g2, completed with g1's best so far
    CHECK(c.GetPairs().size() == 3);
    CHECK(space.IsValid(c));
}

void TestNeighbours()
{
    Coulomb3dSpace s;
    s.tuner.InitializeConfigurationData(s.kernel);
    std::vector<ktt::KernelParameterInfo> params;  // rebuild the same space standalone for inspection
    auto base = s.tuner.CreateConfiguration(s.kernel, {{"WORK_GROUP_SIZE_X", uint64_t{32}}, {"WORK_GROUP_SIZE_Y", uint64_t{4}},
        {"Z_ITERATIONS", uint64_t{16}}, {"INNER_UNROLL_FACTOR", uint64_t{0}}});
    CHECK(base.GetPairs().size() == 8);

    class Probe : public ktt::Searcher
    {
    public:
        std::vector<ktt::KernelConfiguration> found;
        ktt::KernelConfiguration start;
        void OnInitialize() override { found = GetNeighbourConfigurations(start, 1, 1000); }
        bool CalculateNextConfiguration(const ktt::KernelResult&) override { return false; }
        ktt::KernelConfiguration GetCurrentConfiguration() const override { return start; }
    };

    auto probe = std::make_unique<Probe>();
    Probe* raw = probe.get();
    raw->start = base;
    s.tuner.SetSearcher(s.kernel, std::move(probe));
    s.tuner.SimulateTuning(s.kernel, {}, 1);
    CHECK(!raw->found.empty());

    for (const auto& n : raw->found)
    {
        int differences = 0;

        for (const auto& pair : n.GetPairs())
        {
            for (const auto& b : base.GetPairs())
            {
                if (b.GetName() == pair.GetName() && !b.HasSameValue(pair))
                {
                    ++differences;
                }
            }
        }

        CHECK(differences == 1);
    }
}

void TestDeterministicSimulationFindsRecordedBest()
{
    Coulomb3dSpace s;
    const auto recorded = Recorded(s.tuner);
    s.tuner.SetSearcher(s.kernel, std::make_unique<ktt::DeterministicSearcher>());
    const auto results = s.tuner.SimulateTuning(s.kernel, recorded);
    CHECK(results.size() == 210);
    ktt::Nanoseconds best = ktt::InvalidDuration;

    for (const auto& r : recorded)
    {
        if (r.IsValid())
        {
            best = std::min(best, r.GetTotalDuration());
        }
    }

    CHECK(best == 769696);  // 769.696 us, the best configuration of the 2080 Ti search
    CHECK(s.tuner.GetBestConfiguration(s.kernel).IsValid());
}

void TestRandomSearcherVisitsEachOnce()
{
    Coulomb3dSpace s;
    const auto recorded = Recorded(s.tuner);
    s.tuner.SetSearcher(s.kernel, std::make_unique<ktt::RandomSearcher>());
    const auto results = s.tuner.SimulateTuning(s.kernel, recorded);
    std::set<std::string> seen;

    for (const auto& r : results)
    {
        seen.insert(Key(r.GetConfiguration()));
    }

    CHECK(results.size() == 210);
    CHECK(seen.size() == 210);
}

void TestMcmcSearcher()
{
    // MCMC over the recorded space: distinct configurations, and with a seeded walk the best
    // configuration (769.696 us) is reached well before the space is exhausted on average.
    int found = 0;
    size_t total = 0;

    for (uint64_t seed = 1; seed <= 20; ++seed)
    {
        Coulomb3dSpace s;
        const auto recorded = Recorded(s.tuner);
        s.tuner.SetSearcher(s.kernel, std::make_unique<ktt::McmcSearcher>(ktt::KernelConfiguration(), seed));
        const auto results = s.tuner.SimulateTuning(s.kernel, recorded, 100);
        std::set<std::string> seen;

        for (const auto& r : results)
        {
            seen.insert(Key(r.GetConfiguration()));
        }

        CHECK(seen.size() == results.size());
        total += results.size();

        for (const auto& r : results)
        {
            if (r.IsValid() && r.GetTotalDuration() <= 775000)
            {
                ++found;
                break;
            }
        }
    }

    CHECK(total == 2000);
    CHECK(found >= 10);  // MCMC beats blind sampling: a random 100 of 210 holds one of the few best in ~50-70% of runs
}

void TestStopConditions()
{
    Coulomb3dSpace s;
    const auto recorded = Recorded(s.tuner);

    auto run = [&](std::unique_ptr<ktt::StopCondition> stop)
    {
        // a stop condition driven by hand over the deterministic order
        stop->Initialize(210);
        size_t n = 0;

        for (const auto& r : recorded)
        {
            stop->Update(r);
            ++n;

            if (stop->IsFulfilled())
            {
                break;
            }
        }

        return n;
    };

    CHECK(run(std::make_unique<ktt::ConfigurationCount>(20)) == 20);
    CHECK(run(std::make_unique<ktt::ConfigurationCount>(1000)) == 210);
    CHECK(run(std::make_unique<ktt::ConfigurationFraction>(0.1)) == 21);
    const size_t byDuration = run(std::make_unique<ktt::ConfigurationDuration>(0.8));  // 0.8 ms
    CHECK(byDuration > 1 && byDuration <= 210);
    CHECK(recorded[byDuration - 1].GetTotalDuration() <= 800000);
    std::vector<std::shared_ptr<ktt::StopCondition>> members{std::make_shared<ktt::ConfigurationCount>(50),
        std::make_shared<ktt::ConfigurationFraction>(0.05)};
    CHECK(run(std::make_unique<ktt::UnionCondition>(members)) == 11);
}

void TestJsonRoundTrip()
{
    Coulomb3dSpace s;
    const auto recorded = Recorded(s.tuner);
    ktt::Tuner::SetTimeUnit(ktt::TimeUnit::Microseconds);
    s.tuner.SaveResults(recorded, workDir + "/roundtrip", ktt::OutputFormat::JSON, {{"device", "RTX 2080 Ti"}});
    ktt::UserData data;
    const auto loaded = s.tuner.LoadResults(workDir + "/roundtrip.json", ktt::OutputFormat::JSON, data);
    CHECK(loaded.size() == recorded.size());
    CHECK(data["device"] == "RTX 2080 Ti");

    for (size_t i = 0; i < std::min(loaded.size(), recorded.size()); ++i)
    {
        CHECK(loaded[i].GetConfiguration() == recorded[i].GetConfiguration());
        CHECK(loaded[i].GetStatus() == recorded[i].GetStatus());
        const double a = static_cast<double>(loaded[i].GetKernelDuration());
        const double b = static_cast<double>(recorded[i].GetKernelDuration());
        CHECK(std::abs(a - b) <= 1.0);
        CHECK(loaded[i].GetResults().at(0).GetGlobalSize() == recorded[i].GetResults().at(0).GetGlobalSize());
    }

    s.tuner.SaveResults(recorded, workDir + "/roundtrip", ktt::OutputFormat::XML);
    std::ifstream xml(workDir + "/roundtrip.xml");
    CHECK(xml.good());
}

void TestErrorConvention()
{
    ktt::Tuner::SetLoggingLevel(ktt::LoggingLevel::Off);
    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    CHECK(tuner.CreateSimpleKernel("k", 12345) == ktt::InvalidKernelId);
    const auto d = tuner.AddKernelDefinition("directCoulombSum", "", ktt::DimensionVector(8), ktt::DimensionVector());
    CHECK(d != ktt::InvalidKernelDefinitionId);
    CHECK(tuner.AddKernelDefinition("directCoulombSum", "", ktt::DimensionVector(8), ktt::DimensionVector())
        == ktt::InvalidKernelDefinitionId);
    const auto k = tuner.CreateSimpleKernel("k", d);
    CHECK(k != ktt::InvalidKernelId);
    CHECK(tuner.CreateSimpleKernel("k", d) == ktt::InvalidKernelId);
    tuner.AddParameter(k, "P", std::vector<uint64_t>{1, 2});
    tuner.AddParameter(k, "P", std::vector<uint64_t>{3});  // duplicate: logged, ignored
    CHECK(tuner.GetConfigurationsCount(k) == 2);
    const std::vector<float> empty;
    CHECK(tuner.AddArgumentVector(empty, ktt::ArgumentAccessType::ReadOnly) == ktt::InvalidArgumentId);
    const auto a = tuner.AddArgumentScalar(3, "atoms");
    CHECK(a == "atoms");
    CHECK(tuner.AddArgumentScalar(4, "atoms") == ktt::InvalidArgumentId);
    tuner.AddParameter(k, "S", std::vector<std::string>{"x", "y"});
    tuner.AddConstraint(k, {"P", "S"}, [](const std::vector<uint64_t>&) { return true; });  // non-integer: rejected
    CHECK(tuner.GetConfigurationsCount(k) == 4);
    tuner.AddGenericConstraint(k, {"P", "S"}, [](const std::vector<const ktt::ParameterValue*>& v)
    {
        return std::get<uint64_t>(*v[0]) == 1 || std::get<std::string>(*v[1]) == "x";
    });
    CHECK(tuner.GetConfigurationsCount(k) == 3);
    ktt::Tuner::SetLoggingLevel(ktt::LoggingLevel::Info);
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        std::cerr << "usage: tuner_cpu_tests <test> [fixture-dir] [work-dir]" << std::endl;
        return 2;
    }

    if (argc > 2) fixtureDir = argv[2];
    if (argc > 3) workDir = argv[3];
    ktt::Tuner::SetLoggingLevel(ktt::LoggingLevel::Warning);

    const std::map<std::string, std::function<void()>> tests{
        {"prefix", TestPrefix},
        {"space", TestCoulombSpaceMatchesRecordedSpace},
        {"subgroup_order", TestSubgroupEnumerationOrder},
        {"groups", TestGroups},
        {"neighbours", TestNeighbours},
        {"deterministic", TestDeterministicSimulationFindsRecordedBest},
        {"random", TestRandomSearcherVisitsEachOnce},
        {"mcmc", TestMcmcSearcher},
        {"stop", TestStopConditions},
        {"json", TestJsonRoundTrip},
        {"errors", TestErrorConvention},
    };

    const auto it = tests.find(argv[1]);

    if (it == tests.end())
    {
        std::cerr << "unknown test " << argv[1] << std::endl;
        return 2;
    }

    it->second();
    return failures == 0 ? 0 : 1;
}
