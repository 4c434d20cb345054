// GPU tests of the ktt:: surface: KTT-style host programs for the Coulomb path, run against the
// sm_100a kernels.  Driven by tests/test_tuner_gpu.py; each test is selected by name.
//
//   tuner_gpu_tests <test> <work-dir>
//
// The programs follow the structure of KTT's examples (Examples/CoulombSum3d/CoulombSum3d.cpp,
// Examples/CoulombSum2d/CoulombSum2d.cpp, Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp):
// the same kernel names, argument lists, tuning parameters, thread modifiers, constraints,
// reference kernels and validation settings.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <iostream>
#include <map>
#include <random>
#include <string>
#include <vector>

#include <Ktt.h>
#include <coulktt.h>

namespace
{

int failures = 0;
std::string workDir = "/tmp";

#define CHECK(cond)                                                                                      \
    do                                                                                                   \
    {                                                                                                    \
        if (!(cond))                                                                                     \
        {                                                                                                \
            std::cerr << __FILE__ << ":" << __LINE__ << ": check failed: " #cond << std::endl;           \
            ++failures;                                                                                  \
        }                                                                                                \
    } while (0)

struct Atoms
{
    std::vector<float> aos;  // x, y, z, w
    std::vector<float> x, y, z, w;
};

Atoms MakeAtoms(const int n, const float extent, const unsigned seed)
{
    Atoms a;
    std::mt19937 engine(seed);
    std::uniform_real_distribution<float> position(0.0f, extent);
    std::uniform_real_distribution<float> charge(-1.0f, 1.0f);

    for (int i = 0; i < n; ++i)
    {
        const float px = position(engine), py = position(engine), pz = position(engine), q = charge(engine);
        a.x.push_back(px);
        a.y.push_back(py);
        a.z.push_back(pz);
        a.w.push_back(q);
        a.aos.insert(a.aos.end(), {px, py, pz, q});
    }

    return a;
}

// FP64 map at the given points, the reference computation registered through SetReferenceComputation.
double PotentialFp64(const Atoms& atoms, const double gx, const double gy, const double gz)
{
    double v = 0.0;

    for (size_t j = 0; j < atoms.w.size(); ++j)
    {
        const double dx = gx - atoms.x[j], dy = gy - atoms.y[j], dz = gz - atoms.z[j];
        v += atoms.w[j] / std::sqrt(dx * dx + dy * dy + dz * dz);
    }

    return v;
}

// Adds the CUDA 3D example's tuning space (Examples/CoulombSum3d/CoulombSum3d.cpp:137-216).
void AddCoulomb3dSpace(ktt::Tuner& tuner, const ktt::KernelId kernel, const ktt::KernelDefinitionId definition)
{
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
    tuner.AddConstraint(kernel, {"INNER_UNROLL_FACTOR", "Z_ITERATIONS"}, [](const std::vector<uint64_t>& v) { return v.at(0) < v.at(1); });
    tuner.AddConstraint(kernel, {"WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"},
        [](const std::vector<uint64_t>& v) { return v.at(0) * v.at(1) >= 64; });
}

// The full KTT 3D space on the 256^3 grid with the reference kernel as validator (SideBySide, 0.01),
// and the launch geometry KTT's thread modifiers give each configuration compared with the sizes
// KTT recorded for the same configuration on the RTX 2080 Ti.
void TestCoulomb3dTuneWithReferenceKernel()
{
    const int gridSize = 256;
    const int atoms = 64;
    const float gridSpacing = 0.5f;
    const Atoms a = MakeAtoms(atoms, 20.0f, 7);
    std::vector<float> energyGrid(static_cast<size_t>(gridSize) * gridSize * gridSize, 0.0f);

    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    tuner.SetGlobalSizeType(ktt::GlobalSizeType::CUDA);
    tuner.SetTimeUnit(ktt::TimeUnit::Microseconds);
    tuner.SetCompilerOptions("-use_fast_math");
    const auto definition = tuner.AddKernelDefinition("directCoulombSum", "", ktt::DimensionVector(gridSize, gridSize, gridSize),
        ktt::DimensionVector());
    const auto referenceDefinition = tuner.AddKernelDefinition("directCoulombSumReference", "",
        ktt::DimensionVector(gridSize / 16, gridSize / 16, gridSize), ktt::DimensionVector(16, 16));
    const auto kernel = tuner.CreateSimpleKernel("CoulombSum", definition);
    const auto referenceKernel = tuner.CreateSimpleKernel("CoulombSumReference", referenceDefinition);
    const auto aiId = tuner.AddArgumentVector(a.aos, ktt::ArgumentAccessType::ReadOnly);
    const auto aixId = tuner.AddArgumentVector(a.x, ktt::ArgumentAccessType::ReadOnly);
    const auto aiyId = tuner.AddArgumentVector(a.y, ktt::ArgumentAccessType::ReadOnly);
    const auto aizId = tuner.AddArgumentVector(a.z, ktt::ArgumentAccessType::ReadOnly);
    const auto aiwId = tuner.AddArgumentVector(a.w, ktt::ArgumentAccessType::ReadOnly);
    const auto aId = tuner.AddArgumentScalar(atoms);
    const auto gsId = tuner.AddArgumentScalar(gridSpacing);
    const auto gridDim = tuner.AddArgumentScalar(gridSize);
    const auto gridId = tuner.AddArgumentVector(energyGrid, ktt::ArgumentAccessType::WriteOnly);
    AddCoulomb3dSpace(tuner, kernel, definition);
    tuner.SetArguments(definition, {aiId, aixId, aiyId, aizId, aiwId, aId, gsId, gridDim, gridId});
    tuner.SetArguments(referenceDefinition, {aiId, aId, gsId, gridDim, gridId});
    tuner.SetReferenceKernel(gridId, referenceKernel, ktt::KernelConfiguration());
    tuner.SetValidationMethod(ktt::ValidationMethod::SideBySideComparison, 0.01);
    tuner.SetSearcher(kernel, std::make_unique<ktt::DeterministicSearcher>());

    const auto results = tuner.Tune(kernel);
    CHECK(results.size() == 210);
    const auto recorded = tuner.LoadResults(workDir + "/coulomb_2080_ktt_format.json", ktt::OutputFormat::JSON);
    CHECK(recorded.size() == 210);
    size_t ok = 0, sizesMatched = 0;

    for (const auto& r : results)
    {
        ok += r.IsValid() ? 1 : 0;

        if (!r.IsValid())
        {
            std::cerr << "failed: " << r.GetConfiguration().GetString() << " status " << static_cast<int>(r.GetStatus()) << std::endl;
        }

        for (const auto& k : recorded)
        {
            if (k.GetConfiguration() == r.GetConfiguration() && !r.GetResults().empty())
            {
                const bool same = k.GetResults()[0].GetGlobalSize() == r.GetResults()[0].GetGlobalSize()
                    && k.GetResults()[0].GetLocalSize() == r.GetResults()[0].GetLocalSize();
                sizesMatched += same ? 1 : 0;

                if (!same)
                {
                    std::cerr << "size mismatch " << r.GetConfiguration().GetString() << ": "
                              << r.GetResults()[0].GetGlobalSize().GetString() << " vs "
                              << k.GetResults()[0].GetGlobalSize().GetString() << std::endl;
                }
            }
        }
    }

    CHECK(ok == 210);
    CHECK(sizesMatched == 210);
    tuner.SaveResults(results, workDir + "/CoulombSumOutput", ktt::OutputFormat::JSON);
    const auto best = tuner.GetBestConfiguration(kernel);
    CHECK(best.IsValid());
    std::cout << "best configuration: " << best.GetString() << std::endl;
}

// FP64 reference computation (SetReferenceComputation), relative side-by-side validation, and Run()
// with an output descriptor, on a map with a non-zero B200-specific configuration.
void TestCoulomb3dReferenceComputationAndRun()
{
    const int gridSize = 48;
    const int atoms = 700;
    const float gridSpacing = 0.5f;
    const Atoms a = MakeAtoms(atoms, 24.0f, 11);
    std::vector<float> energyGrid(static_cast<size_t>(gridSize) * gridSize * gridSize, 0.0f);

    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    tuner.SetGlobalSizeType(ktt::GlobalSizeType::CUDA);
    const auto definition = tuner.AddKernelDefinition("directCoulombSum", "", ktt::DimensionVector(gridSize, gridSize, gridSize),
        ktt::DimensionVector());
    const auto kernel = tuner.CreateSimpleKernel("CoulombSum", definition);
    const auto aiId = tuner.AddArgumentVector(a.aos, ktt::ArgumentAccessType::ReadOnly);
    const auto aixId = tuner.AddArgumentVector(a.x, ktt::ArgumentAccessType::ReadOnly);
    const auto aiyId = tuner.AddArgumentVector(a.y, ktt::ArgumentAccessType::ReadOnly);
    const auto aizId = tuner.AddArgumentVector(a.z, ktt::ArgumentAccessType::ReadOnly);
    const auto aiwId = tuner.AddArgumentVector(a.w, ktt::ArgumentAccessType::ReadOnly);
    const auto aId = tuner.AddArgumentScalar(atoms);
    const auto gsId = tuner.AddArgumentScalar(gridSpacing);
    const auto gridDim = tuner.AddArgumentScalar(gridSize);
    const auto gridId = tuner.AddArgumentVector(energyGrid, ktt::ArgumentAccessType::WriteOnly);
    tuner.SetArguments(definition, {aiId, aixId, aiyId, aizId, aiwId, aId, gsId, gridDim, gridId});
    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_X", std::vector<uint64_t>{32});
    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_Y", std::vector<uint64_t>{4});
    tuner.AddParameter(kernel, "Z_ITERATIONS", std::vector<uint64_t>{8, 16});
    tuner.AddParameter(kernel, "X_POINTS", std::vector<uint64_t>{1, 2, 4});
    tuner.AddParameter(kernel, "PRECISION", std::vector<uint64_t>{0, 2});
    tuner.AddParameter(kernel, "RSQRT_SOFT", std::vector<uint64_t>{0, 2});

    tuner.SetReferenceComputation(gridId, [&](void* buffer)
    {
        float* out = static_cast<float*>(buffer);

        for (int z = 0; z < gridSize; ++z)
            for (int y = 0; y < gridSize; ++y)
                for (int x = 0; x < gridSize; ++x)
                    out[(static_cast<size_t>(z) * gridSize + y) * gridSize + x] = static_cast<float>(
                        PotentialFp64(a, gridSpacing * x, gridSpacing * y, gridSpacing * z));
    });
    tuner.SetValidationMethod(ktt::ValidationMethod::SideBySideRelativeComparison, 1e-4);
    const auto results = tuner.Tune(kernel);
    CHECK(!results.empty());
    size_t ok = 0, notCompiled = 0;

    for (const auto& r : results)
    {
        ok += r.IsValid() ? 1 : 0;
        // a configuration with no ahead-of-time compiled variant reports CompilationFailed, as a
        // configuration whose source fails to compile does in KTT; it must never fail validation
        notCompiled += r.GetStatus() == ktt::ResultStatus::CompilationFailed ? 1 : 0;
        CHECK(r.GetStatus() == ktt::ResultStatus::Ok || r.GetStatus() == ktt::ResultStatus::CompilationFailed);
    }

    CHECK(results.size() == 2 * 3 * 2 * 2);
    CHECK(ok + notCompiled == results.size());
    CHECK(ok >= 20);

    // Run a chosen configuration and download the map through an output descriptor.
    const auto configuration = tuner.CreateConfiguration(kernel, {{"Z_ITERATIONS", uint64_t{8}}, {"X_POINTS", uint64_t{2}},
        {"RSQRT_SOFT", uint64_t{2}}});
    std::vector<float> map(energyGrid.size(), -1.0f);
    const auto run = tuner.Run(kernel, configuration, {ktt::BufferOutputDescriptor(gridId, map.data())});
    CHECK(run.IsValid());
    CHECK(run.GetKernelDuration() > 0);
    double maxRel = 0.0, maxRef = 0.0;

    for (int i = 0; i < 500; ++i)
    {
        const size_t p = (static_cast<size_t>(i) * 2654435761u) % map.size();
        const int x = static_cast<int>(p % gridSize), y = static_cast<int>((p / gridSize) % gridSize),
                  z = static_cast<int>(p / (static_cast<size_t>(gridSize) * gridSize));
        const double ref = PotentialFp64(a, gridSpacing * x, gridSpacing * y, gridSpacing * z);
        maxRef = std::max(maxRef, std::fabs(ref));
        maxRel = std::max(maxRel, std::fabs(map[p] - ref));
    }

    CHECK(maxRel / maxRef < 1e-5);
}

// The 2D example's space (Examples/CoulombSum2d/CoulombSum2d.cpp:42-136): OpenCL-style global size
// 512 x 512, OUTER_UNROLL_FACTOR dividing the x size, random searcher, 2D reference kernel.
void TestCoulomb2dRandomSearch()
{
    const ktt::DimensionVector ndRange(512, 512);
    const int numberOfAtoms = 4000;
    const float gridSpacing = 0.5f;
    Atoms a = MakeAtoms(numberOfAtoms, 40.0f, 3);

    for (int i = 0; i < numberOfAtoms; ++i)
    {
        // the 2D kernels read the squared z distance to the slice from the atom's z field
        const float dz = 8.0f - a.z[i];
        a.z[i] = dz * dz;
        a.aos[4 * i + 2] = a.z[i];
    }

    std::vector<float> energyGrid(ndRange.GetTotalSize(), 0.0f);
    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    const auto definition = tuner.AddKernelDefinition("directCoulombSum", "", ndRange, ktt::DimensionVector());
    const auto kernel = tuner.CreateSimpleKernel("CoulombSum", definition);
    const auto referenceDefinition = tuner.AddKernelDefinition("directCoulombSumReference", "", ndRange, ktt::DimensionVector(16, 16));
    const auto referenceKernel = tuner.CreateSimpleKernel("CoulombSumReference", referenceDefinition);
    tuner.AddParameter(kernel, "INNER_UNROLL_FACTOR", std::vector<uint64_t>{0, 1, 2, 4, 8, 16, 32});
    tuner.AddParameter(kernel, "USE_CONSTANT_MEMORY", std::vector<uint64_t>{0, 1});
    tuner.AddParameter(kernel, "VECTOR_TYPE", std::vector<uint64_t>{1, 2, 4, 8});
    tuner.AddParameter(kernel, "USE_SOA", std::vector<uint64_t>{0, 1, 2});
    tuner.AddConstraint(kernel, {"VECTOR_TYPE", "USE_SOA"}, [](const std::vector<uint64_t>& v) { return v[0] > 1 || v[1] != 2; });
    tuner.AddParameter(kernel, "OUTER_UNROLL_FACTOR", std::vector<uint64_t>{1, 2, 4, 8});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::X, "OUTER_UNROLL_FACTOR",
        ktt::ModifierAction::Divide);
    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_X", std::vector<uint64_t>{4, 8, 16, 32});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::X, "WORK_GROUP_SIZE_X",
        ktt::ModifierAction::Multiply);
    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_Y", std::vector<uint64_t>{1, 2, 4, 8, 16, 32});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
        ktt::ModifierAction::Multiply);
    const auto atomInfoId = tuner.AddArgumentVector(a.aos, ktt::ArgumentAccessType::ReadOnly);
    const auto xId = tuner.AddArgumentVector(a.x, ktt::ArgumentAccessType::ReadOnly);
    const auto yId = tuner.AddArgumentVector(a.y, ktt::ArgumentAccessType::ReadOnly);
    const auto zId = tuner.AddArgumentVector(a.z, ktt::ArgumentAccessType::ReadOnly);
    const auto wId = tuner.AddArgumentVector(a.w, ktt::ArgumentAccessType::ReadOnly);
    const auto nId = tuner.AddArgumentScalar(numberOfAtoms);
    const auto hId = tuner.AddArgumentScalar(gridSpacing);
    const auto gridId = tuner.AddArgumentVector(energyGrid, ktt::ArgumentAccessType::ReadWrite);
    tuner.SetArguments(definition, {atomInfoId, xId, yId, zId, wId, nId, hId, gridId});
    tuner.SetArguments(referenceDefinition, {atomInfoId, nId, hId, gridId});
    tuner.SetSearcher(kernel, std::make_unique<ktt::RandomSearcher>());
    tuner.SetValidationMethod(ktt::ValidationMethod::SideBySideComparison, 0.01);
    tuner.SetReferenceKernel(gridId, referenceKernel, ktt::KernelConfiguration());
    const auto results = tuner.Tune(kernel, std::make_unique<ktt::ConfigurationCount>(40));
    CHECK(results.size() == 40);
    size_t ok = 0, limits = 0;

    for (const auto& r : results)
    {
        ok += r.IsValid() ? 1 : 0;
        limits += r.GetStatus() == ktt::ResultStatus::DeviceLimitsExceeded ? 1 : 0;
        CHECK(r.GetStatus() != ktt::ResultStatus::ValidationFailed);
        CHECK(r.GetStatus() != ktt::ResultStatus::ComputationFailed);
    }

    CHECK(ok > 0);
    CHECK(ok + limits == results.size());
}

// A custom launcher (Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp:146-184): the 3D map
// as one 2D-slice launch per z plane, the launcher recomputing dz^2 on the host and replacing the
// atom buffer and the zIndex scalar before each launch; validated against the 3D reference kernel.
void TestIterativeLauncher()
{
    const int gridSize = 40;
    const int atoms = 300;
    const float gridSpacing = 0.5f;
    const Atoms a = MakeAtoms(atoms, 20.0f, 5);
    std::vector<float> atomInfoPrecomp = a.aos;
    std::vector<float> atomInfoZ2(atoms);
    std::vector<float> energyGrid(static_cast<size_t>(gridSize) * gridSize * gridSize, 0.0f);
    int zIndex = 0;

    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    const auto definition = tuner.AddKernelDefinition("directCoulombSum", "", ktt::DimensionVector(gridSize, gridSize),
        ktt::DimensionVector());
    const auto kernel = tuner.CreateSimpleKernel("CoulombSum", definition);
    const auto referenceDefinition = tuner.AddKernelDefinition("directCoulombSumReference", "",
        ktt::DimensionVector(gridSize, gridSize, gridSize), ktt::DimensionVector());
    const auto referenceKernel = tuner.CreateSimpleKernel("CoulombSumReference", referenceDefinition);
    const auto atomInfoId = tuner.AddArgumentVector(a.aos, ktt::ArgumentAccessType::ReadOnly);
    const auto precompId = tuner.AddArgumentVector(atomInfoPrecomp, ktt::ArgumentAccessType::ReadOnly);
    const auto xId = tuner.AddArgumentVector(a.x, ktt::ArgumentAccessType::ReadOnly);
    const auto yId = tuner.AddArgumentVector(a.y, ktt::ArgumentAccessType::ReadOnly);
    const auto z2Id = tuner.AddArgumentVector(atomInfoZ2, ktt::ArgumentAccessType::ReadOnly);
    const auto wId = tuner.AddArgumentVector(a.w, ktt::ArgumentAccessType::ReadOnly);
    const auto nId = tuner.AddArgumentScalar(atoms);
    const auto hId = tuner.AddArgumentScalar(gridSpacing);
    const auto zId = tuner.AddArgumentScalar(zIndex);
    const auto gridId = tuner.AddArgumentVector(energyGrid, ktt::ArgumentAccessType::ReadWrite);
    tuner.SetArguments(definition, {precompId, xId, yId, z2Id, wId, nId, hId, zId, gridId});
    tuner.SetArguments(referenceDefinition, {atomInfoId, nId, hId, gridId});
    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_X", std::vector<uint64_t>{8, 16, 32});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::X, "WORK_GROUP_SIZE_X",
        ktt::ModifierAction::Multiply);
    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_Y", std::vector<uint64_t>{2, 4});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
        ktt::ModifierAction::Multiply);
    tuner.AddParameter(kernel, "USE_SOA", std::vector<uint64_t>{0, 1});
    tuner.AddParameter(kernel, "OUTER_UNROLL_FACTOR", std::vector<uint64_t>{1, 2, 4});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::X, "OUTER_UNROLL_FACTOR",
        ktt::ModifierAction::Divide);
    tuner.SetValidationMethod(ktt::ValidationMethod::SideBySideComparison, 0.01);
    tuner.SetReferenceKernel(gridId, referenceKernel, ktt::KernelConfiguration());
    size_t launches = 0;

    tuner.SetLauncher(kernel, [&](ktt::ComputeInterface& interface) mutable
    {
        ktt::DimensionVector globalSize = interface.GetCurrentGlobalSize(definition);
        const ktt::DimensionVector& localSize = interface.GetCurrentLocalSize(definition);
        const auto& pairs = interface.GetCurrentConfiguration().GetPairs();
        globalSize.SetSizeZ(1);

        for (int i = 0; i < gridSize; ++i)
        {
            const float z = gridSpacing * static_cast<float>(i);

            if (ktt::ParameterPair::GetParameterValue<uint64_t>(pairs, "USE_SOA") == 0)
            {
                for (int j = 0; j < atoms; ++j)
                {
                    atomInfoPrecomp[4 * j + 2] = (z - a.z[j]) * (z - a.z[j]);
                }

                interface.UpdateBuffer(precompId, atomInfoPrecomp.data());
            }
            else
            {
                for (int j = 0; j < atoms; ++j)
                {
                    atomInfoZ2[j] = (z - a.z[j]) * (z - a.z[j]);
                }

                interface.UpdateBuffer(z2Id, atomInfoZ2.data());
            }

            interface.UpdateScalarArgument(zId, &i);
            interface.RunKernel(definition, globalSize, localSize);
            ++launches;
        }
    });

    const auto results = tuner.Tune(kernel);
    CHECK(results.size() == 3 * 2 * 2 * 3);

    for (const auto& r : results)
    {
        CHECK(r.IsValid());
        CHECK(r.GetResults().size() == 1);
        CHECK(r.GetKernelDuration() > 0);
    }

    CHECK(launches == results.size() * gridSize);
}

// Device buffers owned by the caller (AddArgumentVector with a ComputeBuffer): the tuner neither
// copies nor frees them, and results land in the caller's memory.
void TestUserDeviceBuffers()
{
    const int gridSize = 32;
    const int atoms = 100;
    const Atoms a = MakeAtoms(atoms, 16.0f, 9);
    coul_ctx* ctx = nullptr;
    CHECK(coul_ctx_create(0, &ctx) == COUL_OK);
    void* dAtoms = nullptr;
    void* dGrid = nullptr;
    const size_t gridBytes = sizeof(float) * gridSize * gridSize * gridSize;
    CHECK(coul_buffer_alloc(ctx, a.aos.size() * sizeof(float), &dAtoms) == COUL_OK);
    CHECK(coul_buffer_alloc(ctx, gridBytes, &dGrid) == COUL_OK);
    CHECK(coul_buffer_upload(ctx, dAtoms, a.aos.data(), a.aos.size() * sizeof(float)) == COUL_OK);
    CHECK(coul_buffer_memset(ctx, dGrid, 0, gridBytes) == COUL_OK);
    CHECK(coul_synchronize(ctx) == COUL_OK);

    {
        ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
        const auto definition = tuner.AddKernelDefinition("directCoulombSumReference", "",
            ktt::DimensionVector(gridSize / 16, gridSize / 16, gridSize), ktt::DimensionVector(16, 16));
        const auto kernel = tuner.CreateSimpleKernel("Reference", definition);
        const auto atomsId = tuner.AddArgumentVector<float>(dAtoms, a.aos.size() * sizeof(float), ktt::ArgumentAccessType::ReadOnly);
        const auto gridId = tuner.AddArgumentVector<float>(dGrid, gridBytes, ktt::ArgumentAccessType::ReadWrite);
        const auto nId = tuner.AddArgumentScalar(atoms);
        const auto hId = tuner.AddArgumentScalar(0.5f);
        const auto gId = tuner.AddArgumentScalar(gridSize);
        tuner.SetArguments(definition, {atomsId, nId, hId, gId, gridId});
        const auto r = tuner.Run(kernel, ktt::KernelConfiguration(), {});
        CHECK(r.IsValid());
    }

    std::vector<float> map(gridSize * gridSize * gridSize);
    CHECK(coul_buffer_download(ctx, map.data(), dGrid, gridBytes) == COUL_OK);
    const double ref = PotentialFp64(a, 0.5 * 3, 0.5 * 5, 0.5 * 7);
    CHECK(std::fabs(map[(7 * gridSize + 5) * gridSize + 3] - ref) < 1e-4 * std::max(1.0, std::fabs(ref)));
    CHECK(coul_buffer_free(ctx, dAtoms) == COUL_OK);
    CHECK(coul_buffer_free(ctx, dGrid) == COUL_OK);
    coul_ctx_destroy(ctx);
}

// KTT's Nbody example (Examples/Nbody/Nbody.cpp:62-240) on 16,384 bodies: its parameters, thread
// modifiers, constraints and argument lists, the tuned kernel validated against the reference
// kernel (SideBySide 0.001) over a random sample of the space; configurations with no compiled
// counterpart end as CompilationFailed / DeviceLimitsExceeded, the rest must validate.
void TestNbodyExample()
{
    const int n = 16 * 1024;
    std::mt19937 engine(42);
    std::uniform_real_distribution<float> dist(0.0f, 20.0f);
    std::vector<float> info(4 * n), px(n), py(n), pz(n), mass(n), newInfo(4 * n, 0.0f);
    std::vector<float> vel(4 * n), vx(n), vy(n), vz(n), newVel(4 * n, 0.0f);

    for (int i = 0; i < n; ++i)
    {
        px[i] = dist(engine);
        py[i] = dist(engine);
        pz[i] = dist(engine);
        mass[i] = dist(engine);
        vx[i] = dist(engine);
        vy[i] = dist(engine);
        vz[i] = dist(engine);
        info[4 * i] = px[i];
        info[4 * i + 1] = py[i];
        info[4 * i + 2] = pz[i];
        info[4 * i + 3] = mass[i];
        vel[4 * i] = vx[i];
        vel[4 * i + 1] = vy[i];
        vel[4 * i + 2] = vz[i];
        vel[4 * i + 3] = 0.0f;
    }

    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    tuner.SetGlobalSizeType(ktt::GlobalSizeType::OpenCL);
    tuner.SetCompilerOptions("-use_fast_math");
    const auto definition = tuner.AddKernelDefinitionFromFile("nbody_kernel", "Nbody.cu", ktt::DimensionVector(n, 1),
        ktt::DimensionVector(1, 1));
    const auto referenceDefinition = tuner.AddKernelDefinitionFromFile("nbody_kernel_reference", "NbodyReference.cu",
        ktt::DimensionVector(n, 1), ktt::DimensionVector(64));
    const auto kernel = tuner.CreateSimpleKernel("Nbody", definition);
    const auto referenceKernel = tuner.CreateSimpleKernel("NbodyReference", referenceDefinition);

    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_X", std::vector<uint64_t>{16, 32, 64, 128, 256, 512});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::X, "WORK_GROUP_SIZE_X",
        ktt::ModifierAction::Multiply);
    tuner.AddParameter(kernel, "WORK_GROUP_SIZE_Y", std::vector<uint64_t>{1, 2, 4, 8, 16});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
        ktt::ModifierAction::Multiply);
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
        ktt::ModifierAction::Multiply);
    tuner.AddParameter(kernel, "OUTER_UNROLL_FACTOR", std::vector<uint64_t>{1, 2, 4, 8});
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::X, "OUTER_UNROLL_FACTOR",
        ktt::ModifierAction::Divide);
    tuner.AddParameter(kernel, "INNER_UNROLL_FACTOR1", std::vector<uint64_t>{0, 1, 2, 4, 8, 16, 32});
    tuner.AddParameter(kernel, "INNER_UNROLL_FACTOR2", std::vector<uint64_t>{0, 1, 2, 4, 8, 16, 32});
    tuner.AddParameter(kernel, "USE_SOA", std::vector<uint64_t>{0, 1});
    tuner.AddParameter(kernel, "LOCAL_MEM", std::vector<uint64_t>{0, 1});
    tuner.AddParameter(kernel, "USE_CONSTANT_MEMORY", std::vector<uint64_t>{0});
    tuner.AddParameter(kernel, "VECTOR_TYPE", std::vector<uint64_t>{1, 2, 4});

    const auto infoId = tuner.AddArgumentVector(info, ktt::ArgumentAccessType::ReadOnly);
    const auto pxId = tuner.AddArgumentVector(px, ktt::ArgumentAccessType::ReadOnly);
    const auto pyId = tuner.AddArgumentVector(py, ktt::ArgumentAccessType::ReadOnly);
    const auto pzId = tuner.AddArgumentVector(pz, ktt::ArgumentAccessType::ReadOnly);
    const auto massId = tuner.AddArgumentVector(mass, ktt::ArgumentAccessType::ReadOnly);
    const auto newInfoId = tuner.AddArgumentVector(newInfo, ktt::ArgumentAccessType::WriteOnly);
    const auto velId = tuner.AddArgumentVector(vel, ktt::ArgumentAccessType::ReadOnly);
    const auto vxId = tuner.AddArgumentVector(vx, ktt::ArgumentAccessType::ReadOnly);
    const auto vyId = tuner.AddArgumentVector(vy, ktt::ArgumentAccessType::ReadOnly);
    const auto vzId = tuner.AddArgumentVector(vz, ktt::ArgumentAccessType::ReadOnly);
    const auto newVelId = tuner.AddArgumentVector(newVel, ktt::ArgumentAccessType::WriteOnly);
    const auto dtId = tuner.AddArgumentScalar(0.001f);
    const auto dampingId = tuner.AddArgumentScalar(0.5f);
    const auto epsId = tuner.AddArgumentScalar(0.1f * 0.1f);
    const auto nId = tuner.AddArgumentScalar(n);

    tuner.AddConstraint(kernel, {"INNER_UNROLL_FACTOR2", "OUTER_UNROLL_FACTOR"},
        [](const std::vector<uint64_t>& v) { return v.at(0) <= v.at(1); });
    tuner.AddConstraint(kernel, {"INNER_UNROLL_FACTOR1", "INNER_UNROLL_FACTOR2"},
        [](const std::vector<uint64_t>& v) { return v.at(0) * v.at(1) <= 256; });
    tuner.AddConstraint(kernel, {"VECTOR_TYPE", "USE_SOA"},
        [](const std::vector<uint64_t>& v) { return (v.at(0) == 1 && v.at(1) == 0) || v.at(1) == 1; });
    tuner.AddConstraint(kernel, {"WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"},
        [](const std::vector<uint64_t>& v) { return v.at(0) * v.at(1) >= 64 && v.at(0) * v.at(1) <= 1024; });

    tuner.SetArguments(definition, {dtId, infoId, pxId, pyId, pzId, massId, newInfoId, velId, vxId, vyId, vzId, newVelId,
        dampingId, epsId, nId});
    tuner.SetArguments(referenceDefinition, {dtId, infoId, newInfoId, velId, newVelId, dampingId, epsId});
    tuner.SetValidationMethod(ktt::ValidationMethod::SideBySideComparison, 0.001);
    tuner.SetReferenceKernel(newVelId, referenceKernel, ktt::KernelConfiguration());
    tuner.SetReferenceKernel(newInfoId, referenceKernel, ktt::KernelConfiguration());
    tuner.SetSearcher(kernel, std::make_unique<ktt::RandomSearcher>());

    const auto results = tuner.Tune(kernel, std::make_unique<ktt::ConfigurationCount>(40));
    CHECK(results.size() == 40);
    int ok = 0;

    for (const auto& r : results)
    {
        const auto s = r.GetStatus();
        CHECK(s == ktt::ResultStatus::Ok || s == ktt::ResultStatus::CompilationFailed
            || s == ktt::ResultStatus::DeviceLimitsExceeded);
        ok += s == ktt::ResultStatus::Ok ? 1 : 0;
    }

    CHECK(ok >= 10);
    std::cout << "nbody: " << ok << " of " << results.size() << " configurations validated" << std::endl;
}

// Counters and KTT's profile-based searcher through the C++ surface: a profiled Run of one
// configuration of this library's directCoulombSum tile space (64^3 map, 2,048 atoms) carries KTT's
// default counters through SaveResults / LoadResults; then SetProfileBasedSearcher with the counter
// model trained (ktt_b200/profile_model.py) from the B200 recording of the same space
// (<work-dir>/b200_64.model.json) runs a search that reruns each batch's fastest with profiling.
void TestProfileBasedSearcher()
{
    const int grid = 64;
    const int n = 2048;
    const float h = 0.5f;
    const Atoms atoms = MakeAtoms(n, grid * h, 3);
    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    tuner.SetGlobalSizeType(ktt::GlobalSizeType::CUDA);
    const auto definition = tuner.AddKernelDefinition("directCoulombSum", "", ktt::DimensionVector(grid, grid, grid),
        ktt::DimensionVector());
    const auto kernel = tuner.CreateSimpleKernel("CoulombSum", definition);
    const std::vector<std::pair<std::string, std::vector<uint64_t>>> space{{"WORK_GROUP_SIZE_X", {16, 32, 64, 128}},
        {"WORK_GROUP_SIZE_Y", {1, 2, 4, 8}}, {"Z_ITERATIONS", {4, 8, 16}}, {"X_POINTS", {1, 2, 4}},
        {"INNER_UNROLL_FACTOR", {0, 2, 4}}, {"RSQRT_SOFT", {0, 1, 2, 3}}, {"PRECISION", {0}}};

    for (const auto& [name, values] : space)
    {
        tuner.AddParameter(kernel, name, values);
    }

    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::X, "WORK_GROUP_SIZE_X",
        ktt::ModifierAction::Multiply);
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Local, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
        ktt::ModifierAction::Multiply);
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::X, "WORK_GROUP_SIZE_X",
        ktt::ModifierAction::DivideCeil);
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::Y, "WORK_GROUP_SIZE_Y",
        ktt::ModifierAction::DivideCeil);
    tuner.AddThreadModifier(kernel, {definition}, ktt::ModifierType::Global, ktt::ModifierDimension::Z, "Z_ITERATIONS",
        ktt::ModifierAction::DivideCeil);
    tuner.AddConstraint(kernel, {"WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"},
        [](const std::vector<uint64_t>& v) { return v[0] * v[1] >= 32 && v[0] * v[1] <= 256; });
    // only the compiled variants
    tuner.AddConstraint(kernel, {"WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y", "Z_ITERATIONS", "X_POINTS",
        "INNER_UNROLL_FACTOR", "RSQRT_SOFT"}, [](const std::vector<uint64_t>& v)
    {
        coul_tune t;
        coul_tune_default(&t);
        t.block_x = static_cast<int>(v[0]);
        t.block_y = static_cast<int>(v[1]);
        t.z_iterations = static_cast<int>(v[2]);
        t.x_points = static_cast<int>(v[3]);
        t.unroll = v[4] <= 1 ? 1 : (v[4] < 4 ? 2 : 4);
        t.rsqrt_soft = static_cast<int>(v[5]);
        return coul_tune_supported(&t) == COUL_OK;
    });

    std::vector<float> energy(static_cast<size_t>(grid) * grid * grid, 0.0f);
    const auto aos = tuner.AddArgumentVector(atoms.aos, ktt::ArgumentAccessType::ReadOnly);
    const auto xs = tuner.AddArgumentVector(atoms.x, ktt::ArgumentAccessType::ReadOnly);
    const auto ys = tuner.AddArgumentVector(atoms.y, ktt::ArgumentAccessType::ReadOnly);
    const auto zs = tuner.AddArgumentVector(atoms.z, ktt::ArgumentAccessType::ReadOnly);
    const auto ws = tuner.AddArgumentVector(atoms.w, ktt::ArgumentAccessType::ReadOnly);
    const auto count = tuner.AddArgumentScalar(n);
    const auto spacing = tuner.AddArgumentScalar(h);
    const auto size = tuner.AddArgumentScalar(grid);
    const auto out = tuner.AddArgumentVector(energy, ktt::ArgumentAccessType::WriteOnly);
    tuner.SetArguments(definition, {aos, xs, ys, zs, ws, count, spacing, size, out});

    // one profiled run
    const auto configuration = tuner.CreateConfiguration(kernel, {{"WORK_GROUP_SIZE_X", uint64_t{32}},
        {"WORK_GROUP_SIZE_Y", uint64_t{4}}, {"Z_ITERATIONS", uint64_t{8}}, {"X_POINTS", uint64_t{2}},
        {"INNER_UNROLL_FACTOR", uint64_t{2}}, {"RSQRT_SOFT", uint64_t{2}}});
    tuner.SetProfiling(true);
    const auto profiled = tuner.Run(kernel, configuration, {});
    tuner.SetProfiling(false);
    CHECK(profiled.IsValid());
    CHECK(!profiled.GetResults().empty() && profiled.GetResults()[0].HasProfilingData());

    if (profiled.GetResults().empty() || !profiled.GetResults()[0].HasProfilingData())
    {
        return;
    }

    const auto& data = profiled.GetResults()[0].GetProfilingData();
    CHECK(data.IsValid() && data.GetCounters().size() >= 30);
    CHECK(data.HasCounter("smsp__inst_executed.sum") && data.GetCounter("smsp__inst_executed.sum").GetValueDouble() > 0.0);
    CHECK(!data.HasCounter("smsp__inst_executed_pipe_fp16.sum"));  // not offered by GB100
    CHECK(profiled.GetProfilingRunsOverhead() > 0);
    const std::string file = workDir + "/profiled_run";
    tuner.SaveResults({profiled}, file, ktt::OutputFormat::JSON);
    const auto loaded = tuner.LoadResults(file + ".json", ktt::OutputFormat::JSON);
    CHECK(loaded.size() == 1 && loaded[0].GetResults()[0].HasProfilingData());
    CHECK(loaded.size() == 1 && loaded[0].GetResults()[0].GetProfilingData().GetCounters().size() == data.GetCounters().size());

    // the profile-based searcher with the B200 model of this space
    tuner.SetProfileBasedSearcher(kernel, workDir + "/b200_64.model.json", true, 5, 100, 10);
    const auto results = tuner.Tune(kernel, std::make_unique<ktt::ConfigurationCount>(18));
    CHECK(results.size() == 18);
    std::vector<size_t> rerun;

    for (size_t i = 0; i < results.size(); ++i)
    {
        CHECK(results[i].IsValid());

        if (!results[i].GetResults().empty() && results[i].GetResults()[0].HasProfilingData())
        {
            rerun.push_back(i);
        }
    }

    // batches of 5, each followed by a profiled rerun of its fastest
    CHECK((rerun == std::vector<size_t>{5, 11, 17}));
    CHECK(!tuner.GetProfiling());
    std::cout << "profile-based: " << results.size() << " runs, profiled reruns at 5, 11, 17" << std::endl;
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        std::cerr << "usage: tuner_gpu_tests <test> [work-dir]" << std::endl;
        return 2;
    }

    if (argc > 2) workDir = argv[2];
    ktt::Tuner::SetLoggingLevel(ktt::LoggingLevel::Warning);
    const std::map<std::string, std::function<void()>> tests{
        {"coulomb3d_tune", TestCoulomb3dTuneWithReferenceKernel},
        {"coulomb3d_reference_computation", TestCoulomb3dReferenceComputationAndRun},
        {"coulomb2d_random", TestCoulomb2dRandomSearch},
        {"iterative_launcher", TestIterativeLauncher},
        {"user_buffers", TestUserDeviceBuffers},
        {"nbody_example", TestNbodyExample},
        {"profile_based", TestProfileBasedSearcher},
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
