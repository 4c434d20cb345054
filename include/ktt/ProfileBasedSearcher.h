// ProfileBasedSearcher.h -- KTT's profile-based searcher, natively, with an open counter model.
//
// KTT 2.1.0 ships this searcher as embedded Python (Scripts/ProfileBasedSearcher.py, installed by
// Tuner::SetProfileBasedSearcher, Source/Tuner.cpp:591-615; J. Filipovic et al., "Using hardware
// performance counters to speed up autotuning convergence on GPUs", JPDC 160, 2021).  Its steps:
//
//   1. run a batch of random configurations, keep the fastest valid one;
//   2. run that one again with profiling on and read its hardware counters;
//   3. analyse the counters into bottleneck scores in [0, 1] (DRAM, L2, L1, shared memory, local
//      memory, occupancy, SM activity, tail effect, too few threads, per-pipe instruction pressure,
//      issue utilisation);
//   4. turn the bottlenecks into a wanted direction and weight per counter (decrease DRAM sectors,
//      increase issue utilisation, ...);
//   5. take candidates -- unexplored neighbours of the best configuration (up to 2 differing
//      parameters) plus random ones -- predict each candidate's counters with a model of the tuning
//      space, and score it by how far its predicted counters move in the wanted directions relative
//      to the best configuration's prediction;
//   6. draw the next batch from the candidates with probability rising steeply with the score
//      (score^8), turn profiling off and repeat.
//
// KTT's model is a pickled scikit-learn ExtraTreesRegressor (Scripts/PrepareModels/
// generate_decision_tree_model.py).  Here the model is the same kind of forest stored as JSON
// (ktt_b200/profile_model.py trains and writes it from results with counters) and evaluated in C++;
// no Python runs inside the tuner.  The analysis follows KTT's branch for compute capability 7.0 and
// newer (the counter names of CUPTI's profiler API; older GPUs' event/metric names do not exist on
// B200).  One addition for B200, off by default: when the XU pipe (MUFU: reciprocal square root and
// the other special functions) is the limiting pipe, fewer XU instructions are wanted, which KTT
// leaves as a to-do (ProfileBasedSearcher.py:385).  On recorded B200 searches of this library's tile
// space it made convergence worse (it pulls toward more FMA-pipe rsqrts than the FMA pipe can take),
// so KTT's rules are the default.
#pragma once

#include <cstdint>
#include <map>
#include <random>
#include <string>
#include <vector>

#include <ktt/Searcher.h>

namespace ktt
{

class Tuner;

// A forest of regression trees predicting counters from tuning parameters.
class KTT_API CounterModel
{
public:
    CounterModel() = default;
    // Reads the JSON written by ktt_b200/profile_model.py.
    static CounterModel Load(const std::string& path);

    // Tuning parameters the model takes, in its order (KTT's metadata "tp").
    const std::vector<std::string>& GetParameters() const { return m_Parameters; }
    // Counters it predicts, in its order (KTT's metadata "pc").
    const std::vector<std::string>& GetCounters() const { return m_Counters; }
    // Compute capability (major + minor / 10) and SM count of the device the training data came from.
    double GetComputeCapability() const { return m_ComputeCapability; }
    uint32_t GetMultiprocessors() const { return m_Multiprocessors; }
    bool IsEmpty() const { return m_Trees.empty(); }

    // Mean over the trees of the leaf reached by the features (in GetParameters() order); a feature
    // goes left when float(x) <= threshold, as scikit-learn compares its float32 inputs.
    std::vector<double> Predict(const std::vector<double>& features) const;
    // The same for a configuration, its parameters looked up by name.
    std::vector<double> Predict(const KernelConfiguration& configuration) const;

private:
    struct Tree
    {
        std::vector<int32_t> feature;            // -1 on leaves
        std::vector<double> threshold;
        std::vector<int32_t> left;
        std::vector<int32_t> right;
        std::vector<std::vector<double>> value;  // per node; filled on leaves
    };

    std::vector<std::string> m_Parameters;
    std::vector<std::string> m_Counters;
    double m_ComputeCapability = 0.0;
    uint32_t m_Multiprocessors = 0;
    std::vector<Tree> m_Trees;
};

// The searcher's arithmetic, one function per step of Scripts/ProfileBasedSearcher.py.
namespace profiling
{

inline constexpr double ReactToInstructionBottlenecks = 0.7; // REACT_TO_INST_BOTTLENECKS (:41)
inline constexpr double Cutoff = -0.25;                      // CUTOFF (:42)
inline constexpr double Exponent = 8.0;                      // EXP (:40)
inline constexpr double MinimumScore = 0.0001;
inline constexpr uint64_t NeighbourDistance = 2;             // NEIGHBOR_DISTANCE (:43)
inline const std::string GlobalSizeCounter = "Global size";
inline const std::string LocalSizeCounter = "Local size";

// analyzeBottlenecks (:110-331), compute capability >= 7.0.  `names` / `values` hold the measured
// counters plus "Global size" (threads) and "Local size" (threads per block); `cores` is the
// device's FP32 lanes in total.  Returns bnDRAMRead, bnDRAMWrite, bnL2Read, bnL2Write, bnTex,
// bnLocal, bnSMRead, bnSMWrite, bnMPparal, bnGparal, bnTailEffect, bnThreads, bnSP, bnDP, bnSFU, bnCF,
// bnLDST, bnTexFu, bnInt, bnMisc, bnBconv, bnInstIssue.  Divisions by zero contribute zero.
KTT_API std::map<std::string, double> AnalyzeBottlenecks(const std::vector<std::string>& names,
    const std::vector<double>& values, const uint32_t multiprocessors, const uint32_t cores,
    const double reactToInstructions = ReactToInstructionBottlenecks);

// computeChanges (:333-418), compute capability >= 7.0: the wanted change of every counter of
// `counters` (negative = decrease), weighted by its bottleneck; counters the list lacks are skipped.
// With xuPipe, a limiting XU pipe asks for fewer XU instructions (smsp__inst_executed_pipe_xu.sum).
KTT_API std::vector<double> ComputeChanges(const std::map<std::string, double>& bottlenecks,
    const std::vector<std::string>& counters, const bool xuPipe = false,
    const double reactToInstructions = ReactToInstructionBottlenecks);

// scoreTuningConfigurationsPredictor (:490-566): score of each candidate from its predicted counters
// against the predicted counters of the current best configuration; `previous` zero marks a
// candidate already explored (its score stays zero).
KTT_API std::vector<double> ScoreCandidates(const std::vector<double>& changes, const std::vector<double>& actual,
    const std::vector<std::vector<double>>& predicted, const std::vector<double>& previous);

// weightedRandomSearchStep (:574-588) with the uniform draw u in [0, 1) given: index i with
// probability scores[i] / sum(scores); with all scores zero, floor(u * n).
KTT_API size_t WeightedRandomStep(const std::vector<double>& scores, const double u);

// FP32 lanes per SM (convertSM2Cores, :850-875, extended with compute capabilities 8.7 to 12.0; 64
// for unknown ones, as KTT defaults).
KTT_API uint32_t CoresPerMultiprocessor(const uint32_t ccMajor, const uint32_t ccMinor);

} // namespace profiling

class KTT_API ProfileBasedSearcher : public Searcher
{
public:
    // batchSize, neighbourSize and randomSize as Tuner::SetProfileBasedSearcher (defaults 5, 100, 10).
    // The searcher switches the tuner's profiling on for the run whose counters it needs and off again.
    ProfileBasedSearcher(Tuner& tuner, const CounterModel& model, const uint32_t batchSize = 5,
        const uint32_t neighbourSize = 100, const uint32_t randomSize = 10, const uint64_t seed = std::random_device{}());

    // The device the counters come from; by default the tuner's device, or the model's when the tuner
    // has none (replaying recorded results on a machine without a GPU).
    void SetDeviceProperties(const uint32_t ccMajor, const uint32_t ccMinor, const uint32_t multiprocessors);
    void SetXuPipeAnalysis(const bool flag) { m_XuPipe = flag; }

    void OnInitialize() override;
    void OnReset() override;
    bool CalculateNextConfiguration(const KernelResult& previousResult) override;
    KernelConfiguration GetCurrentConfiguration() const override;

    // How many batches were drawn from scored candidates so far.
    uint64_t GetScoredBatches() const { return m_ScoredBatches; }

private:
    Tuner& m_Tuner;
    CounterModel m_Model;
    uint32_t m_BatchSize;
    uint32_t m_NeighbourSize;
    uint32_t m_RandomSize;
    std::mt19937_64 m_Generator;
    std::uniform_real_distribution<double> m_Uniform;
    bool m_XuPipe = false;
    uint32_t m_CcMajor = 0;
    uint32_t m_CcMinor = 0;
    uint32_t m_Multiprocessors = 0;

    std::vector<KernelConfiguration> m_Batch;
    KernelConfiguration m_Current;
    KernelConfiguration m_BestConfiguration;
    bool m_HasBest = false;
    bool m_ProfilingRequested = false;
    Nanoseconds m_BestDuration = 0;
    uint64_t m_ScoredBatches = 0;

    void ResolveDevice();
    KernelConfiguration RandomUnexplored();
    std::vector<KernelConfiguration> UniqueConfigurations(const std::vector<KernelConfiguration>& list) const;
    void FillRandomBatch(const uint64_t size);
    void ScoreAndSelect(const KernelResult& profiled);
};

} // namespace ktt
