// ProfileBasedSearcher.cpp -- see include/ktt/ProfileBasedSearcher.h.  Each function below restates
// one step of KTT 2.1.0 Scripts/ProfileBasedSearcher.py (cited by line); the searcher class follows
// PyProfilingSearcher (:616-848).
#include <algorithm>
#include <cmath>
#include <fstream>
#include <limits>
#include <numeric>
#include <set>
#include <sstream>
#include <stdexcept>

#include <ktt/ProfileBasedSearcher.h>
#include <ktt/Tuner.h>

#include "Json.h"
#include "Logger.h"

namespace ktt
{

// ---- counter model --------------------------------------------------------------------------

namespace
{

std::vector<std::string> Strings(const json::Json* list, const char* what)
{
    if (list == nullptr || list->kind != json::Json::Kind::Array)
    {
        throw std::runtime_error(std::string("counter model lacks the list ") + what);
    }

    std::vector<std::string> result;

    for (const auto& item : list->items)
    {
        result.push_back(item.text);
    }

    return result;
}

double NumberOf(const json::Json& j)
{
    return j.integral ? static_cast<double>(j.integer) : j.number;
}

template <typename T>
std::vector<T> Numbers(const json::Json* list, const char* what)
{
    if (list == nullptr || list->kind != json::Json::Kind::Array)
    {
        throw std::runtime_error(std::string("counter model tree lacks ") + what);
    }

    std::vector<T> result;
    result.reserve(list->items.size());

    for (const auto& item : list->items)
    {
        result.push_back(static_cast<T>(NumberOf(item)));
    }

    return result;
}

double ParameterAsDouble(const ParameterValue& value)
{
    if (std::holds_alternative<int64_t>(value)) return static_cast<double>(std::get<int64_t>(value));
    if (std::holds_alternative<uint64_t>(value)) return static_cast<double>(std::get<uint64_t>(value));
    if (std::holds_alternative<double>(value)) return std::get<double>(value);
    if (std::holds_alternative<bool>(value)) return std::get<bool>(value) ? 1.0 : 0.0;
    throw std::runtime_error("string-valued parameters cannot be model features");
}

} // namespace

CounterModel CounterModel::Load(const std::string& path)
{
    std::ifstream file(path);

    if (!file)
    {
        throw std::runtime_error("Unable to open counter model " + path);
    }

    std::stringstream text;
    text << file.rdbuf();
    const json::Json root = json::Parser(text.str()).Parse();

    if (root.StringOr("format", "") != "ktt_b200.counter_forest/1")
    {
        throw std::runtime_error(path + " is not a counter model written by ktt_b200/profile_model.py");
    }

    CounterModel model;
    model.m_Parameters = Strings(root.Find("tp"), "tp");
    model.m_Counters = Strings(root.Find("pc"), "pc");
    model.m_ComputeCapability = root.NumberOr("cc", 0.0);
    model.m_Multiprocessors = static_cast<uint32_t>(root.NumberOr("multiprocessors", 0.0));
    const json::Json* trees = root.Find("trees");

    if (trees == nullptr || trees->items.empty())
    {
        throw std::runtime_error("counter model " + path + " has no trees");
    }

    for (const auto& t : trees->items)
    {
        Tree tree;
        tree.feature = Numbers<int32_t>(t.Find("feature"), "feature");
        tree.threshold = Numbers<double>(t.Find("threshold"), "threshold");
        tree.left = Numbers<int32_t>(t.Find("left"), "left");
        tree.right = Numbers<int32_t>(t.Find("right"), "right");
        const json::Json* values = t.Find("value");
        const size_t nodes = tree.feature.size();

        if (nodes == 0 || values == nullptr || values->items.size() != nodes || tree.threshold.size() != nodes
            || tree.left.size() != nodes || tree.right.size() != nodes)
        {
            throw std::runtime_error("counter model tree arrays differ in length");
        }

        tree.value.resize(nodes);

        for (size_t n = 0; n < nodes; ++n)
        {
            const int32_t f = tree.feature[n];

            if (f < 0)
            {
                tree.value[n] = Numbers<double>(&values->items[n], "leaf value");

                if (tree.value[n].size() != model.m_Counters.size())
                {
                    throw std::runtime_error("counter model leaf predicts a different number of counters");
                }
            }
            else if (static_cast<size_t>(f) >= model.m_Parameters.size() || tree.left[n] <= static_cast<int32_t>(n)
                || tree.right[n] <= static_cast<int32_t>(n) || static_cast<size_t>(tree.left[n]) >= nodes
                || static_cast<size_t>(tree.right[n]) >= nodes)
            {
                // children always follow their parent in scikit-learn's node order, so every walk ends
                throw std::runtime_error("counter model tree has an invalid node");
            }
        }

        model.m_Trees.push_back(std::move(tree));
    }

    return model;
}

std::vector<double> CounterModel::Predict(const std::vector<double>& features) const
{
    if (features.size() != m_Parameters.size())
    {
        throw std::runtime_error("counter model takes " + std::to_string(m_Parameters.size()) + " parameters");
    }

    std::vector<double> sum(m_Counters.size(), 0.0);

    for (const auto& tree : m_Trees)
    {
        size_t node = 0;

        while (tree.feature[node] >= 0)
        {
            const double x = static_cast<double>(static_cast<float>(features[static_cast<size_t>(tree.feature[node])]));
            node = static_cast<size_t>(x <= tree.threshold[node] ? tree.left[node] : tree.right[node]);
        }

        for (size_t c = 0; c < sum.size(); ++c)
        {
            sum[c] += tree.value[node][c];
        }
    }

    for (auto& v : sum)
    {
        v /= static_cast<double>(m_Trees.size());
    }

    return sum;
}

std::vector<double> CounterModel::Predict(const KernelConfiguration& configuration) const
{
    // the configuration's parameters reordered into the model's order (reorderList, :598-600)
    std::vector<double> features;
    const auto& pairs = configuration.GetPairs();

    for (const auto& name : m_Parameters)
    {
        const auto it = std::find_if(pairs.cbegin(), pairs.cend(), [&name](const auto& p) { return p.GetName() == name; });

        if (it == pairs.cend())
        {
            throw std::runtime_error("configuration lacks the model parameter " + name);
        }

        features.push_back(ParameterAsDouble(it->GetValue()));
    }

    return Predict(features);
}

// ---- analysis -------------------------------------------------------------------------------

namespace profiling
{

namespace
{

double Ratio(const double a, const double b)
{
    return b != 0.0 && std::isfinite(a / b) ? a / b : 0.0;
}

class Counters
{
public:
    Counters(const std::vector<std::string>& names, const std::vector<double>& values) : m_Names(names), m_Values(values)
    {
        if (names.size() != values.size())
        {
            throw std::runtime_error("counter names and values differ in number");
        }
    }

    // missing counters read as zero (KTT's list.index would raise instead)
    double operator[](const std::string& name) const
    {
        const auto it = std::find(m_Names.cbegin(), m_Names.cend(), name);
        return it == m_Names.cend() ? 0.0 : m_Values[static_cast<size_t>(it - m_Names.cbegin())];
    }

    // position of a name in the list (read by KTT's local-memory estimate, see below)
    double Position(const std::string& name) const
    {
        const auto it = std::find(m_Names.cbegin(), m_Names.cend(), name);
        return it == m_Names.cend() ? 0.0 : static_cast<double>(it - m_Names.cbegin());
    }

private:
    const std::vector<std::string>& m_Names;
    const std::vector<double>& m_Values;
};

} // namespace

std::map<std::string, double> AnalyzeBottlenecks(const std::vector<std::string>& names, const std::vector<double>& values,
    const uint32_t multiprocessors, const uint32_t cores, const double react)
{
    const Counters c(names, values);
    std::map<std::string, double> bn;

    // global memory (:113-128)
    const double dramUtil = c["dram__throughput.avg.pct_of_peak_sustained_elapsed"] / 10.0;
    const double dramLoad = c["dram__sectors_read.sum"];
    const double dramStore = c["dram__sectors_write.sum"];
    const bool dramActive = dramLoad + dramStore > 0.0 && dramUtil > 0.0;
    bn["bnDRAMRead"] = dramActive ? dramLoad / (dramLoad + dramStore) * (dramUtil / 10.0) : 0.0;
    bn["bnDRAMWrite"] = dramActive ? dramStore / (dramLoad + dramStore) * (dramUtil / 10.0) : 0.0;

    // caches (:131-152)
    const double l2Util = c["lts__t_sectors.avg.pct_of_peak_sustained_elapsed"] / 10.0;
    const double l2Load = c["lts__t_sectors_op_read.sum"];
    const double l2Store = c["lts__t_sectors_op_write.sum"];
    const double texUtil = c["l1tex__t_requests_pipe_lsu_mem_global_op_ld.avg.pct_of_peak_sustained_active"] / 10.0;
    bn["bnL2Read"] = Ratio(l2Load, l2Load + l2Store) * (l2Util / 10.0);
    bn["bnL2Write"] = Ratio(l2Store, l2Load + l2Store) * (l2Util / 10.0);
    bn["bnTex"] = texUtil / 10.0;

    // local memory (:155-160).  KTT divides the POSITION of the local-store counter in the counter
    // list (not its value) by the L2 store sectors, marked there as experimental; kept as it is so
    // that the scores match KTT's for the same counters.
    const double localOverhead = Ratio(100.0 * c.Position("l1tex__t_sectors_pipe_lsu_mem_local_op_st.sum"), l2Store);
    bn["bnLocal"] = localOverhead / 100.0 * std::max({dramUtil / 10.0, l2Util / 10.0, texUtil / 10.0});

    // shared memory (:163-183)
    const double smUtil = c["l1tex__data_pipe_lsu_wavefronts_mem_shared.avg.pct_of_peak_sustained_elapsed"] / 10.0;
    const double smLoad = c["l1tex__data_pipe_lsu_wavefronts_mem_shared_op_ld.sum"];
    const double smStore = c["l1tex__data_pipe_lsu_wavefronts_mem_shared_op_st.sum"];
    const bool smActive = smLoad + smStore > 0.0;
    bn["bnSMRead"] = smActive ? smLoad / (smLoad + smStore) * (smUtil / 10.0) : 0.0;
    bn["bnSMWrite"] = smActive ? smStore / (smLoad + smStore) * (smUtil / 10.0) : 0.0;

    // parallelism (:186-208)
    bn["bnMPparal"] = 1.0 - c["sm__warps_active.avg.pct_of_peak_sustained_active"] / 100.0;
    bn["bnGparal"] = (100.0 - c["smsp__cycles_active.avg.pct_of_peak_sustained_elapsed"]) / 100.0;
    const double blocks = Ratio(c[GlobalSizeCounter], c[LocalSizeCounter]);
    const double mp = static_cast<double>(multiprocessors);
    // (blocks + mp - 1) / mp is a true division in KTT's Python 3, so this is 1 - blocks / (blocks + mp - 1)
    bn["bnTailEffect"] = 1.0 - Ratio(blocks, (blocks + mp - 1.0) / mp * mp);
    const double threadTarget = static_cast<double>(cores) * 5.0;
    bn["bnThreads"] = std::max(0.0, Ratio(threadTarget - c[GlobalSizeCounter], threadTarget));

    // instructions (:212-321)
    const double spInstr = c["smsp__sass_thread_inst_executed_op_fp32_pred_on.sum"];
    const double dpInstr = c["smsp__sass_thread_inst_executed_op_fp64_pred_on.sum"];
    const double intInstr = c["smsp__sass_thread_inst_executed_op_integer_pred_on.sum"];
    const double miscInstr = c["smsp__sass_thread_inst_executed_op_misc_pred_on.sum"];
    const double ldstInstr = c["smsp__sass_thread_inst_executed_op_memory_pred_on.sum"];
    const double ctrlInstr = c["smsp__sass_thread_inst_executed_op_control_pred_on.sum"];
    const double bconvInstr = c["smsp__sass_thread_inst_executed_op_conversion_pred_on.sum"];
    const double execInstr = c["smsp__inst_executed.sum"];
    const double sfuUtil = c["smsp__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active"] / 10.0;
    const double texFuUtil = c["smsp__inst_executed_pipe_tex.avg.pct_of_peak_sustained_active"] / 10.0;
    const double slotUtil = c["smsp__issue_active.avg.pct_of_peak_sustained_active"];
    const double effExec = c["smsp__thread_inst_executed_per_inst_executed.ratio"] * 100.0 / 32.0;
    const double effPred = c["smsp__thread_inst_executed_per_inst_executed.pct"];
    const double fitted = execInstr * 32.0 * Ratio(100.0, effExec) * Ratio(100.0, effPred);
    const double utilFitted = std::min(1.0, slotUtil / 50.0);
    auto approx = [&](const double instr) { return Ratio(instr, fitted) * utilFitted; };
    const double sp = approx(spInstr), dp = approx(dpInstr), ldst = approx(ldstInstr), cf = approx(ctrlInstr);
    const double in = approx(intInstr), misc = approx(miscInstr), bconv = approx(bconvInstr);
    bn["bnSP"] = sp;
    bn["bnDP"] = dp;
    bn["bnSFU"] = sfuUtil / 10.0;
    bn["bnCF"] = cf;
    bn["bnLDST"] = ldst;
    bn["bnTexFu"] = texFuUtil / 10.0;
    bn["bnInt"] = in;
    bn["bnMisc"] = misc;
    bn["bnBconv"] = bconv;

    const double maxUtil = std::max({Ratio(sp, utilFitted), Ratio(dp, utilFitted), sfuUtil / 10.0, Ratio(cf, utilFitted),
        Ratio(ldst, utilFitted), Ratio(in, utilFitted), Ratio(misc, utilFitted), Ratio(bconv, utilFitted)});
    const double issueWeight = maxUtil > react ? (maxUtil - react) / (1.0 - react) : 0.0;
    bn["bnInstIssue"] = (100.0 - slotUtil) / 100.0 * issueWeight;
    return bn;
}

std::vector<double> ComputeChanges(const std::map<std::string, double>& bn, const std::vector<std::string>& counters,
    const bool xuPipe, const double react)
{
    std::vector<double> change(counters.size(), 0.0);
    auto set = [&](const std::string& counter, const double value)
    {
        const auto it = std::find(counters.cbegin(), counters.cend(), counter);

        if (it != counters.cend())
        {
            change[static_cast<size_t>(it - counters.cbegin())] = value;
        }
    };
    auto get = [&bn](const char* name)
    {
        const auto it = bn.find(name);
        return it == bn.cend() ? 0.0 : it->second;
    };
    // above the reaction threshold, rescaled to [0, 1] (:391-402)
    auto scaled = [react](const double b) { return (b - react) / (1.0 - react); };

    // memory subsystem (:349-358)
    set("dram__sectors_read.sum", -get("bnDRAMRead"));
    set("dram__sectors_write.sum", -get("bnDRAMWrite"));
    set("lts__t_sectors_op_read.sum", -get("bnL2Read"));
    set("lts__t_sectors_op_write.sum", -get("bnL2Write"));
    set("l1tex__t_requests_pipe_lsu_mem_global_op_ld.sum", -get("bnTex"));
    set("l1tex__t_sectors_pipe_lsu_mem_local_op_ld.sum", -get("bnLocal"));
    set("l1tex__t_sectors_pipe_lsu_mem_local_op_st.sum", -get("bnLocal"));
    set("l1tex__data_pipe_lsu_wavefronts_mem_shared_op_ld.sum", -get("bnSMRead"));
    set("l1tex__data_pipe_lsu_wavefronts_mem_shared_op_st.sum", -get("bnSMWrite"));

    // instructions (:380-402); FP32 and FP64 take the bottleneck itself, the others its rescaled excess
    if (get("bnSP") > react) set("smsp__sass_thread_inst_executed_op_fp32_pred_on.sum", -get("bnSP"));
    if (get("bnDP") > react) set("smsp__sass_thread_inst_executed_op_fp64_pred_on.sum", -get("bnDP"));
    if (get("bnCF") > react) set("smsp__sass_thread_inst_executed_op_control_pred_on.sum", -scaled(get("bnCF")));
    if (get("bnLDST") > react) set("smsp__sass_thread_inst_executed_op_memory_pred_on.sum", -scaled(get("bnLDST")));
    if (get("bnInt") > react) set("smsp__sass_thread_inst_executed_op_integer_pred_on.sum", -scaled(get("bnInt")));
    if (get("bnMisc") > react) set("smsp__sass_thread_inst_executed_op_misc_pred_on.sum", -scaled(get("bnMisc")));
    if (get("bnBconv") > react) set("smsp__sass_thread_inst_executed_op_conversion_pred_on.sum", -scaled(get("bnBconv")));
    // B200 addition: a saturated XU pipe asks for fewer XU instructions, like FP32 for the FMA pipe
    if (xuPipe && get("bnSFU") > react) set("smsp__inst_executed_pipe_xu.sum", -get("bnSFU"));
    set("smsp__issue_active.avg.pct_of_peak_sustained_active", get("bnInstIssue"));

    // parallelism (:405-412)
    set("smsp__cycles_active.avg.pct_of_peak_sustained_elapsed", get("bnGparal"));
    set(GlobalSizeCounter, get("bnThreads"));
    return change;
}

std::vector<double> ScoreCandidates(const std::vector<double>& changes, const std::vector<double>& actual,
    const std::vector<std::vector<double>>& predicted, const std::vector<double>& previous)
{
    if (predicted.size() != previous.size())
    {
        throw std::runtime_error("one previous score per candidate is needed");
    }

    // the change list is cut to the model's output length (:521-523)
    const size_t width = std::min(changes.size(), actual.size());
    std::vector<double> score(predicted.size(), 0.0);

    for (size_t i = 0; i < predicted.size(); ++i)
    {
        if (predicted[i].size() < width)
        {
            throw std::runtime_error("a candidate's prediction is shorter than the counter list");
        }

        for (size_t j = 0; j < width; ++j)
        {
            // sign(change * (p - a)) * |change * 2 (p - a) / (p + a)|, NaN (0 / 0) counted as zero and
            // infinities clamped to the largest double, as numpy's nan_to_num does (:525-537)
            const double diff = predicted[i][j] - actual[j];
            const double product = changes[j] * diff;
            const double sign = product > 0.0 ? 1.0 : (product < 0.0 ? -1.0 : 0.0);
            double term = sign * std::fabs(changes[j] * 2.0 * diff / (predicted[i][j] + actual[j]));

            if (std::isnan(term))
            {
                term = 0.0;
            }
            else if (std::isinf(term))
            {
                term = term > 0.0 ? std::numeric_limits<double>::max() : -std::numeric_limits<double>::max();
            }

            score[i] += term;
        }
    }

    if (score.empty())
    {
        return score;
    }

    // normalisation, cut-off and exponent (:539-556)
    const double minScore = *std::min_element(score.cbegin(), score.cend());
    const double maxScore = *std::max_element(score.cbegin(), score.cend());

    for (size_t i = 0; i < score.size(); ++i)
    {
        double s = score[i];

        if (s < Cutoff)
        {
            s = MinimumScore;
        }
        else
        {
            if (s < 0.0)
            {
                s = 1.0 - s / minScore;
            }
            else if (s > 0.0)
            {
                s = 1.0 + s / maxScore;
            }

            s = std::pow(s, Exponent);
        }

        if (s < MinimumScore)
        {
            s = MinimumScore;
        }

        if (previous[i] == 0.0)
        {
            s = 0.0;
        }

        score[i] = s;
    }

    return score;
}

size_t WeightedRandomStep(const std::vector<double>& scores, const double u)
{
    if (scores.empty())
    {
        return 0;
    }

    const double total = std::accumulate(scores.cbegin(), scores.cend(), 0.0);

    if (total == 0.0)
    {
        return std::min(scores.size() - 1, static_cast<size_t>(u * static_cast<double>(scores.size())));
    }

    const double draw = u * total;
    double running = 0.0;
    size_t index = 0;

    for (const double s : scores)
    {
        running += s;

        if (draw < running)
        {
            break;
        }

        ++index;
    }

    return std::min(index, scores.size() - 1);
}

uint32_t CoresPerMultiprocessor(const uint32_t ccMajor, const uint32_t ccMinor)
{
    static const std::map<uint32_t, uint32_t> cores{{0x30, 192}, {0x32, 192}, {0x35, 192}, {0x37, 192}, {0x50, 128},
        {0x52, 128}, {0x53, 128}, {0x60, 64}, {0x61, 128}, {0x62, 128}, {0x70, 64}, {0x72, 64}, {0x75, 64}, {0x80, 64},
        {0x86, 128}, {0x87, 128}, {0x89, 128}, {0x90, 128}, {0xa0, 128}, {0xa1, 128}, {0xc0, 128}};
    const auto it = cores.find((ccMajor << 4) + ccMinor);

    if (it == cores.cend())
    {
        log::Warning("Unknown number of cores for SM " + std::to_string(ccMajor) + "." + std::to_string(ccMinor)
            + ", using default value of 64");
        return 64;
    }

    return it->second;
}

} // namespace profiling

// ---- searcher -------------------------------------------------------------------------------

ProfileBasedSearcher::ProfileBasedSearcher(Tuner& tuner, const CounterModel& model, const uint32_t batchSize,
    const uint32_t neighbourSize, const uint32_t randomSize, const uint64_t seed) :
    m_Tuner(tuner), m_Model(model), m_BatchSize(std::max<uint32_t>(1, batchSize)), m_NeighbourSize(neighbourSize),
    m_RandomSize(randomSize), m_Generator(seed), m_Uniform(0.0, 1.0)
{
    if (m_Model.IsEmpty())
    {
        throw std::runtime_error("The profile-based searcher needs a counter model");
    }
}

void ProfileBasedSearcher::SetDeviceProperties(const uint32_t ccMajor, const uint32_t ccMinor, const uint32_t multiprocessors)
{
    m_CcMajor = ccMajor;
    m_CcMinor = ccMinor;
    m_Multiprocessors = multiprocessors;
}

void ProfileBasedSearcher::ResolveDevice()
{
    if (m_Multiprocessors != 0)
    {
        return;
    }

    // Configure (:669-699): compute capability and SM count of the tuner's device
    const DeviceInfo info = m_Tuner.GetCurrentDeviceInfo();

    if (info.GetMaxComputeUnits() != 0)
    {
        SetDeviceProperties(info.GetCudaComputeCapabilityMajor(), info.GetCudaComputeCapabilityMinor(), info.GetMaxComputeUnits());
        return;
    }

    const double cc = m_Model.GetComputeCapability();
    const uint32_t major = static_cast<uint32_t>(cc);
    SetDeviceProperties(major, static_cast<uint32_t>(std::lround((cc - major) * 10.0)), m_Model.GetMultiprocessors());
    log::Info("Profile-based searcher uses the model's device: compute capability " + std::to_string(cc) + ", "
        + std::to_string(m_Multiprocessors) + " SMs");
}

KernelConfiguration ProfileBasedSearcher::RandomUnexplored()
{
    const uint64_t count = GetConfigurationsCount();
    const auto& explored = GetExploredIndices();
    auto draw = [this](const uint64_t n) { return std::min<uint64_t>(n - 1, static_cast<uint64_t>(m_Uniform(m_Generator) * n)); };

    for (int attempt = 0; attempt < 64; ++attempt)
    {
        const uint64_t index = draw(count);

        if (explored.count(index) == 0)
        {
            return GetConfiguration(index);
        }
    }

    std::vector<uint64_t> open;

    for (uint64_t i = 0; i < count; ++i)
    {
        if (explored.count(i) == 0)
        {
            open.push_back(i);
        }
    }

    return GetConfiguration(open.empty() ? draw(count) : open[draw(open.size())]);
}

std::vector<KernelConfiguration> ProfileBasedSearcher::UniqueConfigurations(const std::vector<KernelConfiguration>& list) const
{
    // GetUniqueConfigurations (:701-713), keeping the first occurrence in order
    std::set<uint64_t> seen;
    std::vector<KernelConfiguration> unique;

    for (const auto& configuration : list)
    {
        if (seen.insert(GetIndex(configuration)).second)
        {
            unique.push_back(configuration);
        }
    }

    return unique;
}

void ProfileBasedSearcher::FillRandomBatch(const uint64_t size)
{
    // distinct random unexplored configurations (:642-649, :737-744)
    m_Batch.clear();
    const uint64_t target = std::min<uint64_t>(size, std::max<uint64_t>(1, GetUnexploredConfigurationsCount()));

    for (int round = 0; m_Batch.size() < target && round < 1000; ++round)
    {
        while (m_Batch.size() < target)
        {
            m_Batch.push_back(RandomUnexplored());
        }

        m_Batch = UniqueConfigurations(m_Batch);
    }
}

void ProfileBasedSearcher::OnInitialize()
{
    ResolveDevice();
    m_HasBest = false;
    m_ProfilingRequested = false;
    m_BestDuration = 0;
    m_ScoredBatches = 0;
    FillRandomBatch(m_BatchSize);
    m_Current = m_Batch.front();
    m_Batch.erase(m_Batch.begin());
}

void ProfileBasedSearcher::OnReset()
{
    m_Batch.clear();
    m_HasBest = false;

    if (m_ProfilingRequested)
    {
        m_Tuner.SetProfiling(false);
        m_ProfilingRequested = false;
    }
}

KernelConfiguration ProfileBasedSearcher::GetCurrentConfiguration() const { return m_Current; }

bool ProfileBasedSearcher::CalculateNextConfiguration(const KernelResult& previousResult)
{
    // CalculateNextConfiguration (:715-845)
    if (!m_ProfilingRequested && previousResult.IsValid()
        && (!m_HasBest || previousResult.GetKernelDuration() < m_BestDuration))
    {
        m_BestDuration = previousResult.GetKernelDuration();
        m_BestConfiguration = m_Current;
        m_HasBest = true;
    }

    if (!m_Batch.empty())
    {
        m_Current = m_Batch.front();
        m_Batch.erase(m_Batch.begin());
    }
    else if (!m_HasBest)
    {
        // every configuration of the batch failed: a new random batch
        FillRandomBatch(m_BatchSize);
        m_Current = m_Batch.front();
        m_Batch.erase(m_Batch.begin());
    }
    else if (!m_ProfilingRequested)
    {
        // run the batch's fastest configuration again, this time with counters
        m_Current = m_BestConfiguration;
        m_ProfilingRequested = true;
        m_Tuner.SetProfiling(true);
    }
    else
    {
        ScoreAndSelect(previousResult);
        m_Current = m_Batch.front();
        m_Batch.erase(m_Batch.begin());
        m_HasBest = false;
        m_ProfilingRequested = false;
        m_Tuner.SetProfiling(false);
    }

    return true;
}

void ProfileBasedSearcher::ScoreAndSelect(const KernelResult& profiled)
{
    // candidates: unexplored neighbours of the best configuration plus random ones (:773-788)
    std::vector<KernelConfiguration> candidates = UniqueConfigurations(
        GetNeighbourConfigurations(m_BestConfiguration, profiling::NeighbourDistance, m_NeighbourSize));
    const uint64_t target = std::min<uint64_t>(candidates.size() + m_RandomSize, GetUnexploredConfigurationsCount());

    for (int round = 0; candidates.size() < target && round < 1000; ++round)
    {
        while (candidates.size() < target)
        {
            candidates.push_back(RandomUnexplored());
        }

        candidates = UniqueConfigurations(candidates);
    }

    if (candidates.empty())
    {
        FillRandomBatch(m_BatchSize);
        return;
    }

    std::vector<double> score(candidates.size(), 1.0);
    const bool counted = !profiled.GetResults().empty() && profiled.GetResults()[0].HasProfilingData()
        && profiled.GetResults()[0].GetProfilingData().IsValid();

    if (counted)
    {
        // counters of the profiled run plus the launch sizes (:756-770)
        const ComputationResult& run = profiled.GetResults()[0];
        std::vector<std::string> names{profiling::GlobalSizeCounter, profiling::LocalSizeCounter};
        std::vector<double> values{static_cast<double>(run.GetGlobalSize().GetTotalSize() * run.GetLocalSize().GetTotalSize()),
            static_cast<double>(run.GetLocalSize().GetTotalSize())};

        for (const auto& counter : run.GetProfilingData().GetCounters())
        {
            names.push_back(counter.GetName());

            switch (counter.GetType())
            {
            case ProfilingCounterType::Int: values.push_back(static_cast<double>(counter.GetValueInt())); break;
            case ProfilingCounterType::UnsignedInt:
            case ProfilingCounterType::Throughput:
            case ProfilingCounterType::UtilizationLevel: values.push_back(static_cast<double>(counter.GetValueUint())); break;
            default: values.push_back(counter.GetValueDouble()); break;
            }
        }

        const uint32_t cores = profiling::CoresPerMultiprocessor(m_CcMajor, m_CcMinor) * m_Multiprocessors;
        const auto bottlenecks = profiling::AnalyzeBottlenecks(names, values, m_Multiprocessors, cores);
        const auto changes = profiling::ComputeChanges(bottlenecks, m_Model.GetCounters(), m_XuPipe);
        const std::vector<double> actual = m_Model.Predict(m_BestConfiguration);
        std::vector<std::vector<double>> predicted;

        for (const auto& candidate : candidates)
        {
            predicted.push_back(m_Model.Predict(candidate));
        }

        score = profiling::ScoreCandidates(changes, actual, predicted, score);
        ++m_ScoredBatches;
    }
    else
    {
        log::Warning("Profile-based searcher: the profiled run of " + m_BestConfiguration.GetString()
            + " has no counters; the next batch is drawn uniformly from the candidates");
    }

    // the next batch, weighted by score without repetition (:800-817)
    m_Batch.clear();

    if (candidates.size() > m_BatchSize)
    {
        std::set<size_t> chosen;

        for (int draws = 0; m_Batch.size() < m_BatchSize; ++draws)
        {
            size_t index = profiling::WeightedRandomStep(score, m_Uniform(m_Generator));

            if (draws > 10000)
            {
                // never reached with scores of at least MinimumScore; keeps the loop finite regardless
                index = 0;

                while (chosen.count(index) != 0)
                {
                    ++index;
                }
            }

            if (chosen.insert(index).second)
            {
                m_Batch.push_back(candidates[index]);
                score[index] = 0.0;
            }
        }
    }
    else
    {
        m_Batch = candidates;
    }
}

} // namespace ktt
