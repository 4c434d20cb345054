// Output.cpp -- tuning results to and from files, in KTT 2.1.0's JSON layout.
//
// Field names, nesting, enum spellings and time conversion follow Source/Output/JsonConverters.cpp:8-394
// (Metadata; Results[] with ComputationResults[], Configuration[] {Name, Value, ValueType}, the
// overheads, Status, TotalDuration, TotalOverhead; optional UserData), so that files written here
// load into KTT's tools and KTT's own result files -- such as the 2080 Ti search-space data of the
// Coulomb example -- load here (fields a file lacks read as zero).  Times are written in the unit
// set by Tuner::SetTimeUnit (default milliseconds) and converted back to nanoseconds when loading.
// The path gets a ".json" / ".xml" extension appended when it has none, as KTT does.
#include <cctype>
#include <chrono>
#include <cmath>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>

#include "Json.h"
#include "Logger.h"
#include "TunerCore.h"

namespace ktt
{

namespace
{

using json::Json;
using json::Parser;

TimeUnit& CurrentUnit()
{
    static TimeUnit unit = TimeUnit::Milliseconds;
    return unit;
}

double UnitScale(const TimeUnit unit)
{
    switch (unit)
    {
    case TimeUnit::Nanoseconds: return 1.0;
    case TimeUnit::Microseconds: return 1e3;
    case TimeUnit::Milliseconds: return 1e6;
    case TimeUnit::Seconds: return 1e9;
    }

    return 1.0;
}

const char* UnitName(const TimeUnit unit)
{
    switch (unit)
    {
    case TimeUnit::Nanoseconds: return "Nanoseconds";
    case TimeUnit::Microseconds: return "Microseconds";
    case TimeUnit::Milliseconds: return "Milliseconds";
    case TimeUnit::Seconds: return "Seconds";
    }

    return "Milliseconds";
}

TimeUnit UnitFromName(const std::string& name)
{
    if (name == "Nanoseconds") return TimeUnit::Nanoseconds;
    if (name == "Microseconds") return TimeUnit::Microseconds;
    if (name == "Seconds") return TimeUnit::Seconds;
    return TimeUnit::Milliseconds;
}

const char* StatusName(const ResultStatus status)
{
    switch (status)
    {
    case ResultStatus::Ok: return "Ok";
    case ResultStatus::ComputationFailed: return "ComputationFailed";
    case ResultStatus::ValidationFailed: return "ValidationFailed";
    case ResultStatus::CompilationFailed: return "CompilationFailed";
    case ResultStatus::DeviceLimitsExceeded: return "DeviceLimitsExceeded";
    }

    return "ComputationFailed";
}

// ProfilingCounterType names of Source/Output/JsonConverters.h:56-64
const char* CounterTypeName(const ProfilingCounterType type)
{
    switch (type)
    {
    case ProfilingCounterType::Int: return "Int";
    case ProfilingCounterType::UnsignedInt: return "UnsignedInt";
    case ProfilingCounterType::Double: return "Double";
    case ProfilingCounterType::Percent: return "Percent";
    case ProfilingCounterType::Throughput: return "Throughput";
    case ProfilingCounterType::UtilizationLevel: return "UtilizationLevel";
    }

    return "Double";
}

// Value written by the counter's type (Source/Output/JsonConverters.cpp:141-166); floating-point
// values with all 17 significant digits, so that a counter reads back bit for bit, NaN as null
std::string CounterValueJson(const KernelProfilingCounter& counter)
{
    switch (counter.GetType())
    {
    case ProfilingCounterType::Int: return std::to_string(counter.GetValueInt());
    case ProfilingCounterType::UnsignedInt:
    case ProfilingCounterType::Throughput:
    case ProfilingCounterType::UtilizationLevel: return std::to_string(counter.GetValueUint());
    default:
    {
        const double v = counter.GetValueDouble();

        if (!std::isfinite(v))
        {
            return "null";
        }

        std::ostringstream text;
        text << std::setprecision(17) << v;
        return text.str();
    }
    }
}

KernelProfilingCounter CounterFromJson(const Json& j)
{
    const std::string name = j.StringOr("Name", "");
    const std::string typeName = j.StringOr("Type", "Double");
    const Json* value = j.Find("Value");
    const double number = value == nullptr || value->kind == Json::Kind::Null
        ? std::nan("") : (value->integral ? static_cast<double>(value->integer) : value->number);

    if (typeName == "Int")
    {
        return KernelProfilingCounter(name, ProfilingCounterType::Int,
            static_cast<int64_t>(value && value->integral ? value->integer : std::llround(number)));
    }

    for (const auto type : {ProfilingCounterType::UnsignedInt, ProfilingCounterType::Throughput,
             ProfilingCounterType::UtilizationLevel})
    {
        if (typeName == CounterTypeName(type))
        {
            return KernelProfilingCounter(name, type,
                static_cast<uint64_t>(value && value->integral ? value->integer : std::llround(number)));
        }
    }

    return KernelProfilingCounter(name, typeName == "Percent" ? ProfilingCounterType::Percent : ProfilingCounterType::Double,
        number);
}

ResultStatus StatusFromName(const std::string& name)
{
    if (name == "Ok") return ResultStatus::Ok;
    if (name == "ValidationFailed") return ResultStatus::ValidationFailed;
    if (name == "CompilationFailed") return ResultStatus::CompilationFailed;
    if (name == "DeviceLimitsExceeded") return ResultStatus::DeviceLimitsExceeded;
    return ResultStatus::ComputationFailed;
}

const char* ValueTypeName(const ParameterValueType type)
{
    switch (type)
    {
    case ParameterValueType::Int: return "Int";
    case ParameterValueType::UnsignedInt: return "UnsignedInt";
    case ParameterValueType::Double: return "Double";
    case ParameterValueType::Bool: return "Bool";
    case ParameterValueType::String: return "String";
    }

    return "UnsignedInt";
}


std::string Escape(const std::string& s)
{
    std::string out;

    for (const char c : s)
    {
        switch (c)
        {
        case '"': out += "\\\""; break;
        case '\\': out += "\\\\"; break;
        case '\n': out += "\\n"; break;
        case '\t': out += "\\t"; break;
        default: out += c; break;
        }
    }

    return out;
}

std::string Number(const double value)
{
    std::ostringstream s;
    s << std::setprecision(15) << value;
    return s.str();
}

std::string Timestamp()
{
    const std::time_t now = std::chrono::system_clock::to_time_t(std::chrono::system_clock::now());
    std::tm tm{};
    gmtime_r(&now, &tm);
    char buffer[64];
    std::strftime(buffer, sizeof buffer, "%Y-%m-%d %H:%M:%S UTC", &tm);
    return buffer;
}

std::string WithExtension(const std::string& path, const std::string& extension)
{
    if (path.size() >= extension.size() && path.compare(path.size() - extension.size(), extension.size(), extension) == 0)
    {
        return path;
    }

    return path + extension;
}

std::string ValueJson(const ParameterValue& value)
{
    switch (ParameterPair::GetTypeFromValue(value))
    {
    case ParameterValueType::Int: return std::to_string(std::get<int64_t>(value));
    case ParameterValueType::UnsignedInt: return std::to_string(std::get<uint64_t>(value));
    case ParameterValueType::Double: return Number(std::get<double>(value));
    case ParameterValueType::Bool: return std::get<bool>(value) ? "true" : "false";
    case ParameterValueType::String: return "\"" + Escape(std::get<std::string>(value)) + "\"";
    }

    return "0";
}

} // namespace

void Tuner::SetTimeUnit(const TimeUnit unit) { CurrentUnit() = unit; }

void Tuner::SaveResults(const std::vector<KernelResult>& results, const std::string& filePath, const OutputFormat format,
    const UserData& data) const
{
    try
    {
        const double scale = UnitScale(CurrentUnit());
        auto t = [scale](const Nanoseconds ns) { return Number(ns == InvalidDuration ? 0.0 : static_cast<double>(ns) / scale); };
        const std::string device = m_Core->DeviceName();
        const std::string sizeType = m_Core->GetGlobalSizeType() == GlobalSizeType::CUDA ? "CUDA" : "OpenCL";

        if (format == OutputFormat::JSON)
        {
            std::ofstream out(WithExtension(filePath, ".json"));

            if (!out)
            {
                throw std::runtime_error("Unable to open " + filePath + " for writing");
            }

            out << "{\n  \"Metadata\": {\n    \"ComputeApi\": \"CUDA\",\n    \"Device\": \"" << Escape(device)
                << "\",\n    \"GlobalSizeType\": \"" << sizeType << "\",\n    \"KttVersion\": \"2.1.0\",\n"
                << "    \"Platform\": \"NVIDIA CUDA\",\n    \"TimeUnit\": \"" << UnitName(CurrentUnit())
                << "\",\n    \"Timestamp\": \"" << Timestamp() << "\"\n  },\n  \"Results\": [";

            for (size_t r = 0; r < results.size(); ++r)
            {
                const KernelResult& result = results[r];
                out << (r ? "," : "") << "\n    {\n      \"ComputationResults\": [";

                for (size_t c = 0; c < result.GetResults().size(); ++c)
                {
                    const ComputationResult& cr = result.GetResults()[c];
                    const auto& g = cr.GetGlobalSize();
                    const auto& l = cr.GetLocalSize();
                    out << (c ? "," : "") << "\n        {\"CompilationOverhead\": " << t(cr.GetCompilationOverhead())
                        << ", \"Duration\": " << t(cr.GetDuration()) << ", \"GlobalSize\": {\"X\": " << g.GetSizeX()
                        << ", \"Y\": " << g.GetSizeY() << ", \"Z\": " << g.GetSizeZ() << "}, \"KernelFunction\": \""
                        << Escape(cr.GetKernelFunction()) << "\", \"LocalSize\": {\"X\": " << l.GetSizeX()
                        << ", \"Y\": " << l.GetSizeY() << ", \"Z\": " << l.GetSizeZ() << "}, \"Overhead\": "
                        << t(cr.GetOverhead());

                    if (cr.HasProfilingData())
                    {
                        const KernelProfilingData& data = cr.GetProfilingData();
                        out << ", \"ProfilingData\": {\"Counters\": [";

                        for (size_t k = 0; k < data.GetCounters().size(); ++k)
                        {
                            const KernelProfilingCounter& counter = data.GetCounters()[k];
                            out << (k ? ", " : "") << "{\"Name\": \"" << Escape(counter.GetName()) << "\", \"Type\": \""
                                << CounterTypeName(counter.GetType()) << "\", \"Value\": " << CounterValueJson(counter) << "}";
                        }

                        out << "], \"RemainingProfilingRuns\": " << data.GetRemainingProfilingRuns() << "}";
                    }

                    out << "}";
                }

                out << "\n      ],\n      \"Configuration\": [";
                const auto& pairs = result.GetConfiguration().GetPairs();

                for (size_t p = 0; p < pairs.size(); ++p)
                {
                    out << (p ? ", " : "") << "{\"Name\": \"" << Escape(pairs[p].GetName()) << "\", \"Value\": "
                        << ValueJson(pairs[p].GetValue()) << ", \"ValueType\": \"" << ValueTypeName(pairs[p].GetValueType())
                        << "\"}";
                }

                out << "],\n      \"DataMovementOverhead\": " << t(result.GetDataMovementOverhead())
                    << ",\n      \"ExtraDuration\": " << t(result.GetExtraDuration())
                    << ",\n      \"FailedKernelOverhead\": " << t(result.GetFailedKernelOverhead())
                    << ",\n      \"KernelName\": \"" << Escape(result.GetKernelName())
                    << "\",\n      \"ProfilingRunsOverhead\": " << t(result.GetProfilingRunsOverhead())
                    << ",\n      \"SearcherOverhead\": " << t(result.GetSearcherOverhead())
                    << ",\n      \"Status\": \"" << StatusName(result.GetStatus())
                    << "\",\n      \"TotalDuration\": " << t(result.GetTotalDuration())
                    << ",\n      \"TotalOverhead\": " << t(result.GetTotalOverhead())
                    << ",\n      \"ValidationOverhead\": " << t(result.GetValidationOverhead()) << "\n    }";
            }

            out << "\n  ]";

            if (!data.empty())
            {
                out << ",\n  \"UserData\": {";
                size_t i = 0;

                for (const auto& [k, v] : data)
                {
                    out << (i++ ? ", " : "") << "\"" << Escape(k) << "\": \"" << Escape(v) << "\"";
                }

                out << "}";
            }

            out << "\n}\n";
            return;
        }

        std::ofstream out(WithExtension(filePath, ".xml"));

        if (!out)
        {
            throw std::runtime_error("Unable to open " + filePath + " for writing");
        }

        out << "<?xml version=\"1.0\"?>\n<TuningData>\n  <Metadata ComputeApi=\"CUDA\" Device=\"" << device
            << "\" GlobalSizeType=\"" << sizeType << "\" KttVersion=\"2.1.0\" Platform=\"NVIDIA CUDA\" TimeUnit=\""
            << UnitName(CurrentUnit()) << "\" Timestamp=\"" << Timestamp() << "\"/>\n  <Results>\n";

        for (const auto& result : results)
        {
            out << "    <Result KernelName=\"" << result.GetKernelName() << "\" Status=\"" << StatusName(result.GetStatus())
                << "\" TotalDuration=\"" << t(result.GetTotalDuration()) << "\" TotalOverhead=\"" << t(result.GetTotalOverhead())
                << "\">\n      <Configuration>\n";

            for (const auto& pair : result.GetConfiguration().GetPairs())
            {
                out << "        <Pair Name=\"" << pair.GetName() << "\" Value=\"" << pair.GetValueString() << "\" ValueType=\""
                    << ValueTypeName(pair.GetValueType()) << "\"/>\n";
            }

            out << "      </Configuration>\n      <ComputationResults>\n";

            for (const auto& cr : result.GetResults())
            {
                out << "        <ComputationResult KernelFunction=\"" << cr.GetKernelFunction() << "\" Duration=\""
                    << t(cr.GetDuration()) << "\" Overhead=\"" << t(cr.GetOverhead()) << "\"";

                if (!cr.HasProfilingData())
                {
                    out << "/>\n";
                    continue;
                }

                // Source/Output/XmlConverters.cpp:438-535: ProfilingData > Counters > Counter
                const KernelProfilingData& profiling = cr.GetProfilingData();
                out << ">\n          <ProfilingData RemainingProfilingRuns=\"" << profiling.GetRemainingProfilingRuns()
                    << "\">\n            <Counters>\n";

                for (const auto& counter : profiling.GetCounters())
                {
                    std::string value = CounterValueJson(counter);
                    value = value == "null" ? "nan" : value;
                    out << "              <Counter Name=\"" << counter.GetName() << "\" Type=\""
                        << CounterTypeName(counter.GetType()) << "\" Value=\"" << value << "\"/>\n";
                }

                out << "            </Counters>\n          </ProfilingData>\n        </ComputationResult>\n";
            }

            out << "      </ComputationResults>\n    </Result>\n";
        }

        out << "  </Results>\n";

        for (const auto& [k, v] : data)
        {
            out << "  <UserData Key=\"" << k << "\" Value=\"" << v << "\"/>\n";
        }

        out << "</TuningData>\n";
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
    }
}

std::vector<KernelResult> Tuner::LoadResults(const std::string& filePath, const OutputFormat format) const
{
    UserData data;
    return LoadResults(filePath, format, data);
}

std::vector<KernelResult> Tuner::LoadResults(const std::string& filePath, const OutputFormat format, UserData& data) const
{
    std::vector<KernelResult> results;

    try
    {
        if (format != OutputFormat::JSON)
        {
            throw std::runtime_error("Results are loaded from JSON files only");
        }

        std::ifstream in(WithExtension(filePath, ".json"));

        if (!in)
        {
            throw std::runtime_error("Unable to open " + filePath);
        }

        std::stringstream buffer;
        buffer << in.rdbuf();
        const std::string text = buffer.str();
        const Json root = Parser(text).Parse();
        const Json* metadata = root.Find("Metadata");
        const TimeUnit unit = metadata ? UnitFromName(metadata->StringOr("TimeUnit", "Milliseconds")) : TimeUnit::Milliseconds;
        const double scale = UnitScale(unit);
        auto ns = [scale](const double v) { return static_cast<Nanoseconds>(std::llround(v * scale)); };
        const Json* list = root.Find("Results");

        if (list == nullptr || list->kind != Json::Kind::Array)
        {
            throw std::runtime_error("File " + filePath + " has no Results array");
        }

        for (const auto& item : list->items)
        {
            std::vector<ParameterPair> pairs;

            if (const Json* configuration = item.Find("Configuration"))
            {
                for (const auto& p : configuration->items)
                {
                    const std::string name = p.StringOr("Name", "");
                    const std::string type = p.StringOr("ValueType", "UnsignedInt");
                    const Json* value = p.Find("Value");
                    ParameterValue v = static_cast<uint64_t>(0);

                    if (value != nullptr)
                    {
                        if (type == "Int") v = static_cast<int64_t>(value->integral ? value->integer : std::llround(value->number));
                        else if (type == "Double") v = value->number;
                        else if (type == "Bool") v = value->boolean;
                        else if (type == "String") v = value->text;
                        else v = static_cast<uint64_t>(value->integral ? value->integer : std::llround(value->number));
                    }

                    pairs.emplace_back(name, v);
                }
            }

            std::vector<ComputationResult> computations;

            if (const Json* crs = item.Find("ComputationResults"))
            {
                for (const auto& c : crs->items)
                {
                    ComputationResult cr(c.StringOr("KernelFunction", ""));
                    cr.SetDurationData(ns(c.NumberOr("Duration", 0.0)), ns(c.NumberOr("Overhead", 0.0)),
                        ns(c.NumberOr("CompilationOverhead", 0.0)));
                    auto size = [&c](const char* key)
                    {
                        const Json* s = c.Find(key);
                        return s ? DimensionVector(static_cast<size_t>(s->NumberOr("X", 1)), static_cast<size_t>(s->NumberOr("Y", 1)),
                                       static_cast<size_t>(s->NumberOr("Z", 1)))
                                 : DimensionVector();
                    };
                    cr.SetSizeData(size("GlobalSize"), size("LocalSize"));

                    if (const Json* profiling = c.Find("ProfilingData"))
                    {
                        const uint64_t remaining = static_cast<uint64_t>(profiling->NumberOr("RemainingProfilingRuns", 0.0));
                        auto data = std::make_unique<KernelProfilingData>(remaining);

                        if (remaining == 0)
                        {
                            std::vector<KernelProfilingCounter> counters;

                            if (const Json* list = profiling->Find("Counters"))
                            {
                                for (const auto& k : list->items)
                                {
                                    counters.push_back(CounterFromJson(k));
                                }
                            }

                            data->SetCounters(counters);
                        }

                        cr.SetProfilingData(std::move(data));
                    }

                    computations.push_back(cr);
                }
            }

            KernelResult result(item.StringOr("KernelName", ""), KernelConfiguration(pairs), computations);
            result.SetStatus(StatusFromName(item.StringOr("Status", "Ok")));
            result.SetExtraDuration(ns(item.NumberOr("ExtraDuration", 0.0)));
            result.SetDataMovementOverhead(ns(item.NumberOr("DataMovementOverhead", 0.0)));
            result.SetValidationOverhead(ns(item.NumberOr("ValidationOverhead", 0.0)));
            result.SetSearcherOverhead(ns(item.NumberOr("SearcherOverhead", 0.0)));
            result.SetFailedKernelOverhead(ns(item.NumberOr("FailedKernelOverhead", 0.0)));
            result.SetProfilingRunsOverhead(ns(item.NumberOr("ProfilingRunsOverhead", 0.0)));
            results.push_back(result);
        }

        if (const Json* user = root.Find("UserData"))
        {
            for (const auto& [k, v] : user->members)
            {
                data[k] = v.text;
            }
        }
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
        results.clear();
    }

    return results;
}

} // namespace ktt
