// TuningLoader.cpp -- KTT JSON tuning scripts on the ktt:: surface (see include/ktt/TuningLoader.h).
//
// The script's sections map onto ktt::Tuner calls as KTT's loader maps them
// (TuningLoader/TuningLoader.cpp:58-212, Commands/*.cpp, Deserialization/JsonCommandConverters.cpp):
//   ConfigurationSpace.TuningParameters -> AddScriptParameter     Conditions -> AddScriptConstraint
//   Budget -> UnionCondition of ConfigurationCount / ConfigurationFraction / TuningDuration
//   Search -> Deterministic / Random / MCMC searcher (ProfileBased: SetProfileBasedSearcher)
//   General -> logging level, time unit, output file and format
//   KernelSpecification -> tuner on the device, kernel definition from the file (relative to the
//   script), global size type, Global/LocalSize modifier scripts, compiler options, profiling,
//   Arguments, ReferenceArguments (reference data + validation method), SharedMemory, and
//   SimulationInput (recorded results replayed by SimulateTuning instead of tuning).
// Each section becomes a step with KTT's command priority; the steps run in that order, ties in
// the order they appear in the script.
#include <ktt/TuningLoader.h>

#include <algorithm>
#include <fstream>
#include <functional>
#include <random>
#include <sstream>
#include <stdexcept>

#include "Json.h"
#include "Logger.h"

namespace ktt
{

namespace
{

using json::Json;

// KTT's command priorities (TuningLoader/CommandPriority.h), lowest first.
enum class Stage
{
    Logging, Initialization, General, Kernel, KernelArgument, SharedMemory, TuningParameter, Constraint, Modifier,
    Searcher, StopCondition, Validation, Tuning, Output
};

[[noreturn]] void Bad(const std::string& what)
{
    throw std::runtime_error("Tuning script: " + what);
}

const Json& Need(const Json& object, const std::string& key, const std::string& where)
{
    const Json* v = object.Find(key);

    if (v == nullptr)
    {
        Bad(where + " lacks \"" + key + "\"");
    }

    return *v;
}

std::string Text(const Json& v, const std::string& what)
{
    if (v.kind != Json::Kind::String)
    {
        Bad(what + " must be a string");
    }

    return v.text;
}

double Num(const Json& v, const std::string& what)
{
    if (v.kind != Json::Kind::Number)
    {
        Bad(what + " must be a number");
    }

    return v.number;
}

const std::vector<Json>& Items(const Json& v, const char* what)
{
    if (v.kind != Json::Kind::Array)
    {
        Bad(std::string(what) + " must be an array");
    }

    return v.items;
}

template <typename E>
E Lookup(const std::string& text, const std::vector<std::pair<const char*, E>>& table, const std::string& what)
{
    for (const auto& [name, value] : table)
    {
        if (text == name)
        {
            return value;
        }
    }

    Bad("unknown " + what + " \"" + text + "\"");
}

ParameterValueType ParameterType(const std::string& t)
{
    // TuningLoader/Commands/ParameterCommand.cpp:27-52
    return Lookup<ParameterValueType>(t, {{"int", ParameterValueType::Int}, {"uint", ParameterValueType::UnsignedInt},
        {"float", ParameterValueType::Double}, {"double", ParameterValueType::Double}, {"bool", ParameterValueType::Bool},
        {"string", ParameterValueType::String}}, "parameter type");
}

ArgumentDataType DataType(const std::string& t)
{
    return Lookup<ArgumentDataType>(t, {{"bool", ArgumentDataType::Char}, {"int8", ArgumentDataType::Char},
        {"uint8", ArgumentDataType::UnsignedChar}, {"int16", ArgumentDataType::Short},
        {"uint16", ArgumentDataType::UnsignedShort}, {"int32", ArgumentDataType::Int},
        {"uint32", ArgumentDataType::UnsignedInt}, {"int64", ArgumentDataType::Long},
        {"uint64", ArgumentDataType::UnsignedLong}, {"half", ArgumentDataType::Half}, {"float", ArgumentDataType::Float},
        {"double", ArgumentDataType::Double}}, "argument type");
}

size_t DataTypeSize(const ArgumentDataType t)
{
    switch (t)
    {
    case ArgumentDataType::Char:
    case ArgumentDataType::UnsignedChar: return 1;
    case ArgumentDataType::Short:
    case ArgumentDataType::UnsignedShort:
    case ArgumentDataType::Half: return 2;
    case ArgumentDataType::Int:
    case ArgumentDataType::UnsignedInt:
    case ArgumentDataType::Float: return 4;
    case ArgumentDataType::Long:
    case ArgumentDataType::UnsignedLong:
    case ArgumentDataType::Double: return 8;
    case ArgumentDataType::Custom: break;
    }

    return 0;
}

// One "Arguments" / "ReferenceArguments" entry (Deserialization/JsonCommandConverters.cpp:33-101).
struct ArgumentSpec
{
    ArgumentId id;
    ArgumentMemoryType memoryType = ArgumentMemoryType::Vector;
    ArgumentDataType dataType = ArgumentDataType::Float;
    size_t size = 0;
    size_t typeSize = 0;
    ArgumentAccessType accessType = ArgumentAccessType::ReadWrite;
    std::string fillType = "Constant";
    float fillValue = 0.0f;
    bool seeded = false;
    int seed = 0;
    std::string dataSource;

    static ArgumentSpec FromJson(const Json& j)
    {
        ArgumentSpec a;

        if (const Json* v = j.Find("Name")) a.id = Text(*v, "argument Name");
        if (const Json* v = j.Find("MemoryType"))
        {
            a.memoryType = Lookup<ArgumentMemoryType>(Text(*v, "MemoryType"), {{"Scalar", ArgumentMemoryType::Scalar},
                {"Vector", ArgumentMemoryType::Vector}, {"Local", ArgumentMemoryType::Local},
                {"Symbol", ArgumentMemoryType::Symbol}}, "memory type");
        }
        if (const Json* v = j.Find("Type")) a.dataType = DataType(Text(*v, "argument Type"));
        if (const Json* v = j.Find("Size")) a.size = static_cast<size_t>(Num(*v, "argument Size"));
        if (const Json* v = j.Find("TypeSize")) a.typeSize = static_cast<size_t>(Num(*v, "argument TypeSize"));
        if (const Json* v = j.Find("AccessType"))
        {
            a.accessType = Lookup<ArgumentAccessType>(Text(*v, "AccessType"), {{"Undefined", ArgumentAccessType::Undefined},
                {"ReadOnly", ArgumentAccessType::ReadOnly}, {"WriteOnly", ArgumentAccessType::WriteOnly},
                {"ReadWrite", ArgumentAccessType::ReadWrite}}, "access type");
        }
        if (const Json* v = j.Find("FillType")) a.fillType = Text(*v, "FillType");

        if (a.fillType == "Constant" || a.fillType == "Random")
        {
            if (const Json* v = j.Find("FillValue"))
            {
                a.fillValue = static_cast<float>(Num(*v, "FillValue"));
            }
            else if (j.Find("TargetName") == nullptr)
            {
                Bad("argument " + a.id + " lacks \"FillValue\"");
            }

            if (const Json* v = j.Find("RandomSeed"))
            {
                a.seeded = true;
                a.seed = static_cast<int>(Num(*v, "RandomSeed"));
            }
        }
        else if (a.fillType == "Generator" || a.fillType == "BinaryRaw")
        {
            a.dataSource = Text(Need(j, "DataSource", "argument " + a.id), "DataSource");
        }
        else
        {
            Bad("argument fill type \"" + a.fillType + "\" is not supported (Constant, Random, Generator, BinaryRaw)");
        }

        return a;
    }
};

} // namespace

struct TuningLoader::Impl
{
    std::string directory;
    std::vector<std::pair<Stage, std::function<void()>>> steps;
    bool loaded = false;

    std::unique_ptr<Tuner> tuner;
    KernelDefinitionId definition = InvalidKernelDefinitionId;
    KernelId kernel = InvalidKernelId;
    std::vector<ArgumentId> arguments;
    std::unique_ptr<StopCondition> stop;
    std::vector<KernelResult> results;

    Tuner& GetTuner()
    {
        if (!tuner)
        {
            Bad("no tuner was created");
        }

        return *tuner;
    }

    std::string FullPath(const std::string& file) const
    {
        // TuningLoader/TunerContext.cpp: paths in the script are relative to the script's directory
        if (directory.empty() || (!file.empty() && file[0] == '/'))
        {
            return file;
        }

        return directory + "/" + file;
    }

    void Add(const Stage stage, std::function<void()> step) { steps.emplace_back(stage, std::move(step)); }

    ArgumentId SubmitArgument(const ArgumentSpec& a)
    {
        Tuner& t = GetTuner();

        if (a.memoryType == ArgumentMemoryType::Local || a.memoryType == ArgumentMemoryType::Symbol)
        {
            Bad("argument " + a.id + ": local and symbol arguments are not supported");
        }

        if (a.memoryType == ArgumentMemoryType::Scalar)
        {
            // TuningLoader/Commands/AddArgumentCommand.cpp:78-88: int or float scalars from FillValue
            if (a.dataType == ArgumentDataType::Int)
            {
                return t.AddArgumentScalar(static_cast<int>(a.fillValue), a.id);
            }

            if (a.dataType == ArgumentDataType::Float)
            {
                return t.AddArgumentScalar(a.fillValue, a.id);
            }

            Bad("scalar argument " + a.id + " must be int32 or float");
        }

        const size_t typeSize = a.typeSize != 0 ? a.typeSize : DataTypeSize(a.dataType);

        if (a.fillType == "Constant")
        {
            return t.AddArgumentVector(std::vector<float>(a.size, a.fillValue), a.accessType, a.id);
        }

        if (a.fillType == "Random")
        {
            // uniform in [0, FillValue), seeded when the script gives RandomSeed
            std::default_random_engine engine(a.seeded ? static_cast<unsigned>(a.seed) : std::random_device{}());
            std::uniform_real_distribution<float> distribution(0.0f, a.fillValue);
            std::vector<float> data(a.size);

            for (auto& x : data)
            {
                x = distribution(engine);
            }

            return t.AddArgumentVector(data, a.accessType, a.id);
        }

        if (a.fillType == "Generator")
        {
            return t.AddArgumentVectorFromGenerator(a.dataSource, a.dataType, a.size * typeSize, typeSize, a.accessType,
                ArgumentMemoryLocation::Device, ArgumentManagementType::Framework, a.id);
        }

        return t.AddArgumentVectorFromFile(FullPath(a.dataSource), a.dataType, typeSize, a.accessType,
            ArgumentMemoryLocation::Device, ArgumentManagementType::Framework, a.id);
    }

    void Deserialize(const Json& root);
};

void TuningLoader::Impl::Deserialize(const Json& root)
{
    if (root.kind != Json::Kind::Object)
    {
        Bad("the document must be a JSON object");
    }

    if (const Json* space = root.Find("ConfigurationSpace"))
    {
        if (const Json* parameters = space->Find("TuningParameters"))
        {
            for (const Json& p : Items(*parameters, "TuningParameters"))
            {
                const std::string name = Text(Need(p, "Name", "a tuning parameter"), "parameter Name");
                const ParameterValueType type = ParameterType(Text(Need(p, "Type", "parameter " + name), "parameter Type"));
                const std::string values = Text(Need(p, "Values", "parameter " + name), "parameter Values");
                Add(Stage::TuningParameter, [this, name, type, values] { GetTuner().AddScriptParameter(kernel, name, type, values); });
            }
        }

        if (const Json* conditions = space->Find("Conditions"))
        {
            for (const Json& c : Items(*conditions, "Conditions"))
            {
                std::vector<std::string> names;

                const Json* listed = c.Find("Parameters");

                if (listed == nullptr)
                {
                    Bad("a condition lacks \"Parameters\"");
                }

                for (const Json& n : Items(*listed, "condition Parameters"))
                {
                    names.push_back(Text(n, "condition parameter"));
                }

                const std::string expression = Text(Need(c, "Expression", "a condition"), "condition Expression");
                Add(Stage::Constraint, [this, names, expression] { GetTuner().AddScriptConstraint(kernel, names, expression); });
            }
        }
    }

    if (const Json* budget = root.Find("Budget"))
    {
        std::vector<std::pair<std::string, double>> budgets;

        for (const Json& b : Items(*budget, "Budget"))
        {
            budgets.emplace_back(Text(Need(b, "Type", "a budget"), "budget Type"), Num(Need(b, "BudgetValue", "a budget"),
                "BudgetValue"));
        }

        Add(Stage::StopCondition, [this, budgets]
        {
            std::vector<std::shared_ptr<StopCondition>> conditions;

            for (const auto& [type, value] : budgets)
            {
                if (type == "ConfigurationCount")
                    conditions.push_back(std::make_shared<ConfigurationCount>(static_cast<uint64_t>(value)));
                else if (type == "ConfigurationFraction")
                    conditions.push_back(std::make_shared<ConfigurationFraction>(value));
                else if (type == "TuningDuration")
                    conditions.push_back(std::make_shared<TuningDuration>(value));
                else
                    Bad("unknown budget type \"" + type + "\"");
            }

            stop = std::make_unique<UnionCondition>(conditions);
        });
    }

    if (const Json* search = root.Find("Search"))
    {
        const std::string name = Text(Need(*search, "Name", "Search"), "searcher Name");
        std::map<std::string, std::string> attributes;

        if (const Json* list = search->Find("Attributes"))
        {
            for (const Json& a : Items(*list, "searcher Attributes"))
            {
                attributes[Text(Need(a, "Name", "a searcher attribute"), "attribute Name")]
                    = Text(Need(a, "Value", "a searcher attribute"), "attribute Value");
            }
        }

        if (name != "Deterministic" && name != "Random" && name != "MCMC" && name != "ProfileBased")
        {
            Bad("unknown searcher \"" + name + "\"");
        }

        Add(Stage::Searcher, [this, name, attributes]
        {
            Tuner& t = GetTuner();

            if (name == "Deterministic") t.SetSearcher(kernel, std::make_unique<DeterministicSearcher>());
            else if (name == "Random") t.SetSearcher(kernel, std::make_unique<RandomSearcher>());
            else if (name == "MCMC") t.SetSearcher(kernel, std::make_unique<McmcSearcher>());
            else
            {
                auto get = [&](const char* key, const uint32_t fallback)
                {
                    auto it = attributes.find(key);
                    return it == attributes.end() ? fallback : static_cast<uint32_t>(std::stoul(it->second));
                };
                auto model = attributes.find("modelPath");
                t.SetProfileBasedSearcher(kernel, model == attributes.end() ? "" : model->second, true, get("batchSize", 5),
                    get("neighborSize", 100), get("randomSize", 10));
            }
        });
    }

    if (const Json* general = root.Find("General"))
    {
        if (const Json* level = general->Find("LoggingLevel"))
        {
            const LoggingLevel l = Lookup<LoggingLevel>(Text(*level, "LoggingLevel"), {{"Off", LoggingLevel::Off},
                {"Error", LoggingLevel::Error}, {"Warning", LoggingLevel::Warning}, {"Info", LoggingLevel::Info},
                {"Debug", LoggingLevel::Debug}}, "logging level");
            Add(Stage::Logging, [l] { Tuner::SetLoggingLevel(l); });
        }

        if (const Json* unit = general->Find("TimeUnit"))
        {
            const TimeUnit u = Lookup<TimeUnit>(Text(*unit, "TimeUnit"), {{"Nanoseconds", TimeUnit::Nanoseconds},
                {"Microseconds", TimeUnit::Microseconds}, {"Milliseconds", TimeUnit::Milliseconds},
                {"Seconds", TimeUnit::Seconds}}, "time unit");
            Add(Stage::General, [u] { Tuner::SetTimeUnit(u); });
        }

        if (const Json* file = general->Find("OutputFile"))
        {
            const std::string path = Text(*file, "OutputFile");
            OutputFormat format = OutputFormat::JSON;

            if (const Json* f = general->Find("OutputFormat"))
            {
                format = Lookup<OutputFormat>(Text(*f, "OutputFormat"), {{"JSON", OutputFormat::JSON}, {"XML", OutputFormat::XML}},
                    "output format");
            }

            Add(Stage::Output, [this, path, format] { GetTuner().SaveResults(results, path, format); });
        }
    }

    const Json* spec = root.Find("KernelSpecification");

    if (spec == nullptr)
    {
        Bad("the script has no KernelSpecification, so there is nothing to tune");
    }

    const std::string language = Text(Need(*spec, "Language", "KernelSpecification"), "Language");

    if (language != "CUDA")
    {
        Bad("kernel language " + language + " is not supported: this library runs CUDA kernels on sm_100a only");
    }

    DeviceIndex device = 0;

    if (const Json* d = spec->Find("Device"))
    {
        if (const Json* id = d->Find("DeviceId"))
        {
            device = static_cast<DeviceIndex>(Num(*id, "DeviceId"));
        }
    }

    Add(Stage::Initialization, [this, device] { tuner = std::make_unique<Tuner>(0, device, ComputeApi::CUDA); });

    const std::string kernelName = Text(Need(*spec, "KernelName", "KernelSpecification"), "KernelName");
    const std::string kernelFile = Text(Need(*spec, "KernelFile", "KernelSpecification"), "KernelFile");
    std::vector<std::string> typeNames;

    if (const Json* names = spec->Find("KernelTypeNames"))
    {
        for (const Json& n : Items(*names, "KernelTypeNames"))
        {
            typeNames.push_back(Text(n, "kernel type name"));
        }
    }

    Add(Stage::Kernel, [this, kernelName, kernelFile, typeNames]
    {
        definition = GetTuner().AddKernelDefinitionFromFile(kernelName, FullPath(kernelFile), typeNames);

        if (definition == InvalidKernelDefinitionId)
        {
            Bad("kernel definition " + kernelName + " could not be added");
        }

        kernel = GetTuner().CreateSimpleKernel(kernelName + "_kernel", definition);
    });

    if (const Json* type = spec->Find("GlobalSizeType"))
    {
        const GlobalSizeType g = Lookup<GlobalSizeType>(Text(*type, "GlobalSizeType"), {{"OpenCL", GlobalSizeType::OpenCL},
            {"CUDA", GlobalSizeType::CUDA}, {"Vulkan", GlobalSizeType::Vulkan}}, "global size type");
        Add(Stage::General, [this, g] { GetTuner().SetGlobalSizeType(g); });
    }

    for (const auto& [section, type] : {std::make_pair("GlobalSize", ModifierType::Global),
             std::make_pair("LocalSize", ModifierType::Local)})
    {
        const Json* sizes = spec->Find(section);

        if (sizes == nullptr)
        {
            continue;
        }

        for (const auto& [key, dimension] : {std::make_pair("X", ModifierDimension::X), std::make_pair("Y", ModifierDimension::Y),
                 std::make_pair("Z", ModifierDimension::Z)})
        {
            if (const Json* s = sizes->Find(key))
            {
                const std::string script = Text(*s, std::string(section) + "." + key);
                const ModifierType modifierType = type;
                const ModifierDimension modifierDimension = dimension;
                Add(Stage::Modifier, [this, script, modifierType, modifierDimension]
                {
                    GetTuner().AddScriptThreadModifier(kernel, {definition}, modifierType, modifierDimension, script);
                });
            }
        }
    }

    if (const Json* options = spec->Find("CompilerOptions"))
    {
        std::string joined;

        for (const Json& o : Items(*options, "CompilerOptions"))
        {
            joined += (joined.empty() ? "" : " ") + Text(o, "compiler option");
        }

        Add(Stage::General, [this, joined] { GetTuner().SetCompilerOptions(joined); });
    }

    if (const Json* profiling = spec->Find("Profiling"))
    {
        if (profiling->kind != Json::Kind::Bool)
        {
            Bad("Profiling must be true or false");
        }

        const bool on = profiling->boolean;
        Add(Stage::General, [this, on] { GetTuner().SetProfiling(on); });
    }

    std::vector<ArgumentSpec> argumentSpecs;

    if (const Json* list = spec->Find("Arguments"))
    {
        for (const Json& a : Items(*list, "Arguments"))
        {
            argumentSpecs.push_back(ArgumentSpec::FromJson(a));
            const ArgumentSpec argument = argumentSpecs.back();
            Add(Stage::KernelArgument, [this, argument]
            {
                const ArgumentId id = SubmitArgument(argument);

                if (id == InvalidArgumentId)
                {
                    Bad("argument " + argument.id + " could not be added");
                }

                arguments.push_back(id);
                GetTuner().SetArguments(definition, arguments);
            });
        }
    }

    if (const Json* list = spec->Find("ReferenceArguments"))
    {
        for (const Json& r : Items(*list, "ReferenceArguments"))
        {
            const ArgumentId target = Text(Need(r, "TargetName", "a reference argument"), "TargetName");
            ArgumentSpec reference = ArgumentSpec::FromJson(r);
            // the reference takes the shape of the argument it validates (ValidationCommand.cpp:29-40)
            auto it = std::find_if(argumentSpecs.cbegin(), argumentSpecs.cend(), [&](const ArgumentSpec& a) { return a.id == target; });

            if (it == argumentSpecs.cend())
            {
                Bad("reference argument " + reference.id + " names an unknown target " + target);
            }

            reference.memoryType = it->memoryType;
            reference.dataType = it->dataType;
            reference.size = it->size;
            reference.typeSize = it->typeSize;
            reference.accessType = it->accessType;
            ValidationMethod method = ValidationMethod::SideBySideComparison;
            double threshold = 1e-4;

            if (const Json* m = r.Find("ValidationMethod"))
            {
                method = Lookup<ValidationMethod>(Text(*m, "ValidationMethod"), {{"AbsoluteDifference",
                    ValidationMethod::AbsoluteDifference}, {"SideBySideComparison", ValidationMethod::SideBySideComparison},
                    {"SideBySideRelativeComparison", ValidationMethod::SideBySideRelativeComparison}}, "validation method");
            }

            if (const Json* v = r.Find("ValidationThreshold"))
            {
                threshold = Num(*v, "ValidationThreshold");
            }

            Add(Stage::Validation, [this, target, reference, method, threshold]
            {
                const ArgumentId id = SubmitArgument(reference);

                if (id == InvalidArgumentId)
                {
                    Bad("reference argument " + reference.id + " could not be added");
                }

                GetTuner().SetValidationMethod(method, threshold);
                GetTuner().SetReferenceArgument(target, id);
            });
        }
    }

    if (const Json* shared = spec->Find("SharedMemory"))
    {
        const double bytes = Num(*shared, "SharedMemory");
        // The built-in kernels size their own shared memory (TMA atom rings); the request is recorded.
        Add(Stage::SharedMemory, [bytes] { log::Debug("SharedMemory " + std::to_string(bytes) + " bytes requested by the script"); });
    }

    std::string simulation;

    if (const Json* input = spec->Find("SimulationInput"))
    {
        simulation = Text(*input, "SimulationInput");
    }

    Add(Stage::Tuning, [this, simulation]
    {
        Tuner& t = GetTuner();

        if (simulation.empty())
        {
            results = t.Tune(kernel, std::move(stop));
        }
        else
        {
            const auto recorded = t.LoadResults(FullPath(simulation), OutputFormat::JSON);
            results = t.SimulateTuning(kernel, recorded, std::move(stop));
        }
    });
}

TuningLoader::TuningLoader() : m_Impl(std::make_unique<Impl>()) {}
TuningLoader::~TuningLoader() = default;

void TuningLoader::LoadTuningFile(const std::string& file, const std::map<std::string, std::string>& parameters)
{
    std::ifstream input(file);

    if (!input)
    {
        throw std::runtime_error("Unable to open file: " + file);
    }

    std::stringstream buffer;
    buffer << input.rdbuf();
    std::string text = buffer.str();

    // "$NAME" placeholders take the given values (TuningLoader.cpp:245-259)
    for (const auto& [name, value] : parameters)
    {
        const std::string token = "$" + name;

        for (size_t pos = text.find(token); pos != std::string::npos; pos = text.find(token, pos + value.size()))
        {
            text.replace(pos, token.size(), value);
        }
    }

    const auto slash = file.find_last_of('/');
    m_Impl->directory = slash == std::string::npos ? "" : file.substr(0, slash);
    m_Impl->steps.clear();
    m_Impl->Deserialize(json::Parser(text).Parse());
    std::stable_sort(m_Impl->steps.begin(), m_Impl->steps.end(),
        [](const auto& a, const auto& b) { return static_cast<int>(a.first) < static_cast<int>(b.first); });
    m_Impl->loaded = true;
}

void TuningLoader::ExecuteCommands()
{
    if (!m_Impl->loaded)
    {
        throw std::runtime_error("ExecuteCommands called before LoadTuningFile");
    }

    for (auto& [stage, step] : m_Impl->steps)
    {
        step();
    }
}

Tuner& TuningLoader::GetTuner() { return m_Impl->GetTuner(); }
KernelId TuningLoader::GetKernelId() const { return m_Impl->kernel; }
const std::vector<KernelResult>& TuningLoader::GetResults() const { return m_Impl->results; }

} // namespace ktt
