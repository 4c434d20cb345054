// CPU test driver for the script evaluator and the JSON tuning-script loader of libktt_b200.so
// (driven by tests/test_loader_cpu.py).
//
//   loader_cpu_tests eval                      expressions on stdin, one per line; prints one typed
//                                              result per line: "int 3", "float 3.5", "bool 1",
//                                              "list [int 1, float 2]" or "error <message>"
//   loader_cpu_tests generator <expr> <n> <file>
//                                              FP32 vector from a generator script, saved raw
//   loader_cpu_tests script <script.json> [NAME=VALUE ...]
//                                              loads and runs a tuning script in the current
//                                              directory; prints "results <n> configurations <m>
//                                              best <NAME=VALUE,...>"
//   loader_cpu_tests space                     parameters/constraints/modifiers given as scripts
//                                              give KTT's 210-configuration CoulombSum3d space
#include <cmath>
#include <cstdio>
#include <iostream>
#include <map>
#include <sstream>
#include <string>

#include <Ktt.h>

#include "ktt/Script.h"

namespace
{

std::string Show(const ktt::script::Value& v)
{
    using K = ktt::script::Value::Kind;
    std::ostringstream out;

    switch (v.kind)
    {
    case K::Int: out << "int " << v.i; break;
    case K::Bool: out << "bool " << v.i; break;
    case K::Float:
    {
        char buffer[64];
        std::snprintf(buffer, sizeof buffer, "float %.17g", v.f);
        out << buffer;
        break;
    }
    case K::List:
        out << "list [";
        for (size_t k = 0; k < v.list.size(); ++k)
        {
            out << (k ? ", " : "") << Show(v.list[k]);
        }
        out << "]";
        break;
    }

    return out.str();
}

int Eval()
{
    std::string line;

    while (std::getline(std::cin, line))
    {
        try
        {
            ktt::script::Environment env;
            env.Set("a", ktt::script::Value::Int(7));
            env.Set("b", ktt::script::Value::Int(-3));
            env.Set("x", ktt::script::Value::Float(2.5));
            std::cout << Show(ktt::script::Expression(line).Evaluate(env)) << "\n";
        }
        catch (const std::exception& e)
        {
            std::string message = e.what();

            for (auto& c : message)
            {
                if (c == '\n') c = ' ';
            }

            std::cout << "error " << message << "\n";
        }
    }

    return 0;
}

int Generator(const std::string& expression, const size_t count, const std::string& file)
{
    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    const ktt::ArgumentId id = tuner.AddArgumentVectorFromGenerator(expression, ktt::ArgumentDataType::Float, count * 4, 4,
        ktt::ArgumentAccessType::ReadOnly);

    if (id == ktt::InvalidArgumentId)
    {
        return 2;
    }

    tuner.SaveArgumentVector(id, file);
    return 0;
}

int Script(const std::string& path, const std::map<std::string, std::string>& parameters)
{
    ktt::TuningLoader loader;
    loader.LoadTuningFile(path, parameters);
    loader.ExecuteCommands();
    const auto& results = loader.GetResults();
    const ktt::KernelResult* best = nullptr;

    for (const auto& r : results)
    {
        if (r.IsValid() && (best == nullptr || r.GetTotalDuration() < best->GetTotalDuration()))
        {
            best = &r;
        }
    }

    std::cout << "results " << results.size() << " configurations "
              << loader.GetTuner().GetConfigurationsCount(loader.GetKernelId()) << " best ";

    if (best != nullptr)
    {
        bool first = true;

        for (const auto& pair : best->GetConfiguration().GetPairs())
        {
            std::cout << (first ? "" : ",") << pair.GetName() << "=" << pair.GetValueString();
            first = false;
        }
    }

    std::cout << "\n";
    return 0;
}

int Space()
{
    ktt::Tuner tuner(0, 0, ktt::ComputeApi::CUDA);
    const auto def = tuner.AddKernelDefinition("directCoulombSum", "", std::vector<std::string>{});
    const auto kernel = tuner.CreateSimpleKernel("CoulombSum", def);
    tuner.AddScriptParameter(kernel, "WORK_GROUP_SIZE_X", ktt::ParameterValueType::UnsignedInt, "[16, 32]");
    tuner.AddScriptParameter(kernel, "WORK_GROUP_SIZE_Y", ktt::ParameterValueType::UnsignedInt, "[2**k for k in range(4)]");
    tuner.AddScriptParameter(kernel, "Z_ITERATIONS", ktt::ParameterValueType::UnsignedInt, "[1, 2, 4, 8, 16, 32]");
    tuner.AddScriptParameter(kernel, "INNER_UNROLL_FACTOR", ktt::ParameterValueType::UnsignedInt, "[0] + [2**k for k in range(6)]");
    tuner.AddScriptParameter(kernel, "USE_SOA", ktt::ParameterValueType::UnsignedInt, "list(range(2))");
    tuner.AddScriptConstraint(kernel, {"INNER_UNROLL_FACTOR", "Z_ITERATIONS"}, "INNER_UNROLL_FACTOR < Z_ITERATIONS");
    tuner.AddScriptConstraint(kernel, {"WORK_GROUP_SIZE_X", "WORK_GROUP_SIZE_Y"}, "WORK_GROUP_SIZE_X * WORK_GROUP_SIZE_Y >= 64");
    tuner.AddScriptThreadModifier(kernel, {def}, ktt::ModifierType::Global, ktt::ModifierDimension::Z, "256 // Z_ITERATIONS");
    const uint64_t count = tuner.GetConfigurationsCount(kernel);
    std::cout << "configurations " << count << "\n";

    // a script naming something that is not a parameter is rejected (logged), leaving the count
    tuner.AddScriptThreadModifier(kernel, {def}, ktt::ModifierType::Local, ktt::ModifierDimension::X, "NOT_A_PARAMETER * 2");
    return count == 210 ? 0 : 3;
}

} // namespace

int main(int argc, char** argv)
{
    ktt::Tuner::SetLoggingLevel(ktt::LoggingLevel::Warning);

    if (argc < 2)
    {
        std::cerr << "usage: loader_cpu_tests eval|generator|script|space ..." << std::endl;
        return 1;
    }

    const std::string mode = argv[1];

    try
    {
        if (mode == "eval") return Eval();
        if (mode == "generator" && argc == 5) return Generator(argv[2], std::stoul(argv[3]), argv[4]);
        if (mode == "space") return Space();

        if (mode == "script" && argc >= 3)
        {
            std::map<std::string, std::string> parameters;

            for (int i = 3; i < argc; ++i)
            {
                const std::string token = argv[i];
                const auto eq = token.find('=');
                parameters[token.substr(0, eq)] = token.substr(eq + 1);
            }

            return Script(argv[2], parameters);
        }
    }
    catch (const std::exception& e)
    {
        std::cout << "error " << e.what() << std::endl;
        return 4;
    }

    std::cerr << "bad arguments" << std::endl;
    return 1;
}
