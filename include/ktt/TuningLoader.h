// TuningLoader.h -- KTT's JSON tuning-script front end on the ktt:: surface.
//
// Same role and interface as KTT 2.1.0's TuningLoader (TuningLoader/TuningLoader.h,
// TuningLoader.cpp:28-263, TuningLauncher.cpp): a script describes the configuration space
// (parameters with Python list scripts, conditions as Python expressions), the searcher, the budget,
// output, and the kernel (name, file, global/local size scripts, arguments with constant, random,
// generated or file data, reference data for validation, an optional recorded-results file for
// simulated tuning).  LoadTuningFile substitutes "$NAME" placeholders with the given parameters,
// checks the script and turns it into steps; ExecuteCommands runs them in KTT's order (logging,
// tuner creation, general settings, kernel, arguments, shared memory, parameters, constraints,
// modifiers, searcher, budget, validation, tuning, output).  Kernels are matched to this library's
// built-in sm_100a implementations by name and argument list, as for any ktt::Tuner program; only
// CUDA scripts are accepted.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include <ktt/Tuner.h>

namespace ktt
{

class KTT_API TuningLoader
{
public:
    TuningLoader();
    ~TuningLoader();

    // Throws std::runtime_error when the file cannot be read or the script is malformed.
    void LoadTuningFile(const std::string& file, const std::map<std::string, std::string>& parameters = {});
    void ExecuteCommands();

    // After ExecuteCommands: the tuner the script created, its kernel and the tuning results.
    Tuner& GetTuner();
    KernelId GetKernelId() const;
    const std::vector<KernelResult>& GetResults() const;

private:
    struct Impl;
    std::unique_ptr<Impl> m_Impl;
};

} // namespace ktt
