// pyktt.cpp -- the Python module of the ktt:: surface, under KTT's module name and method names.
//
// KTT ships its Python API as the pybind11 module "pyktt" (Source/Python/PythonModule.cpp:16,
// PythonTuner.cpp, PythonDataHolders.cpp, PythonEnums.cpp, PythonSearchers.cpp,
// PythonStopConditions.cpp, PythonComputeInterface.cpp).  This module binds libktt_b200.so the same
// way, so a KTT Python host program for the Coulomb path runs with
//
//     from ktt_b200 import pyktt as ktt        # instead of: import pyktt as ktt
//
// Types and typed entry points keep KTT's Python names (AddArgumentVectorFloat,
// AddArgumentScalarInt, AddParameter, BufferOutputDescriptor(id, buffer), SetReferenceComputation(id,
// size, function(memoryview)), ...).  Vector arguments are taken from any buffer-protocol object
// (NumPy arrays, array.array, lists are converted); long calls (Tune, TuneIteration, Run,
// SimulateTuning) release the GIL, and Python callbacks (constraints, modifiers, launchers,
// reference computations) take it back.  Searchers and stop conditions passed to the tuner are
// owned by it afterwards, as in C++.
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <Ktt.h>

namespace py = pybind11;

namespace
{

// Python subclasses of StopCondition (KTT: PythonStopConditions.cpp:12-36).
class PyStopCondition : public ktt::StopCondition, public py::trampoline_self_life_support
{
public:
    using ktt::StopCondition::StopCondition;

    bool IsFulfilled() const override { PYBIND11_OVERRIDE_PURE(bool, ktt::StopCondition, IsFulfilled); }
    void Initialize(const uint64_t count) override { PYBIND11_OVERRIDE_PURE(void, ktt::StopCondition, Initialize, count); }
    void Update(const ktt::KernelResult& result) override { PYBIND11_OVERRIDE_PURE(void, ktt::StopCondition, Update, result); }
    std::string GetStatusString() const override { PYBIND11_OVERRIDE_PURE(std::string, ktt::StopCondition, GetStatusString); }
};

template <typename T>
std::vector<T> VectorFrom(const py::array_t<T, py::array::c_style | py::array::forcecast>& data)
{
    const T* p = data.data();
    return std::vector<T>(p, p + data.size());
}

template <typename T, typename C>
void BindVectorArgument(C& tuner, const char* name)
{
    tuner.def(name,
        [](ktt::Tuner& t, const py::array_t<T, py::array::c_style | py::array::forcecast>& data,
            const ktt::ArgumentAccessType access, const ktt::ArgumentId& customId)
        {
            return t.AddArgumentVector(VectorFrom<T>(data), access, customId);
        },
        py::arg("data"), py::arg("accessType"), py::arg("customId") = ktt::ArgumentId());
}

template <typename T, typename C>
void BindScalarArgument(C& tuner, const char* name)
{
    tuner.def(name, [](ktt::Tuner& t, const T value, const ktt::ArgumentId& customId) { return t.AddArgumentScalar(value, customId); },
        py::arg("data"), py::arg("customId") = ktt::ArgumentId());
}

template <typename T, typename C>
void BindLocalArgument(C& tuner, const char* name)
{
    tuner.def(name, [](ktt::Tuner& t, const size_t size, const ktt::ArgumentId& customId) { return t.AddArgumentLocal<T>(size, customId); },
        py::arg("localMemorySize"), py::arg("customId") = ktt::ArgumentId());
}

// Keyword names as KTT's module gives them (data, symbolName, customId), each passed to its C++ meaning.
template <typename T, typename C>
void BindSymbolArgument(C& tuner, const char* name)
{
    tuner.def(name, [](ktt::Tuner& t, const T value, const std::string& symbolName, const ktt::ArgumentId& customId)
        { return t.AddArgumentSymbol<T>(value, customId, symbolName); },
        py::arg("data"), py::arg("symbolName") = std::string(), py::arg("customId") = ktt::ArgumentId());
}

template <typename T, typename C>
void BindScalarUpdate(C& ci, const char* name)
{
    ci.def(name, [](ktt::ComputeInterface& c, const ktt::ArgumentId& id, const T value) { c.UpdateScalarArgument(id, &value); });
}

} // namespace

PYBIND11_MODULE(pyktt, m)
{
    m.doc() = "B200-native ktt:: surface for the direct Coulomb summation path (KTT 2.1.0 Python API names)";
    m.def("GetKttVersion", [] { return (2u << 16) | (1u << 8); });
    m.def("GetKttVersionString", [] { return std::string("2.1.0"); });
    m.attr("InvalidQueueId") = ktt::InvalidQueueId;
    m.attr("InvalidKernelDefinitionId") = ktt::InvalidKernelDefinitionId;
    m.attr("InvalidKernelId") = ktt::InvalidKernelId;
    m.attr("InvalidArgumentId") = ktt::InvalidArgumentId;
    m.attr("InvalidDuration") = ktt::InvalidDuration;

    // ---- enums (PythonEnums.cpp) ----
    py::enum_<ktt::ArgumentAccessType>(m, "ArgumentAccessType")
        .value("Undefined", ktt::ArgumentAccessType::Undefined).value("ReadOnly", ktt::ArgumentAccessType::ReadOnly)
        .value("WriteOnly", ktt::ArgumentAccessType::WriteOnly).value("ReadWrite", ktt::ArgumentAccessType::ReadWrite);
    py::enum_<ktt::ArgumentDataType>(m, "ArgumentDataType")
        .value("Char", ktt::ArgumentDataType::Char).value("UnsignedChar", ktt::ArgumentDataType::UnsignedChar)
        .value("Short", ktt::ArgumentDataType::Short).value("UnsignedShort", ktt::ArgumentDataType::UnsignedShort)
        .value("Int", ktt::ArgumentDataType::Int).value("UnsignedInt", ktt::ArgumentDataType::UnsignedInt)
        .value("Long", ktt::ArgumentDataType::Long).value("UnsignedLong", ktt::ArgumentDataType::UnsignedLong)
        .value("Half", ktt::ArgumentDataType::Half).value("Float", ktt::ArgumentDataType::Float)
        .value("Double", ktt::ArgumentDataType::Double).value("Custom", ktt::ArgumentDataType::Custom);
    py::enum_<ktt::ArgumentManagementType>(m, "ArgumentManagementType")
        .value("Framework", ktt::ArgumentManagementType::Framework).value("User", ktt::ArgumentManagementType::User);
    py::enum_<ktt::ArgumentMemoryLocation>(m, "ArgumentMemoryLocation")
        .value("Undefined", ktt::ArgumentMemoryLocation::Undefined).value("Device", ktt::ArgumentMemoryLocation::Device)
        .value("Host", ktt::ArgumentMemoryLocation::Host).value("HostZeroCopy", ktt::ArgumentMemoryLocation::HostZeroCopy)
        .value("Unified", ktt::ArgumentMemoryLocation::Unified);
    py::enum_<ktt::ArgumentMemoryType>(m, "ArgumentMemoryType")
        .value("Scalar", ktt::ArgumentMemoryType::Scalar).value("Vector", ktt::ArgumentMemoryType::Vector)
        .value("Local", ktt::ArgumentMemoryType::Local).value("Symbol", ktt::ArgumentMemoryType::Symbol);
    py::enum_<ktt::ComputeApi>(m, "ComputeApi")
        .value("OpenCL", ktt::ComputeApi::OpenCL).value("CUDA", ktt::ComputeApi::CUDA).value("Vulkan", ktt::ComputeApi::Vulkan);
    py::enum_<ktt::ExceptionReason>(m, "ExceptionReason")
        .value("General", ktt::ExceptionReason::General).value("CompilerError", ktt::ExceptionReason::CompilerError)
        .value("DeviceLimitsExceeded", ktt::ExceptionReason::DeviceLimitsExceeded);
    py::enum_<ktt::GlobalSizeType>(m, "GlobalSizeType")
        .value("OpenCL", ktt::GlobalSizeType::OpenCL).value("CUDA", ktt::GlobalSizeType::CUDA)
        .value("Vulkan", ktt::GlobalSizeType::Vulkan);
    py::enum_<ktt::KernelRunMode>(m, "KernelRunMode")
        .value("Running", ktt::KernelRunMode::Running).value("OfflineTuning", ktt::KernelRunMode::OfflineTuning)
        .value("OnlineTuning", ktt::KernelRunMode::OnlineTuning).value("ResultValidation", ktt::KernelRunMode::ResultValidation);
    py::enum_<ktt::DeviceType>(m, "DeviceType")
        .value("CPU", ktt::DeviceType::CPU)
        .value("GPU", ktt::DeviceType::GPU)
        .value("Custom", ktt::DeviceType::Custom);

    py::enum_<ktt::LoggingLevel>(m, "LoggingLevel")
        .value("Off", ktt::LoggingLevel::Off).value("Error", ktt::LoggingLevel::Error).value("Warning", ktt::LoggingLevel::Warning)
        .value("Info", ktt::LoggingLevel::Info).value("Debug", ktt::LoggingLevel::Debug);
    py::enum_<ktt::ModifierAction>(m, "ModifierAction")
        .value("Add", ktt::ModifierAction::Add).value("Subtract", ktt::ModifierAction::Subtract)
        .value("Multiply", ktt::ModifierAction::Multiply).value("Divide", ktt::ModifierAction::Divide)
        .value("DivideCeil", ktt::ModifierAction::DivideCeil);
    py::enum_<ktt::ModifierDimension>(m, "ModifierDimension")
        .value("X", ktt::ModifierDimension::X).value("Y", ktt::ModifierDimension::Y).value("Z", ktt::ModifierDimension::Z);
    py::enum_<ktt::ModifierType>(m, "ModifierType")
        .value("Global", ktt::ModifierType::Global).value("Local", ktt::ModifierType::Local);
    py::enum_<ktt::OutputFormat>(m, "OutputFormat").value("JSON", ktt::OutputFormat::JSON).value("XML", ktt::OutputFormat::XML);
    py::enum_<ktt::ParameterValueType>(m, "ParameterValueType")
        .value("Int", ktt::ParameterValueType::Int).value("UnsignedInt", ktt::ParameterValueType::UnsignedInt)
        .value("Double", ktt::ParameterValueType::Double).value("Bool", ktt::ParameterValueType::Bool)
        .value("String", ktt::ParameterValueType::String);
    py::enum_<ktt::ResultStatus>(m, "ResultStatus")
        .value("Ok", ktt::ResultStatus::Ok).value("ComputationFailed", ktt::ResultStatus::ComputationFailed)
        .value("ValidationFailed", ktt::ResultStatus::ValidationFailed)
        .value("CompilationFailed", ktt::ResultStatus::CompilationFailed)
        .value("DeviceLimitsExceeded", ktt::ResultStatus::DeviceLimitsExceeded);
    py::enum_<ktt::TimeUnit>(m, "TimeUnit")
        .value("Nanoseconds", ktt::TimeUnit::Nanoseconds).value("Microseconds", ktt::TimeUnit::Microseconds)
        .value("Milliseconds", ktt::TimeUnit::Milliseconds).value("Seconds", ktt::TimeUnit::Seconds);
    py::enum_<ktt::ValidationMethod>(m, "ValidationMethod")
        .value("AbsoluteDifference", ktt::ValidationMethod::AbsoluteDifference)
        .value("SideBySideComparison", ktt::ValidationMethod::SideBySideComparison)
        .value("SideBySideRelativeComparison", ktt::ValidationMethod::SideBySideRelativeComparison);
    py::enum_<ktt::ValidationMode>(m, "ValidationMode", py::arithmetic())
        .value("None", ktt::ValidationMode::None).value("Running", ktt::ValidationMode::Running)
        .value("OfflineTuning", ktt::ValidationMode::OfflineTuning).value("OnlineTuning", ktt::ValidationMode::OnlineTuning)
        .value("All", ktt::ValidationMode::All);

    // ---- data holders (PythonDataHolders.cpp) ----
    py::class_<ktt::DimensionVector>(m, "DimensionVector")
        .def(py::init<>())
        .def(py::init<const size_t>())
        .def(py::init<const size_t, const size_t>())
        .def(py::init<const size_t, const size_t, const size_t>())
        .def(py::init<const std::vector<size_t>&>())
        .def("SetSizeX", &ktt::DimensionVector::SetSizeX)
        .def("SetSizeY", &ktt::DimensionVector::SetSizeY)
        .def("SetSizeZ", &ktt::DimensionVector::SetSizeZ)
        .def("SetSize", &ktt::DimensionVector::SetSize)
        .def("Multiply", &ktt::DimensionVector::Multiply)
        .def("Divide", &ktt::DimensionVector::Divide)
        .def("RoundUp", &ktt::DimensionVector::RoundUp)
        .def("ModifyByValue", &ktt::DimensionVector::ModifyByValue)
        .def("GetSizeX", &ktt::DimensionVector::GetSizeX)
        .def("GetSizeY", &ktt::DimensionVector::GetSizeY)
        .def("GetSizeZ", &ktt::DimensionVector::GetSizeZ)
        .def("GetSize", &ktt::DimensionVector::GetSize)
        .def("GetTotalSize", &ktt::DimensionVector::GetTotalSize)
        .def("GetVector", &ktt::DimensionVector::GetVector)
        .def("GetString", &ktt::DimensionVector::GetString)
        .def("__eq__", &ktt::DimensionVector::operator==)
        .def("__ne__", &ktt::DimensionVector::operator!=)
        .def("__repr__", &ktt::DimensionVector::GetString);

    py::class_<ktt::ParameterPair>(m, "ParameterPair")
        .def(py::init<>())
        .def(py::init<const std::string&, const ktt::ParameterValue&>())
        .def("SetValue", &ktt::ParameterPair::SetValue)
        .def("GetName", &ktt::ParameterPair::GetName)
        .def("GetString", &ktt::ParameterPair::GetString)
        .def("GetValueString", &ktt::ParameterPair::GetValueString)
        .def("GetValue", &ktt::ParameterPair::GetValue)
        .def("GetValueUint", &ktt::ParameterPair::GetValueUint)
        .def("GetValueType", &ktt::ParameterPair::GetValueType)
        .def("HasSameValue", &ktt::ParameterPair::HasSameValue)
        .def_static("GetTypeFromValue", &ktt::ParameterPair::GetTypeFromValue)
        .def("__repr__", &ktt::ParameterPair::GetString);

    py::class_<ktt::KernelConfiguration>(m, "KernelConfiguration")
        .def(py::init<>())
        .def(py::init<const std::vector<ktt::ParameterPair>&>())
        .def("GetPairs", &ktt::KernelConfiguration::GetPairs)
        .def("IsValid", &ktt::KernelConfiguration::IsValid)
        .def("GeneratePrefix", &ktt::KernelConfiguration::GeneratePrefix)
        .def("GetString", &ktt::KernelConfiguration::GetString)
        .def("Merge", &ktt::KernelConfiguration::Merge)
        .def("__eq__", &ktt::KernelConfiguration::operator==)
        .def("__ne__", &ktt::KernelConfiguration::operator!=)
        .def("__repr__", &ktt::KernelConfiguration::GetString);

    py::class_<ktt::DeviceInfo>(m, "DeviceInfo")
        .def(py::init<const ktt::DeviceIndex, const std::string&>())
        .def("GetIndex", &ktt::DeviceInfo::GetIndex)
        .def("GetName", &ktt::DeviceInfo::GetName)
        .def("GetVendor", &ktt::DeviceInfo::GetVendor)
        .def("GetExtensions", &ktt::DeviceInfo::GetExtensions)
        .def("GetDeviceType", &ktt::DeviceInfo::GetDeviceType)
        .def("GetDeviceTypeString", &ktt::DeviceInfo::GetDeviceTypeString)
        .def("GetGlobalMemorySize", &ktt::DeviceInfo::GetGlobalMemorySize)
        .def("GetLocalMemorySize", &ktt::DeviceInfo::GetLocalMemorySize)
        .def("GetMaxConstantBufferSize", &ktt::DeviceInfo::GetMaxConstantBufferSize)
        .def("GetMaxWorkGroupSize", &ktt::DeviceInfo::GetMaxWorkGroupSize)
        .def("GetMaxComputeUnits", &ktt::DeviceInfo::GetMaxComputeUnits)
        .def("GetCudaComputeCapabilityMajor", &ktt::DeviceInfo::GetCudaComputeCapabilityMajor)
        .def("GetCudaComputeCapabilityMinor", &ktt::DeviceInfo::GetCudaComputeCapabilityMinor)
        .def("GetString", &ktt::DeviceInfo::GetString)
        .def("SetVendor", &ktt::DeviceInfo::SetVendor)
        .def("SetExtensions", &ktt::DeviceInfo::SetExtensions)
        .def("SetDeviceType", &ktt::DeviceInfo::SetDeviceType)
        .def("SetGlobalMemorySize", &ktt::DeviceInfo::SetGlobalMemorySize)
        .def("SetLocalMemorySize", &ktt::DeviceInfo::SetLocalMemorySize)
        .def("SetMaxConstantBufferSize", &ktt::DeviceInfo::SetMaxConstantBufferSize)
        .def("SetMaxWorkGroupSize", &ktt::DeviceInfo::SetMaxWorkGroupSize)
        .def("SetMaxComputeUnits", &ktt::DeviceInfo::SetMaxComputeUnits)
        .def("SetCudaComputeCapabilityMajor", &ktt::DeviceInfo::SetCudaComputeCapabilityMajor)
        .def("SetCudaComputeCapabilityMinor", &ktt::DeviceInfo::SetCudaComputeCapabilityMinor)
        .def("__repr__", &ktt::DeviceInfo::GetString);

    py::class_<ktt::PlatformInfo>(m, "PlatformInfo")
        .def(py::init<const ktt::PlatformIndex, const std::string&>())
        .def("GetIndex", &ktt::PlatformInfo::GetIndex)
        .def("GetName", &ktt::PlatformInfo::GetName)
        .def("GetVendor", &ktt::PlatformInfo::GetVendor)
        .def("GetVersion", &ktt::PlatformInfo::GetVersion)
        .def("GetExtensions", &ktt::PlatformInfo::GetExtensions)
        .def("GetString", &ktt::PlatformInfo::GetString)
        .def("SetVendor", &ktt::PlatformInfo::SetVendor)
        .def("SetVersion", &ktt::PlatformInfo::SetVersion)
        .def("SetExtensions", &ktt::PlatformInfo::SetExtensions)
        .def("__repr__", &ktt::PlatformInfo::GetString);

    // The caller's buffer must outlive the descriptor's use in Run / TuneIteration (as in KTT).
    py::class_<ktt::BufferOutputDescriptor>(m, "BufferOutputDescriptor")
        .def(py::init([](const ktt::ArgumentId& id, py::buffer buffer)
            {
                const py::buffer_info info = buffer.request(true);
                return ktt::BufferOutputDescriptor(id, info.ptr, static_cast<size_t>(info.size * info.itemsize));
            }), py::keep_alive<1, 3>())
        .def(py::init([](const ktt::ArgumentId& id, py::buffer buffer, const size_t size)
            {
                return ktt::BufferOutputDescriptor(id, buffer.request(true).ptr, size);
            }), py::keep_alive<1, 3>())
        .def("GetArgumentId", &ktt::BufferOutputDescriptor::GetArgumentId)
        .def("GetOutputSize", &ktt::BufferOutputDescriptor::GetOutputSize);

    py::enum_<ktt::ProfilingCounterType>(m, "ProfilingCounterType")
        .value("Int", ktt::ProfilingCounterType::Int)
        .value("UnsignedInt", ktt::ProfilingCounterType::UnsignedInt)
        .value("Double", ktt::ProfilingCounterType::Double)
        .value("Percent", ktt::ProfilingCounterType::Percent)
        .value("Throughput", ktt::ProfilingCounterType::Throughput)
        .value("UtilizationLevel", ktt::ProfilingCounterType::UtilizationLevel);

    py::class_<ktt::KernelProfilingCounter>(m, "KernelProfilingCounter")
        .def(py::init<>())
        .def(py::init<const std::string&, const ktt::ProfilingCounterType, const int64_t>())
        .def(py::init<const std::string&, const ktt::ProfilingCounterType, const uint64_t>())
        .def(py::init<const std::string&, const ktt::ProfilingCounterType, const double>())
        .def("GetName", &ktt::KernelProfilingCounter::GetName)
        .def("GetType", &ktt::KernelProfilingCounter::GetType)
        .def("GetValueInt", &ktt::KernelProfilingCounter::GetValueInt)
        .def("GetValueUint", &ktt::KernelProfilingCounter::GetValueUint)
        .def("GetValueDouble", &ktt::KernelProfilingCounter::GetValueDouble)
        .def("__eq__", &ktt::KernelProfilingCounter::operator==)
        .def("__ne__", &ktt::KernelProfilingCounter::operator!=)
        .def("__lt__", &ktt::KernelProfilingCounter::operator<);

    py::class_<ktt::KernelProfilingData>(m, "KernelProfilingData")
        .def(py::init<>())
        .def(py::init<const uint64_t>())
        .def(py::init<const std::vector<ktt::KernelProfilingCounter>&>())
        .def("IsValid", &ktt::KernelProfilingData::IsValid)
        .def("HasCounter", &ktt::KernelProfilingData::HasCounter)
        .def("GetCounter", &ktt::KernelProfilingData::GetCounter, py::return_value_policy::copy)
        .def("GetCounters", &ktt::KernelProfilingData::GetCounters, py::return_value_policy::copy)
        .def("SetCounters", &ktt::KernelProfilingData::SetCounters)
        .def("AddCounter", &ktt::KernelProfilingData::AddCounter)
        .def("HasRemainingProfilingRuns", &ktt::KernelProfilingData::HasRemainingProfilingRuns)
        .def("GetRemainingProfilingRuns", &ktt::KernelProfilingData::GetRemainingProfilingRuns)
        .def("DecreaseRemainingProfilingRuns", &ktt::KernelProfilingData::DecreaseRemainingProfilingRuns);

    py::class_<ktt::ComputationResult>(m, "ComputationResult")
        .def(py::init<>())
        .def(py::init<const std::string&>())
        .def(py::init<const ktt::ComputationResult&>())
        .def("SetDurationData", &ktt::ComputationResult::SetDurationData, py::arg("duration"), py::arg("overhead"),
            py::arg("compilationOverhead") = 0)
        .def("SetSizeData", &ktt::ComputationResult::SetSizeData)
        .def("SetProfilingData", [](ktt::ComputationResult& r, const ktt::KernelProfilingData& data)
            {
                r.SetProfilingData(std::make_unique<ktt::KernelProfilingData>(data));
            })
        .def("GetProfilingData", &ktt::ComputationResult::GetProfilingData, py::return_value_policy::copy)
        .def("HasRemainingProfilingRuns", &ktt::ComputationResult::HasRemainingProfilingRuns)
        .def("GetKernelFunction", &ktt::ComputationResult::GetKernelFunction)
        .def("GetGlobalSize", &ktt::ComputationResult::GetGlobalSize)
        .def("GetLocalSize", &ktt::ComputationResult::GetLocalSize)
        .def("GetDuration", &ktt::ComputationResult::GetDuration)
        .def("GetOverhead", &ktt::ComputationResult::GetOverhead)
        .def("GetCompilationOverhead", &ktt::ComputationResult::GetCompilationOverhead)
        .def("HasCompilationData", &ktt::ComputationResult::HasCompilationData)
        .def("HasProfilingData", &ktt::ComputationResult::HasProfilingData)
        .def("HasPowerData", &ktt::ComputationResult::HasPowerData);

    py::class_<ktt::KernelResult>(m, "KernelResult")
        .def(py::init<>())
        .def(py::init<const std::string&, const ktt::KernelConfiguration&>())
        .def(py::init<const std::string&, const ktt::KernelConfiguration&, const std::vector<ktt::ComputationResult>&>())
        .def("SetStatus", &ktt::KernelResult::SetStatus)
        .def("SetExtraDuration", &ktt::KernelResult::SetExtraDuration)
        .def("SetDataMovementOverhead", &ktt::KernelResult::SetDataMovementOverhead)
        .def("SetValidationOverhead", &ktt::KernelResult::SetValidationOverhead)
        .def("SetSearcherOverhead", &ktt::KernelResult::SetSearcherOverhead)
        .def("GetProfilingRunsOverhead", &ktt::KernelResult::GetProfilingRunsOverhead)
        .def("HasRemainingProfilingRuns", &ktt::KernelResult::HasRemainingProfilingRuns)
        .def("GetKernelName", &ktt::KernelResult::GetKernelName)
        .def("GetResults", &ktt::KernelResult::GetResults)
        .def("GetConfiguration", &ktt::KernelResult::GetConfiguration)
        .def("GetStatus", &ktt::KernelResult::GetStatus)
        .def("GetKernelDuration", &ktt::KernelResult::GetKernelDuration)
        .def("GetKernelOverhead", &ktt::KernelResult::GetKernelOverhead)
        .def("GetExtraDuration", &ktt::KernelResult::GetExtraDuration)
        .def("GetDataMovementOverhead", &ktt::KernelResult::GetDataMovementOverhead)
        .def("GetValidationOverhead", &ktt::KernelResult::GetValidationOverhead)
        .def("GetSearcherOverhead", &ktt::KernelResult::GetSearcherOverhead)
        .def("GetTotalDuration", &ktt::KernelResult::GetTotalDuration)
        .def("GetTotalOverhead", &ktt::KernelResult::GetTotalOverhead)
        .def("IsValid", &ktt::KernelResult::IsValid);

    // ---- searchers and stop conditions (owned by the tuner once passed to it) ----
    py::classh<ktt::Searcher>(m, "Searcher");
    py::classh<ktt::DeterministicSearcher, ktt::Searcher>(m, "DeterministicSearcher").def(py::init<>());
    py::classh<ktt::RandomSearcher, ktt::Searcher>(m, "RandomSearcher").def(py::init<>());
    py::classh<ktt::McmcSearcher, ktt::Searcher>(m, "McmcSearcher")
        .def(py::init<>())
        .def(py::init<const ktt::KernelConfiguration&>())
        .def(py::init<const ktt::KernelConfiguration&, const uint64_t>(), py::arg("start"), py::arg("seed"));

    // the profile-based searcher and its counter model (native; KTT runs it as embedded Python)
    py::class_<ktt::CounterModel>(m, "CounterModel")
        .def(py::init<>())
        .def_static("Load", &ktt::CounterModel::Load)
        .def("GetParameters", &ktt::CounterModel::GetParameters)
        .def("GetCounters", &ktt::CounterModel::GetCounters)
        .def("GetComputeCapability", &ktt::CounterModel::GetComputeCapability)
        .def("GetMultiprocessors", &ktt::CounterModel::GetMultiprocessors)
        .def("IsEmpty", &ktt::CounterModel::IsEmpty)
        .def("Predict", py::overload_cast<const std::vector<double>&>(&ktt::CounterModel::Predict, py::const_))
        .def("PredictConfiguration", py::overload_cast<const ktt::KernelConfiguration&>(&ktt::CounterModel::Predict,
            py::const_));
    py::classh<ktt::ProfileBasedSearcher, ktt::Searcher>(m, "ProfileBasedSearcher")
        .def(py::init<ktt::Tuner&, const ktt::CounterModel&, const uint32_t, const uint32_t, const uint32_t, const uint64_t>(),
            py::arg("tuner"), py::arg("model"), py::arg("batchSize") = 5, py::arg("neighborSize") = 100,
            py::arg("randomSize") = 10, py::arg("seed") = 0, py::keep_alive<1, 2>())
        .def("SetDeviceProperties", &ktt::ProfileBasedSearcher::SetDeviceProperties)
        .def("SetXuPipeAnalysis", &ktt::ProfileBasedSearcher::SetXuPipeAnalysis)
        .def("GetScoredBatches", &ktt::ProfileBasedSearcher::GetScoredBatches);
    py::module_ profiling = m.def_submodule("profiling", "steps of the profile-based searcher");
    profiling.def("AnalyzeBottlenecks", &ktt::profiling::AnalyzeBottlenecks, py::arg("names"), py::arg("values"),
        py::arg("multiprocessors"), py::arg("cores"), py::arg("reactToInstructions") = ktt::profiling::ReactToInstructionBottlenecks);
    profiling.def("ComputeChanges", &ktt::profiling::ComputeChanges, py::arg("bottlenecks"), py::arg("counters"),
        py::arg("xuPipe") = false, py::arg("reactToInstructions") = ktt::profiling::ReactToInstructionBottlenecks);
    profiling.def("ScoreCandidates", &ktt::profiling::ScoreCandidates);
    profiling.def("WeightedRandomStep", &ktt::profiling::WeightedRandomStep);
    profiling.def("CoresPerMultiprocessor", &ktt::profiling::CoresPerMultiprocessor);

    py::classh<ktt::StopCondition, PyStopCondition>(m, "StopCondition")
        .def(py::init<>())
        .def("IsFulfilled", &ktt::StopCondition::IsFulfilled)
        .def("Initialize", &ktt::StopCondition::Initialize)
        .def("Update", &ktt::StopCondition::Update)
        .def("GetStatusString", &ktt::StopCondition::GetStatusString);
    py::classh<ktt::ConfigurationCount, ktt::StopCondition>(m, "ConfigurationCount").def(py::init<const uint64_t>());
    py::classh<ktt::ConfigurationDuration, ktt::StopCondition>(m, "ConfigurationDuration").def(py::init<const double>());
    py::classh<ktt::ConfigurationFraction, ktt::StopCondition>(m, "ConfigurationFraction").def(py::init<const double>());
    py::classh<ktt::TuningDuration, ktt::StopCondition>(m, "TuningDuration").def(py::init<const double>());

    // ---- compute interface for launchers (PythonComputeInterface.cpp) ----
    py::class_<ktt::ComputeInterface> ci(m, "ComputeInterface");
    ci.def("RunKernel", py::overload_cast<const ktt::KernelDefinitionId>(&ktt::ComputeInterface::RunKernel))
        .def("RunKernel", py::overload_cast<const ktt::KernelDefinitionId, const ktt::DimensionVector&,
            const ktt::DimensionVector&>(&ktt::ComputeInterface::RunKernel))
        .def("RunKernelAsync", py::overload_cast<const ktt::KernelDefinitionId, const ktt::QueueId>(
            &ktt::ComputeInterface::RunKernelAsync))
        .def("WaitForComputeAction", &ktt::ComputeInterface::WaitForComputeAction)
        .def("RunKernelWithProfiling", py::overload_cast<const ktt::KernelDefinitionId>(
            &ktt::ComputeInterface::RunKernelWithProfiling))
        .def("RunKernelWithProfiling", py::overload_cast<const ktt::KernelDefinitionId, const ktt::DimensionVector&,
            const ktt::DimensionVector&>(&ktt::ComputeInterface::RunKernelWithProfiling))
        .def("GetRemainingProfilingRuns", py::overload_cast<const ktt::KernelDefinitionId>(
            &ktt::ComputeInterface::GetRemainingProfilingRuns, py::const_))
        .def("GetRemainingProfilingRuns", py::overload_cast<>(&ktt::ComputeInterface::GetRemainingProfilingRuns, py::const_))
        .def("GetDefaultQueue", &ktt::ComputeInterface::GetDefaultQueue)
        .def("GetAllQueues", &ktt::ComputeInterface::GetAllQueues)
        .def("SynchronizeQueue", &ktt::ComputeInterface::SynchronizeQueue)
        .def("SynchronizeQueues", &ktt::ComputeInterface::SynchronizeQueues)
        .def("SynchronizeDevice", &ktt::ComputeInterface::SynchronizeDevice)
        .def("GetCurrentGlobalSize", &ktt::ComputeInterface::GetCurrentGlobalSize, py::return_value_policy::copy)
        .def("GetCurrentLocalSize", &ktt::ComputeInterface::GetCurrentLocalSize, py::return_value_policy::copy)
        .def("GetCurrentConfiguration", &ktt::ComputeInterface::GetCurrentConfiguration, py::return_value_policy::copy)
        .def("GetRunMode", &ktt::ComputeInterface::GetRunMode)
        .def("ChangeArguments", &ktt::ComputeInterface::ChangeArguments)
        .def("SwapArguments", &ktt::ComputeInterface::SwapArguments)
        .def("UploadBuffer", &ktt::ComputeInterface::UploadBuffer)
        .def("DownloadBuffer", [](ktt::ComputeInterface& c, const ktt::ArgumentId& id, py::buffer destination)
            {
                const py::buffer_info info = destination.request(true);
                c.DownloadBuffer(id, info.ptr, static_cast<size_t>(info.size * info.itemsize));
            })
        .def("UpdateBuffer", [](ktt::ComputeInterface& c, const ktt::ArgumentId& id, py::buffer data)
            {
                const py::buffer_info info = data.request();
                c.UpdateBuffer(id, info.ptr, static_cast<size_t>(info.size * info.itemsize));
            })
        .def("CopyBuffer", &ktt::ComputeInterface::CopyBuffer)
        .def("ClearBuffer", &ktt::ComputeInterface::ClearBuffer)
        .def("HasBuffer", &ktt::ComputeInterface::HasBuffer)
        .def("UploadBufferAsync", &ktt::ComputeInterface::UploadBufferAsync)
        .def("DownloadBufferAsync", [](ktt::ComputeInterface& c, const ktt::ArgumentId& id, const ktt::QueueId queue,
            py::buffer destination)
            {
                const py::buffer_info info = destination.request(true);
                return c.DownloadBufferAsync(id, queue, info.ptr, static_cast<size_t>(info.size * info.itemsize));
            })
        .def("UpdateBufferAsync", [](ktt::ComputeInterface& c, const ktt::ArgumentId& id, const ktt::QueueId queue,
            py::buffer data)
            {
                const py::buffer_info info = data.request();
                return c.UpdateBufferAsync(id, queue, info.ptr, static_cast<size_t>(info.size * info.itemsize));
            })
        .def("CopyBufferAsync", &ktt::ComputeInterface::CopyBufferAsync, py::arg("destination"), py::arg("source"),
            py::arg("queue"), py::arg("dataSize") = 0)
        .def("WaitForTransferAction", &ktt::ComputeInterface::WaitForTransferAction)
        .def("ResizeBuffer", &ktt::ComputeInterface::ResizeBuffer)
        .def("UpdateLocalArgument", &ktt::ComputeInterface::UpdateLocalArgument)
        .def("GetProfiling", &ktt::ComputeInterface::GetProfiling);
    BindScalarUpdate<int8_t>(ci, "UpdateScalarArgumentChar");
    BindScalarUpdate<int16_t>(ci, "UpdateScalarArgumentShort");
    BindScalarUpdate<int32_t>(ci, "UpdateScalarArgumentInt");
    BindScalarUpdate<int64_t>(ci, "UpdateScalarArgumentLong");
    BindScalarUpdate<float>(ci, "UpdateScalarArgumentFloat");
    BindScalarUpdate<double>(ci, "UpdateScalarArgumentDouble");

    // ---- tuner (PythonTuner.cpp) ----
    // The caller's CUDA context and streams as integers (CUcontext / CUstream handles, e.g. from ctypes).
    py::class_<ktt::ComputeApiInitializer>(m, "ComputeApiInitializer")
        .def(py::init([](const uintptr_t context, const std::vector<uintptr_t>& queues)
            {
                std::vector<ktt::ComputeQueue> q;

                for (const auto queue : queues)
                {
                    q.push_back(reinterpret_cast<ktt::ComputeQueue>(queue));
                }

                return ktt::ComputeApiInitializer(reinterpret_cast<ktt::ComputeContext>(context), q);
            }), py::arg("context"), py::arg("queues"))
        .def("GetContext", [](const ktt::ComputeApiInitializer& i) { return reinterpret_cast<uintptr_t>(i.GetContext()); })
        .def("GetQueues", [](const ktt::ComputeApiInitializer& i)
            {
                std::vector<uintptr_t> q;

                for (const auto queue : i.GetQueues())
                {
                    q.push_back(reinterpret_cast<uintptr_t>(queue));
                }

                return q;
            });

    py::class_<ktt::Tuner> tuner(m, "Tuner");
    tuner.def(py::init<const ktt::PlatformIndex, const ktt::DeviceIndex, const ktt::ComputeApi>())
        .def(py::init<const ktt::PlatformIndex, const ktt::DeviceIndex, const ktt::ComputeApi, const uint32_t>())
        .def(py::init<const ktt::ComputeApi, const ktt::ComputeApiInitializer&>())
        .def("AddKernelDefinition", py::overload_cast<const std::string&, const std::string&, const ktt::DimensionVector&,
            const ktt::DimensionVector&, const std::vector<std::string>&>(&ktt::Tuner::AddKernelDefinition),
            py::arg("name"), py::arg("source"), py::arg("globalSize"), py::arg("localSize"),
            py::arg("typeNames") = std::vector<std::string>{})
        .def("AddKernelDefinition", py::overload_cast<const std::string&, const std::string&, const std::vector<std::string>&>(
            &ktt::Tuner::AddKernelDefinition), py::arg("name"), py::arg("source"), py::arg("typeNames") = std::vector<std::string>{})
        .def("AddKernelDefinitionFromFile", py::overload_cast<const std::string&, const std::string&, const ktt::DimensionVector&,
            const ktt::DimensionVector&, const std::vector<std::string>&>(&ktt::Tuner::AddKernelDefinitionFromFile),
            py::arg("name"), py::arg("filePath"), py::arg("globalSize"), py::arg("localSize"),
            py::arg("typeNames") = std::vector<std::string>{})
        .def("AddKernelDefinitionFromFile", py::overload_cast<const std::string&, const std::string&,
            const std::vector<std::string>&>(&ktt::Tuner::AddKernelDefinitionFromFile), py::arg("name"), py::arg("filePath"),
            py::arg("typeNames") = std::vector<std::string>{})
        .def("GetKernelDefinitionId", &ktt::Tuner::GetKernelDefinitionId, py::arg("name"),
            py::arg("typeNames") = std::vector<std::string>{})
        .def("RemoveKernelDefinition", &ktt::Tuner::RemoveKernelDefinition)
        .def("SetArguments", &ktt::Tuner::SetArguments)
        .def("CreateSimpleKernel", &ktt::Tuner::CreateSimpleKernel)
        // Python launchers receive the ComputeInterface by reference (a pointer on the C++ side; the
        // interface cannot be copied), as KTT's module passes it (Source/Python/PythonTuner.cpp:80-88)
        .def("CreateCompositeKernel", [](ktt::Tuner& t, const std::string& name, const std::vector<ktt::KernelDefinitionId>& ids,
            std::function<void(ktt::ComputeInterface*)> launcher)
            {
                ktt::KernelLauncher wrapped;

                if (launcher)
                {
                    wrapped = [launcher](ktt::ComputeInterface& ci) { launcher(&ci); };
                }

                return t.CreateCompositeKernel(name, ids, wrapped);
            }, py::arg("name"), py::arg("definitionIds"), py::arg("launcher") = nullptr)
        .def("RemoveKernel", &ktt::Tuner::RemoveKernel)
        .def("SetLauncher", [](ktt::Tuner& t, const ktt::KernelId id, std::function<void(ktt::ComputeInterface*)> launcher)
            {
                ktt::KernelLauncher wrapped;

                if (launcher)
                {
                    wrapped = [launcher](ktt::ComputeInterface& ci) { launcher(&ci); };
                }

                t.SetLauncher(id, wrapped);
            }, py::arg("id"), py::arg("launcher"))
        .def("AddParameter", [](ktt::Tuner& t, const ktt::KernelId id, const std::string& name, const std::vector<uint64_t>& values,
            const std::string& group) { t.AddParameter(id, name, values, group); },
            py::arg("id"), py::arg("name"), py::arg("values"), py::arg("group") = std::string())
        .def("AddParameterInt", [](ktt::Tuner& t, const ktt::KernelId id, const std::string& name, const std::vector<int64_t>& values,
            const std::string& group) { t.AddParameter(id, name, values, group); },
            py::arg("id"), py::arg("name"), py::arg("values"), py::arg("group") = std::string())
        .def("AddParameterUint", [](ktt::Tuner& t, const ktt::KernelId id, const std::string& name, const std::vector<uint64_t>& values,
            const std::string& group) { t.AddParameter(id, name, values, group); },
            py::arg("id"), py::arg("name"), py::arg("values"), py::arg("group") = std::string())
        .def("AddParameterDouble", [](ktt::Tuner& t, const ktt::KernelId id, const std::string& name,
            const std::vector<double>& values, const std::string& group) { t.AddParameter(id, name, values, group); },
            py::arg("id"), py::arg("name"), py::arg("values"), py::arg("group") = std::string())
        .def("AddParameterBool", [](ktt::Tuner& t, const ktt::KernelId id, const std::string& name, const std::vector<bool>& values,
            const std::string& group) { t.AddParameter(id, name, values, group); },
            py::arg("id"), py::arg("name"), py::arg("values"), py::arg("group") = std::string())
        .def("AddParameterString", [](ktt::Tuner& t, const ktt::KernelId id, const std::string& name,
            const std::vector<std::string>& values, const std::string& group) { t.AddParameter(id, name, values, group); },
            py::arg("id"), py::arg("name"), py::arg("values"), py::arg("group") = std::string())
        .def("AddScriptParameter", &ktt::Tuner::AddScriptParameter, py::arg("id"), py::arg("name"), py::arg("valueType"),
            py::arg("valueScript"), py::arg("group") = std::string())
        .def("AddThreadModifier", py::overload_cast<const ktt::KernelId, const std::vector<ktt::KernelDefinitionId>&,
            const ktt::ModifierType, const ktt::ModifierDimension, const std::vector<std::string>&, ktt::ModifierFunction>(
            &ktt::Tuner::AddThreadModifier))
        .def("AddThreadModifier", py::overload_cast<const ktt::KernelId, const std::vector<ktt::KernelDefinitionId>&,
            const ktt::ModifierType, const ktt::ModifierDimension, const std::string&, const ktt::ModifierAction>(
            &ktt::Tuner::AddThreadModifier))
        .def("AddScriptThreadModifier", &ktt::Tuner::AddScriptThreadModifier)
        .def("AddConstraint", &ktt::Tuner::AddConstraint)
        .def("AddGenericConstraint", [](ktt::Tuner& t, const ktt::KernelId id, const std::vector<std::string>& names,
            std::function<bool(const std::vector<ktt::ParameterValue>&)> function)
            {
                t.AddGenericConstraint(id, names, [function](const std::vector<const ktt::ParameterValue*>& values)
                {
                    std::vector<ktt::ParameterValue> copies;

                    for (const auto* v : values)
                    {
                        copies.push_back(*v);
                    }

                    return function(copies);
                });
            })
        .def("AddScriptConstraint", &ktt::Tuner::AddScriptConstraint)
        .def("AddArgumentVectorFromFile", &ktt::Tuner::AddArgumentVectorFromFile, py::arg("filePath"), py::arg("dataType"),
            py::arg("elementSize"), py::arg("accessType"), py::arg("memoryLocation") = ktt::ArgumentMemoryLocation::Device,
            py::arg("managementType") = ktt::ArgumentManagementType::Framework, py::arg("customId") = ktt::ArgumentId())
        .def("AddArgumentVectorFromGenerator", &ktt::Tuner::AddArgumentVectorFromGenerator, py::arg("generatorFunction"),
            py::arg("dataType"), py::arg("bufferSize"), py::arg("elementSize"), py::arg("accessType"),
            py::arg("memoryLocation") = ktt::ArgumentMemoryLocation::Device,
            py::arg("managementType") = ktt::ArgumentManagementType::Framework, py::arg("customId") = ktt::ArgumentId())
        .def("SaveArgumentVector", &ktt::Tuner::SaveArgumentVector)
        .def("RemoveArgument", &ktt::Tuner::RemoveArgument)
        .def("SetReadOnlyArgumentCache", &ktt::Tuner::SetReadOnlyArgumentCache);
    BindVectorArgument<int8_t>(tuner, "AddArgumentVectorChar");
    BindVectorArgument<int16_t>(tuner, "AddArgumentVectorShort");
    BindVectorArgument<int32_t>(tuner, "AddArgumentVectorInt");
    BindVectorArgument<int64_t>(tuner, "AddArgumentVectorLong");
    BindVectorArgument<float>(tuner, "AddArgumentVectorFloat");
    BindVectorArgument<double>(tuner, "AddArgumentVectorDouble");
    BindScalarArgument<int8_t>(tuner, "AddArgumentScalarChar");
    BindScalarArgument<int16_t>(tuner, "AddArgumentScalarShort");
    BindScalarArgument<int32_t>(tuner, "AddArgumentScalarInt");
    BindScalarArgument<int64_t>(tuner, "AddArgumentScalarLong");
    BindScalarArgument<float>(tuner, "AddArgumentScalarFloat");
    BindScalarArgument<double>(tuner, "AddArgumentScalarDouble");
    BindLocalArgument<int8_t>(tuner, "AddArgumentLocalChar");
    BindLocalArgument<int16_t>(tuner, "AddArgumentLocalShort");
    BindLocalArgument<int32_t>(tuner, "AddArgumentLocalInt");
    BindLocalArgument<int64_t>(tuner, "AddArgumentLocalLong");
    BindLocalArgument<float>(tuner, "AddArgumentLocalFloat");
    BindLocalArgument<double>(tuner, "AddArgumentLocalDouble");
    BindSymbolArgument<int8_t>(tuner, "AddArgumentSymbolChar");
    BindSymbolArgument<int16_t>(tuner, "AddArgumentSymbolShort");
    BindSymbolArgument<int32_t>(tuner, "AddArgumentSymbolInt");
    BindSymbolArgument<int64_t>(tuner, "AddArgumentSymbolLong");
    BindSymbolArgument<float>(tuner, "AddArgumentSymbolFloat");
    BindSymbolArgument<double>(tuner, "AddArgumentSymbolDouble");

    tuner.def("Run", &ktt::Tuner::Run, py::call_guard<py::gil_scoped_release>())
        .def("SetProfiling", &ktt::Tuner::SetProfiling)
        .def("SetProfilingCounters", &ktt::Tuner::SetProfilingCounters)
        .def("SetProfiledDefinitions", &ktt::Tuner::SetProfiledDefinitions)
        .def("GetProfiling", &ktt::Tuner::GetProfiling)
        .def("SetValidationMethod", &ktt::Tuner::SetValidationMethod)
        .def("SetValidationMode", &ktt::Tuner::SetValidationMode)
        .def("SetValidationRange", &ktt::Tuner::SetValidationRange)
        .def("SetReferenceComputation", [](ktt::Tuner& t, const ktt::ArgumentId& id, const size_t referenceSize,
            std::function<void(py::memoryview)> reference)
            {
                t.SetReferenceComputation(id, [reference, referenceSize](void* buffer)
                {
                    py::gil_scoped_acquire acquire;
                    reference(py::memoryview::from_memory(buffer, static_cast<py::ssize_t>(referenceSize)));
                });
            })
        .def("SetReferenceKernel", &ktt::Tuner::SetReferenceKernel)
        .def("SetReferenceArgument", &ktt::Tuner::SetReferenceArgument)
        .def("Tune", [](ktt::Tuner& t, const ktt::KernelId id, std::unique_ptr<ktt::StopCondition> stop)
            {
                py::gil_scoped_release release;
                return t.Tune(id, std::move(stop));
            }, py::arg("id"), py::arg("stopCondition") = nullptr)
        .def("TuneIteration", &ktt::Tuner::TuneIteration, py::call_guard<py::gil_scoped_release>(), py::arg("id"),
            py::arg("output"), py::arg("recomputeReference") = false)
        .def("SimulateTuning", [](ktt::Tuner& t, const ktt::KernelId id, const std::vector<ktt::KernelResult>& results,
            std::unique_ptr<ktt::StopCondition> stop)
            {
                py::gil_scoped_release release;
                return t.SimulateTuning(id, results, std::move(stop));
            }, py::arg("id"), py::arg("results"), py::arg("stopCondition") = nullptr)
        .def("SetSearcher", [](ktt::Tuner& t, const ktt::KernelId id, std::unique_ptr<ktt::Searcher> searcher)
            {
                t.SetSearcher(id, std::move(searcher));
            })
        .def("SetProfileBasedSearcher", &ktt::Tuner::SetProfileBasedSearcher, py::arg("id"), py::arg("modelPath"),
            py::arg("useBuiltinModule") = true, py::arg("batchSize") = 5, py::arg("neighborSize") = 100,
            py::arg("randomSize") = 10)
        .def("InitializeConfigurationData", &ktt::Tuner::InitializeConfigurationData, py::call_guard<py::gil_scoped_release>())
        .def("ClearConfigurationData", &ktt::Tuner::ClearConfigurationData)
        .def("ClearData", &ktt::Tuner::ClearConfigurationData)
        .def("GetConfigurationsCount", &ktt::Tuner::GetConfigurationsCount)
        .def("GetBestConfiguration", &ktt::Tuner::GetBestConfiguration)
        .def("CreateConfiguration", &ktt::Tuner::CreateConfiguration)
        .def("GetKernelSource", &ktt::Tuner::GetKernelSource)
        .def("GetKernelDefinitionSource", &ktt::Tuner::GetKernelDefinitionSource)
        .def_static("SetTimeUnit", &ktt::Tuner::SetTimeUnit)
        .def("SaveResults", &ktt::Tuner::SaveResults, py::arg("results"), py::arg("filePath"), py::arg("format"),
            py::arg("data") = ktt::UserData{})
        .def("LoadResults", py::overload_cast<const std::string&, const ktt::OutputFormat>(&ktt::Tuner::LoadResults, py::const_))
        .def("AddComputeQueue", [](ktt::Tuner& t, const uintptr_t queue) { return t.AddComputeQueue(reinterpret_cast<ktt::ComputeQueue>(queue)); })
        .def("RemoveComputeQueue", &ktt::Tuner::RemoveComputeQueue)
        .def("WaitForComputeAction", &ktt::Tuner::WaitForComputeAction)
        .def("WaitForTransferAction", &ktt::Tuner::WaitForTransferAction)
        .def("SynchronizeQueue", &ktt::Tuner::SynchronizeQueue)
        .def("SynchronizeQueues", &ktt::Tuner::SynchronizeQueues)
        .def("SynchronizeDevice", &ktt::Tuner::SynchronizeDevice)
        .def("SetCompilerOptions", &ktt::Tuner::SetCompilerOptions, py::arg("options"), py::arg("overrideDefault") = false)
        .def("SetGlobalSizeType", &ktt::Tuner::SetGlobalSizeType)
        .def("SetAutomaticGlobalSizeCorrection", &ktt::Tuner::SetAutomaticGlobalSizeCorrection)
        .def("SetKernelCacheCapacity", &ktt::Tuner::SetKernelCacheCapacity)
        .def("GetPlatformInfo", &ktt::Tuner::GetPlatformInfo)
        .def("GetDeviceInfo", &ktt::Tuner::GetDeviceInfo)
        .def("GetCurrentDeviceInfo", &ktt::Tuner::GetCurrentDeviceInfo)
        .def_static("SetLoggingLevel", &ktt::Tuner::SetLoggingLevel)
        .def_static("GetLoggingLevel", &ktt::Tuner::GetLoggingLevel)
        .def_static("SetLoggingTarget", py::overload_cast<const std::string&>(&ktt::Tuner::SetLoggingTarget));

    // ---- the JSON tuning-script loader ----
    py::class_<ktt::TuningLoader>(m, "TuningLoader")
        .def(py::init<>())
        .def("LoadTuningFile", &ktt::TuningLoader::LoadTuningFile, py::arg("file"),
            py::arg("parameters") = std::map<std::string, std::string>{})
        .def("ExecuteCommands", &ktt::TuningLoader::ExecuteCommands, py::call_guard<py::gil_scoped_release>())
        .def("GetTuner", &ktt::TuningLoader::GetTuner, py::return_value_policy::reference_internal)
        .def("GetKernelId", &ktt::TuningLoader::GetKernelId)
        .def("GetResults", &ktt::TuningLoader::GetResults);
}
