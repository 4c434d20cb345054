// Tuner.cpp -- the public ktt::Tuner facade.
//
// Every method forwards to TunerCore inside a try block; failures are logged at Error level and
// turned into the invalid return values of KTT 2.1.0 (Source/Tuner.cpp:40-150): InvalidKernelId,
// InvalidKernelDefinitionId, InvalidArgumentId, an empty configuration, or a KernelResult whose
// status says what went wrong.
#include <algorithm>
#include <cstring>
#include <fstream>
#include <iterator>
#include <memory>
#include <sstream>

#include <ktt/ProfileBasedSearcher.h>

#include "Logger.h"
#include "Script.h"
#include "TunerCore.h"

namespace ktt
{

namespace
{

template <typename F, typename R>
R Guarded(F&& f, R fallback)
{
    try
    {
        return f();
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
        return fallback;
    }
}

template <typename F>
void GuardedVoid(F&& f)
{
    try
    {
        f();
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
    }
}

} // namespace

// ---- DeviceInfo, PlatformInfo ---------------------------------------------------------------------

DeviceInfo::DeviceInfo(const DeviceIndex index, const std::string& name) : m_Index(index), m_Name(name) {}

DeviceInfo::DeviceInfo(const DeviceIndex index, const std::string& name, const uint64_t globalMemorySize, const uint32_t smCount,
    const uint32_t ccMajor, const uint32_t ccMinor) :
    m_Index(index), m_Name(name), m_GlobalMemorySize(globalMemorySize), m_SmCount(smCount), m_CcMajor(ccMajor),
    m_CcMinor(ccMinor)
{}

DeviceIndex DeviceInfo::GetIndex() const { return m_Index; }
const std::string& DeviceInfo::GetName() const { return m_Name; }
const std::string& DeviceInfo::GetVendor() const { return m_Vendor; }
const std::string& DeviceInfo::GetExtensions() const { return m_Extensions; }
DeviceType DeviceInfo::GetDeviceType() const { return m_DeviceType; }
uint64_t DeviceInfo::GetGlobalMemorySize() const { return m_GlobalMemorySize; }
uint64_t DeviceInfo::GetLocalMemorySize() const { return m_LocalMemorySize; }
uint64_t DeviceInfo::GetMaxConstantBufferSize() const { return m_MaxConstantBufferSize; }
uint64_t DeviceInfo::GetMaxWorkGroupSize() const { return m_MaxWorkGroupSize; }
uint32_t DeviceInfo::GetMaxComputeUnits() const { return m_SmCount; }
uint32_t DeviceInfo::GetCudaComputeCapabilityMajor() const { return m_CcMajor; }
uint32_t DeviceInfo::GetCudaComputeCapabilityMinor() const { return m_CcMinor; }

std::string DeviceInfo::GetDeviceTypeString() const
{
    switch (m_DeviceType)
    {
    case DeviceType::CPU:
        return "CPU";
    case DeviceType::GPU:
        return "GPU";
    default:
        return "Custom";
    }
}

// The same fields, labels and order as KTT's DeviceInfo::GetString (DeviceInfo.cpp:96-113).
std::string DeviceInfo::GetString() const
{
    std::string result;
    result += "Information about device with index: " + std::to_string(m_Index) + "\n";
    result += "Name: " + m_Name + "\n";
    result += "Vendor: " + m_Vendor + "\n";
    result += "Device type: " + GetDeviceTypeString() + "\n";
    result += "Global memory size: " + std::to_string(m_GlobalMemorySize) + "\n";
    result += "Local memory size: " + std::to_string(m_LocalMemorySize) + "\n";
    result += "Maximum constant buffer size: " + std::to_string(m_MaxConstantBufferSize) + "\n";
    result += "Maximum work-group size: " + std::to_string(m_MaxWorkGroupSize) + "\n";
    result += "Maximum parallel compute units: " + std::to_string(m_SmCount) + "\n";
    result += "Extensions: " + m_Extensions + "\n";
    result += "CUDA compute capability: " + std::to_string(m_CcMajor) + "." + std::to_string(m_CcMinor) + "\n";
    return result;
}

void DeviceInfo::SetVendor(const std::string& vendor) { m_Vendor = vendor; }
void DeviceInfo::SetExtensions(const std::string& extensions) { m_Extensions = extensions; }
void DeviceInfo::SetDeviceType(const DeviceType deviceType) { m_DeviceType = deviceType; }
void DeviceInfo::SetGlobalMemorySize(const uint64_t size) { m_GlobalMemorySize = size; }
void DeviceInfo::SetLocalMemorySize(const uint64_t size) { m_LocalMemorySize = size; }
void DeviceInfo::SetMaxConstantBufferSize(const uint64_t size) { m_MaxConstantBufferSize = size; }
void DeviceInfo::SetMaxWorkGroupSize(const uint64_t size) { m_MaxWorkGroupSize = size; }
void DeviceInfo::SetMaxComputeUnits(const uint32_t units) { m_SmCount = units; }
void DeviceInfo::SetCudaComputeCapabilityMajor(const uint32_t major) { m_CcMajor = major; }
void DeviceInfo::SetCudaComputeCapabilityMinor(const uint32_t minor) { m_CcMinor = minor; }

PlatformInfo::PlatformInfo(const PlatformIndex index, const std::string& name) : m_Index(index), m_Name(name) {}
PlatformIndex PlatformInfo::GetIndex() const { return m_Index; }
const std::string& PlatformInfo::GetName() const { return m_Name; }
const std::string& PlatformInfo::GetVendor() const { return m_Vendor; }
const std::string& PlatformInfo::GetVersion() const { return m_Version; }
const std::string& PlatformInfo::GetExtensions() const { return m_Extensions; }
void PlatformInfo::SetVendor(const std::string& vendor) { m_Vendor = vendor; }
void PlatformInfo::SetVersion(const std::string& version) { m_Version = version; }
void PlatformInfo::SetExtensions(const std::string& extensions) { m_Extensions = extensions; }

// KTT's PlatformInfo::GetString layout (PlatformInfo.cpp:36-47).
std::string PlatformInfo::GetString() const
{
    std::string result;
    result += "Information about platform with index: " + std::to_string(m_Index) + "\n";
    result += "Name: " + m_Name + "\n";
    result += "Vendor: " + m_Vendor + "\n";
    result += "Compute API version: " + m_Version + "\n";
    result += "Extensions: " + m_Extensions + "\n";
    return result;
}

// ---- Tuner ------------------------------------------------------------------------------------

Tuner::Tuner(const PlatformIndex platform, const DeviceIndex device, const ComputeApi api) : Tuner(platform, device, api, 1) {}

Tuner::Tuner([[maybe_unused]] const PlatformIndex platform, const DeviceIndex device, const ComputeApi api,
    [[maybe_unused]] const uint32_t computeQueueCount) :
    m_Core(std::make_unique<TunerCore>(device, api))
{}

Tuner::Tuner(const ComputeApi api, const ComputeApiInitializer& initializer) :
    m_Core(std::make_unique<TunerCore>(0, api))
{
    std::vector<QueueId> ignored;
    m_Core->AdoptContext(initializer, ignored);
}

Tuner::Tuner(const ComputeApi api, const ComputeApiInitializer& initializer, std::vector<QueueId>& assignedQueueIds) :
    m_Core(std::make_unique<TunerCore>(0, api))
{
    m_Core->AdoptContext(initializer, assignedQueueIds);
}

Tuner::~Tuner() = default;

ComputeApiInitializer::ComputeApiInitializer(ComputeContext context, const std::vector<ComputeQueue>& queues) :
    m_Context(context), m_Queues(queues)
{}

ComputeContext ComputeApiInitializer::GetContext() const { return m_Context; }
const std::vector<ComputeQueue>& ComputeApiInitializer::GetQueues() const { return m_Queues; }

KernelDefinitionId Tuner::AddKernelDefinition(const std::string& name, const std::string& source, const DimensionVector& globalSize,
    const DimensionVector& localSize, const std::vector<std::string>& typeNames)
{
    return Guarded([&] { return m_Core->AddDefinition(name, source, globalSize, localSize, typeNames); },
        InvalidKernelDefinitionId);
}

KernelDefinitionId Tuner::AddKernelDefinitionFromFile(const std::string& name, const std::string& filePath,
    const DimensionVector& globalSize, const DimensionVector& localSize, const std::vector<std::string>& typeNames)
{
    return Guarded([&]
    {
        std::ifstream file(filePath);
        std::string source;

        if (file)
        {
            source.assign(std::istreambuf_iterator<char>(file), std::istreambuf_iterator<char>());
        }
        else
        {
            // The kernel runs from its built-in sm_100a implementation; the source text is only kept
            // for GetKernelSource, so a missing file is reported but not fatal.
            log::Warning("Kernel source file " + filePath + " was not found; the definition keeps an empty source");
        }

        return m_Core->AddDefinition(name, source, globalSize, localSize, typeNames);
    }, InvalidKernelDefinitionId);
}

KernelDefinitionId Tuner::AddKernelDefinition(const std::string& name, const std::string& source,
    const std::vector<std::string>& typeNames)
{
    return AddKernelDefinition(name, source, DimensionVector(), DimensionVector(), typeNames);
}

KernelDefinitionId Tuner::AddKernelDefinitionFromFile(const std::string& name, const std::string& filePath,
    const std::vector<std::string>& typeNames)
{
    return AddKernelDefinitionFromFile(name, filePath, DimensionVector(), DimensionVector(), typeNames);
}

KernelDefinitionId Tuner::GetKernelDefinitionId(const std::string& name, const std::vector<std::string>& typeNames) const
{
    return m_Core->GetDefinitionId(name, typeNames);
}

void Tuner::RemoveKernelDefinition(const KernelDefinitionId id) { GuardedVoid([&] { m_Core->RemoveDefinition(id); }); }

void Tuner::SetArguments(const KernelDefinitionId id, const std::vector<ArgumentId>& argumentIds)
{
    GuardedVoid([&] { m_Core->SetArguments(id, argumentIds); });
}

KernelId Tuner::CreateSimpleKernel(const std::string& name, const KernelDefinitionId definitionId)
{
    return Guarded([&] { return m_Core->CreateKernel(name, {definitionId}, nullptr); }, InvalidKernelId);
}

KernelId Tuner::CreateCompositeKernel(const std::string& name, const std::vector<KernelDefinitionId>& definitionIds,
    KernelLauncher launcher)
{
    return Guarded([&] { return m_Core->CreateKernel(name, definitionIds, launcher); }, InvalidKernelId);
}

void Tuner::RemoveKernel(const KernelId id) { GuardedVoid([&] { m_Core->RemoveKernel(id); }); }
void Tuner::SetLauncher(const KernelId id, KernelLauncher launcher) { GuardedVoid([&] { m_Core->SetLauncher(id, launcher); }); }

void Tuner::AddParameterInternal(const KernelId id, const std::string& name, const std::vector<ParameterValue>& values,
    const std::string& group)
{
    GuardedVoid([&] { m_Core->AddParameter(id, name, values, group); });
}

void Tuner::AddThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds, const ModifierType type,
    const ModifierDimension dimension, const std::vector<std::string>& parameters, ModifierFunction function)
{
    GuardedVoid([&]
    {
        ModifierData data;
        data.type = type;
        data.dimension = dimension;
        data.definitions = definitionIds;
        data.parameters = parameters;
        data.function = function;
        m_Core->AddModifier(id, data);
    });
}

void Tuner::AddThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds, const ModifierType type,
    const ModifierDimension dimension, const std::string& parameter, const ModifierAction action)
{
    AddThreadModifier(id, definitionIds, type, dimension, std::vector<std::string>{parameter},
        [action, dimension](const uint64_t size, const std::vector<uint64_t>& values)
        {
            DimensionVector v;
            v.SetSize(dimension, static_cast<size_t>(size));
            v.ModifyByValue(static_cast<size_t>(values.at(0)), action, dimension);
            return static_cast<uint64_t>(v.GetSize(dimension));
        });
}

void Tuner::AddConstraint(const KernelId id, const std::vector<std::string>& parameters, ConstraintFunction function)
{
    GuardedVoid([&]
    {
        m_Core->AddConstraint(id, parameters, [function](const std::vector<const ParameterValue*>& values)
        {
            std::vector<uint64_t> plain;

            for (const auto* v : values)
            {
                plain.push_back(std::get<uint64_t>(*v));
            }

            return function(plain);
        }, true);
    });
}

void Tuner::AddGenericConstraint(const KernelId id, const std::vector<std::string>& parameters, GenericConstraintFunction function)
{
    GuardedVoid([&] { m_Core->AddConstraint(id, parameters, function, false); });
}

// ---- script forms (Source/Tuner.h:233-336 of KTT; evaluated by Script.cpp) ----------------------

namespace
{

script::Value ScriptValue(const ParameterValue& v, const std::string& name)
{
    if (const auto* p = std::get_if<uint64_t>(&v)) return script::Value::Int(static_cast<int64_t>(*p));
    if (const auto* p = std::get_if<int64_t>(&v)) return script::Value::Int(*p);
    if (const auto* p = std::get_if<double>(&v)) return script::Value::Float(*p);
    if (const auto* p = std::get_if<bool>(&v)) return script::Value::Bool(*p);
    throw std::runtime_error("string parameter " + name + " cannot be used in a script");
}

ParameterValue ParameterFromScript(const script::Value& v, const ParameterValueType type, const std::string& name)
{
    switch (type)
    {
    case ParameterValueType::UnsignedInt:
        if (v.kind == script::Value::Kind::Float || v.AsInt() < 0)
        {
            throw std::runtime_error("value " + v.Repr() + " of parameter " + name + " is not an unsigned integer");
        }
        return static_cast<uint64_t>(v.AsInt());
    case ParameterValueType::Int:
        if (v.kind == script::Value::Kind::Float)
        {
            throw std::runtime_error("value " + v.Repr() + " of parameter " + name + " is not an integer");
        }
        return v.AsInt();
    case ParameterValueType::Double: return v.AsDouble();
    case ParameterValueType::Bool: return v.Truthy();
    case ParameterValueType::String: break;
    }

    throw std::runtime_error("string parameters cannot be produced by a values script (parameter " + name + ")");
}

template <typename T>
void AppendBytes(std::vector<uint8_t>& out, const T value)
{
    const auto* p = reinterpret_cast<const uint8_t*>(&value);
    out.insert(out.end(), p, p + sizeof(T));
}

size_t DataTypeSize(const ArgumentDataType type)
{
    switch (type)
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
    case ArgumentDataType::Custom: return 0;
    }

    return 0;
}

} // namespace

void Tuner::AddScriptParameter(const KernelId id, const std::string& name, const ParameterValueType valueType,
    const std::string& valueScript, const std::string& group)
{
    GuardedVoid([&]
    {
        const script::Expression expression(valueScript);
        const script::Value list = expression.Evaluate(script::Environment());

        if (list.kind != script::Value::Kind::List || list.list.empty())
        {
            throw std::runtime_error("the values script of parameter " + name + " must yield a non-empty list");
        }

        std::vector<ParameterValue> values;

        for (const auto& v : list.list)
        {
            values.push_back(ParameterFromScript(v, valueType, name));
        }

        m_Core->AddParameter(id, name, values, group);
    });
}

void Tuner::AddScriptThreadModifier(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds,
    const ModifierType type, const ModifierDimension dimension, const std::string& script)
{
    GuardedVoid([&]
    {
        auto expression = std::make_shared<script::Expression>(script);
        std::vector<std::string> names;

        for (const auto& free : expression->FreeNames())
        {
            if (free == "defaultSize")
            {
                continue;
            }

            const auto& parameters = m_Core->Kernel(id).parameters;
            const bool known = std::any_of(parameters.cbegin(), parameters.cend(),
                [&](const KernelParameterInfo& p) { return p.name == free; });

            if (!known)
            {
                throw std::runtime_error("thread modifier script '" + script + "' reads " + free
                    + ", which is not a tuning parameter of the kernel");
            }

            names.push_back(free);
        }

        ModifierData data;
        data.type = type;
        data.dimension = dimension;
        data.definitions = definitionIds;
        data.parameters = names;
        data.function = [expression, names](const uint64_t defaultSize, const std::vector<uint64_t>& values)
        {
            script::Environment env;
            env.Set("defaultSize", script::Value::Int(static_cast<int64_t>(defaultSize)));

            for (size_t k = 0; k < names.size(); ++k)
            {
                env.Set(names[k], script::Value::Int(static_cast<int64_t>(values[k])));
            }

            const int64_t size = expression->Evaluate(env).AsInt();

            if (size < 0)
            {
                throw std::runtime_error("thread modifier script '" + expression->Source() + "' gave a negative size");
            }

            return static_cast<uint64_t>(size);
        };
        m_Core->AddModifier(id, data);
    });
}

void Tuner::AddScriptConstraint(const KernelId id, const std::vector<std::string>& parameters, const std::string& script)
{
    GuardedVoid([&]
    {
        auto expression = std::make_shared<script::Expression>(script);
        m_Core->AddConstraint(id, parameters, [expression, parameters](const std::vector<const ParameterValue*>& values)
        {
            script::Environment env;

            for (size_t k = 0; k < parameters.size(); ++k)
            {
                env.Set(parameters[k], ScriptValue(*values[k], parameters[k]));
            }

            return expression->Evaluate(env).Truthy();
        }, false);
    });
}

ArgumentId Tuner::AddArgumentVectorFromFile(const std::string& filePath, const ArgumentDataType dataType, const size_t elementSize,
    const ArgumentAccessType accessType, [[maybe_unused]] const ArgumentMemoryLocation memoryLocation,
    [[maybe_unused]] const ArgumentManagementType managementType, const ArgumentId& customId)
{
    std::vector<uint8_t> data;

    try
    {
        std::ifstream file(filePath, std::ios::binary);

        if (!file)
        {
            throw std::runtime_error("Unable to open argument data file " + filePath);
        }

        data.assign(std::istreambuf_iterator<char>(file), std::istreambuf_iterator<char>());

        if (elementSize == 0 || data.size() % elementSize != 0)
        {
            throw std::runtime_error("File " + filePath + " holds " + std::to_string(data.size())
                + " bytes, not a whole number of " + std::to_string(elementSize) + "-byte elements");
        }
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
        return InvalidArgumentId;
    }

    return AddArgumentWithOwnedData(elementSize, dataType, ArgumentMemoryType::Vector, accessType, data.data(), data.size(),
        customId);
}

ArgumentId Tuner::AddArgumentVectorFromGenerator(const std::string& generatorFunction, const ArgumentDataType dataType,
    const size_t bufferSize, const size_t elementSize, const ArgumentAccessType accessType,
    [[maybe_unused]] const ArgumentMemoryLocation memoryLocation, [[maybe_unused]] const ArgumentManagementType managementType,
    const ArgumentId& customId)
{
    std::vector<uint8_t> data;

    try
    {
        if (elementSize == 0 || DataTypeSize(dataType) != elementSize || bufferSize % elementSize != 0)
        {
            throw std::runtime_error("Generated argument: element size " + std::to_string(elementSize)
                + " does not match its data type, or the buffer size " + std::to_string(bufferSize)
                + " is not a whole number of elements");
        }

        const script::Expression expression(generatorFunction);
        const size_t count = bufferSize / elementSize;
        data.reserve(bufferSize);
        script::Environment env;

        for (size_t i = 0; i < count; ++i)
        {
            env.Set("i", script::Value::Int(static_cast<int64_t>(i)));
            const script::Value v = expression.Evaluate(env);

            switch (dataType)
            {
            case ArgumentDataType::Float: AppendBytes(data, static_cast<float>(v.AsDouble())); break;
            case ArgumentDataType::Double: AppendBytes(data, v.AsDouble()); break;
            case ArgumentDataType::Char: AppendBytes(data, static_cast<int8_t>(v.AsInt())); break;
            case ArgumentDataType::UnsignedChar: AppendBytes(data, static_cast<uint8_t>(v.AsInt())); break;
            case ArgumentDataType::Short: AppendBytes(data, static_cast<int16_t>(v.AsInt())); break;
            case ArgumentDataType::UnsignedShort: AppendBytes(data, static_cast<uint16_t>(v.AsInt())); break;
            case ArgumentDataType::Int: AppendBytes(data, static_cast<int32_t>(v.AsInt())); break;
            case ArgumentDataType::UnsignedInt: AppendBytes(data, static_cast<uint32_t>(v.AsInt())); break;
            case ArgumentDataType::Long: AppendBytes(data, static_cast<int64_t>(v.AsInt())); break;
            case ArgumentDataType::UnsignedLong: AppendBytes(data, static_cast<uint64_t>(v.AsInt())); break;
            default: throw std::runtime_error("Generated arguments of this data type are not supported");
            }
        }
    }
    catch (const std::exception& e)
    {
        log::Error(e.what());
        return InvalidArgumentId;
    }

    return AddArgumentWithOwnedData(elementSize, dataType, ArgumentMemoryType::Vector, accessType, data.data(), data.size(),
        customId);
}

void Tuner::SaveArgumentVector(const ArgumentId& id, const std::string& filePath)
{
    GuardedVoid([&]
    {
        ArgumentData& argument = m_Core->Argument(id);

        if (argument.memoryType != ArgumentMemoryType::Vector)
        {
            throw std::runtime_error("Argument " + id + " is not a vector");
        }

        std::vector<uint8_t> bytes(argument.bytes);

        if (argument.ownership == ArgumentOwnership::User || argument.deviceCurrent)
        {
            m_Core->DownloadArgument(argument, bytes.data(), bytes.size());
        }
        else
        {
            std::memcpy(bytes.data(), argument.HostData(), bytes.size());
        }

        std::ofstream file(filePath, std::ios::binary);

        if (!file)
        {
            throw std::runtime_error("Unable to write " + filePath);
        }

        file.write(reinterpret_cast<const char*>(bytes.data()), static_cast<std::streamsize>(bytes.size()));
    });
}

ArgumentId Tuner::AddArgumentWithOwnedData(const size_t elementSize, const ArgumentDataType dataType,
    const ArgumentMemoryType memoryType, const ArgumentAccessType accessType, const void* data, const size_t dataSize,
    const ArgumentId& customId)
{
    return Guarded([&]
    {
        ArgumentData argument;
        argument.dataType = dataType;
        argument.memoryType = memoryType;
        argument.accessType = accessType;
        argument.ownership = ArgumentOwnership::Owned;
        argument.elementSize = elementSize;
        argument.bytes = dataSize;
        argument.owned.assign(static_cast<const uint8_t*>(data), static_cast<const uint8_t*>(data) + dataSize);
        return m_Core->AddArgument(std::move(argument), customId);
    }, InvalidArgumentId);
}

ArgumentId Tuner::AddArgumentScalar(const void* data, const size_t dataSize, const ArgumentId& customId)
{
    if (data == nullptr || dataSize == 0)
    {
        log::Error("Scalar argument data must not be empty");
        return InvalidArgumentId;
    }

    return AddArgumentWithOwnedData(dataSize, ArgumentDataType::Custom, ArgumentMemoryType::Scalar, ArgumentAccessType::ReadOnly,
        data, dataSize, customId);
}

ArgumentId Tuner::AddSpecialArgument(const size_t elementSize, const ArgumentDataType dataType,
    const ArgumentMemoryType memoryType, const void* data, const size_t dataSize, const std::string& symbolName,
    const ArgumentId& customId)
{
    return Guarded([&]
    {
        if (dataSize == 0)
        {
            throw std::runtime_error(memoryType == ArgumentMemoryType::Local ? "Local memory size must be positive"
                : "Symbol argument data must not be empty");
        }

        ArgumentData argument;
        argument.dataType = dataType;
        argument.memoryType = memoryType;
        argument.accessType = ArgumentAccessType::ReadOnly;
        argument.ownership = ArgumentOwnership::Owned;
        argument.elementSize = elementSize;
        argument.bytes = dataSize;
        argument.symbolName = symbolName;

        if (data != nullptr)
        {
            argument.owned.assign(static_cast<const uint8_t*>(data), static_cast<const uint8_t*>(data) + dataSize);
        }

        return m_Core->AddArgument(std::move(argument), customId);
    }, InvalidArgumentId);
}

ArgumentId Tuner::AddArgumentWithReferencedData(const size_t elementSize, const ArgumentDataType dataType,
    const ArgumentAccessType accessType, void* data, const size_t dataSize, const ArgumentId& customId)
{
    return Guarded([&]
    {
        ArgumentData argument;
        argument.dataType = dataType;
        argument.memoryType = ArgumentMemoryType::Vector;
        argument.accessType = accessType;
        argument.ownership = ArgumentOwnership::Referenced;
        argument.elementSize = elementSize;
        argument.bytes = dataSize;
        argument.referenced = data;
        return m_Core->AddArgument(std::move(argument), customId);
    }, InvalidArgumentId);
}

ArgumentId Tuner::AddUserArgument(ComputeBuffer buffer, const size_t elementSize, const ArgumentDataType dataType,
    const ArgumentAccessType accessType, const size_t bufferSize, const ArgumentId& customId)
{
    return Guarded([&]
    {
        ArgumentData argument;
        argument.dataType = dataType;
        argument.memoryType = ArgumentMemoryType::Vector;
        argument.accessType = accessType;
        argument.ownership = ArgumentOwnership::User;
        argument.elementSize = elementSize;
        argument.bytes = bufferSize;
        argument.userDevice = buffer;
        argument.deviceCurrent = true;
        return m_Core->AddArgument(std::move(argument), customId);
    }, InvalidArgumentId);
}

void Tuner::RemoveArgument(const ArgumentId& id) { GuardedVoid([&] { m_Core->RemoveArgument(id); }); }
void Tuner::SetReadOnlyArgumentCache(const bool flag) { m_Core->SetReadOnlyCache(flag); }

KernelResult Tuner::Run(const KernelId id, const KernelConfiguration& configuration, const std::vector<BufferOutputDescriptor>& output)
{
    return Guarded([&] { return m_Core->Run(id, configuration, output, KernelRunMode::Running); },
        [&] { KernelResult r("", configuration); r.SetStatus(ResultStatus::ComputationFailed); return r; }());
}

void Tuner::SetProfiling(const bool flag) { m_Core->SetProfiling(flag); }

void Tuner::SetProfilingCounters(const std::vector<std::string>& counters)
{
    GuardedVoid([&] { m_Core->SetProfilingCounters(counters); });
}

void Tuner::SetProfiledDefinitions(const KernelId id, const std::vector<KernelDefinitionId>& definitionIds)
{
    GuardedVoid([&] { m_Core->SetProfiledDefinitions(id, definitionIds); });
}

bool Tuner::GetProfiling() { return m_Core->GetProfiling(); }

void Tuner::SetValidationMethod(const ValidationMethod method, const double toleranceThreshold)
{
    GuardedVoid([&] { m_Core->SetValidationMethod(method, toleranceThreshold); });
}

void Tuner::SetValidationMode(const ValidationMode mode) { m_Core->SetValidationMode(mode); }

void Tuner::SetValidationRange(const ArgumentId& id, const size_t range)
{
    GuardedVoid([&] { m_Core->Validation(id).range = range; });
}

void Tuner::SetValueComparator(const ArgumentId& id, ValueComparator comparator)
{
    GuardedVoid([&] { m_Core->Validation(id).comparator = comparator; });
}

void Tuner::SetReferenceComputation(const ArgumentId& id, ReferenceComputation computation)
{
    GuardedVoid([&]
    {
        ValidationData& data = m_Core->Validation(id);
        data.computation = computation;
        data.referenceKernel = InvalidKernelId;
        data.referenceArgument.clear();
        data.computed = false;
    });
}

void Tuner::SetReferenceKernel(const ArgumentId& id, const KernelId referenceId, const KernelConfiguration& configuration)
{
    GuardedVoid([&]
    {
        (void)m_Core->Kernel(referenceId);
        ValidationData& data = m_Core->Validation(id);
        data.computation = nullptr;
        data.referenceKernel = referenceId;
        data.referenceConfiguration = configuration;
        data.referenceArgument.clear();
        data.computed = false;
    });
}

void Tuner::SetReferenceArgument(const ArgumentId& id, const ArgumentId& referenceId)
{
    GuardedVoid([&]
    {
        (void)m_Core->Argument(referenceId);
        ValidationData& data = m_Core->Validation(id);
        data.computation = nullptr;
        data.referenceKernel = InvalidKernelId;
        data.referenceArgument = referenceId;
        data.computed = false;
    });
}

std::vector<KernelResult> Tuner::Tune(const KernelId id, std::unique_ptr<StopCondition> stopCondition)
{
    return Guarded([&] { return m_Core->Tune(id, std::move(stopCondition)); }, std::vector<KernelResult>{});
}

KernelResult Tuner::TuneIteration(const KernelId id, const std::vector<BufferOutputDescriptor>& output, const bool recomputeReference)
{
    return Guarded([&] { return m_Core->TuneIteration(id, output, recomputeReference); },
        [&] { KernelResult r; r.SetStatus(ResultStatus::ComputationFailed); return r; }());
}

std::vector<KernelResult> Tuner::SimulateTuning(const KernelId id, const std::vector<KernelResult>& results, const uint64_t iterations)
{
    return Guarded([&] { return m_Core->SimulateTuning(id, results, iterations, nullptr); }, std::vector<KernelResult>{});
}

std::vector<KernelResult> Tuner::SimulateTuning(const KernelId id, const std::vector<KernelResult>& results,
    std::unique_ptr<StopCondition> stopCondition)
{
    return Guarded([&] { return m_Core->SimulateTuning(id, results, 0, stopCondition.get()); }, std::vector<KernelResult>{});
}

void Tuner::SetSearcher(const KernelId id, std::unique_ptr<Searcher> searcher)
{
    GuardedVoid([&] { m_Core->SetSearcher(id, std::move(searcher)); });
}

void Tuner::SetProfileBasedSearcher(const KernelId id, const std::string& modelPath,
    [[maybe_unused]] const bool useBuiltinModule, const uint32_t batchSize, const uint32_t neighborSize,
    const uint32_t randomSize)
{
    // Source/Tuner.cpp:591-615 imports the Python searcher module and a pickled model; here the
    // searcher is native and the model is the JSON forest written by ktt_b200/profile_model.py, read
    // from modelPath or, for a KTT model path such as "X.sav", from "X.sav.json".
    GuardedVoid([&]
    {
        CounterModel model;
        std::string error;

        for (const auto& path : {modelPath, modelPath + ".json"})
        {
            try
            {
                model = CounterModel::Load(path);
                break;
            }
            catch (const std::exception& e)
            {
                error += std::string(error.empty() ? "" : "; ") + e.what();
            }
        }

        if (model.IsEmpty())
        {
            throw std::runtime_error("No counter model for the profile-based searcher (" + error
                + "); pickled scikit-learn models are not loaded, convert them with ktt_b200/profile_model.py");
        }

        m_Core->SetSearcher(id, std::make_unique<ProfileBasedSearcher>(*this, model, batchSize, neighborSize, randomSize));
    });
}

void Tuner::InitializeConfigurationData(const KernelId id) { GuardedVoid([&] { (void)m_Core->Space(id); }); }
void Tuner::ClearConfigurationData(const KernelId id) { GuardedVoid([&] { m_Core->ClearSpace(id); }); }

uint64_t Tuner::GetConfigurationsCount(const KernelId id) const
{
    return Guarded([&] { return m_Core->Space(id).GetConfigurationsCount(); }, uint64_t{0});
}

KernelConfiguration Tuner::GetBestConfiguration(const KernelId id) const
{
    return Guarded([&] { return m_Core->Space(id).GetBestConfiguration(); }, KernelConfiguration());
}

KernelConfiguration Tuner::CreateConfiguration(const KernelId id, const ParameterInput& parameters) const
{
    return Guarded([&] { return m_Core->CreateConfiguration(id, parameters); }, KernelConfiguration());
}

std::string Tuner::GetKernelSource(const KernelId id, const KernelConfiguration& configuration) const
{
    return Guarded([&] { return m_Core->GetKernelSource(id, configuration); }, std::string());
}

std::string Tuner::GetKernelDefinitionSource(const KernelDefinitionId id, const KernelConfiguration& configuration) const
{
    return Guarded([&] { return m_Core->GetDefinitionSource(id, configuration); }, std::string());
}

QueueId Tuner::AddComputeQueue(ComputeQueue queue)
{
    return Guarded([&] { return m_Core->AddQueue(queue); }, InvalidQueueId);
}

void Tuner::RemoveComputeQueue(const QueueId id) { GuardedVoid([&] { m_Core->RemoveQueue(id); }); }
void Tuner::WaitForComputeAction([[maybe_unused]] const ComputeActionId id) { GuardedVoid([&] { m_Core->Synchronize(); }); }
void Tuner::WaitForTransferAction([[maybe_unused]] const TransferActionId id) { GuardedVoid([&] { m_Core->Synchronize(); }); }
void Tuner::SynchronizeQueue(const QueueId id) { GuardedVoid([&] { m_Core->SynchronizeQueue(id); }); }

void Tuner::SynchronizeQueues()
{
    GuardedVoid([&]
    {
        for (const auto id : m_Core->QueueIds())
        {
            m_Core->SynchronizeQueue(id);
        }
    });
}

void Tuner::SynchronizeDevice() { GuardedVoid([&] { m_Core->Synchronize(); }); }
void Tuner::SetCompilerOptions(const std::string& options, [[maybe_unused]] const bool overrideDefault)
{
    m_Core->SetCompilerOptions(options);
}

void Tuner::SetGlobalSizeType(const GlobalSizeType type) { m_Core->SetGlobalSizeType(type); }
void Tuner::SetAutomaticGlobalSizeCorrection([[maybe_unused]] const bool flag) {}
void Tuner::SetKernelCacheCapacity([[maybe_unused]] const uint64_t capacity) {}

std::vector<PlatformInfo> Tuner::GetPlatformInfo() const
{
    return Guarded([&] { return m_Core->GetPlatformInfo(); }, std::vector<PlatformInfo>{});
}

std::vector<DeviceInfo> Tuner::GetDeviceInfo(const PlatformIndex platform) const
{
    return Guarded([&] { return m_Core->GetDeviceInfo(platform); }, std::vector<DeviceInfo>{});
}

DeviceInfo Tuner::GetCurrentDeviceInfo() const
{
    return Guarded([&] { return m_Core->GetDeviceInfo(); }, DeviceInfo(0, "unavailable", 0, 0, 0, 0));
}

void Tuner::SetLoggingLevel(const LoggingLevel level) { log::state().level = level; }
LoggingLevel Tuner::GetLoggingLevel() { return log::state().level; }

void Tuner::SetLoggingTarget(std::ostream& outputTarget)
{
    log::state().file.reset();
    log::state().stream = &outputTarget;
}

void Tuner::SetLoggingTarget(const std::string& filePath)
{
    auto file = std::make_unique<std::ofstream>(filePath);

    if (!*file)
    {
        log::Error("Unable to open log file " + filePath);
        return;
    }

    log::state().stream = file.get();
    log::state().file = std::move(file);
}

} // namespace ktt
