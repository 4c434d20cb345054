// Configuration.cpp -- DimensionVector, ParameterPair, KernelConfiguration (see include/ktt/Configuration.h).
//
// Semantics follow KTT 2.1.0 Source/Api/Configuration/DimensionVector.cpp (ModifyByValue,
// DivideCeil rounding up, "(x, y, z)" strings), ParameterPair.cpp ("NAME VALUE" strings, values
// compared by type) and KernelConfiguration.cpp (GeneratePrefix, GetString, Merge,
// GenerateNeighbours).
#include <algorithm>
#include <stdexcept>

#include <ktt/Configuration.h>

namespace ktt
{

DimensionVector::DimensionVector() : DimensionVector(1, 1, 1) {}
DimensionVector::DimensionVector(const size_t sizeX) : DimensionVector(sizeX, 1, 1) {}
DimensionVector::DimensionVector(const size_t sizeX, const size_t sizeY) : DimensionVector(sizeX, sizeY, 1) {}
DimensionVector::DimensionVector(const size_t sizeX, const size_t sizeY, const size_t sizeZ) :
    m_SizeX(sizeX), m_SizeY(sizeY), m_SizeZ(sizeZ)
{}

DimensionVector::DimensionVector(const std::vector<size_t>& vector) : DimensionVector()
{
    if (vector.size() > 3)
    {
        throw std::runtime_error("Dimension vector has at most three dimensions");
    }

    if (vector.size() > 0) m_SizeX = vector[0];
    if (vector.size() > 1) m_SizeY = vector[1];
    if (vector.size() > 2) m_SizeZ = vector[2];
}

void DimensionVector::SetSizeX(const size_t sizeX) { m_SizeX = sizeX; }
void DimensionVector::SetSizeY(const size_t sizeY) { m_SizeY = sizeY; }
void DimensionVector::SetSizeZ(const size_t sizeZ) { m_SizeZ = sizeZ; }

void DimensionVector::SetSize(const ModifierDimension dimension, const size_t size)
{
    switch (dimension)
    {
    case ModifierDimension::X: m_SizeX = size; break;
    case ModifierDimension::Y: m_SizeY = size; break;
    case ModifierDimension::Z: m_SizeZ = size; break;
    }
}

void DimensionVector::Multiply(const DimensionVector& factor)
{
    m_SizeX *= factor.m_SizeX;
    m_SizeY *= factor.m_SizeY;
    m_SizeZ *= factor.m_SizeZ;
}

void DimensionVector::Divide(const DimensionVector& divisor)
{
    m_SizeX /= divisor.m_SizeX;
    m_SizeY /= divisor.m_SizeY;
    m_SizeZ /= divisor.m_SizeZ;
}

void DimensionVector::RoundUp(const DimensionVector& multiple)
{
    auto up = [](size_t v, size_t m) { return m == 0 ? v : ((v + m - 1) / m) * m; };
    m_SizeX = up(m_SizeX, multiple.m_SizeX);
    m_SizeY = up(m_SizeY, multiple.m_SizeY);
    m_SizeZ = up(m_SizeZ, multiple.m_SizeZ);
}

void DimensionVector::ModifyByValue(const size_t value, const ModifierAction action, const ModifierDimension dimension)
{
    size_t size = GetSize(dimension);

    switch (action)
    {
    case ModifierAction::Add: size += value; break;
    case ModifierAction::Subtract: size -= value; break;
    case ModifierAction::Multiply: size *= value; break;
    case ModifierAction::Divide: size /= value; break;
    case ModifierAction::DivideCeil: size = (size + value - 1) / value; break;
    }

    SetSize(dimension, size);
}

size_t DimensionVector::GetSizeX() const { return m_SizeX; }
size_t DimensionVector::GetSizeY() const { return m_SizeY; }
size_t DimensionVector::GetSizeZ() const { return m_SizeZ; }

size_t DimensionVector::GetSize(const ModifierDimension dimension) const
{
    switch (dimension)
    {
    case ModifierDimension::X: return m_SizeX;
    case ModifierDimension::Y: return m_SizeY;
    case ModifierDimension::Z: return m_SizeZ;
    }

    return 0;
}

size_t DimensionVector::GetTotalSize() const { return m_SizeX * m_SizeY * m_SizeZ; }
std::vector<size_t> DimensionVector::GetVector() const { return {m_SizeX, m_SizeY, m_SizeZ}; }

std::string DimensionVector::GetString() const
{
    return "(" + std::to_string(m_SizeX) + ", " + std::to_string(m_SizeY) + ", " + std::to_string(m_SizeZ) + ")";
}

bool DimensionVector::operator==(const DimensionVector& other) const
{
    return m_SizeX == other.m_SizeX && m_SizeY == other.m_SizeY && m_SizeZ == other.m_SizeZ;
}

bool DimensionVector::operator!=(const DimensionVector& other) const { return !(*this == other); }

// ---- ParameterPair --------------------------------------------------------------------------

ParameterPair::ParameterPair() : m_Name(""), m_Value(static_cast<uint64_t>(0)) {}
ParameterPair::ParameterPair(const std::string& name, const ParameterValue& value) : m_Name(name), m_Value(value) {}

void ParameterPair::SetValue(const ParameterValue& value) { m_Value = value; }
const std::string& ParameterPair::GetName() const { return m_Name; }
std::string ParameterPair::GetString() const { return m_Name + " " + GetValueString(); }

std::string ParameterPair::GetValueString() const
{
    switch (GetValueType())
    {
    case ParameterValueType::Int: return std::to_string(std::get<int64_t>(m_Value));
    case ParameterValueType::UnsignedInt: return std::to_string(std::get<uint64_t>(m_Value));
    case ParameterValueType::Double: return std::to_string(std::get<double>(m_Value));
    case ParameterValueType::Bool: return std::get<bool>(m_Value) ? "true" : "false";
    case ParameterValueType::String: return std::get<std::string>(m_Value);
    }

    return "";
}

const ParameterValue& ParameterPair::GetValue() const { return m_Value; }

uint64_t ParameterPair::GetValueUint() const
{
    switch (GetValueType())
    {
    case ParameterValueType::UnsignedInt: return std::get<uint64_t>(m_Value);
    case ParameterValueType::Int: return static_cast<uint64_t>(std::get<int64_t>(m_Value));
    case ParameterValueType::Bool: return std::get<bool>(m_Value) ? 1 : 0;
    case ParameterValueType::Double: return static_cast<uint64_t>(std::get<double>(m_Value));
    default: throw std::runtime_error("Parameter " + m_Name + " does not hold a numeric value");
    }
}

ParameterValueType ParameterPair::GetValueType() const { return GetTypeFromValue(m_Value); }

bool ParameterPair::HasSameValue(const ParameterPair& other) const
{
    if (GetValueType() != other.GetValueType())
    {
        return false;
    }

    return m_Value == other.m_Value;
}

ParameterValueType ParameterPair::GetTypeFromValue(const ParameterValue& value)
{
    if (std::holds_alternative<int64_t>(value)) return ParameterValueType::Int;
    if (std::holds_alternative<uint64_t>(value)) return ParameterValueType::UnsignedInt;
    if (std::holds_alternative<double>(value)) return ParameterValueType::Double;
    if (std::holds_alternative<bool>(value)) return ParameterValueType::Bool;
    return ParameterValueType::String;
}

// ---- KernelConfiguration ----------------------------------------------------------------------

KernelConfiguration::KernelConfiguration() = default;
KernelConfiguration::KernelConfiguration(const std::vector<ParameterPair>& pairs) : m_Pairs(pairs) {}

const std::vector<ParameterPair>& KernelConfiguration::GetPairs() const { return m_Pairs; }
bool KernelConfiguration::IsValid() const { return !m_Pairs.empty(); }

std::string KernelConfiguration::GeneratePrefix() const
{
    std::string result;

    for (const auto& pair : m_Pairs)
    {
        result += "#define " + pair.GetString() + "\n";
    }

    return result;
}

std::string KernelConfiguration::GetString() const
{
    if (m_Pairs.empty())
    {
        return "empty";
    }

    std::string result;

    for (size_t i = 0; i < m_Pairs.size(); ++i)
    {
        result += m_Pairs[i].GetString();

        if (i + 1 != m_Pairs.size())
        {
            result += ", ";
        }
    }

    return result;
}

void KernelConfiguration::Merge(const KernelConfiguration& other)
{
    for (const auto& pair : other.m_Pairs)
    {
        const bool present = std::any_of(m_Pairs.cbegin(), m_Pairs.cend(),
            [&pair](const auto& own) { return own.GetName() == pair.GetName(); });

        if (!present)
        {
            m_Pairs.push_back(pair);
        }
    }
}

std::vector<KernelConfiguration> KernelConfiguration::GenerateNeighbours(const std::string& parameter,
    const std::vector<ParameterPair>& pairs) const
{
    size_t index = m_Pairs.size();

    for (size_t i = 0; i < m_Pairs.size(); ++i)
    {
        if (m_Pairs[i].GetName() == parameter)
        {
            index = i;
            break;
        }
    }

    if (index == m_Pairs.size())
    {
        throw std::runtime_error("Configuration has no parameter " + parameter);
    }

    std::vector<KernelConfiguration> result;

    for (const auto& pair : pairs)
    {
        if (pair.HasSameValue(m_Pairs[index]))
        {
            continue;
        }

        auto newPairs = m_Pairs;
        newPairs[index] = pair;
        result.emplace_back(newPairs);
    }

    return result;
}

bool KernelConfiguration::operator==(const KernelConfiguration& other) const
{
    if (m_Pairs.size() != other.m_Pairs.size())
    {
        return false;
    }

    for (const auto& pair : m_Pairs)
    {
        const bool found = std::any_of(other.m_Pairs.cbegin(), other.m_Pairs.cend(),
            [&pair](const auto& o) { return o.GetName() == pair.GetName() && o.HasSameValue(pair); });

        if (!found)
        {
            return false;
        }
    }

    return true;
}

bool KernelConfiguration::operator!=(const KernelConfiguration& other) const { return !(*this == other); }

} // namespace ktt
