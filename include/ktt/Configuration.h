// Configuration.h -- DimensionVector, ParameterPair and KernelConfiguration of the ktt:: surface.
//
// Interfaces of KTT 2.1.0 Source/Api/Configuration/DimensionVector.h, ParameterPair.h and
// KernelConfiguration.h (same member names and semantics: DivideCeil rounds up, GeneratePrefix
// emits "#define NAME VALUE\n" per pair in pair order, GetString joins "NAME: VALUE" with ", ").
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include <ktt/KttTypes.h>

namespace ktt
{

class KTT_API DimensionVector
{
public:
    DimensionVector();
    explicit DimensionVector(const size_t sizeX);
    explicit DimensionVector(const size_t sizeX, const size_t sizeY);
    explicit DimensionVector(const size_t sizeX, const size_t sizeY, const size_t sizeZ);
    explicit DimensionVector(const std::vector<size_t>& vector);

    void SetSizeX(const size_t sizeX);
    void SetSizeY(const size_t sizeY);
    void SetSizeZ(const size_t sizeZ);
    void SetSize(const ModifierDimension dimension, const size_t size);
    void Multiply(const DimensionVector& factor);
    void Divide(const DimensionVector& divisor);
    void RoundUp(const DimensionVector& multiple);
    void ModifyByValue(const size_t value, const ModifierAction action, const ModifierDimension dimension);

    size_t GetSizeX() const;
    size_t GetSizeY() const;
    size_t GetSizeZ() const;
    size_t GetSize(const ModifierDimension dimension) const;
    size_t GetTotalSize() const;
    std::vector<size_t> GetVector() const;
    std::string GetString() const;

    bool operator==(const DimensionVector& other) const;
    bool operator!=(const DimensionVector& other) const;

private:
    size_t m_SizeX;
    size_t m_SizeY;
    size_t m_SizeZ;
};

class KTT_API ParameterPair
{
public:
    ParameterPair();
    explicit ParameterPair(const std::string& name, const ParameterValue& value);

    void SetValue(const ParameterValue& value);
    const std::string& GetName() const;
    std::string GetString() const;
    std::string GetValueString() const;
    const ParameterValue& GetValue() const;
    uint64_t GetValueUint() const;
    ParameterValueType GetValueType() const;
    bool HasSameValue(const ParameterPair& other) const;

    static ParameterValueType GetTypeFromValue(const ParameterValue& value);

    template <typename T>
    static T GetParameterValue(const std::vector<ParameterPair>& pairs, const std::string& name)
    {
        for (const auto& pair : pairs)
        {
            if (pair.GetName() == name)
            {
                return std::get<T>(pair.GetValue());
            }
        }

        throw std::runtime_error("No parameter with name " + name);
    }

    template <typename T>
    static std::vector<T> GetParameterValues(const std::vector<ParameterPair>& pairs, const std::vector<std::string>& names)
    {
        std::vector<T> result;

        for (const auto& name : names)
        {
            result.push_back(GetParameterValue<T>(pairs, name));
        }

        return result;
    }

private:
    std::string m_Name;
    ParameterValue m_Value;
};

class KTT_API KernelConfiguration
{
public:
    KernelConfiguration();
    explicit KernelConfiguration(const std::vector<ParameterPair>& pairs);

    const std::vector<ParameterPair>& GetPairs() const;
    bool IsValid() const;
    std::string GeneratePrefix() const;
    std::string GetString() const;
    void Merge(const KernelConfiguration& other);
    std::vector<KernelConfiguration> GenerateNeighbours(const std::string& parameter,
        const std::vector<ParameterPair>& pairs) const;

    bool operator==(const KernelConfiguration& other) const;
    bool operator!=(const KernelConfiguration& other) const;

private:
    std::vector<ParameterPair> m_Pairs;
};

} // namespace ktt
