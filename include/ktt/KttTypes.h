// KttTypes.h -- type aliases, enumerations and constants of the ktt:: surface.
//
// Same names, values and meaning as KTT 2.1.0 (Source/KttTypes.h:22-160 and the enum headers under
// Source/Api, Source/Kernel, Source/KernelArgument, Source/KernelRunner, Source/Output), so that
// KTT host programs for the Coulomb path compile against this header unchanged.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <limits>
#include <map>
#include <string>
#include <utility>
#include <variant>
#include <vector>

#if defined(__GNUC__)
#define KTT_API __attribute__((visibility("default")))
#else
#define KTT_API
#endif

namespace ktt
{

class ComputeInterface;
class DimensionVector;

using PlatformIndex = uint32_t;
using DeviceIndex = uint32_t;
using QueueId = uint32_t;
using KernelDefinitionId = uint64_t;
using KernelId = uint64_t;
using ArgumentId = std::string;
using ParameterValue = std::variant<int64_t, uint64_t, double, bool, std::string>;
using ParameterInput = std::vector<std::pair<std::string, ParameterValue>>;
using UserData = std::map<std::string, std::string>;
using Nanoseconds = uint64_t;
using ComputeActionId = uint64_t;
using TransferActionId = uint64_t;
using ModifierFunction = std::function<uint64_t(const uint64_t /*defaultSize*/, const std::vector<uint64_t>& /*values*/)>;
using ConstraintFunction = std::function<bool(const std::vector<uint64_t>& /*values*/)>;
using GenericConstraintFunction = std::function<bool(const std::vector<const ParameterValue*>& /*values*/)>;
using KernelLauncher = std::function<void(ComputeInterface& /*interface*/)>;
using ReferenceComputation = std::function<void(void* /*buffer*/)>;
using ValueComparator = std::function<bool(const void* /*result*/, const void* /*reference*/)>;
using UnifiedBufferMemory = void*;
using ComputeContext = void*;
using ComputeQueue = void*;
using ComputeBuffer = void*;

inline const QueueId InvalidQueueId = std::numeric_limits<QueueId>::max();
inline const KernelDefinitionId InvalidKernelDefinitionId = std::numeric_limits<KernelDefinitionId>::max();
inline const KernelId InvalidKernelId = std::numeric_limits<KernelId>::max();
inline const ArgumentId InvalidArgumentId = ArgumentId();
inline const Nanoseconds InvalidDuration = std::numeric_limits<Nanoseconds>::max();

enum class ComputeApi { OpenCL, CUDA, Vulkan };
enum class GlobalSizeType { OpenCL, CUDA, Vulkan };
enum class ModifierType { Global, Local };
enum class ModifierDimension { X, Y, Z };
enum class ModifierAction { Add, Subtract, Multiply, Divide, DivideCeil };
enum class ParameterValueType { Int, UnsignedInt, Double, Float = Double, Bool, String };
enum class ArgumentDataType { Char, UnsignedChar, Short, UnsignedShort, Int, UnsignedInt, Long, UnsignedLong, Half, Float, Double, Custom };
enum class ArgumentMemoryType { Scalar, Vector, Local, Symbol };
enum class ArgumentAccessType { Undefined, ReadOnly, WriteOnly, ReadWrite };
enum class ArgumentMemoryLocation { Undefined, Device, Host, HostZeroCopy, Unified };
enum class ArgumentManagementType { Framework, User };
enum class ValidationMethod { AbsoluteDifference, SideBySideComparison, SideBySideRelativeComparison };
enum class ValidationMode { None = 0, Running = (1 << 0), OfflineTuning = (1 << 1), OnlineTuning = (1 << 2),
    All = Running | OfflineTuning | OnlineTuning };
enum class KernelRunMode { Running, OfflineTuning, OnlineTuning, ResultValidation };
enum class ResultStatus { Ok, ComputationFailed, ValidationFailed, CompilationFailed, DeviceLimitsExceeded };
enum class TimeUnit { Nanoseconds, Microseconds, Milliseconds, Seconds };
enum class OutputFormat { JSON, XML };
enum class LoggingLevel { Off, Error, Warning, Info, Debug };
enum class DeviceType { CPU, GPU, Custom };
enum class ExceptionReason { General, CompilerError, DeviceLimitsExceeded };

inline ValidationMode operator|(ValidationMode a, ValidationMode b)
{
    return static_cast<ValidationMode>(static_cast<int>(a) | static_cast<int>(b));
}

inline bool HasFlag(ValidationMode mode, ValidationMode flag)
{
    return (static_cast<int>(mode) & static_cast<int>(flag)) != 0;
}

} // namespace ktt
