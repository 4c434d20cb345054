// ComputeInterface.h -- the interface a custom kernel launcher drives.
//
// Interface of KTT 2.1.0 Source/Api/ComputeInterface.h (the subset a launcher for the Coulomb
// path uses: run a kernel definition with the current or given sizes, replace scalar arguments,
// update / download / copy / clear buffers, synchronise, query the current configuration and
// sizes).  Every RunKernel call adds its event-timed duration to the configuration's result, as
// KTT sums the durations of all launches made by a launcher (Source/Api/Output/KernelResult.cpp:108-118).
#pragma once

#include <vector>

#include <ktt/Configuration.h>

namespace ktt
{

class KTT_API ComputeInterface
{
public:
    virtual ~ComputeInterface() = default;

    virtual void RunKernel(const KernelDefinitionId id) = 0;
    virtual void RunKernel(const KernelDefinitionId id, const DimensionVector& globalSize, const DimensionVector& localSize) = 0;
    virtual ComputeActionId RunKernelAsync(const KernelDefinitionId id, const QueueId queue) = 0;
    virtual ComputeActionId RunKernelAsync(const KernelDefinitionId id, const QueueId queue, const DimensionVector& globalSize,
        const DimensionVector& localSize) = 0;
    virtual void WaitForComputeAction(const ComputeActionId id) = 0;
    // Profiled launches (Source/Api/ComputeInterface.h:82-119).  Here the counter passes replay the
    // launcher's whole execution before its timed run (Tuner::SetProfiling), so these run the
    // definition like RunKernel and no profiling runs ever remain.
    virtual void RunKernelWithProfiling(const KernelDefinitionId id) = 0;
    virtual void RunKernelWithProfiling(const KernelDefinitionId id, const DimensionVector& globalSize,
        const DimensionVector& localSize) = 0;
    virtual uint64_t GetRemainingProfilingRuns(const KernelDefinitionId id) const = 0;
    virtual uint64_t GetRemainingProfilingRuns() const = 0;

    virtual QueueId GetDefaultQueue() const = 0;
    virtual std::vector<QueueId> GetAllQueues() const = 0;
    virtual void SynchronizeQueue(const QueueId queue) = 0;
    virtual void SynchronizeQueues() = 0;
    virtual void SynchronizeDevice() = 0;

    virtual const DimensionVector& GetCurrentGlobalSize(const KernelDefinitionId id) const = 0;
    virtual const DimensionVector& GetCurrentLocalSize(const KernelDefinitionId id) const = 0;
    virtual const KernelConfiguration& GetCurrentConfiguration() const = 0;
    virtual KernelRunMode GetRunMode() const = 0;

    virtual void ChangeArguments(const KernelDefinitionId id, const std::vector<ArgumentId>& arguments) = 0;
    virtual void SwapArguments(const KernelDefinitionId id, const ArgumentId& first, const ArgumentId& second) = 0;
    virtual void UpdateScalarArgument(const ArgumentId& id, const void* data) = 0;

    virtual void UploadBuffer(const ArgumentId& id) = 0;
    virtual void DownloadBuffer(const ArgumentId& id, void* destination, const size_t dataSize = 0) = 0;
    virtual void UpdateBuffer(const ArgumentId& id, const void* data, const size_t dataSize = 0) = 0;
    virtual void CopyBuffer(const ArgumentId& destination, const ArgumentId& source, const size_t dataSize = 0) = 0;
    virtual void ClearBuffer(const ArgumentId& id) = 0;
    virtual bool HasBuffer(const ArgumentId& id) = 0;

    // Transfers on a queue (Source/Api/ComputeInterface.h:216-310).  They complete before the call
    // returns; the action ids exist for WaitForTransferAction, as in KTT.
    virtual TransferActionId UploadBufferAsync(const ArgumentId& id, const QueueId queue) = 0;
    virtual TransferActionId DownloadBufferAsync(const ArgumentId& id, const QueueId queue, void* destination,
        const size_t dataSize = 0) = 0;
    virtual TransferActionId UpdateBufferAsync(const ArgumentId& id, const QueueId queue, const void* data,
        const size_t dataSize = 0) = 0;
    virtual TransferActionId CopyBufferAsync(const ArgumentId& destination, const ArgumentId& source, const QueueId queue,
        const size_t dataSize = 0) = 0;
    virtual void WaitForTransferAction(const TransferActionId id) = 0;
    // New size of a vector argument's device buffer owned by the tuner (user buffers cannot be resized),
    // keeping the first min(old, new) bytes when preserveData; the other bytes are zero.
    virtual void ResizeBuffer(const ArgumentId& id, const size_t newDataSize, const bool preserveData) = 0;
    // New size of a local-memory argument.
    virtual void UpdateLocalArgument(const ArgumentId& id, const size_t dataSize) = 0;
    // Unified-memory arguments are not offered by this build: the call reports an error.
    virtual void GetUnifiedMemoryBufferHandle(const ArgumentId& id, UnifiedBufferMemory& memoryHandle) = 0;
    virtual bool GetProfiling(const KernelId id) = 0;
};

} // namespace ktt
