// ComputeApiInitializer.h -- a tuner on the caller's own CUDA context and streams
// (KTT: Source/Api/ComputeApiInitializer.h:16-45).
#pragma once

#include <vector>

#include <ktt/KttTypes.h>

namespace ktt
{

class KTT_API ComputeApiInitializer
{
public:
    // context: a CUcontext; queues: CUstreams of that context (at least one).  The tuner uses them
    // and never destroys them; they must outlive the tuner.
    explicit ComputeApiInitializer(ComputeContext context, const std::vector<ComputeQueue>& queues);

    ComputeContext GetContext() const;
    const std::vector<ComputeQueue>& GetQueues() const;

private:
    ComputeContext m_Context;
    std::vector<ComputeQueue> m_Queues;
};

} // namespace ktt
