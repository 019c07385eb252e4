// ReconParts.h -- the application's split of a volume into z-parts and its
// answer to a device allocation failure (JEngine/JEngine.cpp:167-175,
// 402-421): try 1, 2, 3, ... parts; build the agent chain for each and get it
// ready; when that fails with "CUDA failed to malloc ", drop the chain and try
// the next count.  Pure host code.
#pragma once

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "Agent.h"

namespace JEngine {

struct ReconPartPlan {
    size_t numReconParts;
    size_t numSlicesPerRecon;
};

// The plans in the order the application tries them: P = 1, 2, ..., Z parts
// of ceil(Z / P) slices, skipping a P whose last part would be empty.
std::vector<ReconPartPlan> ReconPartPlans(size_t numPixelsZ);

// The failure the retry answers: a message that starts "CUDA failed to malloc ".
bool IsDeviceAllocationFailure(const std::string& message);

// For each plan in turn: makeAgents(plan), then SetPipes and GetReady of every
// agent.  A device allocation failure drops the agents and their pipes and
// moves on; any other exception propagates, and so does the allocation
// failure of the last plan.  Returns the plan that got ready; `agents` and
// `pipes` then hold its chain.
ReconPartPlan PrepareAgentsWithRetry(
    size_t numPixelsZ, const std::function<std::vector<std::shared_ptr<AgentBase>>(const ReconPartPlan&)>& makeAgents,
    std::vector<std::shared_ptr<AgentBase>>& agents, std::vector<std::shared_ptr<PipeBase>>& pipes);

}  // namespace JEngine
