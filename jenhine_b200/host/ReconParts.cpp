// ReconParts.cpp -- z-part plans and the allocation-failure retry
// (include/jengine/ReconParts.h).
#include "../../include/jengine/ReconParts.h"

#include <cstring>
#include <sstream>

namespace JEngine {

std::vector<ReconPartPlan> ReconPartPlans(size_t Z) {
    std::vector<ReconPartPlan> plans;
    for (size_t parts = 1; parts <= Z; ++parts) {
        const size_t slices = (Z - 1) / parts + 1;
        if (slices * (parts - 1) >= Z) continue;  // the last part would hold no slice
        plans.push_back({parts, slices});
    }
    return plans;
}

bool IsDeviceAllocationFailure(const std::string& message) {
    static const char kPrefix[] = "CUDA failed to malloc ";
    return message.compare(0, sizeof(kPrefix) - 1, kPrefix) == 0;
}

ReconPartPlan PrepareAgentsWithRetry(
    size_t Z, const std::function<std::vector<std::shared_ptr<AgentBase>>(const ReconPartPlan&)>& makeAgents,
    std::vector<std::shared_ptr<AgentBase>>& agents, std::vector<std::shared_ptr<PipeBase>>& pipes) {
    const std::vector<ReconPartPlan> plans = ReconPartPlans(Z);
    for (size_t i = 0; i < plans.size(); ++i) {
        const ReconPartPlan& plan = plans[i];
        if (plan.numReconParts > 1) {
            std::ostringstream ss;
            ss << "try to split recon into " << plan.numReconParts << " parts, " << plan.numSlicesPerRecon
               << " slices per recon part";
            GLog(ss.str());
        }
        try {
            agents = makeAgents(plan);
            pipes.clear();
            for (auto& a : agents) a->SetPipes(pipes);
            for (auto& a : agents) a->GetReady();
            return plan;
        } catch (Exception& e) {
            if (!IsDeviceAllocationFailure(e.What()) || i + 1 == plans.size()) throw;
            GLog("Fail to prepare recon due to CUDA malloc error");
            agents.clear();
            pipes.clear();
        }
    }
    ThrowExceptionAndLog("no z-part plan for an empty volume");
}

}  // namespace JEngine
