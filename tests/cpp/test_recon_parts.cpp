// test_recon_parts.cpp -- the z-part plans and the allocation-failure retry
// (include/jengine/ReconParts.h) on CPU, with agents whose GetReady fails the
// way a device allocation does.
#include <cstdio>

#include "jengine/ReconParts.h"

using namespace JEngine;

static int failures = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            ++failures;                                            \
        }                                                          \
    } while (0)

class FakeAgent : public SequentialAgentBase {
public:
    FakeAgent(const ReconPartPlan& plan, size_t minParts, const char* error)
        : SequentialAgentBase("BPCUDAAgent", 1), plan(plan), minParts(minParts), error(error) {}
    void GetReady() override {
        if (plan.numReconParts < minParts) ThrowException(error);
    }
    ReconPartPlan plan;

private:
    void SetPipesImpl() override {}
    void WorkFlow0() override {}
    size_t minParts;
    const char* error;
};

static bool same(const std::vector<ReconPartPlan>& a, const std::vector<ReconPartPlan>& b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (a[i].numReconParts != b[i].numReconParts || a[i].numSlicesPerRecon != b[i].numSlicesPerRecon) return false;
    return true;
}

int main() {
    SetGLogSink([](const std::string&) {});
    CHECK(same(ReconPartPlans(10), {{1, 10}, {2, 5}, {3, 4}, {4, 3}, {5, 2}, {10, 1}}));
    CHECK(same(ReconPartPlans(7), {{1, 7}, {2, 4}, {3, 3}, {4, 2}, {7, 1}}));
    CHECK(same(ReconPartPlans(1), {{1, 1}}));
    CHECK(ReconPartPlans(0).empty());
    CHECK(IsDeviceAllocationFailure("CUDA failed to malloc 64 bytes for the sum volume"));
    CHECK(!IsDeviceAllocationFailure("jfdk: CUDA failed to malloc"));

    const char* oom = "CUDA failed to malloc 1048576 bytes for the backprojection sum volume";
    std::vector<std::shared_ptr<AgentBase>> agents;
    std::vector<std::shared_ptr<PipeBase>> pipes;
    // fits from 3 parts on
    {
        std::vector<size_t> tried;
        auto plan = PrepareAgentsWithRetry(
            10,
            [&](const ReconPartPlan& p) {
                tried.push_back(p.numReconParts);
                return std::vector<std::shared_ptr<AgentBase>>{std::make_shared<FakeAgent>(p, 3, oom)};
            },
            agents, pipes);
        CHECK(plan.numReconParts == 3 && plan.numSlicesPerRecon == 4);
        CHECK((tried == std::vector<size_t>{1, 2, 3}));
        CHECK(agents.size() == 1 && std::static_pointer_cast<FakeAgent>(agents[0])->plan.numReconParts == 3);
    }
    // any other failure is not retried
    {
        size_t calls = 0;
        bool threw = false;
        try {
            PrepareAgentsWithRetry(
                10,
                [&](const ReconPartPlan& p) {
                    ++calls;
                    return std::vector<std::shared_ptr<AgentBase>>{std::make_shared<FakeAgent>(p, 3, "bad PTM")};
                },
                agents, pipes);
        } catch (Exception& e) {
            threw = e.What() == "bad PTM";
        }
        CHECK(threw && calls == 1);
    }
    // nothing fits: the last allocation failure propagates
    {
        size_t calls = 0;
        bool threw = false;
        try {
            PrepareAgentsWithRetry(
                7,
                [&](const ReconPartPlan& p) {
                    ++calls;
                    return std::vector<std::shared_ptr<AgentBase>>{std::make_shared<FakeAgent>(p, 100, oom)};
                },
                agents, pipes);
        } catch (Exception& e) {
            threw = IsDeviceAllocationFailure(e.What());
        }
        CHECK(threw && calls == 5);
    }
    std::printf("OK (%d failures)\n", failures);
    return failures ? 1 : 0;
}
