// test_pipeline.cpp -- the Pipe / Agent runtime on the CPU (no GPU).
//
// Behaviours checked are those the reference's own runtime tests exercise
// (UnitTests/UTPipeline/UTPipe.cpp, UTAgentBase.cpp, UTSequentialAgent.cpp):
// token order and shot flags, read overlap, shots never merged in one read,
// blocking on a full ring, close / drain, deadlock detection, in-order
// release, a multi-threaded agent chain, and an exception in one agent
// closing the whole chain (failure injected on the host).
#include <atomic>
#include <chrono>
#include <cstdio>
#include <future>
#include <thread>

#include "jengine/Agent.h"

using namespace JEngine;

static int failures = 0;
#define CHECK(c)                                                              \
    do {                                                                      \
        if (!(c)) {                                                           \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);          \
            ++failures;                                                       \
        }                                                                     \
    } while (0)

template <class F>
static bool finishes_within(F f, double seconds) {
    auto fut = std::async(std::launch::async, f);
    return fut.wait_for(std::chrono::duration<double>(seconds)) == std::future_status::ready;
}

static std::shared_ptr<Pipe<int>> make_pipe(size_t readers, size_t readSize, size_t overlap, size_t writers,
                                             size_t writeSize, size_t buffer = 0) {
    auto p = std::make_shared<Pipe<int>>("p");
    if (buffer) p->SetBufferSize(buffer);
    p->SetTemplate(0, {1});
    p->SetConsumer("c", readers, readSize, overlap);
    p->SetProducer("w", writers, writeSize);
    return p;
}

static void test_order_and_shot_flags() {
    auto p = make_pipe(1, 1, 0, 1, 1, 16);
    for (int i = 0; i < 5; ++i) {
        auto w = p->GetWriteToken(1, i == 4);
        w.GetBuffer(0) = 10 + i;
        CHECK(w.IsShotStart() == (i == 0));
    }
    for (int i = 0; i < 5; ++i) {
        auto r = p->GetReadToken();
        CHECK(r.GetStartIndex() == (size_t)i);
        CHECK(r.GetBuffer(0) == 10 + i);
        CHECK(r.IsShotStart() == (i == 0));
        CHECK(r.IsShotEnd() == (i == 4));
    }
}

static void test_overlap_and_shots() {
    auto p = make_pipe(1, 3, 1, 1, 1, 32);
    for (int i = 0; i < 10; ++i) p->GetWriteToken(1, i == 9).GetBuffer(0) = i;
    for (int i = 0; i < 5; ++i) p->GetWriteToken(1, i == 4).GetBuffer(0) = 100 + i;  // second shot
    const size_t starts[] = {0, 2, 4, 6, 8, 10, 12};
    const size_t sizes[] = {3, 3, 3, 3, 2, 3, 3};
    for (int k = 0; k < 7; ++k) {
        auto r = p->GetReadToken();
        CHECK(r.GetStartIndex() == starts[k]);
        CHECK(r.GetSize() == sizes[k]);
        CHECK(r.IsShotStart() == (k == 0 || k == 5));
        CHECK(r.IsShotEnd() == (k == 4 || k == 6));
        CHECK(r.GetOverlapSize() == ((k == 0 || k == 5) ? 0u : 1u));
        if (k == 5) CHECK(r.GetBuffer(0) == 100);   // reads never span two shots
    }
}

static void test_blocking_on_full_ring() {
    auto p = make_pipe(1, 1, 0, 1, 1, 2);
    p->GetWriteToken(1, false).GetBuffer(0) = 1;
    p->GetWriteToken(1, false).GetBuffer(0) = 2;
    std::atomic<bool> wrote{false};
    auto th = std::async(std::launch::async, [&] {
        p->GetWriteToken(1, true).GetBuffer(0) = 3;
        wrote = true;
    });
    std::this_thread::sleep_for(std::chrono::milliseconds(100));
    CHECK(!wrote);                    // ring full: the writer waits
    { auto r = p->GetReadToken(); CHECK(r.GetBuffer(0) == 1); }
    th.wait();
    CHECK(wrote);
    CHECK(p->GetReadToken().GetBuffer(0) == 2);
    CHECK(p->GetReadToken().GetBuffer(0) == 3);
}

static void test_close_and_drain() {
    auto p = make_pipe(1, 1, 0, 1, 1, 8);
    p->GetWriteToken(1, true).GetBuffer(0) = 7;
    p->Close();
    CHECK(p->GetReadToken().GetBuffer(0) == 7);   // drained first
    bool signalled = false;
    try { p->GetReadToken(); } catch (PipeClosedAndEmptySignal&) { signalled = true; }
    CHECK(signalled);
    bool threw = false;
    try { p->GetWriteToken(1, false); } catch (Exception&) { threw = true; }
    CHECK(threw);
}

static void test_deadlock_detected() {
    auto p = make_pipe(1, 5, 0, 1, 1, 4);   // a read needs 5 slots, the ring has 4
    bool threw = false;
    CHECK(finishes_within([&] {
        try {
            for (int i = 0; i < 8; ++i) p->GetWriteToken(1, false);
        } catch (Exception& e) {
            threw = std::string(e.what()) == "Pipe deadlock";
        }
    }, 5.0));
    CHECK(threw);
}

static void test_release_in_order() {
    auto p = make_pipe(1, 1, 0, 2, 1, 8);
    auto a = p->GetWriteToken(1, false);
    auto b = p->GetWriteToken(1, true);
    b.Reset();                                   // second token done first
    CHECK(p->GetWriteDonePos() == 0);
    a.Reset();
    CHECK(p->GetWriteDonePos() == 2);
}

// ---- agents ------------------------------------------------------------------

class SourceAgent : public SequentialAgentBase {
public:
    explicit SourceAgent(int n) : SequentialAgentBase("SourceAgent", 1), n(n) {}

private:
    void SetPipesImpl() override {
        out = CreateNewPipe<int>("Num");
        out->SetTemplate(0, {1});
        out->SetProducer(GetAgentName(), 1, 1);
        MergePipeToTrunk(out);
    }
    void WorkFlow0() override {
        for (int i = 1; i <= n; ++i) out->GetWriteToken(1, i == n).GetBuffer(0) = i;
        out->Close();
    }
    int n;
    std::shared_ptr<Pipe<int>> out;
};

class SquareAgent : public ConcurrentAgentBase {
public:
    SquareAgent(size_t threads, int failAt) : ConcurrentAgentBase("SquareAgent", threads), failAt(failAt) {}

private:
    struct Task : TaskBase {
        Pipe<int>::ReadToken r;
        Pipe<int>::WriteToken w;
    };
    void SetPipesImpl() override {
        in = BranchPipeFromTrunk<int>("Num");
        in->SetConsumer(GetAgentName(), GetNumThreads(), 1, 0);
        out = CreateNewPipe<int>("Num");
        out->SetTemplate(0, {1});
        out->SetProducer(GetAgentName(), GetNumThreads(), 1);
        MergePipeToTrunk(out);
    }
    void ManagerWorkFlow() override {
        try {
            while (true) {
                WaitIdleWorkerIndex();
                Task t;
                t.r = in->GetReadToken();
                t.w = out->GetWriteToken(1, t.r.IsShotEnd());
                SubmitTask(std::make_unique<Task>(t));
            }
        } catch (PipeClosedAndEmptySignal&) {
            out->Close();
        }
    }
    void ProcessTask(size_t, std::unique_ptr<TaskBase> base) override {
        Task* t = static_cast<Task*>(base.get());
        const int v = t->r.GetBuffer(0);
        if (v == failAt) ThrowException("injected failure");
        std::this_thread::sleep_for(std::chrono::microseconds(200 * (v % 3)));  // finish out of order
        t->w.GetBuffer(0) = v * v;
    }
    int failAt;
    std::shared_ptr<Pipe<int>> in, out;
};

class SinkAgent : public SequentialAgentBase {
public:
    SinkAgent() : SequentialAgentBase("SinkAgent", 1) {}
    std::vector<int> got;
    bool sawClose = false;

private:
    void SetPipesImpl() override {
        in = BranchPipeFromTrunk<int>("Num");
        in->SetConsumer(GetAgentName(), 1, 1, 0);
    }
    void WorkFlow0() override {
        try {
            while (true) got.push_back(in->GetReadToken().GetBuffer(0));
        } catch (PipeClosedAndEmptySignal&) {
            sawClose = true;
        }
    }
    std::shared_ptr<Pipe<int>> in;
};

static void run_chain(int n, int failAt, SinkAgent& sink) {
    SetGLogSink([](const std::string&) {});
    std::vector<std::shared_ptr<AgentBase>> agents{std::make_shared<SourceAgent>(n),
                                                   std::make_shared<SquareAgent>(4, failAt)};
    std::vector<std::shared_ptr<PipeBase>> trunk;
    for (auto& a : agents) a->SetPipes(trunk);
    sink.SetPipes(trunk);
    for (auto& a : agents) a->Start();
    sink.Start();
    for (auto& a : agents) a->Join();
    sink.Join();
}

static void test_agent_chain() {
    SinkAgent sink;
    CHECK(finishes_within([&] { run_chain(200, -1, sink); }, 30.0));
    CHECK(sink.got.size() == 200);
    bool ordered = true;
    for (size_t i = 0; i < sink.got.size(); ++i) ordered &= sink.got[i] == (int)((i + 1) * (i + 1));
    CHECK(ordered);   // pipes keep stream order although workers finish out of order
}

static void test_failure_closes_chain() {
    SinkAgent sink;
    CHECK(finishes_within([&] { run_chain(200, 57, sink); }, 30.0));
    CHECK(sink.sawClose);
    CHECK(sink.got.size() < 200);
}

int main() {
    test_order_and_shot_flags();
    test_overlap_and_shots();
    test_blocking_on_full_ring();
    test_close_and_drain();
    test_deadlock_detected();
    test_release_in_order();
    test_agent_chain();
    test_failure_closes_chain();
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
