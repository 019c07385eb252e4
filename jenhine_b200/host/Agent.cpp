// Agent.cpp -- AgentBase, ConcurrentAgentBase, SequentialAgentBase and the
// shared utilities of Common.h.
#include "jengine/Agent.h"

#include <iostream>
#include <sstream>

namespace JEngine {

// ---- logging and exceptions ------------------------------------------------

namespace {
std::mutex g_log_mutex;
std::function<void(const std::string&)>& log_sink() {
    static std::function<void(const std::string&)> sink = [](const std::string& m) { std::cerr << m << "\n"; };
    return sink;
}
}  // namespace

void GLogWrite(const std::string& msg) {
    std::lock_guard<std::mutex> lk(g_log_mutex);
    if (log_sink()) log_sink()(msg);
}

void SetGLogSink(std::function<void(const std::string&)> sink) {
    std::lock_guard<std::mutex> lk(g_log_mutex);
    log_sink() = std::move(sink);
}

Exception::Exception(const std::string& file, size_t line, const std::string& msg, bool log) : message(msg) {
    if (log) GLogWrite("An exception is thrown in line " + std::to_string(line) + ", \"" + file + "\": " + msg);
}

// ---- AgentBase -----------------------------------------------------------

AgentBase::AgentBase(const std::string& name) : name(name) {}

void AgentBase::SetPipes(std::vector<std::shared_ptr<PipeBase>>& pipes) {
    trunk = pipes;
    SetPipesImpl();
    pipes = trunk;
}

void AgentBase::CloseAllConnectedPipes() {
    std::lock_guard<std::mutex> lk(closeMutex);
    for (auto& p : connected)
        if (!p->Closed()) {
            GLog(name + ": " + p->GetName() + " is forced closed");
            p->Close();
        }
}

void AgentBase::ThreadOccupiedScope::Release() {
    const double span = timer.Toc();
    std::lock_guard<std::mutex> lk(owner->timeMutex);
    owner->occupied += span;
    if (span > owner->maxOccupied) owner->maxOccupied = span;
}

AgentBase::WaitAsyncScope::WaitAsyncScope(ThreadOccupiedScope* occupied) : occ(occupied) {
    occ->Release();  // the asynchronous part does not occupy the thread
}

AgentBase::WaitAsyncScope::~WaitAsyncScope() {
    {
        std::lock_guard<std::mutex> lk(occ->owner->timeMutex);
        occ->owner->asyncWait += timer.Toc();
    }
    occ->timer.Tic();
}

// ---- ConcurrentAgentBase ---------------------------------------------------

ConcurrentAgentBase::ConcurrentAgentBase(const std::string& name, size_t numThreads)
    : AgentBase(name), numWorkers(numThreads), nextTask(1), idleWorkers(0) {
    if (numThreads == 0) ThrowExceptionAndLog(name + ": needs at least one worker thread");
}

void ConcurrentAgentBase::Start() {
    manager = std::async(std::launch::async, &ConcurrentAgentBase::ManagerWrapped, this);
    for (size_t i = 0; i < numWorkers; ++i)
        workers.emplace_back(std::async(std::launch::async, &ConcurrentAgentBase::WorkerWrapped, this, i));
}

void ConcurrentAgentBase::Join() {
    manager.get();
    nextTask.Close();
    for (auto& w : workers) w.get();
    CloseAllConnectedPipes();
}

size_t ConcurrentAgentBase::WaitIdleWorkerIndex() { return idleWorkers.Pop(); }

void ConcurrentAgentBase::SubmitTask(std::unique_ptr<TaskBase>&& task) { nextTask.Push(std::move(task)); }

void ConcurrentAgentBase::ManagerWrapped() {
    try {
        ManagerWorkFlow();
    } catch (SyncQueueClosedAndEmptySignal&) {
        GLog(GetAgentName() + " workers are quit.");
    } catch (std::exception& e) {
        idleWorkers.Close();
        GLog(GetAgentName() + " manager die, " + e.what());
    } catch (...) {
        idleWorkers.Close();
        GLog(GetAgentName() + " manager die, unknown exception.");
    }
    CloseAllConnectedPipes();
}

void ConcurrentAgentBase::WorkerWrapped(size_t threadIndex) {
    try {
        while (true) {
            idleWorkers.Push(threadIndex);            // "I am ready"
            std::unique_ptr<TaskBase> task = nextTask.Pop();
            ProcessTask(threadIndex, std::move(task));
        }
    } catch (SyncQueueClosedAndEmptySignal&) {
        // normal end
    } catch (std::exception& e) {
        idleWorkers.Close();
        GLog(GetAgentName() + " #" + std::to_string(threadIndex) + " die, " + e.what());
        CloseAllConnectedPipes();
    } catch (...) {
        idleWorkers.Close();
        GLog(GetAgentName() + " #" + std::to_string(threadIndex) + " die, unknown exception.");
        CloseAllConnectedPipes();
    }
}

// ---- SequentialAgentBase ---------------------------------------------------

SequentialAgentBase::SequentialAgentBase(const std::string& name, int numSteps)
    : AgentBase(name), numSteps(numSteps) {
    if (numSteps < 1 || numSteps > 10) ThrowException("SequentialAgentBase can only contain 1 to 10 steps");
}

void SequentialAgentBase::Start() {
    for (int i = 0; i < numSteps; ++i)
        workers.emplace_back(std::async(std::launch::async, &SequentialAgentBase::StepWrapped, this, i));
}

void SequentialAgentBase::Join() {
    for (auto& w : workers) w.get();
    CloseAllConnectedPipes();
}

void SequentialAgentBase::StepWrapped(int index) {
    try {
        switch (index) {
            case 0: WorkFlow0(); break;
            case 1: WorkFlow1(); break;
            case 2: WorkFlow2(); break;
            case 3: WorkFlow3(); break;
            case 4: WorkFlow4(); break;
            case 5: WorkFlow5(); break;
            case 6: WorkFlow6(); break;
            case 7: WorkFlow7(); break;
            case 8: WorkFlow8(); break;
            default: WorkFlow9(); break;
        }
    } catch (PipeClosedAndEmptySignal&) {
        // upstream finished
    } catch (std::exception& e) {
        GLog(GetAgentName() + " step #" + std::to_string(index) + " die, " + e.what());
        CloseAllConnectedPipes();
    } catch (...) {
        GLog(GetAgentName() + " step #" + std::to_string(index) + " die, unknown exception.");
        CloseAllConnectedPipes();
    }
}

}  // namespace JEngine
