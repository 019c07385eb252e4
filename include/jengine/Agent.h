// Agent.h -- working units of the pipeline.
//
// Names and behaviour of the reference's Pipeline/AgentBase.h,
// ConcurrentAgentBase.h and SequentialAgentBase.h, written for this library:
//  * SetPipes(trunk): the agent takes the pipes it consumes from the trunk
//    (BranchPipeFromTrunk<T>(name)) and puts the pipes it produces back
//    (CreateNewPipe<T>(name) + MergePipeToTrunk), AgentBase.h:54-63,133-168;
//  * any exception in an agent thread closes every pipe the agent touches, so
//    the whole chain drains and stops (AgentBase.cpp:25-36);
//  * ConcurrentAgentBase: one manager thread (ManagerWorkFlow) hands tasks to
//    N worker threads through a one-deep queue and an idle-worker queue
//    (ConcurrentAgentBase.cpp:9-133);
//  * SequentialAgentBase: up to 10 step threads WorkFlow0..9
//    (SequentialAgentBase.cpp:17-90);
//  * ThreadOccupiedScope / WaitAsyncScope accumulate busy and asynchronous
//    wait time per agent (AgentBase.h:101-131).
#pragma once

#include <atomic>
#include <future>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "Pipe.h"

namespace JEngine {

class AgentBase {
public:
    explicit AgentBase(const std::string& name);
    virtual ~AgentBase() = default;
    AgentBase(const AgentBase&) = delete;
    AgentBase& operator=(const AgentBase&) = delete;

    void SetPipes(std::vector<std::shared_ptr<PipeBase>>& pipes);
    virtual void GetReady() {}
    virtual void Start() = 0;
    virtual void Join() = 0;

    std::string GetAgentName() const { return name; }
    virtual size_t GetNumThreads() const = 0;
    double GetOccupiedTime() const { return occupied; }
    double GetAsyncTime() const { return asyncWait; }
    double GetMaxOccupiedTime() const { return maxOccupied; }

    class ThreadOccupiedScope;
    class WaitAsyncScope;

protected:
    template <class T>
    std::shared_ptr<Pipe<T>> BranchPipeFromTrunk(const std::string& pipeName) {
        for (auto it = trunk.begin(); it != trunk.end(); ++it) {
            if ((*it)->GetName() == pipeName) {
                auto p = std::dynamic_pointer_cast<Pipe<T>>(*it);
                if (!p) ThrowExceptionAndLog(name + ": pipe " + pipeName + " carries another element type");
                connected.insert(*it);
                trunk.erase(it);
                return p;
            }
        }
        ThrowExceptionAndLog(name + ": Pipe trunk does not contain a pipe named " + pipeName);
    }
    template <class T>
    std::shared_ptr<Pipe<T>> CreateNewPipe(const std::string& pipeName) {
        auto p = std::make_shared<Pipe<T>>(pipeName);
        connected.insert(p);
        return p;
    }
    template <class T>
    void MergePipeToTrunk(std::shared_ptr<Pipe<T>> p) {
        if (!connected.count(p)) ThrowExceptionAndLog("Please use CreateNewPipe<PipeType>() to create a pipe");
        trunk.push_back(p);
    }
    void CloseAllConnectedPipes();

private:
    virtual void SetPipesImpl() = 0;
    friend class ThreadOccupiedScope;
    friend class WaitAsyncScope;

    const std::string name;
    std::vector<std::shared_ptr<PipeBase>> trunk;
    std::set<std::shared_ptr<PipeBase>> connected;
    std::mutex closeMutex, timeMutex;
    double occupied = 0.0, maxOccupied = 0.0, asyncWait = 0.0;
};

class AgentBase::ThreadOccupiedScope {
public:
    explicit ThreadOccupiedScope(AgentBase* owner) : owner(owner) {}
    ~ThreadOccupiedScope() { Release(); }
    ThreadOccupiedScope(const ThreadOccupiedScope&) = delete;

private:
    friend class WaitAsyncScope;
    void Release();
    AgentBase* owner;
    Timer timer;
};

class AgentBase::WaitAsyncScope {
public:
    explicit WaitAsyncScope(ThreadOccupiedScope* occupied);
    ~WaitAsyncScope();
    WaitAsyncScope(const WaitAsyncScope&) = delete;

private:
    ThreadOccupiedScope* occ;
    Timer timer;
};

class ConcurrentAgentBase : public AgentBase {
public:
    ConcurrentAgentBase(const std::string& name, size_t numThreads);
    void Start() override final;
    void Join() override final;
    size_t GetNumThreads() const override final { return numWorkers; }

protected:
    struct TaskBase {
        virtual ~TaskBase() = default;
    };
    virtual void ManagerWorkFlow() = 0;
    size_t WaitIdleWorkerIndex();
    void SubmitTask(std::unique_ptr<TaskBase>&& task);

private:
    virtual void ProcessTask(size_t threadIndex, std::unique_ptr<TaskBase> task) = 0;
    void ManagerWrapped();
    void WorkerWrapped(size_t threadIndex);

    const size_t numWorkers;
    std::future<void> manager;
    std::vector<std::future<void>> workers;
    SyncQueue<std::unique_ptr<TaskBase>> nextTask;
    SyncQueue<size_t> idleWorkers;
};

class SequentialAgentBase : public AgentBase {
public:
    SequentialAgentBase(const std::string& name, int numSteps);
    void Start() override final;
    void Join() override final;
    size_t GetNumThreads() const override final { return 1; }

protected:
    virtual void WorkFlow0() = 0;
    virtual void WorkFlow1() {}
    virtual void WorkFlow2() {}
    virtual void WorkFlow3() {}
    virtual void WorkFlow4() {}
    virtual void WorkFlow5() {}
    virtual void WorkFlow6() {}
    virtual void WorkFlow7() {}
    virtual void WorkFlow8() {}
    virtual void WorkFlow9() {}

private:
    void StepWrapped(int index);
    const int numSteps;
    std::vector<std::future<void>> workers;
};

}  // namespace JEngine
