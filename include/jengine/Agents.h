// Agents.h -- the FDK hot-path agents, backed by libjfdk.so (include/jfdk.h).
//
// Constructor signatures and pipe wiring follow the reference agents so they
// drop into the same agent list (JEngine/JEngine.cpp:186-314):
//   PreProcessingAgent  PreProcessingAgent/PreProcessingAgent.h:17-30   "Proj" UINT16Vec -> FloatVec
//   CompositeAgent      CompositeAgent/CompositeAgent.h:15-55           "Proj" FloatVec pairs -> FloatVec (2W)
//   FilterAgent         FilterAgent/FilterAgent.h:19-33                 "Proj" FloatVec  -> FloatVec
//   ZFilterAgent        FilterAgent/ZFilterAgent.h                      "Proj" FloatVec  -> FloatVec
//   DeviceUploadAgent   (Tex2DUploadAgent, CUDA/Tex2DUploadAgent.h)     "Proj" FloatVec  -> DeviceMemory<float>
//   BPCUDAAgent         BPCUDAAgent/BPCUDAAgent.h:22-33                 "Proj" DeviceMemory<float> -> "Slice" DeviceMemory<float>
//   DeviceMemoryDownloadAgent  CUDA/DeviceMemoryDownloadAgent.h        "Slice" DeviceMemory<float> -> FloatVec
//   CTNumAgent          CTNumAgent/CTNumAgent.h:17-24                   "Slice" FloatVec -> FloatVec
// Each worker thread owns a CUDA stream and a jfdk context.  Differences from
// the reference, by design: FilterAgent processes a whole view per task (the
// GPU parallelises over rows, nRowsPerThread is accepted and unused);
// BPCUDAAgent reads `viewsPerChunk` frames per token and accumulates them in
// one launch, keeps the whole volume on the device (numReconParts > 1 is
// accepted; slices come out in order) and backprojects the weight alongside
// the data, so it needs no weight-cache file (tempFileFolder is unused).
#pragma once

#include <filesystem>
#include <memory>
#include <vector>

#include "Agent.h"
#include "DeviceMemory.h"
#include "Geometry.h"

struct jfdk_ctx;

namespace JEngine {

class StageContext;  // a jfdk context + its stream (Agents.cpp)
class PinnedSlots;   // page-locked slots of a host pipe (Agents.cpp)

class PreProcessingAgent : public ConcurrentAgentBase {
public:
    PreProcessingAgent(size_t numThreads, size_t packSize, size_t inputSizeX, size_t inputSizeY, size_t borderSizeUp,
                       size_t borderSizeBottom, size_t borderSizeLeft, size_t borderSizeRight, size_t outputSizeX,
                       size_t outputSizeY, float brightField, const FloatVec& BeamHardeningParams);
    ~PreProcessingAgent() override;

private:
    struct Task : TaskBase {
        Pipe<UINT16Vec>::ReadToken ReadToken;
        Pipe<FloatVec>::WriteToken WriteToken;
    };
    void SetPipesImpl() override;
    void ManagerWorkFlow() override;
    void ProcessTask(size_t threadIndex, std::unique_ptr<TaskBase> task) override;

    const size_t packSize, inputSizeX, inputSizeY, outputSizeX, outputSizeY;
    std::vector<std::unique_ptr<StageContext>> stages;
    std::shared_ptr<Pipe<UINT16Vec>> pipeIn;
    std::shared_ptr<Pipe<FloatVec>> pipeOut;
};

// Reads (direct, conjugate) frame pairs -- the order InputAgent writes them,
// JEngine/InputAgent.cpp:45-90 -- and writes one 2W-wide composite frame per
// pair (jfdk_composite_frames).
class CompositeAgent : public ConcurrentAgentBase {
public:
    CompositeAgent(size_t numThreads, size_t inputWidth, size_t inputHeight, bool detectorAtTheRight,
                   float sourceOriginDistance, const std::vector<ProjectionMatrix>& projectionMatrices);
    ~CompositeAgent() override;

private:
    struct Task : TaskBase {
        Pipe<FloatVec>::ReadToken ReadToken;
        Pipe<FloatVec>::WriteToken WriteToken;
    };
    void SetPipesImpl() override;
    void ManagerWorkFlow() override;
    void ProcessTask(size_t threadIndex, std::unique_ptr<TaskBase> task) override;

    const size_t width, height, numViewsPerRot;
    std::vector<std::unique_ptr<StageContext>> stages;
    std::shared_ptr<Pipe<FloatVec>> pipeIn, pipeOut;
};

class FilterAgent : public ConcurrentAgentBase {
public:
    FilterAgent(size_t nThreads, size_t nRowsPerThread, size_t nInputWidth, size_t nInputHeight, size_t nOutputWidth,
                bool detectorAtTheRight, float HalfSampleRate, float FilterCutOffStart, float FilterCutOffEnd,
                const FloatVec& AdjustPoints, const FloatVec& AdjustLevelInDB,
                const std::vector<ProjectionMatrix>& ptms, float DSO);
    ~FilterAgent() override;

private:
    struct Task : TaskBase {
        Pipe<FloatVec>::ReadToken ReadToken;
        Pipe<FloatVec>::WriteToken WriteToken;
    };
    void SetPipesImpl() override;
    void ManagerWorkFlow() override;
    void ProcessTask(size_t threadIndex, std::unique_ptr<TaskBase> task) override;

    const size_t inputWidth, height, outputWidth, numViewsPerRot;
    std::vector<std::unique_ptr<StageContext>> stages;
    std::shared_ptr<Pipe<FloatVec>> pipeIn, pipeOut;
};

class ZFilterAgent : public ConcurrentAgentBase {
public:
    ZFilterAgent(size_t nThreads, size_t nWidth, size_t nHeight);
    ~ZFilterAgent() override;

private:
    struct Task : TaskBase {
        Pipe<FloatVec>::ReadToken ReadToken;
        Pipe<FloatVec>::WriteToken WriteToken;
    };
    void SetPipesImpl() override;
    void ManagerWorkFlow() override;
    void ProcessTask(size_t threadIndex, std::unique_ptr<TaskBase> task) override;

    const size_t width, height;
    std::vector<std::unique_ptr<StageContext>> stages;
    std::shared_ptr<Pipe<FloatVec>> pipeIn, pipeOut;
};

// Host frames -> device frames.  The slots of the host pipe are page-locked
// in GetReady, so each frame goes to the device as one asynchronous DMA on the
// agent's own stream, straight from the pipe slot (no driver staging copy).
class DeviceUploadAgent : public SequentialAgentBase {
public:
    DeviceUploadAgent(const std::string& pipeName, size_t width, size_t height);
    ~DeviceUploadAgent() override;
    void GetReady() override;
    size_t NumPinnedSlots() const;

private:
    void SetPipesImpl() override;
    void WorkFlow0() override;
    const std::string pipeName;
    const size_t width, height;
    std::unique_ptr<PinnedSlots> pinned;
    void* stream = nullptr;  // cudaStream_t
    std::shared_ptr<Pipe<FloatVec>> pipeIn;
    std::shared_ptr<Pipe<DeviceMemory<float>>> pipeOut;
};

// The volume is reconstructed in numReconParts parts of numSlicesPerRecon
// slices (the last part may be shorter): shot i of the input pipe is
// backprojected into part i mod numReconParts only, and that part's slices
// are written out at its end, the last slice of the volume marking the shot
// end (BPCUDAAgent/BPCUDAAgent.cpp:84-111, 231-287); the input agent repeats
// the views once per part.  The accumulators hold one part; GetReady
// allocates them, so a volume that does not fit fails there with "CUDA failed
// to malloc ", which the application's retry loop answers with more parts
// (PrepareAgentsWithRetry).  deviceMemoryBudget (an addition: 0 = no bound)
// bounds the device memory the backprojection may take on top of its
// context's fixed tables: the accumulators of one part and the packed store
// of one chunk of views.  The reference's cache file
// of precomputed weights has no counterpart: the weights are accumulated in
// the same pass as the values.
class BPCUDAAgent : public SequentialAgentBase {
public:
    BPCUDAAgent(const std::vector<ProjectionMatrix>& projectionMatrices, size_t numDetectorsU, size_t numDetectorsV,
                size_t volumeSizeX, size_t volumeSizeY, size_t volumeSizeZ, float pitchXY, float pitchZ,
                size_t numSlicesPerRecon, size_t numReconParts, const std::filesystem::path& tempFileFolder,
                size_t viewsPerChunk = 16, size_t deviceMemoryBudget = 0);
    ~BPCUDAAgent() override;
    void GetReady() override;

private:
    void SetPipesImpl() override;
    void WorkFlow0() override;

    const std::vector<ProjectionMatrix> projectionMatrices;
    const size_t numDetectorsU, numDetectorsV, volumeSizeX, volumeSizeY, volumeSizeZ;
    const float pitchXY, pitchZ;
    const size_t numSlicesPerRecon, numReconParts;
    const size_t viewsPerChunk, deviceMemoryBudget;
    size_t shot = 0;
    std::unique_ptr<StageContext> stage;
    std::unique_ptr<DeviceMemory<float>> staging;
    std::shared_ptr<Pipe<DeviceMemory<float>>> pipeIn, pipeOut;
};

// Device slices -> host slices, into page-locked slots of its output pipe
// (the mirror of DeviceUploadAgent).
class DeviceMemoryDownloadAgent : public SequentialAgentBase {
public:
    DeviceMemoryDownloadAgent(const std::string& pipeName, size_t width, size_t height);
    ~DeviceMemoryDownloadAgent() override;
    void GetReady() override;
    size_t NumPinnedSlots() const;

private:
    void SetPipesImpl() override;
    void WorkFlow0() override;
    const std::string pipeName;
    const size_t width, height;
    std::unique_ptr<PinnedSlots> pinned;
    void* stream = nullptr;  // cudaStream_t
    std::shared_ptr<Pipe<DeviceMemory<float>>> pipeIn;
    std::shared_ptr<Pipe<FloatVec>> pipeOut;
};

class CTNumAgent : public ConcurrentAgentBase {
public:
    CTNumAgent(size_t numThreads, size_t width, size_t height, float norm0, float norm1, float muWater);
    ~CTNumAgent() override;

private:
    struct Task : TaskBase {
        Pipe<FloatVec>::ReadToken ReadToken;
        Pipe<FloatVec>::WriteToken WriteToken;
    };
    void SetPipesImpl() override;
    void ManagerWorkFlow() override;
    void ProcessTask(size_t threadIndex, std::unique_ptr<TaskBase> task) override;

    const size_t width, height;
    std::vector<std::unique_ptr<StageContext>> stages;
    std::shared_ptr<Pipe<FloatVec>> pipeIn, pipeOut;
};

}  // namespace JEngine
