// Agents.cpp -- the hot-path agents over the C ABI (include/jfdk.h).
#include "jengine/Agents.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/jfdk.h"

namespace JEngine {

// ---- device memory ------------------------------------------------------------

void* DeviceAlloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        ThrowExceptionAndLog("CUDA failed to malloc " + std::to_string(bytes) + " bytes");
    }
    return p;
}
void DeviceFree(void* p) noexcept {
    if (p) cudaFree(p);
}
static void copy(void* d, const void* s, size_t n, cudaMemcpyKind k) {
    if (n && cudaMemcpy(d, s, n, k) != cudaSuccess) ThrowExceptionAndLog("CUDA copy failed");
}
void DeviceCopy(void* d, const void* s, size_t n) { copy(d, s, n, cudaMemcpyDeviceToDevice); }
void CopyToDevice(void* d, const void* s, size_t n) { copy(d, s, n, cudaMemcpyHostToDevice); }
void CopyToHost(void* d, const void* s, size_t n) { copy(d, s, n, cudaMemcpyDeviceToHost); }

// ---- a jfdk context with its own stream and staging buffers ------------------

class StageContext {
public:
    StageContext(const jfdk_scan_params& s, const jfdk_recon_params& r, const std::vector<float>& ptms) {
        if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
            ThrowExceptionAndLog("CUDA failed to create a stream");
        const jfdk_status st = jfdk_create(&ctx, &s, &r, ptms.data(), JFDK_PRECISION_FP32, stream);
        if (st != JFDK_OK) {
            const std::string msg = ctx ? jfdk_last_error(ctx) : "jfdk_create failed";
            jfdk_destroy(ctx);
            ctx = nullptr;
            cudaStreamDestroy(stream);
            ThrowExceptionAndLog(msg);
        }
    }
    ~StageContext() {
        jfdk_destroy(ctx);
        for (void* b : buf) DeviceFree(b);
        cudaStreamDestroy(stream);
    }
    // An out-of-memory failure keeps its "CUDA failed to malloc " message
    // unprefixed: the application's retry loop matches it
    // (JEngine/JEngine.cpp:413-421).
    void Check(jfdk_status st) const {
        if (st == JFDK_ERR_OOM) ThrowExceptionAndLog(jfdk_last_error(ctx));
        if (st != JFDK_OK) ThrowExceptionAndLog(std::string("jfdk: ") + jfdk_last_error(ctx));
    }
    void Sync() const { Check(jfdk_sync(ctx)); }
    // Staging buffer `i` of at least `bytes` (grown on demand).
    void* Buffer(int i, size_t bytes) {
        if (cap[i] < bytes) {
            DeviceFree(buf[i]);
            buf[i] = DeviceAlloc(bytes);
            cap[i] = bytes;
        }
        return buf[i];
    }
    void Upload(void* d, const void* h, size_t n) const {
        if (cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, stream) != cudaSuccess)
            ThrowExceptionAndLog("CUDA upload failed");
    }
    void Download(void* h, const void* d, size_t n) const {
        if (cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
            ThrowExceptionAndLog("CUDA download failed");
    }
    jfdk_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;

private:
    void* buf[2] = {nullptr, nullptr};
    size_t cap[2] = {0, 0};
};

namespace {

std::vector<float> flatten(const std::vector<ProjectionMatrix>& p) {
    std::vector<float> f;
    for (const auto& m : p) f.insert(f.end(), m.Data(), m.Data() + 12);
    return f;
}

// Stages that use neither the orbit nor the volume (preprocessing, Z-filter,
// CT numbers) still get a complete, valid context: a one-view placeholder
// projection matrix with an invertible transform and a 1-voxel volume.
std::vector<float> placeholder_ptm(size_t w, size_t h) {
    return {1.0f, 0.0f, 0.01f, 0.5f * w, 0.0f, 0.01f, 1.0f, 0.5f * h, 0.001f, 0.0f, 0.0f, 1.0f};
}

jfdk_scan_params scan_defaults(size_t views, size_t u, size_t v) {
    jfdk_scan_params s{};
    s.num_views = (int)views;
    s.dso = 500.0f;
    s.dsd = 800.0f;
    s.num_dets_u = (int)u;
    s.num_dets_v = (int)v;
    s.detector_pixel_size = 1.0f;
    s.bright_field = 1.0f;
    s.beam_hardening[0] = 1.0f;
    s.half_sample_rate = 1.0f;
    return s;
}

jfdk_recon_params recon_defaults(size_t x, size_t y, size_t z) {
    jfdk_recon_params r{};
    r.num_pixels_x = (int)x;
    r.num_pixels_y = (int)y;
    r.num_pixels_z = (int)z;
    r.pitch_xy = 1.0f;
    r.pitch_z = 1.0f;
    r.ct_norm0 = 1.0f;
    r.ct_norm1 = 1.0f;
    r.mu_water = 0.02f;
    return r;
}

}  // namespace

// ---- PreProcessingAgent (PreProcessingAgent/PreProcessingAgent.cpp:9-110) ----

PreProcessingAgent::PreProcessingAgent(size_t numThreads, size_t packSize, size_t inputSizeX, size_t inputSizeY,
                                       size_t borderSizeUp, size_t borderSizeBottom, size_t borderSizeLeft,
                                       size_t borderSizeRight, size_t outputSizeX, size_t outputSizeY,
                                       float brightField, const FloatVec& bhc)
    : ConcurrentAgentBase("PreProcessingAgent", numThreads), packSize(packSize), inputSizeX(inputSizeX),
      inputSizeY(inputSizeY), outputSizeX(outputSizeX), outputSizeY(outputSizeY) {
    if (outputSizeX != inputSizeX - borderSizeLeft - borderSizeRight ||
        outputSizeY != inputSizeY - borderSizeUp - borderSizeBottom)
        ThrowExceptionAndLog("PreProcessingAgent: resizing the cropped frame is not supported");
    if (bhc.size() != 3) ThrowException("The number of parameters in BeamHardeningParams should be 3.");
    jfdk_scan_params s = scan_defaults(1, inputSizeX, inputSizeY);
    s.border_up = (int)borderSizeUp;
    s.border_down = (int)borderSizeBottom;
    s.border_left = (int)borderSizeLeft;
    s.border_right = (int)borderSizeRight;
    s.bright_field = brightField;
    for (int i = 0; i < 3; ++i) s.beam_hardening[i] = bhc[i];
    for (size_t t = 0; t < numThreads; ++t)
        stages.emplace_back(new StageContext(s, recon_defaults(1, 1, 1), placeholder_ptm(outputSizeX, outputSizeY)));
}
PreProcessingAgent::~PreProcessingAgent() = default;

void PreProcessingAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<UINT16Vec>("Proj");
    pipeIn->SetConsumer(GetAgentName(), GetNumThreads(), packSize, 0);
    pipeOut = CreateNewPipe<FloatVec>("Proj");
    pipeOut->SetTemplate(FloatVec(outputSizeX * outputSizeY, 0.0f), {outputSizeX, outputSizeY});
    pipeOut->SetProducer(GetAgentName(), GetNumThreads(), packSize);
    MergePipeToTrunk(pipeOut);
}

void PreProcessingAgent::ManagerWorkFlow() {
    try {
        while (true) {
            WaitIdleWorkerIndex();
            Task task;
            task.ReadToken = pipeIn->GetReadToken();
            task.WriteToken = pipeOut->GetWriteToken(task.ReadToken.GetSize(), task.ReadToken.IsShotEnd());
            SubmitTask(std::make_unique<Task>(task));
        }
    } catch (PipeClosedAndEmptySignal&) {
    }
    pipeIn->Close();
    pipeOut->Close();
}

void PreProcessingAgent::ProcessTask(size_t ti, std::unique_ptr<TaskBase> base) {
    Task* task = static_cast<Task*>(base.get());
    ThreadOccupiedScope occupied(this);
    StageContext& st = *stages[ti];
    const size_t n = task->ReadToken.GetSize(), in = inputSizeX * inputSizeY, out = outputSizeX * outputSizeY;
    auto* d_raw = static_cast<uint16_t*>(st.Buffer(0, n * in * sizeof(uint16_t)));
    auto* d_out = static_cast<float*>(st.Buffer(1, n * out * sizeof(float)));
    for (size_t i = 0; i < n; ++i) st.Upload(d_raw + i * in, task->ReadToken.GetBuffer(i).data(), in * 2);
    st.Check(jfdk_preprocess_frames(st.ctx, d_raw, (int)n, d_out));
    for (size_t i = 0; i < n; ++i) st.Download(task->WriteToken.GetBuffer(i).data(), d_out + i * out, out * 4);
    WaitAsyncScope wait(&occupied);
    st.Sync();
}

// ---- CompositeAgent (CompositeAgent/CompositeAgent.cpp:9-83) --------------------

CompositeAgent::CompositeAgent(size_t numThreads, size_t inputWidth, size_t inputHeight, bool detectorAtTheRight,
                               float sourceOriginDistance, const std::vector<ProjectionMatrix>& projectionMatrices)
    : ConcurrentAgentBase("CompositeAgent", numThreads), width(inputWidth), height(inputHeight),
      numViewsPerRot(projectionMatrices.size()) {
    jfdk_scan_params s = scan_defaults(projectionMatrices.size(), inputWidth, inputHeight);
    s.dso = sourceOriginDistance;
    s.detector_on_right = detectorAtTheRight ? 1 : 0;
    s.filter_input_width = (int)(2 * inputWidth);   // a compositing context
    const std::vector<float> p = flatten(projectionMatrices);
    for (size_t t = 0; t < numThreads; ++t) stages.emplace_back(new StageContext(s, recon_defaults(1, 1, 1), p));
}
CompositeAgent::~CompositeAgent() = default;

void CompositeAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<FloatVec>("Proj");
    pipeIn->SetConsumer(GetAgentName(), GetNumThreads(), 2, 0);
    pipeOut = CreateNewPipe<FloatVec>("Proj");
    pipeOut->SetProducer(GetAgentName(), GetNumThreads(), 1);
    pipeOut->SetTemplate(FloatVec(width * height * 2, 0.0f), {width * 2, height});
    MergePipeToTrunk(pipeOut);
}

void CompositeAgent::ManagerWorkFlow() {
    try {
        while (true) {
            WaitIdleWorkerIndex();
            Task task;
            task.ReadToken = pipeIn->GetReadToken();
            task.WriteToken = pipeOut->GetWriteToken(1, task.ReadToken.IsShotEnd());
            SubmitTask(std::make_unique<Task>(task));
        }
    } catch (PipeClosedAndEmptySignal&) {
        pipeOut->Close();
    }
}

void CompositeAgent::ProcessTask(size_t ti, std::unique_ptr<TaskBase> base) {
    Task* task = static_cast<Task*>(base.get());
    ThreadOccupiedScope occupied(this);
    StageContext& st = *stages[ti];
    // token i holds frames 2i (view i) and 2i + 1 (its conjugate)
    const int view = (int)((task->ReadToken.GetStartIndex() / 2) % numViewsPerRot);
    const size_t px = width * height;
    auto* d_in = static_cast<float*>(st.Buffer(0, px * 2 * 4));
    auto* d_out = static_cast<float*>(st.Buffer(1, px * 2 * 4));
    st.Upload(d_in, task->ReadToken.GetBuffer(0).data(), px * 4);
    st.Upload(d_in + px, task->ReadToken.GetBuffer(1).data(), px * 4);
    st.Check(jfdk_composite_frames(st.ctx, d_in, d_in + px, view, 1, d_out));
    st.Download(task->WriteToken.GetBuffer(0).data(), d_out, px * 2 * 4);
    WaitAsyncScope wait(&occupied);
    st.Sync();
}

// ---- FilterAgent (FilterAgent/FilterAgent.cpp:10-192) --------------------------

FilterAgent::FilterAgent(size_t nThreads, size_t /*nRowsPerThread*/, size_t nInputWidth, size_t nInputHeight,
                         size_t nOutputWidth, bool detectorAtTheRight, float HalfSampleRate, float FilterCutOffStart,
                         float FilterCutOffEnd, const FloatVec& AdjustPoints, const FloatVec& AdjustLevelInDB,
                         const std::vector<ProjectionMatrix>& ptms, float DSO)
    : ConcurrentAgentBase("FilterAgent", nThreads), inputWidth(nInputWidth), height(nInputHeight),
      outputWidth(nOutputWidth), numViewsPerRot(ptms.size()) {
    if (AdjustPoints.size() != AdjustLevelInDB.size())
        ThrowExceptionAndLog("FilterAgent: adjust points and levels differ in length");
    jfdk_scan_params s = scan_defaults(ptms.size(), nOutputWidth, nInputHeight);
    s.dso = DSO;
    s.half_sample_rate = HalfSampleRate;
    s.detector_on_right = detectorAtTheRight ? 1 : 0;
    s.filter_input_width = (int)nInputWidth;
    jfdk_recon_params r = recon_defaults(1, 1, 1);
    r.filter_cutoff_start = FilterCutOffStart;
    r.filter_cutoff_end = FilterCutOffEnd;
    r.num_adjust = (int)AdjustPoints.size();
    r.adjust_points = AdjustPoints.data();
    r.adjust_level_db = AdjustLevelInDB.data();
    const std::vector<float> p = flatten(ptms);
    for (size_t t = 0; t < nThreads; ++t) stages.emplace_back(new StageContext(s, r, p));
}
FilterAgent::~FilterAgent() = default;

void FilterAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<FloatVec>("Proj");
    pipeIn->SetConsumer(GetAgentName(), GetNumThreads() + 1, 1, 0);
    pipeOut = CreateNewPipe<FloatVec>("Proj");
    pipeOut->SetTemplate(FloatVec(outputWidth * height, 0.0f), {outputWidth, height});
    pipeOut->SetProducer(GetAgentName(), GetNumThreads() + 1, 1);
    MergePipeToTrunk(pipeOut);
}

void FilterAgent::ManagerWorkFlow() {
    try {
        while (true) {
            WaitIdleWorkerIndex();
            Task task;
            task.ReadToken = pipeIn->GetReadToken();
            task.WriteToken = pipeOut->GetWriteToken(1, task.ReadToken.IsShotEnd());
            SubmitTask(std::make_unique<Task>(task));
        }
    } catch (PipeClosedAndEmptySignal&) {
        pipeOut->Close();
    }
}

void FilterAgent::ProcessTask(size_t ti, std::unique_ptr<TaskBase> base) {
    Task* task = static_cast<Task*>(base.get());
    ThreadOccupiedScope occupied(this);
    StageContext& st = *stages[ti];
    // the view's index within the rotation selects its 9-view pre-weight group
    const int view = (int)(task->ReadToken.GetStartIndex() % numViewsPerRot);
    auto* d_in = static_cast<float*>(st.Buffer(0, inputWidth * height * 4));
    auto* d_out = static_cast<float*>(st.Buffer(1, outputWidth * height * 4));
    st.Upload(d_in, task->ReadToken.GetBuffer(0).data(), inputWidth * height * 4);
    st.Check(jfdk_filter_frames(st.ctx, d_in, view, 1, d_out));
    st.Download(task->WriteToken.GetBuffer(0).data(), d_out, outputWidth * height * 4);
    WaitAsyncScope wait(&occupied);
    st.Sync();
}

// ---- ZFilterAgent (FilterAgent/ZFilterAgent.cpp:8-71) ---------------------------

ZFilterAgent::ZFilterAgent(size_t nThreads, size_t nWidth, size_t nHeight)
    : ConcurrentAgentBase("ZFilterAgent", nThreads), width(nWidth), height(nHeight) {
    for (size_t t = 0; t < nThreads; ++t)
        stages.emplace_back(
            new StageContext(scan_defaults(1, nWidth, nHeight), recon_defaults(1, 1, 1), placeholder_ptm(nWidth, nHeight)));
}
ZFilterAgent::~ZFilterAgent() = default;

void ZFilterAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<FloatVec>("Proj");
    pipeIn->SetConsumer(GetAgentName(), GetNumThreads(), 1, 0);
    pipeOut = CreateNewPipe<FloatVec>("Proj");
    pipeOut->SetProducer(GetAgentName(), GetNumThreads(), 1);
    pipeOut->SetTemplate(FloatVec(width * height), {width, height});
    MergePipeToTrunk(pipeOut);
}

void ZFilterAgent::ManagerWorkFlow() {
    try {
        while (true) {
            WaitIdleWorkerIndex();
            Task task;
            task.ReadToken = pipeIn->GetReadToken();
            task.WriteToken = pipeOut->GetWriteToken(1, task.ReadToken.IsShotEnd());
            SubmitTask(std::make_unique<Task>(task));
        }
    } catch (PipeClosedAndEmptySignal&) {
        pipeOut->Close();
    }
}

void ZFilterAgent::ProcessTask(size_t ti, std::unique_ptr<TaskBase> base) {
    Task* task = static_cast<Task*>(base.get());
    ThreadOccupiedScope occupied(this);
    StageContext& st = *stages[ti];
    auto* d = static_cast<float*>(st.Buffer(0, width * height * 4));
    st.Upload(d, task->ReadToken.GetBuffer(0).data(), width * height * 4);
    st.Check(jfdk_zfilter_frames(st.ctx, d, 1));
    st.Download(task->WriteToken.GetBuffer(0).data(), d, width * height * 4);
    WaitAsyncScope wait(&occupied);
    st.Sync();
}

// ---- page-locked pipe slots ------------------------------------------------------

// Registers every slot of a host pipe with cudaHostRegister, so that copies to
// and from the slots are DMA from / to them directly.  A slot the driver does
// not register (e.g. a small one sharing a page with another registration)
// stays pageable: its copies are still correct, through the driver's staging.
class PinnedSlots {
public:
    template <class T>
    explicit PinnedSlots(Pipe<std::vector<T>>& p) {
        for (size_t i = 0; i < p.NumSlots(); ++i) {
            std::vector<T>& s = p.Slot(i);
            if (s.empty()) continue;
            if (cudaHostRegister(s.data(), s.size() * sizeof(T), cudaHostRegisterDefault) == cudaSuccess)
                ptrs.push_back(s.data());
            else
                cudaGetLastError();
        }
    }
    ~PinnedSlots() {
        for (void* p : ptrs) cudaHostUnregister(p);
    }
    size_t Count() const { return ptrs.size(); }

private:
    std::vector<void*> ptrs;
};

static cudaStream_t new_stream() {
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        ThrowExceptionAndLog("CUDA failed to create a stream");
    }
    return s;
}

// One frame, asynchronously on `stream`, complete when this returns (the
// pipe token that owns the memory is released right after).
static void copy_frame(void* d, const void* s, size_t n, cudaMemcpyKind k, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(d, s, n, k, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        ThrowExceptionAndLog("CUDA frame copy failed");
    }
}

// ---- DeviceUploadAgent (CUDA/Tex2DUploadAgent.cpp:19-67) ------------------------

DeviceUploadAgent::DeviceUploadAgent(const std::string& pipeName, size_t width, size_t height)
    : SequentialAgentBase("DeviceUploadAgent", 1), pipeName(pipeName), width(width), height(height) {}
DeviceUploadAgent::~DeviceUploadAgent() {
    pinned.reset();
    if (stream) cudaStreamDestroy(static_cast<cudaStream_t>(stream));
}
void DeviceUploadAgent::GetReady() {
    pinned.reset(new PinnedSlots(*pipeIn));
    if (!stream) stream = new_stream();
}
size_t DeviceUploadAgent::NumPinnedSlots() const { return pinned ? pinned->Count() : 0; }

void DeviceUploadAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<FloatVec>(pipeName);
    pipeIn->SetConsumer(GetAgentName(), 1, 1, 0);
    pipeOut = CreateNewPipe<DeviceMemory<float>>(pipeName);
    pipeOut->SetTemplate(DeviceMemory<float>(width * height), {width, height});
    pipeOut->SetProducer(GetAgentName(), 1, 1);
    MergePipeToTrunk(pipeOut);
}

void DeviceUploadAgent::WorkFlow0() {
    try {
        while (true) {
            auto rt = pipeIn->GetReadToken();
            auto wt = pipeOut->GetWriteToken(1, rt.IsShotEnd());
            ThreadOccupiedScope occupied(this);
            copy_frame(wt.GetBuffer(0).Data(), rt.GetBuffer(0).data(), width * height * sizeof(float),
                       cudaMemcpyHostToDevice, stream);
        }
    } catch (PipeClosedAndEmptySignal&) {
        pipeOut->Close();
    }
}

// ---- BPCUDAAgent (BPCUDAAgent/BPCUDAAgent.cpp:49-287) ----------------------------

BPCUDAAgent::BPCUDAAgent(const std::vector<ProjectionMatrix>& ptms, size_t numDetectorsU, size_t numDetectorsV,
                         size_t volumeSizeX, size_t volumeSizeY, size_t volumeSizeZ, float pitchXY, float pitchZ,
                         size_t numSlicesPerRecon, size_t numReconParts,
                         const std::filesystem::path& /*tempFileFolder*/, size_t viewsPerChunk,
                         size_t deviceMemoryBudget)
    : SequentialAgentBase("BPCUDAAgent", 1), projectionMatrices(ptms), numDetectorsU(numDetectorsU),
      numDetectorsV(numDetectorsV), volumeSizeX(volumeSizeX), volumeSizeY(volumeSizeY), volumeSizeZ(volumeSizeZ),
      pitchXY(pitchXY), pitchZ(pitchZ),
      numSlicesPerRecon(std::min(std::max<size_t>(1, numSlicesPerRecon), volumeSizeZ)),
      numReconParts(std::max<size_t>(1, numReconParts)), viewsPerChunk(std::max<size_t>(1, viewsPerChunk)),
      deviceMemoryBudget(deviceMemoryBudget) {
    if (this->numSlicesPerRecon * this->numReconParts < volumeSizeZ)
        ThrowExceptionAndLog("BPCUDAAgent: numReconParts x numSlicesPerRecon does not cover the volume");
}
BPCUDAAgent::~BPCUDAAgent() = default;

void BPCUDAAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<DeviceMemory<float>>("Proj");
    pipeIn->SetConsumer(GetAgentName(), 1, viewsPerChunk, 0);
    pipeOut = CreateNewPipe<DeviceMemory<float>>("Slice");
    pipeOut->SetTemplate(DeviceMemory<float>(volumeSizeX * volumeSizeY), {volumeSizeX, volumeSizeY});
    pipeOut->SetProducer(GetAgentName(), 1, 1);
    MergePipeToTrunk(pipeOut);
}

void BPCUDAAgent::GetReady() {
    jfdk_scan_params s = scan_defaults(projectionMatrices.size(), numDetectorsU, numDetectorsV);
    jfdk_recon_params r = recon_defaults(volumeSizeX, volumeSizeY, volumeSizeZ);
    r.pitch_xy = pitchXY;
    r.pitch_z = pitchZ;
    stage.reset(new StageContext(s, r, flatten(projectionMatrices)));
    if (deviceMemoryBudget)
        stage->Check(jfdk_set_option(stage->ctx, JFDK_OPT_DEVICE_MEMORY_LIMIT,
                                     jfdk_device_bytes(stage->ctx) + (long long)deviceMemoryBudget));
    // the accumulators of one part (BPCUDACore's accumulatedVol)
    stage->Check(jfdk_bp_set_slab(stage->ctx, 0, (int)numSlicesPerRecon));
    stage->Check(jfdk_bp_reserve(stage->ctx, (int)std::min(viewsPerChunk, projectionMatrices.size())));
    staging.reset(new DeviceMemory<float>(viewsPerChunk * numDetectorsU * numDetectorsV));
    shot = 0;
}

void BPCUDAAgent::WorkFlow0() {
    const size_t frame = numDetectorsU * numDetectorsV;
    try {
        while (true) {
            auto rt = pipeIn->GetReadToken();
            ThreadOccupiedScope occupied(this);
            const size_t part = shot % numReconParts;
            const size_t z0 = std::min(part * numSlicesPerRecon, volumeSizeZ - 1);
            const size_t nz = std::min(numSlicesPerRecon, volumeSizeZ - z0);
            if (rt.IsShotStart()) {
                stage->Check(jfdk_bp_set_slab(stage->ctx, (int)z0, (int)nz));
                stage->Check(jfdk_bp_reset(stage->ctx));
            }
            const size_t n = rt.GetSize();
            const int view = (int)(rt.GetStartIndex() % projectionMatrices.size());
            for (size_t i = 0; i < n; ++i)
                if (cudaMemcpyAsync(staging->Data() + i * frame, rt.GetBuffer(i).CData(), frame * sizeof(float),
                                    cudaMemcpyDeviceToDevice, stage->stream) != cudaSuccess)
                    ThrowExceptionAndLog("CUDA staging copy failed");
            stage->Check(jfdk_bp_accumulate(stage->ctx, staging->Data(), view, (int)n));
            {
                WaitAsyncScope wait(&occupied);
                stage->Sync();   // the read token (frames) is released only after the kernels read it
            }
            if (rt.IsShotEnd()) {
                for (size_t z = z0; z < z0 + nz; ++z) {  // the part's slices, one token each
                    auto wt = pipeOut->GetWriteToken(1, z + 1 == volumeSizeZ);
                    stage->Check(jfdk_finalize(stage->ctx, (int)z, 1, 0, wt.GetBuffer(0).Data(), nullptr));
                    stage->Sync();
                }
                ++shot;
            }
        }
    } catch (PipeClosedAndEmptySignal&) {
        pipeOut->Close();
    }
}

// ---- DeviceMemoryDownloadAgent (CUDA/DeviceMemoryDownloadAgent.cpp:19-69) --------

DeviceMemoryDownloadAgent::DeviceMemoryDownloadAgent(const std::string& pipeName, size_t width, size_t height)
    : SequentialAgentBase("DeviceMemoryDownloadAgent", 1), pipeName(pipeName), width(width), height(height) {}
DeviceMemoryDownloadAgent::~DeviceMemoryDownloadAgent() {
    pinned.reset();
    if (stream) cudaStreamDestroy(static_cast<cudaStream_t>(stream));
}
void DeviceMemoryDownloadAgent::GetReady() {
    pinned.reset(new PinnedSlots(*pipeOut));
    if (!stream) stream = new_stream();
}
size_t DeviceMemoryDownloadAgent::NumPinnedSlots() const { return pinned ? pinned->Count() : 0; }

void DeviceMemoryDownloadAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<DeviceMemory<float>>(pipeName);
    pipeIn->SetConsumer(GetAgentName(), 1, 1, 0);
    pipeOut = CreateNewPipe<FloatVec>(pipeName);
    pipeOut->SetTemplate(FloatVec(width * height), {width, height});
    pipeOut->SetProducer(GetAgentName(), 1, 1);
    MergePipeToTrunk(pipeOut);
}

void DeviceMemoryDownloadAgent::WorkFlow0() {
    try {
        while (true) {
            auto rt = pipeIn->GetReadToken();
            auto wt = pipeOut->GetWriteToken(1, rt.IsShotEnd());
            ThreadOccupiedScope occupied(this);
            copy_frame(wt.GetBuffer(0).data(), rt.GetBuffer(0).CData(), width * height * sizeof(float),
                       cudaMemcpyDeviceToHost, stream);
        }
    } catch (PipeClosedAndEmptySignal&) {
        pipeOut->Close();
    }
}

// ---- CTNumAgent (CTNumAgent/CTNumAgent.cpp:7-69) ---------------------------------

CTNumAgent::CTNumAgent(size_t numThreads, size_t width, size_t height, float norm0, float norm1, float muWater)
    : ConcurrentAgentBase("CTNumAgent", numThreads), width(width), height(height) {
    jfdk_recon_params r = recon_defaults(width, height, 1);
    r.ct_norm0 = norm0;
    r.ct_norm1 = norm1;
    r.mu_water = muWater;
    for (size_t t = 0; t < numThreads; ++t)
        stages.emplace_back(new StageContext(scan_defaults(1, 8, 8), r, placeholder_ptm(8, 8)));
}
CTNumAgent::~CTNumAgent() = default;

void CTNumAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<FloatVec>("Slice");
    pipeIn->SetConsumer(GetAgentName(), GetNumThreads(), 1, 0);
    pipeOut = CreateNewPipe<FloatVec>("Slice");
    pipeOut->SetProducer(GetAgentName(), GetNumThreads(), 1);
    pipeOut->SetTemplate(FloatVec(width * height), {width, height});
    MergePipeToTrunk(pipeOut);
}

void CTNumAgent::ManagerWorkFlow() {
    try {
        while (true) {
            auto rt = pipeIn->GetReadToken();
            WaitIdleWorkerIndex();
            auto wt = pipeOut->GetWriteToken(1, rt.IsShotEnd());
            Task task;
            task.ReadToken = rt;
            task.WriteToken = wt;
            SubmitTask(std::make_unique<Task>(task));
        }
    } catch (PipeClosedAndEmptySignal&) {
        pipeOut->Close();
    }
}

void CTNumAgent::ProcessTask(size_t ti, std::unique_ptr<TaskBase> base) {
    Task* task = static_cast<Task*>(base.get());
    ThreadOccupiedScope occupied(this);
    StageContext& st = *stages[ti];
    const size_t n = width * height;
    auto* d = static_cast<float*>(st.Buffer(0, n * 4));
    st.Upload(d, task->ReadToken.GetBuffer(0).data(), n * 4);
    st.Check(jfdk_ctnum(st.ctx, d, n));
    st.Download(task->WriteToken.GetBuffer(0).data(), d, n * 4);
    WaitAsyncScope wait(&occupied);
    st.Sync();
}

}  // namespace JEngine
