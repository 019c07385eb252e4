// IO.cpp -- on-disk formats of the reference application (include/jengine/IO.h).
#include "../../include/jengine/IO.h"

#include <chrono>
#include <cstdio>
#include <thread>

namespace JEngine {

std::string FormatName(const std::string& t, size_t index) {
    std::vector<char> buf(t.size() + 32);
    const int n = std::snprintf(buf.data(), buf.size(), t.c_str(), (int)index);
    if (n < 0) ThrowExceptionAndLog("bad file name template: " + t);
    if ((size_t)n >= buf.size()) {
        buf.resize((size_t)n + 1);
        std::snprintf(buf.data(), buf.size(), t.c_str(), (int)index);
    }
    return std::string(buf.data());
}

std::vector<ProjectionMatrix> ReadPTMFile(const std::filesystem::path& fullPath, size_t nViews) {
    if (!std::filesystem::exists(fullPath)) ThrowExceptionAndLog(fullPath.string() + " does not exist");
    PTMReader r(fullPath, nViews);
    std::vector<ProjectionMatrix> out(nViews);
    for (auto& p : out) r.ReadNextView(p);
    if (!r.Good()) ThrowExceptionAndLog("PTM file " + fullPath.string() + " holds fewer than " + std::to_string(nViews) + " views");
    return out;
}

// ---- InputAgent (JEngine/InputAgent.cpp:9-90) ------------------------------------

InputAgent::InputAgent(size_t nDetSizeX, size_t nDetSizeY, size_t nViews, size_t nRounds,
                       const std::filesystem::path& f, const std::string& t, bool withConjugates)
    : SequentialAgentBase("InputAgent", 1), detX(nDetSizeX), detY(nDetSizeY), numViews(nViews), rounds(nRounds),
      folder(f), nameTemplate(t), conjugates(withConjugates) {
    if (!std::filesystem::exists(folder)) ThrowExceptionAndLog(folder.string() + " does not exist.");
    if (!std::filesystem::is_directory(folder)) ThrowExceptionAndLog(folder.string() + " is not a folder");
}

void InputAgent::SetPipesImpl() {
    pipeOut = CreateNewPipe<UINT16Vec>("Proj");
    pipeOut->SetTemplate(UINT16Vec(detX * detY), {detX, detY});
    pipeOut->SetProducer(GetAgentName(), 1, 1);
    MergePipeToTrunk(pipeOut);
}

void InputAgent::ReadFrame(size_t index, UINT16Vec& dst) const {
    const std::filesystem::path p = folder / FormatName(nameTemplate, index);
    std::ifstream ifs(p, std::ios::binary);
    if (!ifs) ThrowExceptionAndLog("cannot open " + p.string());
    ifs.read(reinterpret_cast<char*>(dst.data()), (std::streamsize)(detX * detY * sizeof(uint16_t)));
    if (!ifs) ThrowExceptionAndLog(p.string() + " is shorter than one frame");
}

void InputAgent::WorkFlow0() {
    for (size_t r = 0; r < rounds; ++r) {
        for (size_t v = 0; v < numViews; ++v) {
            const bool last = v + 1 == numViews;
            {
                auto wt = pipeOut->GetWriteToken(1, last && !conjugates);
                ThreadOccupiedScope occupied(this);
                WaitAsyncScope wait(&occupied);
                ReadFrame(v, wt.GetBuffer(0));
            }
            if (conjugates) {
                auto wt = pipeOut->GetWriteToken(1, last);
                ThreadOccupiedScope occupied(this);
                WaitAsyncScope wait(&occupied);
                ReadFrame((v + numViews / 2) % numViews, wt.GetBuffer(0));
            }
        }
    }
    pipeOut->Close();
}

// ---- OutputAgent (JEngine/OutputAgent.cpp:9-82) ----------------------------------

OutputAgent::OutputAgent(size_t nWidth, size_t nHeight, const std::filesystem::path& f, const std::string& t)
    : SequentialAgentBase("OutputAgent", 1), width(nWidth), height(nHeight), folder(f), nameTemplate(t) {
    if (!std::filesystem::exists(folder)) ThrowExceptionAndLog(folder.string() + " does not exist.");
}

void OutputAgent::SetPipesImpl() {
    pipeIn = BranchPipeFromTrunk<FloatVec>("Slice");
    pipeIn->SetConsumer(GetAgentName(), GetNumThreads(), 1, 0);
}

void OutputAgent::WorkFlow0() {
    size_t index = 0;
    try {
        while (true) {
            auto rt = pipeIn->GetReadToken();
            ThreadOccupiedScope occupied(this);
            const std::filesystem::path p = folder / FormatName(nameTemplate, index);
            WaitAsyncScope wait(&occupied);
            // three attempts, a second apart, as the reference does
            for (int attempt = 0; attempt < 3; ++attempt) {
                std::ofstream ofs(p, std::ios::binary);
                if (ofs.good()) {
                    ofs.write(reinterpret_cast<const char*>(rt.GetBuffer(0).data()),
                              (std::streamsize)(sizeof(float) * width * height));
                    ++index;
                    break;
                }
                GLog("Fail to write file " + p.string());
                if (attempt == 2) ThrowExceptionAndLog("Error writing output file #" + std::to_string(index));
                std::this_thread::sleep_for(std::chrono::seconds(1));
            }
        }
    } catch (PipeClosedAndEmptySignal&) {
    }
}

}  // namespace JEngine
