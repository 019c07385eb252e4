// test_agents_gpu.cpp -- the reference's GPU agent chain on libjfdk.so:
// Source -> PreProcessingAgent -> [CompositeAgent] -> FilterAgent ->
// DeviceUploadAgent -> BPCUDAAgent -> DeviceMemoryDownloadAgent -> CTNumAgent
// -> Sink (the order of JEngine/JEngine.cpp:186-314).
//
// usage: test_agents_gpu <case.bin> <out.bin> [folder|-] [parts|retry]
//   With a folder, the frames come from its Proj_%d.prj files and the
//   orbit from its PTM.dat (InputAgent, ReadPTMFile), and the slices go to
//   slice_%d.slc files there (OutputAgent) -- the application's file chain.
//   parts: the volume in that many z-parts; retry: the application's part
//   loop under a device-memory budget that only 3 or more parts fit.
//   case.bin: int32 header [views, detU, detV, X, Y, Z, comp] (comp: -1 no
//   compositing, else 1 when the detector is on the right), float32 [dso, hsr,
//   bright, bhc0, bhc1, bhc2, pitchXY, pitchZ, norm0, norm1, cutStart,
//   cutEnd, nAdj], nAdj adjust points, nAdj levels, views*12 PTM floats,
//   views*detV*detU uint16 frames.  out.bin: Z*Y*X float32 HU.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

#include "jengine/Agents.h"
#include "jengine/IO.h"
#include "jengine/ReconParts.h"

using namespace JEngine;

class FrameSource : public SequentialAgentBase {
public:
    // pairs: write view k and then view (k + N/2) % N, as InputAgent does for
    // compositing (JEngine/InputAgent.cpp:45-90)
    FrameSource(const std::vector<UINT16Vec>& frames, size_t w, size_t h, int shots, bool pairs)
        : SequentialAgentBase("InputAgent", 1), frames(frames), w(w), h(h), shots(shots), pairs(pairs) {}

private:
    void SetPipesImpl() override {
        out = CreateNewPipe<UINT16Vec>("Proj");
        out->SetTemplate(UINT16Vec(w * h), {w, h});
        out->SetProducer(GetAgentName(), 1, 1);
        MergePipeToTrunk(out);
    }
    void WorkFlow0() override {
        const size_t n = frames.size();
        for (int s = 0; s < shots; ++s)
            for (size_t i = 0; i < n; ++i) {
                if (!pairs) {
                    out->GetWriteToken(1, i + 1 == n).GetBuffer(0) = frames[i];
                } else {
                    out->GetWriteToken(1, false).GetBuffer(0) = frames[i];
                    out->GetWriteToken(1, i + 1 == n).GetBuffer(0) = frames[(i + n / 2) % n];
                }
            }
        out->Close();
    }
    const std::vector<UINT16Vec>& frames;
    size_t w, h;
    int shots;
    bool pairs;
    std::shared_ptr<Pipe<UINT16Vec>> out;
};

class SliceSink : public SequentialAgentBase {
public:
    explicit SliceSink(size_t n) : SequentialAgentBase("OutputAgent", 1), n(n) {}
    std::vector<FloatVec> slices;

private:
    void SetPipesImpl() override {
        in = BranchPipeFromTrunk<FloatVec>("Slice");
        in->SetConsumer(GetAgentName(), 1, 1, 0);
    }
    void WorkFlow0() override {
        try {
            while (true) slices.push_back(in->GetReadToken().GetBuffer(0));
        } catch (PipeClosedAndEmptySignal&) {
        }
    }
    size_t n;
    std::shared_ptr<Pipe<FloatVec>> in;
};

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    std::ifstream f(argv[1], std::ios::binary);
    int hdr[7];
    float prm[13];
    f.read((char*)hdr, sizeof hdr);
    f.read((char*)prm, sizeof prm);
    const size_t V = hdr[0], U = hdr[1], H = hdr[2], X = hdr[3], Y = hdr[4], Z = hdr[5];
    const bool comp = hdr[6] >= 0, detRight = hdr[6] == 1;
    const int nAdj = (int)prm[12];
    FloatVec adjP(nAdj), adjL(nAdj);
    f.read((char*)adjP.data(), 4 * nAdj);
    f.read((char*)adjL.data(), 4 * nAdj);
    std::vector<ProjectionMatrix> ptms(V);
    for (auto& p : ptms) f.read((char*)p.Data(), 48);
    std::vector<UINT16Vec> frames(V, UINT16Vec(U * H));
    for (auto& fr : frames) f.read((char*)fr.data(), 2 * U * H);
    if (!f) return 3;
    const std::filesystem::path folder = (argc > 3 && std::string(argv[3]) != "-") ? argv[3] : "";
    if (!folder.empty()) {
        try {
            auto fromFile = ReadPTMFile(folder / "PTM.dat", V);
            for (size_t v = 0; v < V; ++v)
                if (std::memcmp(fromFile[v].Data(), ptms[v].Data(), 48) != 0) {
                    std::printf("PTM.dat view %zu differs\n", v);
                    return 7;
                }
            ptms = fromFile;
        } catch (std::exception& e) {
            std::printf("exception: %s\n", e.what());
            return 4;
        }
    }

    // z-parts: a count, or "retry" -- the application's loop over part counts
    // with the backprojection's device memory bounded so that the
    // accumulators of ceil(Z / 3) slices fit and those of ceil(Z / 2) do not
    const std::string partsArg = argc > 4 ? argv[4] : "1";
    const bool retry = partsArg == "retry";
    const size_t chunk = 7;
    size_t budget = 0;
    // (accumulators: 2 floats a voxel; packed store: 16 bytes a pixel a view;
    // margin: half a slice of accumulators)
    if (retry) budget = 2 * X * Y * ((Z + 2) / 3) * 4 + chunk * H * U * 16 + X * Y * 4;

    const int scans = 2;  // two scans back to back: the second must not see the first
    std::shared_ptr<SliceSink> sink;
    std::shared_ptr<DeviceUploadAgent> upload;
    std::shared_ptr<DeviceMemoryDownloadAgent> download;
    auto makeAgents = [&](const ReconPartPlan& plan) {
        std::vector<std::shared_ptr<AgentBase>> agents;
        const int shots = scans * (int)plan.numReconParts;  // the views once per part
        if (folder.empty())
            agents.push_back(std::make_shared<FrameSource>(frames, U, H, shots, comp));
        else
            agents.push_back(std::make_shared<InputAgent>(U, H, V, shots, folder, "Proj_%d.prj", comp));
        agents.push_back(std::make_shared<PreProcessingAgent>(2, 1, U, H, 0, 0, 0, 0, U, H, prm[2],
                                                              FloatVec{prm[3], prm[4], prm[5]}));
        if (comp) agents.push_back(std::make_shared<CompositeAgent>(2, U, H, detRight, prm[0], ptms));
        agents.push_back(std::make_shared<FilterAgent>(2, 240, comp ? 2 * U : U, H, U, detRight, prm[1], prm[10],
                                                       prm[11], adjP, adjL, ptms, prm[0]));
        upload = std::make_shared<DeviceUploadAgent>("Proj", U, H);
        agents.push_back(upload);
        agents.push_back(std::make_shared<BPCUDAAgent>(ptms, U, H, X, Y, Z, prm[6], prm[7], plan.numSlicesPerRecon,
                                                       plan.numReconParts, "", chunk, budget));
        download = std::make_shared<DeviceMemoryDownloadAgent>("Slice", X, Y);
        agents.push_back(download);
        agents.push_back(std::make_shared<CTNumAgent>(2, X, Y, prm[8], prm[9], 0.02f));
        sink = std::make_shared<SliceSink>(Z);
        if (folder.empty())
            agents.push_back(sink);
        else
            agents.push_back(std::make_shared<OutputAgent>(X, Y, folder, "slice_%d.slc"));
        return agents;
    };

    std::vector<std::shared_ptr<AgentBase>> agents;
    std::vector<std::shared_ptr<PipeBase>> trunk;
    try {
        ReconPartPlan plan{1, Z};
        if (retry) {
            plan = PrepareAgentsWithRetry(Z, makeAgents, agents, trunk);
        } else {
            const size_t parts = std::stoul(partsArg);
            plan = {parts, (Z - 1) / parts + 1};
            agents = makeAgents(plan);
            for (auto& a : agents) a->SetPipes(trunk);
            for (auto& a : agents) a->GetReady();
        }
        std::printf("plan: %zu parts of %zu slices\n", plan.numReconParts, plan.numSlicesPerRecon);
        std::printf("pinned slots: upload %zu, download %zu\n", upload->NumPinnedSlots(), download->NumPinnedSlots());
        if (upload->NumPinnedSlots() == 0 || download->NumPinnedSlots() == 0) return 8;
        for (auto& a : agents) a->Start();
        for (auto& a : agents) a->Join();
    } catch (std::exception& e) {
        std::printf("exception: %s\n", e.what());
        return 4;
    }
    const size_t shots = scans;
    if (!folder.empty()) {  // the slice files, numbered on across both scans
        for (size_t s = 0; s < shots * Z; ++s) {
            std::ifstream in(folder / FormatName("slice_%d.slc", s), std::ios::binary);
            FloatVec x(X * Y);
            in.read((char*)x.data(), 4 * X * Y);
            if (!in) break;
            sink->slices.push_back(x);
        }
    }
    std::printf("slices received: %zu (expected %zu)\n", sink->slices.size(), shots * Z);
    if (sink->slices.size() != shots * Z) return 5;
    std::ofstream o(argv[2], std::ios::binary);
    for (size_t s = (shots - 1) * Z; s < shots * Z; ++s) o.write((const char*)sink->slices[s].data(), 4 * X * Y);
    // both scans identical -> identical volumes
    for (size_t z = 0; z < Z; ++z)
        if (sink->slices[z] != sink->slices[Z + z]) {
            std::printf("scan 2 differs from scan 1 at slice %zu\n", z);
            return 6;
        }
    return 0;
}
