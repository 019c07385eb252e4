// test_io.cpp -- the on-disk format agents (include/jengine/IO.h) on CPU:
// InputAgent reads frames in (view, conjugate) order, OutputAgent writes one
// float file per slice, ReadPTMFile parses 12 numbers per view.
#include <cstdio>
#include <filesystem>
#include <fstream>

#include "jengine/IO.h"

using namespace JEngine;

static int failures = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            ++failures;                                            \
        }                                                          \
    } while (0)

class Collect : public SequentialAgentBase {
public:
    Collect() : SequentialAgentBase("Collect", 1) {}
    std::vector<UINT16Vec> frames;

private:
    void SetPipesImpl() override {
        in = BranchPipeFromTrunk<UINT16Vec>("Proj");
        in->SetConsumer(GetAgentName(), 1, 1, 0);
    }
    void WorkFlow0() override {
        try {
            while (true) frames.push_back(in->GetReadToken().GetBuffer(0));
        } catch (PipeClosedAndEmptySignal&) {
        }
    }
    std::shared_ptr<Pipe<UINT16Vec>> in;
};

class Slices : public SequentialAgentBase {
public:
    Slices(size_t w, size_t h, size_t n) : SequentialAgentBase("Slices", 1), w(w), h(h), n(n) {}

private:
    void SetPipesImpl() override {
        out = CreateNewPipe<FloatVec>("Slice");
        out->SetTemplate(FloatVec(w * h), {w, h});
        out->SetProducer(GetAgentName(), 1, 1);
        MergePipeToTrunk(out);
    }
    void WorkFlow0() override {
        for (size_t s = 0; s < n; ++s) {
            auto wt = out->GetWriteToken(1, s + 1 == n);
            for (size_t i = 0; i < w * h; ++i) wt.GetBuffer(0)[i] = (float)(s * 100000 + i) * 0.5f;
        }
        out->Close();
    }
    size_t w, h, n;
    std::shared_ptr<Pipe<FloatVec>> out;
};

template <class... A>
static void run(std::vector<std::shared_ptr<AgentBase>> agents) {
    std::vector<std::shared_ptr<PipeBase>> trunk;
    for (auto& a : agents) a->SetPipes(trunk);
    for (auto& a : agents) a->GetReady();
    for (auto& a : agents) a->Start();
    for (auto& a : agents) a->Join();
}

int main(int argc, char** argv) {
    const std::filesystem::path dir = argc > 1 ? argv[1] : std::filesystem::temp_directory_path() / "jfdk_io";
    std::filesystem::create_directories(dir);
    const size_t W = 7, H = 5, N = 6;
    for (size_t v = 0; v < N; ++v) {
        std::ofstream f(dir / FormatName("Proj_%d.prj", v), std::ios::binary);
        for (size_t i = 0; i < W * H; ++i) {
            const uint16_t x = (uint16_t)(v * 1000 + i);
            f.write(reinterpret_cast<const char*>(&x), 2);
        }
    }
    // frames in (view, conjugate) order, two rounds
    {
        auto c = std::make_shared<Collect>();
        run({std::make_shared<InputAgent>(W, H, N, 2, dir, "Proj_%d.prj"), c});
        CHECK(c->frames.size() == 2 * 2 * N);
        for (size_t k = 0; k < c->frames.size(); ++k) {
            const size_t v = (k / 2) % N, expect = (k % 2 == 0) ? v : (v + N / 2) % N;
            CHECK(c->frames[k][0] == expect * 1000 && c->frames[k][W * H - 1] == expect * 1000 + W * H - 1);
        }
    }
    {
        auto c = std::make_shared<Collect>();
        run({std::make_shared<InputAgent>(W, H, N, 1, dir, "Proj_%d.prj", false), c});
        CHECK(c->frames.size() == N);
        for (size_t k = 0; k < N; ++k) CHECK(c->frames[k][3] == k * 1000 + 3);
    }
    // slices out
    {
        run({std::make_shared<Slices>(W, H, 4), std::make_shared<OutputAgent>(W, H, dir, "slice_%d.slc")});
        for (size_t s = 0; s < 4; ++s) {
            std::ifstream f(dir / FormatName("slice_%d.slc", s), std::ios::binary);
            FloatVec x(W * H);
            f.read(reinterpret_cast<char*>(x.data()), (std::streamsize)(4 * W * H));
            CHECK(f.good());
            CHECK(x[0] == (float)(s * 100000) * 0.5f && x[W * H - 1] == (float)(s * 100000 + W * H - 1) * 0.5f);
        }
    }
    // PTM text
    {
        std::ofstream f(dir / "PTM.dat");
        for (size_t v = 0; v < 3; ++v) {
            for (int i = 0; i < 12; ++i) f << (v * 12 + i) * 0.25 << (i == 11 ? "\n" : " ");
        }
        f.close();
        auto p = ReadPTMFile(dir / "PTM.dat", 3);
        CHECK(p.size() == 3 && p[2][11] == (2 * 12 + 11) * 0.25f && p[1][0] == 12 * 0.25f);
        bool threw = false;
        try {
            ReadPTMFile(dir / "PTM.dat", 4);
        } catch (Exception&) {
            threw = true;
        }
        CHECK(threw);
    }
    std::printf("OK (%d failures)\n", failures);
    return failures ? 1 : 0;
}
