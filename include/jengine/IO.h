// IO.h -- the reference application's on-disk formats, as agents and a reader:
//   InputAgent   JEngine/InputAgent.cpp:9-90    uint16 frames, one file per view
//                (printf-style name template, e.g. "Proj_%d.prj", no header),
//                each view followed by its conjugate (view + N/2) % N, as the
//                compositing chain reads them; "Proj" UINT16Vec out
//   OutputAgent  JEngine/OutputAgent.cpp:9-82   float slices, one file per slice
//                ("slice_%d.slc", no header, numbered from 0); "Slice" FloatVec in
//   PTMReader    JEngine/PTMReader.h:9-30        text, 12 numbers per view
// Pure host code (no CUDA); the reference's wide-character paths become
// std::filesystem paths and std::string templates.
#pragma once

#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "Agent.h"
#include "Geometry.h"

namespace JEngine {

class PTMReader {
public:
    PTMReader(const std::filesystem::path& fullPath, size_t /*nViews*/) : fs(fullPath) {}
    void ReadNextView(ProjectionMatrix& ptm) {
        for (size_t i = 0; i < 12; ++i) fs >> ptm[i];
    }
    bool Good() const { return fs.good(); }

private:
    std::ifstream fs;
};

// All views of a PTM file (the reference reads them the same way, one view
// after another, JEngine/JEngine.cpp:129-137).
std::vector<ProjectionMatrix> ReadPTMFile(const std::filesystem::path& fullPath, size_t nViews);

class InputAgent : public SequentialAgentBase {
public:
    // withConjugates: write view k and then view (k + N/2) % N for every k
    // (the reference always does; false writes each view once).
    InputAgent(size_t nDetSizeX, size_t nDetSizeY, size_t numViews, size_t numRoundsPerIteration,
               const std::filesystem::path& folder, const std::string& fileNameTemplate, bool withConjugates = true);

private:
    void SetPipesImpl() override;
    void WorkFlow0() override;
    void ReadFrame(size_t index, UINT16Vec& dst) const;

    const size_t detX, detY, numViews, rounds;
    const std::filesystem::path folder;
    const std::string nameTemplate;
    const bool conjugates;
    std::shared_ptr<Pipe<UINT16Vec>> pipeOut;
};

class OutputAgent : public SequentialAgentBase {
public:
    OutputAgent(size_t nWidth, size_t nHeight, const std::filesystem::path& folder, const std::string& fileNameTemplate);

private:
    void SetPipesImpl() override;
    void WorkFlow0() override;

    const size_t width, height;
    const std::filesystem::path folder;
    const std::string nameTemplate;
    std::shared_ptr<Pipe<FloatVec>> pipeIn;
};

// "Proj_%d.prj" with index 7 -> "Proj_7.prj".
std::string FormatName(const std::string& fileNameTemplate, size_t index);

}  // namespace JEngine
