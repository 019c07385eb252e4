// Geometry.h -- projection matrices and the scan / reconstruction parameter
// structs the hot-path agents are built from.
//
// Same names, layout and float arithmetic as the reference:
//   ProjectionMatrix / TransformMatrix  TransformMatrix/TransformMatrixBase.h:9-63
//     (row-major, (r, c) = r * 4 + c), ProjectionMatrix.h:11-19;
//   ProjectionMatrixModifier            TransformMatrix/ProjectionMatrixModifier.cpp:5-43;
//   MatrixConvertor                     TransformMatrix/MatrixConvertor.cpp:8-32;
//   ScanParams / ReconParams            Config/ScanParams.h:13-40, Config/ReconParams.h:14-68
//     (the fields on the FDK path).
#pragma once

#include <cstring>
#include <vector>

#include "Common.h"

namespace JEngine {

class TransformMatrixBase {
public:
    explicit TransformMatrixBase(size_t n) : m(n, 0.0f) {}
    TransformMatrixBase(size_t n, const float* p) : m(p, p + n) {}
    float& operator[](size_t i) { return m[i]; }
    const float& operator[](size_t i) const { return m[i]; }
    float& operator()(size_t r, size_t c) { return m[r * 4 + c]; }
    const float& operator()(size_t r, size_t c) const { return m[r * 4 + c]; }
    float* Data() { return m.data(); }
    const float* Data() const { return m.data(); }
    bool operator==(const TransformMatrixBase& o) const { return m == o.m; }

private:
    std::vector<float> m;
};

// (x, y, z, 1) -> (u w, v w, w)
class ProjectionMatrix : public TransformMatrixBase {
public:
    ProjectionMatrix() : TransformMatrixBase(12) {}
    explicit ProjectionMatrix(const float* p) : TransformMatrixBase(12, p) {}
};

class TransformMatrix : public TransformMatrixBase {
public:
    TransformMatrix() : TransformMatrixBase(16) {}
    explicit TransformMatrix(const float* p) : TransformMatrixBase(16, p) {}
};

namespace ProjectionMatrixModifier {
inline void MoveUAxis(ProjectionMatrix& p, float u) { for (size_t j = 0; j < 4; ++j) p(0, j) -= p(2, j) * u; }
inline void MoveVAxis(ProjectionMatrix& p, float v) { for (size_t j = 0; j < 4; ++j) p(1, j) -= p(2, j) * v; }
inline void ReverseXAxis(ProjectionMatrix& p) { for (size_t j = 0; j < 3; ++j) p(j, 0) *= -1.0f; }
inline void ReverseYAxis(ProjectionMatrix& p) { for (size_t j = 0; j < 3; ++j) p(j, 1) *= -1.0f; }
inline void MoveZAxis(ProjectionMatrix& p, float z) { for (size_t i = 0; i < 3; ++i) p(i, 3) += p(i, 2) * z; }
}  // namespace ProjectionMatrixModifier

class MatrixConvertor {
public:
    explicit MatrixConvertor(float dso) {
        const float far_ = (1.0f + 1.0f / dso) * dso, near_ = (1.0f - 1.0f / dso) * dso;
        s20 = (far_ + near_) / (far_ - near_);
        s23 = ((far_ + near_) - 2.0f * far_ * near_ / dso) / (far_ - near_) / dso;
    }
    void PTM2TM(TransformMatrix& tm, const ProjectionMatrix& p) const {
        std::memcpy(tm.Data(), p.Data(), 8 * sizeof(float));
        tm(2, 0) = s20 * p(2, 0);
        tm(2, 1) = s20 * p(2, 1);
        tm(2, 2) = 0.0f;
        tm(2, 3) = s23 * p(2, 3);
        std::memcpy(tm.Data() + 12, p.Data() + 8, 4 * sizeof(float));
    }
    void TM2PTM(ProjectionMatrix& p, const TransformMatrix& tm) const {
        std::memcpy(p.Data(), tm.Data(), 8 * sizeof(float));
        std::memcpy(p.Data() + 8, tm.Data() + 12, 4 * sizeof(float));
    }

private:
    float s20, s23;
};

struct ScanParams {
    size_t NumViews = 0;
    float DSO = 0.0f;
    float DSD = 0.0f;
    size_t NumDetsU = 0;
    size_t NumDetsV = 0;
    float DetectorPixelSize = 0.0f;
    size_t BorderSizeUp = 0, BorderSizeDown = 0, BorderSizeLeft = 0, BorderSizeRight = 0;
    float BrightField = 0.0f;
    FloatVec BeamHardeningParams{1.0f, 0.0f, 0.0f};
    // derived (Config/ConfigHelper.cpp:52-63)
    float HalfSampleRate = 0.0f;
    size_t NumUsedDetsU = 0;
    size_t NumUsedDetsV = 0;

    void Derive() {
        const float detectorSizeAtISO = DetectorPixelSize / DSD * DSO;
        HalfSampleRate = 0.5f * (1.0f / detectorSizeAtISO);
        NumUsedDetsU = NumDetsU - BorderSizeLeft - BorderSizeRight;
        NumUsedDetsV = NumDetsV - BorderSizeUp - BorderSizeDown;
    }
};

struct ReconParams {
    size_t NumPixelsX = 0, NumPixelsY = 0, NumPixelsZ = 0;
    float PitchXY = 0.0f, PitchZ = 0.0f;
    bool MirroringY = false;
    float CenterZ = 0.0f;
    float CTNumNorm0 = 1.0f, CTNumNorm1 = 1.0f;
    float FilterCutOffStart = 0.0f, FilterCutOffEnd = 0.0f;
    FloatVec FilterAdjustPoints, FilterAdjustLevelInDB;
    float MuWater = 0.02f;  // Config/ConfigHelper.cpp:70
};

}  // namespace JEngine
