// ref_driver.cpp -- C entry points that run the reference's own Core classes
// (compiled from the JEngine sources by oracle/build.py) on caller buffers.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/ (second oracle, used to pin the
// restatement in fdk_oracle.c) and by bench.py's CPU baseline.  The threading
// mirrors the reference agents:
//   FilterAgent  -- rows of a view split over threads, pre-weight regenerated
//                   every 9 views from view min(v+4, N-1)
//                   (FilterAgent/FilterAgent.cpp:99-192)
//   BPAgent      -- one view at a time, slices split over threads, a barrier
//                   per view (BPAgent/BPAgent.cpp:60-108)
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "BPAgent/BPCore.h"
#include "CompositeAgent/CompositeCore.h"
#include "CTNumAgent/CTNumCore.h"
#include "FilterAgent/FilterCore.h"
#include "FilterAgent/PreFilterWeightGenerator.h"
#include "PreProcessingAgent/PreProcessingCore.h"
#include "TransformMatrix/MatrixConvertor.h"
#include "TransformMatrix/ProjectionMatrixModifier.h"

using namespace JEngine;

static std::vector<ProjectionMatrix> to_ptms(const float* p, int n) {
    std::vector<ProjectionMatrix> v;
    v.reserve(n);
    for (int i = 0; i < n; ++i) v.emplace_back(p + 12 * (size_t)i);
    return v;
}

template <class F>
static void parallel_for(int n, int nthreads, F f) {
    nthreads = std::max(1, std::min(nthreads, n));
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([=] {
            for (int i = (int)((long)n * t / nthreads); i < (int)((long)n * (t + 1) / nthreads); ++i) f(t, i);
        });
    for (auto& x : th) x.join();
}

extern "C" {

int jref_ptm2tm(float* tm16, const float* ptm12, float dso) {
    MatrixConvertor c(dso);
    ProjectionMatrix p(ptm12);
    TransformMatrix t;
    c.PTM2TM(t, p);
    std::memcpy(tm16, t.Data(), 16 * sizeof(float));
    return 0;
}

// op: 0 MoveU(a), 1 MoveV(a), 2 ReverseX, 3 ReverseY, 4 MoveZ(a)
int jref_ptm_modify(float* ptm12, int op, float a) {
    ProjectionMatrix p(ptm12);
    switch (op) {
        case 0: ProjectionMatrixModifier::MoveUAxis(p, a); break;
        case 1: ProjectionMatrixModifier::MoveVAxis(p, a); break;
        case 2: ProjectionMatrixModifier::ReverseXAxis(p); break;
        case 3: ProjectionMatrixModifier::ReverseYAxis(p); break;
        case 4: ProjectionMatrixModifier::MoveZAxis(p, a); break;
        default: return -1;
    }
    std::memcpy(ptm12, p.Data(), 12 * sizeof(float));
    return 0;
}

int jref_preprocess(float* out, const uint16_t* in, int nViews, int inW, int inH, int bUp,
                    int bDown, int bLeft, int bRight, int outW, int outH, float brightField,
                    const float* bhc3, int nthreads) {
    FloatVec bhc(bhc3, bhc3 + 3);
    std::vector<std::unique_ptr<PreProcessingCore>> cores;
    nthreads = std::max(1, std::min(nthreads, nViews));
    for (int t = 0; t < nthreads; ++t)
        cores.emplace_back(new PreProcessingCore(inW, inH, bUp, bDown, bLeft, bRight, outW, outH, brightField, bhc));
    parallel_for(nViews, nthreads, [&](int t, int v) {
        UINT16Vec src(in + (size_t)v * inW * inH, in + (size_t)(v + 1) * inW * inH);
        FloatVec dst((size_t)outW * outH);
        cores[t]->Process(dst, src);
        std::memcpy(out + (size_t)v * outW * outH, dst.data(), dst.size() * sizeof(float));
    });
    return 0;
}

int jref_preweight(float* weights, const float* ptms, int nViews, int inputWidth, int height,
                   int detOnRight, float dso, int viewIndex) {
    PreFilterWeightGenerator g(to_ptms(ptms, nViews), inputWidth, height, detOnRight != 0, dso);
    g.Generate(weights, viewIndex);
    return 0;
}

// FilterAgent + FilterCore over views [0, nViews): in [nViews][H][W] -> out
// [nViews][H][Wout].  ptms are all views of the rotation (pre-weight source).
int jref_filter(float* out, const float* in, int nViews, int W, int H, int Wout, int mirror,
                float hsr, float cutStart, float cutEnd, const float* adjPts, const float* adjDB,
                int nAdj, const float* ptms, int numViewsPerRot, float dso, int nthreads) {
    FloatVec ap(adjPts, adjPts + nAdj), ad(adjDB, adjDB + nAdj);
    FilterCore core(W, H, Wout, mirror != 0, hsr, cutStart, cutEnd, ap, ad);
    PreFilterWeightGenerator gen(to_ptms(ptms, numViewsPerRot), W, H, mirror != 0, dso);
    const size_t L = FilterCore::CalFFTLength(W);
    FloatVec pw(L * H);
    nthreads = std::max(1, nthreads);
    std::vector<FloatVec> bs(nthreads), bc(nthreads);
    for (int t = 0; t < nthreads; ++t) core.InitBuffer(bs[t], bc[t]);
    for (int v = 0; v < nViews; ++v) {
        const size_t vi = (size_t)v % numViewsPerRot;
        if (vi % 9 == 0) gen.Generate(pw.data(), std::min(vi + 9 / 2, (size_t)numViewsPerRot - 1));
        parallel_for(H, nthreads, [&](int t, int r) {
            core.ProcessRow(out + ((size_t)v * H + r) * Wout, in + ((size_t)v * H + r) * W,
                            pw.data() + (size_t)r * L, bs[t].data(), bc[t].data());
        });
    }
    return 0;
}

// FilterCore::ProcessRow without a pre-weight, one row per call batch.
int jref_filter_rows_noweight(float* out, const float* in, int rows, int W, int Wout, int mirror,
                              float hsr, float cutStart, float cutEnd, const float* adjPts,
                              const float* adjDB, int nAdj) {
    FloatVec ap(adjPts, adjPts + nAdj), ad(adjDB, adjDB + nAdj);
    FilterCore core(W, rows, Wout, mirror != 0, hsr, cutStart, cutEnd, ap, ad);
    FloatVec bs, bc;
    core.InitBuffer(bs, bc);
    for (int r = 0; r < rows; ++r) core.ProcessRow(out + (size_t)r * Wout, in + (size_t)r * W, bs.data(), bc.data());
    return 0;
}

// BPAgent + BPCore: proj [nViews][V][U] (filtered, not tapered; copied, since
// InitView tapers in place) -> out [Z][Y][X] = sum / count.
int jref_bp(float* out, const float* proj, const float* ptms, int nViews,
            int U, int V, int X, int Y, int Z, float pitchXY, float pitchZ, int nthreads) {
    BPCore core(U, V, X, Y, Z, pitchXY, pitchZ, to_ptms(ptms, nViews));
    nthreads = std::max(1, nthreads);
    std::vector<FloatVec> bufs(nthreads, core.InitBuffer());
    core.InitShot();
    FloatVec p((size_t)U * V);
    const int slicesPerTask = 10;  // BPAgent.cpp:25
    const int nTasks = (Z + slicesPerTask - 1) / slicesPerTask;
    for (int v = 0; v < nViews; ++v) {
        std::memcpy(p.data(), proj + (size_t)v * U * V, p.size() * sizeof(float));
        core.InitView(v, p);
        parallel_for(nTasks, nthreads, [&](int t, int task) {
            for (int z = task * slicesPerTask; z < std::min(Z, (task + 1) * slicesPerTask); ++z)
                core.ProcessSlice(p, z, bufs[t]);
        });
    }
    FloatVec s((size_t)X * Y);
    for (int z = 0; z < Z; ++z) {
        core.DoneSlice(s, z);
        std::memcpy(out + (size_t)z * X * Y, s.data(), s.size() * sizeof(float));
    }
    return 0;
}

int jref_ctnum(float* inout, int width, int height, int nSlices, float norm0, float norm1, float muWater) {
    CTNumCore core(width, height, norm0, norm1, muWater);
    for (int s = 0; s < nSlices; ++s) core.Process(inout + (size_t)s * width * height);
    return 0;
}

// CompositeAgent + CompositeCore over views [v0, v0 + nv): pre holds the
// preprocessed frames of the whole rotation [N][H][W]; out [nv][H][2W].  View
// k is composited with view (k + N/2) % N, as InputAgent pairs them
// (JEngine/InputAgent.cpp:45-90, CompositeAgent.cpp:72-83).
int jref_composite(float* out, const float* pre, int v0, int nv, const float* ptms, int N, int W, int H,
                   int detRight, float dso, int nthreads) {
    std::vector<std::unique_ptr<CompositeCore>> cores;
    nthreads = std::max(1, std::min(nthreads, nv));
    const std::vector<ProjectionMatrix> pm = to_ptms(ptms, N);   // the cores keep a reference to it
    for (int t = 0; t < nthreads; ++t) cores.emplace_back(new CompositeCore(W, H, detRight != 0, dso, pm));
    const size_t px = (size_t)W * H;
    parallel_for(nv, nthreads, [&](int t, int i) {
        const int k = (v0 + i) % N, kc = (k + N / 2) % N;
        FloatVec o(px * 2), d(pre + px * k, pre + px * (k + 1)), c(pre + px * kc, pre + px * (kc + 1));
        cores[t]->Process(o, d, c, (size_t)k);
        std::memcpy(out + px * 2 * i, o.data(), sizeof(float) * px * 2);
    });
    return 0;
}

int jref_fft_length(int w) { return (int)FilterCore::CalFFTLength(w); }

}  // extern "C"
