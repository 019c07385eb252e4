// bpcuda_driver.cpp -- runs the reference's own GPU backprojector
// (BPCUDAAgent/BPCUDACore.cu + BPCUDACore.cpp, compiled unchanged from the
// JEngine sources by oracle/build.py into baseline/_ref) on caller buffers,
// through the host loop BPCUDAAgent drives it with.
//
// BASELINE INFRASTRUCTURE ONLY: loaded by bench.py to time the reference's
// GPU kernel beside the engine.  Nothing under jenhine_b200/ loads it.
//
// The loop follows BPCUDAAgent (BPCUDAAgent/BPCUDAAgent.cpp):
//   setup (untimed: the agent caches it in a weight file and loads it back)
//     PreCalculateWeight -- per view PreCalculate_Synced, DeployBackProjWeight,
//     SyncBackProjWeight, then BackupAccumulatedWeight (:193-215);
//   timed, one volume in one part (numReconParts = 1)
//     BackProjectAndAccumulate -- InitShot_Synced, then per view
//     PreCalculate_Synced, DeployBackProj, SyncBackProj (:217-253);
//     NormalizeAndOutput -- per slice DeployUpdateOutput, SyncUpdateOutput
//     (:255-274).
// Each view's filtered projection is uploaded into its own Tex2D<float>
// before the timed loop (the reference's Tex2DUploadAgent does that on
// another thread while the backprojector runs).
#include <chrono>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "BPCUDAAgent/BPCUDACore.h"
#include "CUDA/DeviceMemory.h"
#include "CUDA/Tex2D.h"
#include "Common/Exception.h"

using namespace JEngine;

static std::string g_err;

extern "C" {

const char* jrefgpu_last_error() { return g_err.c_str(); }

// filt: [nv][V][U] host floats (filtered projections); ptms: [nv][12].
// Writes the normalised volume [Z][Y][X] to out (host) when out != NULL, and
// the timings (ms): t[0] backprojection of every view, t[1] normalisation
// and output of every slice -- the means of `reps` timed runs after `warm`
// untimed ones (host clock; the reference synchronises its stream after
// every kernel) -- and t[2] the setup (texture uploads and weights).
int jrefgpu_bp(float* out, const float* filt, const float* ptms, int nv, int U, int V, int X, int Y, int Z,
               float pitch_xy, float pitch_z, int warm, int reps, double* t) {
    try {
        std::vector<ProjectionMatrix> p;
        p.reserve(nv);
        for (int i = 0; i < nv; ++i) p.emplace_back(ptms + 12 * (size_t)i);
        const auto c0 = std::chrono::steady_clock::now();
        BPCUDACore core(p, U, V, X, Y, Z, Z, pitch_xy, pitch_z);
        std::vector<std::unique_ptr<Tex2D<float>>> tex;
        tex.reserve(nv);
        for (int i = 0; i < nv; ++i) {
            tex.emplace_back(new Tex2D<float>(U, V));
            tex.back()->Set(filt + (size_t)i * U * V);
        }
        // weights, as PreCalculateWeight does for part 0
        core.InitShot_Synced();
        for (int v = 0; v < nv; ++v) {
            core.PreCalculate_Synced(0, v);
            core.DeployBackProjWeight(0, v);
            core.SyncBackProjWeight();
        }
        core.BackupAccumulatedWeight(0);
        cudaDeviceSynchronize();
        const auto c1 = std::chrono::steady_clock::now();
        t[2] = std::chrono::duration<double, std::milli>(c1 - c0).count();
        DeviceMemory<float> slice((size_t)X * Y);
        t[0] = t[1] = 0.0;
        for (int r = 0; r < warm + reps; ++r) {
            const auto a = std::chrono::steady_clock::now();
            core.InitShot_Synced();
            for (int v = 0; v < nv; ++v) {
                core.PreCalculate_Synced(0, v);
                core.DeployBackProj(*tex[v], 0, v);
                core.SyncBackProj();
            }
            const auto b = std::chrono::steady_clock::now();
            for (int z = 0; z < Z; ++z) {
                core.DeployUpdateOutput(slice, 0, z);
                core.SyncUpdateOutput();
                if (out && r == warm + reps - 1)
                    cudaMemcpy(out + (size_t)z * X * Y, slice.Data(), sizeof(float) * X * Y, cudaMemcpyDeviceToHost);
            }
            const auto c = std::chrono::steady_clock::now();
            if (r >= warm) {
                t[0] += std::chrono::duration<double, std::milli>(b - a).count() / reps;
                t[1] += std::chrono::duration<double, std::milli>(c - b).count() / reps;
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
}

}  // extern "C"
