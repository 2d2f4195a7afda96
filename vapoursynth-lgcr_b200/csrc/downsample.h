// Downsample filter (the reference's standalone 4:4:4 -> 4:2:0 guided
// downsampler, src/downsample.cpp): device descriptor and launch.
#pragma once

#include <cuda_runtime.h>

#include "recon.cuh"

namespace lgcr_b200 {

// Candidate planes of quality 2 (generateCandidateRow,
// src/downsample.cpp:524-569), each cw x ch floats.
enum DsCandidatePlane : int {
    kDsBaseU = 0, kDsBaseV = 1, kDsGate = 2, kDsCandU = 3, kDsCandV = 7, kDsPlanes = 11
};

struct DownsampleJob {
    int W, H;                           // source (4:4:4) size, both even
    int cw, ch;                         // output chroma size W / 2, H / 2
    int kind;                           // kU8 / kU16 / kF32 (input and output)
    float inScale, chromaOffset;        // SourcePlane scale, chroma offset
    float outScale, outOffset;          // OutputPlane scale and offset
    int maxCode;
    const void *in[3];
    long long inPitch[3];
    void *out[2];                       // output U, V (cw x ch)
    long long outPitch[2];
    int hSup, vSup;                     // polyphase tables of the base
    const int *hStart, *vStart;
    const float *hW, *vW;
    float2 *rows;                       // H x cw horizontal pass (U, V)
    float *cand;                        // kDsPlanes x cw x ch (quality 2)
    int quality;
    float strength, shiftX, shiftY;
};

cudaError_t launchDownsample(const DownsampleJob &J, cudaStream_t s);

} // namespace lgcr_b200
