// Sharpen filter (the reference's SharpenData / sharpenPlane,
// src/lgcr.h:968-980, src/algos.cpp:595-659): device descriptor and launch.
#pragma once

#include <cuda_runtime.h>

#include "recon.cuh"

namespace lgcr_b200 {

struct SharpenJob {
    int sw, sh, cw, ch;
    int kind;                           // kU8 / kU16 / kF32 (input and output)
    double yScale, cOffset;             // planeToFloat scale, chroma offset
    float qScale, qOffC;                // floatToPlane scale, chroma offset
    int maxCode;
    const void *in[3];
    long long inPitch[3];
    void *out[3];
    long long outPitch[3];
    float *Ys;                          // sw x sh sharpened luma (chroma guide)
    float alpha, sigma, sratio, invG2, margin;
    int clampHull;                      // ar >= 0
    int guided;                         // chroma subsampled: guided by the luma
    double rw, rh, shiftX, shiftY;      // sw / cw, sh / ch, left siting
    const int *lcXb, *lcXe, *lcYb, *lcYe;   // luma footprint of each chroma sample
};

cudaError_t launchSharpen(const SharpenJob &J, cudaStream_t s);

} // namespace lgcr_b200
