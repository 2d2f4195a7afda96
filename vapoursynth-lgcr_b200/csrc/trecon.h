// TRecon preparation stages (tReconGetFrame src/plugin.cpp:796-840): the
// frames' float planes, the neighbours' footprint luma maps, 16x16 block
// matching on luma (blockMatch src/algos.cpp:683-755) and the per-block
// chroma-consistency confidence (applyChromaConsistency
// src/algos.cpp:757-807). Their outputs feed the guided pass's temporal
// taps (TemporalView).
#pragma once

#include <cuda_runtime.h>

#include "recon.cuh"

namespace lgcr_b200 {

constexpr int kTReconMaxFrames = 17;        // the frame and up to 2 * 8 neighbours
constexpr int kTReconBlock = 16;            // block size of the motion search

struct TReconPrep {
    int sw, sh, cw, ch;
    int kind;                               // kU8 / kU16 / kF32
    int frames;                             // 1 + neighbours
    double yScale, cOffset;                 // planeToFloat
    const void *in[kTReconMaxFrames][3];
    long long inPitch[kTReconMaxFrames][3];
    float *f[kTReconMaxFrames][3];          // float planes; index 0 is the frame
    float *lc[kTReconMaxFrames];            // neighbours' footprint maps (index >= 1)
    short *mvx[kTReconMaxFrames], *mvy[kTReconMaxFrames];
    float *conf[kTReconMaxFrames];
    int bw, bh;                             // block grid
    int search;                             // tsearch
    float tsad;
    double rw, rh;
    const int *lcXb, *lcXe, *lcYb, *lcYe;   // footprint extents at the frame's siting
};

// Enqueues conversion, footprint maps, block matching and the consistency
// check for neighbours 1 .. frames - 1. Returns the number of launches, or
// -1 when a launch failed.
int launchTReconPrep(const TReconPrep &P, cudaStream_t s);

} // namespace lgcr_b200
