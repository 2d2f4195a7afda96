// Host-side geometry of the Recon path: kernel profiles, polyphase tables,
// chroma sampling axes and radial (jinc) phase tables. Built once per
// filter/geometry in double precision on the host and uploaded resident.
//
// Each builder follows the reference's arithmetic step for step because the
// device kernels index these tables and must see identical float values:
//   kernelEval/sinc/jincWindowed/kernelSupport   src/lgcr.h:53-117
//   buildWeights                                 src/kernels.cpp:135-167
//   buildChromaAxisUncached                      src/kernels.cpp:337-404
//   buildBilinAxis (index/fraction part)         src/maps.cpp:190-208
//   collectPhases / buildRadialWeights           src/kernels.cpp:449-526
//   lutLookup                                    src/lgcr.h:636-641
//   buildLcMap footprint extents                 src/maps.cpp:429-447
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace lgcr_b200 {

enum class Kernel : int { Bilinear = 0, Bicubic = 1, Lanczos = 2, Spline16 = 3, Spline36 = 4, Jinc = 5 };

double sincd(double x);
double kernelEval(Kernel k, double x, double p1, double p2);
double jincWindowed(double x, double taps);
float lutLookup(const float *lut, int n, float idx);

struct KernelSpec {
    Kernel kernel = Kernel::Lanczos;
    double kp1 = 3.0, kp2 = 0.6;
    double support = 3.0;
    bool radial = false;
    std::vector<float> lut;     // jinc profile, 1024 entries per unit
    float lutScale = 0.0f;
};

struct WeightTable {
    int n = 0, sup = 0;
    std::vector<int> start;
    std::vector<float> w;       // n * sup
};

WeightTable buildWeights(int srcN, int dstN, const KernelSpec &k, double shift);

struct BilinAxis {
    std::vector<int> i0;
    std::vector<float> f;
};

BilinAxis buildBilinAxis(const std::vector<float> &pos, int srcN);

struct ChromaAxis {
    int n = 0, sup = 0;
    std::vector<int> start;
    std::vector<float> w;        // n * sup (normalized; zero for radial)
    std::vector<uint8_t> am;     // n * sup activity (0/1)
    std::vector<float> weightSum, absoluteWeightSum;
    std::vector<float> pos, lpos;
    BilinAxis chromaBilin, lumaBilin;
};

ChromaAxis buildChromaAxis(int srcLumaN, int dstLumaN, double r, double sitShift,
                           const KernelSpec &k);

struct RadialTable {
    bool valid = false;          // false: evaluate the LUT per tap
    int supportX = 0, supportY = 0, phaseCountX = 0, phaseCountY = 0;
    std::vector<uint16_t> xPhase, yPhase;
    std::vector<float> weights;
    std::vector<double> weightSum, absoluteWeightSum;
    // per phase pair: the guided rescue's kappa (max |w|)^2 / (sum w^2 + 1e-12)
    // over the active taps, in float and in tap order (rows, then columns)
    std::vector<float> kappa;
};

RadialTable buildRadialTable(const KernelSpec &k, const ChromaAxis &ax, const ChromaAxis &ay,
                             int sourceWidth, int sourceHeight);

// Per index of a separable chroma axis: the largest |weight| and the sum of
// squared weights over the active taps (the guided rescue term's kappa
// factors), in float and in tap order as the guided pass evaluates them.
void rescueFactors(const ChromaAxis &a, std::vector<float> &mx, std::vector<float> &ss);

// Footprint extents of each chroma sample on the luma grid.
void lcExtents(int lumaN, int chromaN, double r, double shift,
               std::vector<int> &begin, std::vector<int> &end);

} // namespace lgcr_b200
