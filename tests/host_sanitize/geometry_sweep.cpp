// Host geometry builders under AddressSanitizer and UndefinedBehaviorSanitizer.
//
// Every table the Recon kernels index on the device (chroma axes with their
// bilinear axes, polyphase luma tables, radial phase tables, lc footprint
// extents, rescue factors) is built here over degenerate and real sizes,
// every kernel profile, integer and half-sample sitings, subsampled and full
// chroma, same size, upscale and downscale. Besides the sanitizers' own
// checks, each table is tested for the structural facts the device code
// relies on (sizes, index ranges, fractions in [0, 1], finite weights).
// Exit status: 0 when every check held; the failures are listed on stderr.
#include "geometry.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

using namespace lgcr_b200;

namespace {

int failures = 0;

#define CHECK(cond, ...)                                                                     \
    do {                                                                                     \
        if (!(cond)) {                                                                       \
            if (++failures <= 50) {                                                          \
                std::fprintf(stderr, "check failed: %s: ", #cond);                           \
                std::fprintf(stderr, __VA_ARGS__);                                           \
                std::fputc('\n', stderr);                                                    \
            }                                                                                \
        }                                                                                    \
    } while (0)

// The kernel profiles as the filter constructor sets them up.
KernelSpec makeSpec(Kernel kind, int taps) {
    KernelSpec k;
    k.kernel = kind;
    switch (kind) {
    case Kernel::Bilinear: k.support = 1.0; break;
    case Kernel::Bicubic: k.support = 2.0; k.kp1 = 0.0; k.kp2 = 0.6; break;
    case Kernel::Lanczos: k.kp1 = taps; k.support = taps; break;
    case Kernel::Spline16: k.support = 2.0; break;
    case Kernel::Spline36: k.support = 3.0; break;
    case Kernel::Jinc: {
        k.radial = true;
        k.kp1 = taps;
        k.support = taps;
        const int n = static_cast<int>(k.support * 1024) + 2;
        k.lut.resize(n);
        for (int i = 0; i < n; ++i)
            k.lut[i] = static_cast<float>(jincWindowed(double(i) / 1024.0, k.support));
        k.lutScale = 1024.0f;
        break;
    }
    }
    return k;
}

void checkBilin(const BilinAxis &b, size_t n, int srcN, const char *what, int src, int dst) {
    CHECK(b.i0.size() == n && b.f.size() == n, "%s sizes (%d -> %d)", what, src, dst);
    const int hi = std::max(0, srcN - 2);
    for (size_t i = 0; i < std::min(n, b.i0.size()); ++i) {
        CHECK(b.i0[i] >= 0 && b.i0[i] <= hi, "%s i0[%zu] = %d, src %d", what, i, b.i0[i], srcN);
        CHECK(b.f[i] >= 0.0f && b.f[i] <= 1.0f, "%s f[%zu] = %g", what, i, double(b.f[i]));
    }
}

void checkAxis(const ChromaAxis &a, int srcLuma, int dst, int r, const KernelSpec &k) {
    const int srcChroma = (srcLuma + r - 1) / r;
    CHECK(a.n == dst && a.sup >= 1, "axis n %d sup %d (%d -> %d)", a.n, a.sup, srcLuma, dst);
    const size_t cells = size_t(a.n) * a.sup;
    CHECK(a.start.size() == size_t(a.n) && a.w.size() == cells && a.am.size() == cells &&
              a.pos.size() == size_t(a.n) && a.lpos.size() == size_t(a.n) &&
              a.weightSum.size() == size_t(a.n) && a.absoluteWeightSum.size() == size_t(a.n),
          "axis table sizes (%d -> %d)", srcLuma, dst);
    const int startHi = std::max(0, srcChroma - a.sup);
    for (int i = 0; i < a.n && size_t(i) < a.start.size(); ++i) {
        CHECK(a.start[i] >= 0 && a.start[i] <= startHi, "axis start[%d] = %d (chroma %d, sup %d)", i,
              a.start[i], srcChroma, a.sup);
        CHECK(std::isfinite(a.pos[i]) && std::isfinite(a.lpos[i]), "axis pos[%d]", i);
        CHECK(std::isfinite(a.weightSum[i]) && std::isfinite(a.absoluteWeightSum[i]),
              "axis sums[%d]", i);
    }
    for (size_t c = 0; c < std::min(cells, a.w.size()); ++c) {
        CHECK(std::isfinite(a.w[c]), "axis w[%zu] = %g", c, double(a.w[c]));
        CHECK(a.am[c] <= 1, "axis am[%zu] = %d", c, int(a.am[c]));
        if (k.radial)
            CHECK(a.w[c] == 0.0f, "radial axis carries a weight at %zu", c);
    }
    checkBilin(a.chromaBilin, size_t(a.n), srcChroma, "chroma bilinear", srcLuma, dst);
    checkBilin(a.lumaBilin, size_t(a.n), srcLuma, "luma bilinear", srcLuma, dst);
    std::vector<float> mx, ss;
    rescueFactors(a, mx, ss);
    CHECK(mx.size() == size_t(a.n) && ss.size() == size_t(a.n), "rescue factor sizes");
    for (size_t i = 0; i < std::min(mx.size(), ss.size()); ++i)
        CHECK(std::isfinite(mx[i]) && std::isfinite(ss[i]) && mx[i] >= 0.0f && ss[i] >= 0.0f,
              "rescue factors[%zu]", i);
}

void checkWeights(const WeightTable &t, int src, int dst) {
    CHECK(t.n == dst && t.sup >= 1, "weights n %d sup %d (%d -> %d)", t.n, t.sup, src, dst);
    CHECK(t.start.size() == size_t(dst) && t.w.size() == size_t(dst) * t.sup,
          "weights sizes (%d -> %d)", src, dst);
    for (size_t i = 0; i < t.start.size(); ++i)
        CHECK(t.start[i] >= -(t.sup - 1) && t.start[i] <= src - 1, "weights start[%zu] = %d", i,
              t.start[i]);
    for (size_t c = 0; c < t.w.size(); ++c)
        CHECK(std::isfinite(t.w[c]), "weights w[%zu]", c);
}

void checkRadial(const RadialTable &t, const ChromaAxis &ax, const ChromaAxis &ay) {
    if (!t.valid)
        return;                                    // the kernels evaluate the LUT per tap
    CHECK(t.xPhase.size() == size_t(ax.n) && t.yPhase.size() == size_t(ay.n), "phase index sizes");
    for (uint16_t p : t.xPhase)
        CHECK(p < t.phaseCountX, "x phase %d of %d", int(p), t.phaseCountX);
    for (uint16_t p : t.yPhase)
        CHECK(p < t.phaseCountY, "y phase %d of %d", int(p), t.phaseCountY);
    const size_t pairs = size_t(t.phaseCountX) * t.phaseCountY;
    CHECK(t.weights.size() == pairs * t.supportX * t.supportY && t.kappa.size() == pairs &&
              t.weightSum.size() == pairs && t.absoluteWeightSum.size() == pairs,
          "radial table sizes");
    for (float w : t.weights)
        CHECK(std::isfinite(w), "radial weight");
    for (float q : t.kappa)
        CHECK(std::isfinite(q) && q >= 0.0f, "radial kappa");
}

void checkExtents(int luma, int chroma, int r, double shift) {
    std::vector<int> b, e;
    lcExtents(luma, chroma, r, shift, b, e);
    CHECK(b.size() == size_t(chroma) && e.size() == size_t(chroma), "extent sizes");
    for (int c = 0; c < chroma && size_t(c) < b.size(); ++c)
        CHECK(b[c] >= 0 && b[c] < e[c] && e[c] <= luma, "extent %d: [%d, %d) of %d", c, b[c], e[c],
              luma);
}

} // namespace

int main() {
    const int sizes[] = {1, 2, 3, 4, 5, 7, 8, 16, 17, 33, 64, 135, 540};
    const double shifts[] = {0.0, 0.5, -0.5};
    const struct { Kernel kind; int taps; } kernels[] = {
        {Kernel::Bilinear, 0}, {Kernel::Bicubic, 0}, {Kernel::Lanczos, 1}, {Kernel::Lanczos, 3},
        {Kernel::Lanczos, 4}, {Kernel::Lanczos, 8}, {Kernel::Spline16, 0}, {Kernel::Spline36, 0},
        {Kernel::Jinc, 1}, {Kernel::Jinc, 3}};
    long tables = 0;
    for (const auto &kd : kernels) {
        const KernelSpec k = makeSpec(kd.kind, kd.taps);
        for (int src : sizes)
            for (int r = 1; r <= 2; ++r) {
                const int chroma = (src + r - 1) / r;
                const int dsts[] = {src, 2 * src, src + src / 2 + 1, std::max(1, src / 2), 3};
                for (int dst : dsts)
                    for (double shift : shifts) {
                        const ChromaAxis a = buildChromaAxis(src, dst, double(r), shift, k);
                        checkAxis(a, src, dst, r, k);
                        ++tables;
                        if (!k.radial) {
                            checkWeights(buildWeights(src, dst, k, shift), src, dst);
                            checkWeights(buildWeights(src, chroma, k, shift), src, chroma);
                            tables += 2;
                        }
                    }
                for (double shift : shifts)
                    checkExtents(src, chroma, r, shift);
            }
        if (!k.radial)
            continue;
        // radial phase tables over pairs of axes (width x height)
        const int pairs[][2] = {{1, 1}, {1, 17}, {17, 1}, {2, 2}, {16, 12}, {33, 17}, {135, 64}};
        for (const auto &wh : pairs)
            for (int r = 1; r <= 2; ++r)
                for (int up = 1; up <= 2; ++up) {
                    const int w = wh[0], h = wh[1];
                    const ChromaAxis ax = buildChromaAxis(w, up * w, double(r), 0.0, k);
                    const ChromaAxis ay = buildChromaAxis(h, up * h, double(r), 0.5, k);
                    checkRadial(buildRadialTable(k, ax, ay, (w + r - 1) / r, (h + r - 1) / r), ax,
                                ay);
                    ++tables;
                }
    }
    std::printf("%ld tables checked, %d failures\n", tables, failures);
    return failures == 0 ? 0 : 1;
}
