// Host geometry tables; see geometry.h for the reference functions each
// builder follows. Compiled without FMA contraction so every double and
// float expression rounds exactly as the reference's x86-64 build does.
#include "geometry.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

namespace lgcr_b200 {

double sincd(double x) {
    if (std::fabs(x) < 1e-8)
        return 1.0;
    x *= M_PI;
    return std::sin(x) / x;
}

double kernelEval(Kernel k, double x, double p1, double p2) {
    x = std::fabs(x);
    switch (k) {
    case Kernel::Bilinear:
        return x < 1.0 ? 1.0 - x : 0.0;
    case Kernel::Bicubic: {
        const double b = p1, c = p2;
        if (x < 1.0)
            return ((12 - 9 * b - 6 * c) * x * x * x + (-18 + 12 * b + 6 * c) * x * x + (6 - 2 * b)) / 6.0;
        if (x < 2.0)
            return ((-b - 6 * c) * x * x * x + (6 * b + 30 * c) * x * x + (-12 * b - 48 * c) * x + (8 * b + 24 * c)) / 6.0;
        return 0.0;
    }
    case Kernel::Lanczos:
        return x < p1 ? sincd(x) * sincd(x / p1) : 0.0;
    case Kernel::Spline16:
        if (x < 1.0)
            return ((x - 9.0 / 5.0) * x - 1.0 / 5.0) * x + 1.0;
        if (x < 2.0)
            return ((-1.0 / 3.0 * (x - 1.0) + 4.0 / 5.0) * (x - 1.0) - 7.0 / 15.0) * (x - 1.0);
        return 0.0;
    case Kernel::Spline36:
        if (x < 1.0)
            return ((13.0 / 11.0 * x - 453.0 / 209.0) * x - 3.0 / 209.0) * x + 1.0;
        if (x < 2.0)
            return ((-6.0 / 11.0 * (x - 1.0) + 270.0 / 209.0) * (x - 1.0) - 156.0 / 209.0) * (x - 1.0);
        if (x < 3.0)
            return ((1.0 / 11.0 * (x - 2.0) - 45.0 / 209.0) * (x - 2.0) + 26.0 / 209.0) * (x - 2.0);
        return 0.0;
    case Kernel::Jinc:
        break;
    }
    return 0.0;
}

double jincWindowed(double x, double taps) {
    x = std::fabs(x);
    if (x >= taps)
        return 0.0;
    const double j = (x < 1e-8) ? 1.0 : 2.0 * std::cyl_bessel_j(1.0, M_PI * x) / (M_PI * x);
    return j * sincd(x / taps);
}

float lutLookup(const float *lut, int n, float idx) {
    int i0 = static_cast<int>(idx);
    i0 = std::clamp(i0, 0, n - 2);
    const float fr = std::min(idx - float(i0), 1.0f);
    return lut[i0] + (lut[i0 + 1] - lut[i0]) * fr;
}

WeightTable buildWeights(int srcN, int dstN, const KernelSpec &k, double shift) {
    WeightTable t;
    t.n = dstN;
    const double scale = double(srcN) / dstN;
    const double sup = (scale > 1.0) ? k.support * scale : k.support;
    const double invScale = (scale > 1.0) ? 1.0 / scale : 1.0;
    t.sup = std::max(1, 2 * static_cast<int>(std::ceil(sup)));
    t.start.resize(dstN);
    t.w.assign(size_t(dstN) * t.sup, 0.0f);
    for (int i = 0; i < dstN; ++i) {
        const double center = (i + 0.5) * scale - 0.5 + shift;
        int first = static_cast<int>(std::ceil(center - sup));
        first = std::clamp(first, -(t.sup) + 1, srcN - 1);
        if (first + t.sup > srcN)
            first = std::max(-(t.sup) + 1, srcN - t.sup);
        t.start[i] = first;
        double sum = 0.0;
        for (int j = 0; j < t.sup; ++j) {
            const double d = (first + j) - center;
            const double w = kernelEval(k.kernel, d * invScale, k.kp1, k.kp2);
            t.w[size_t(i) * t.sup + j] = static_cast<float>(w);
            sum += w;
        }
        if (std::fabs(sum) > 1e-9)
            for (int j = 0; j < t.sup; ++j)
                t.w[size_t(i) * t.sup + j] /= static_cast<float>(sum);
    }
    return t;
}

BilinAxis buildBilinAxis(const std::vector<float> &pos, int srcN) {
    BilinAxis a;
    const int n = static_cast<int>(pos.size());
    a.i0.assign(n, 0);
    a.f.assign(n, 0.0f);
    if (srcN == 1)
        return a;
    for (int i = 0; i < n; ++i) {
        const float x = pos[i];
        int j = static_cast<int>(std::floor(x));
        float fr = x - j;
        if (j < 0) { j = 0; fr = 0.0f; }
        if (j > srcN - 2) { j = srcN - 2; fr = 1.0f; }
        a.i0[i] = j;
        a.f[i] = fr;
    }
    return a;
}

ChromaAxis buildChromaAxis(int srcLumaN, int dstLumaN, double r, double sitShift,
                           const KernelSpec &k) {
    ChromaAxis a;
    a.n = dstLumaN;
    const double scaleC = (double(srcLumaN) / r) / dstLumaN;
    const double widenC = k.radial ? std::max(1.0, scaleC) : 1.0;
    a.sup = std::max(1, 2 * static_cast<int>(std::ceil(k.support * widenC)));
    a.start.resize(a.n);
    a.pos.resize(a.n);
    a.lpos.resize(a.n);
    a.w.assign(size_t(a.n) * a.sup, 0.0f);
    a.am.assign(size_t(a.n) * a.sup, 0);
    a.weightSum.assign(a.n, 0.0f);
    a.absoluteWeightSum.assign(a.n, 0.0f);
    // Chroma sample count implied by the integer ratio (as the reference
    // derives it; equal to the chroma width whenever the ratio is integral).
    const int srcChromaN = (srcLumaN + static_cast<int>(r) - 1) / static_cast<int>(r);
    const double scale = double(srcLumaN) / dstLumaN;
    for (int i = 0; i < a.n; ++i) {
        const double lx = (i + 0.5) * scale - 0.5;
        const double sc = (lx + 0.5 - sitShift) / r - 0.5;
        a.pos[i] = static_cast<float>(sc);
        a.lpos[i] = static_cast<float>(lx);
        int first = static_cast<int>(std::ceil(sc - k.support * widenC));
        first = std::clamp(first, 0, std::max(0, srcChromaN - a.sup));
        a.start[i] = first;
        for (int j = 0; j < a.sup; ++j)
            if (std::fabs((first + j) - sc) < k.support * widenC)
                a.am[size_t(i) * a.sup + j] = 1;
        if (k.radial)
            continue;
        double sum = 0.0;
        for (int j = 0; j < a.sup; ++j) {
            const double dist = (first + j) - sc;
            const double w = kernelEval(k.kernel, dist, k.kp1, k.kp2);
            a.w[size_t(i) * a.sup + j] = static_cast<float>(w);
            sum += w;
        }
        if (std::fabs(sum) > 1e-9)
            for (int j = 0; j < a.sup; ++j)
                a.w[size_t(i) * a.sup + j] /= static_cast<float>(sum);
        for (int j = 0; j < a.sup; ++j) {
            if (a.am[size_t(i) * a.sup + j] == 0)
                continue;
            const float weight = a.w[size_t(i) * a.sup + j];
            a.weightSum[i] += weight;
            a.absoluteWeightSum[i] += std::fabs(weight);
        }
    }
    a.chromaBilin = buildBilinAxis(a.pos, srcChromaN);
    a.lumaBilin = buildBilinAxis(a.lpos, srcLumaN);
    return a;
}

namespace {

struct PhaseKey {
    uint32_t offsetBits;
    uint64_t activity;
    bool operator==(const PhaseKey &o) const {
        return offsetBits == o.offsetBits && activity == o.activity;
    }
};
struct PhaseKeyHash {
    size_t operator()(const PhaseKey &k) const {
        return std::hash<uint64_t>{}(k.activity) * 1000003u ^ k.offsetBits;
    }
};

// Phase ids are assigned in order of first occurrence along the axis.
bool collectPhases(const ChromaAxis &axis, std::vector<uint16_t> &indices,
                   std::vector<float> &offsets, std::vector<uint64_t> &activity) {
    if (axis.sup > 64)
        return false;
    std::unordered_map<PhaseKey, uint16_t, PhaseKeyHash> unique;
    indices.resize(axis.n);
    for (int x = 0; x < axis.n; ++x) {
        const float offset = axis.start[x] - axis.pos[x];
        uint32_t bits;
        std::memcpy(&bits, &offset, sizeof(bits));
        uint64_t mask = 0;
        for (int tap = 0; tap < axis.sup; ++tap)
            if (axis.am[size_t(x) * axis.sup + tap] != 0)
                mask |= uint64_t{1} << tap;
        const PhaseKey key{bits, mask};
        const uint16_t next = static_cast<uint16_t>(unique.size());
        auto [it, inserted] = unique.emplace(key, next);
        if (inserted) {
            if (unique.size() > 64)
                return false;
            offsets.push_back(offset);
            activity.push_back(mask);
        }
        indices[x] = it->second;
    }
    return true;
}

} // namespace

RadialTable buildRadialTable(const KernelSpec &k, const ChromaAxis &ax, const ChromaAxis &ay,
                             int sourceWidth, int sourceHeight) {
    RadialTable t;
    t.supportX = ax.sup;
    t.supportY = ay.sup;
    std::vector<float> xOffsets, yOffsets;
    std::vector<uint64_t> xActivity, yActivity;
    if (!collectPhases(ax, t.xPhase, xOffsets, xActivity) ||
        !collectPhases(ay, t.yPhase, yOffsets, yActivity))
        return t;
    const size_t phasePairs = xOffsets.size() * yOffsets.size();
    const size_t perPhase = size_t(ax.sup) * ay.sup;
    if (phasePairs > 1024 || phasePairs * perPhase > 262144)
        return t;
    t.valid = true;
    t.phaseCountX = int(xOffsets.size());
    t.phaseCountY = int(yOffsets.size());
    t.weights.assign(phasePairs * perPhase, 0.0f);
    t.weightSum.resize(phasePairs);
    t.absoluteWeightSum.resize(phasePairs);
    t.kappa.resize(phasePairs);
    const float invX = float(std::min(1.0, double(ax.n) / sourceWidth));
    const float invY = float(std::min(1.0, double(ay.n) / sourceHeight));
    const int lutN = int(k.lut.size());
    for (int py = 0; py < t.phaseCountY; ++py)
        for (int px = 0; px < t.phaseCountX; ++px) {
            float *w = t.weights.data() + (size_t(py) * t.phaseCountX + px) * perPhase;
            for (int j = 0; j < ay.sup; ++j)
                for (int i = 0; i < ax.sup; ++i) {
                    if ((xActivity[px] & (uint64_t{1} << i)) == 0 ||
                        (yActivity[py] & (uint64_t{1} << j)) == 0)
                        continue;
                    const float dx = (xOffsets[px] + i) * invX;
                    const float dy = (yOffsets[py] + j) * invY;
                    w[size_t(j) * ax.sup + i] =
                        lutLookup(k.lut.data(), lutN, std::sqrt(dx * dx + dy * dy) * k.lutScale);
                }
            const size_t phase = size_t(py) * t.phaseCountX + px;
            double sum = 0.0, absSum = 0.0;
            for (size_t i = 0; i < perPhase; ++i) {
                sum += w[i];
                absSum += std::fabs(w[i]);
            }
            t.weightSum[phase] = sum;
            t.absoluteWeightSum[phase] = absSum;
            float m = 0.0f, q = 0.0f;
            for (int j = 0; j < ay.sup; ++j)
                for (int i = 0; i < ax.sup; ++i) {
                    if ((xActivity[px] & (uint64_t{1} << i)) == 0 ||
                        (yActivity[py] & (uint64_t{1} << j)) == 0)
                        continue;
                    const float wv = w[size_t(j) * ax.sup + i];
                    m = (m < std::fabs(wv)) ? std::fabs(wv) : m;
                    q += wv * wv;
                }
            t.kappa[phase] = (m * m) / (q + 1e-12f);
        }
    return t;
}

void rescueFactors(const ChromaAxis &a, std::vector<float> &mx, std::vector<float> &ss) {
    mx.assign(a.n, 0.0f);
    ss.assign(a.n, 0.0f);
    if (a.w.empty())
        return;                                   // radial axes carry no weights
    for (int i = 0; i < a.n; ++i) {
        float m = 0.0f, q = 0.0f;
        for (int j = 0; j < a.sup; ++j) {
            if (a.am[size_t(i) * a.sup + j] == 0)
                continue;
            const float w = a.w[size_t(i) * a.sup + j];
            m = (m < std::fabs(w)) ? std::fabs(w) : m;
            q += w * w;
        }
        mx[i] = m;
        ss[i] = q;
    }
}

void lcExtents(int lumaN, int chromaN, double r, double shift,
               std::vector<int> &begin, std::vector<int> &end) {
    begin.resize(chromaN);
    end.resize(chromaN);
    for (int c = 0; c < chromaN; ++c) {
        const double l = (c + 0.5) * r - 0.5 + shift;
        int first = static_cast<int>(std::ceil(l - 0.5 * r));
        int last = static_cast<int>(std::ceil(l + 0.5 * r));
        first = std::clamp(first, 0, lumaN - 1);
        last = std::clamp(last, first + 1, lumaN);
        begin[c] = first;
        end[c] = last;
    }
}

} // namespace lgcr_b200
